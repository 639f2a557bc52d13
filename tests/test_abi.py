"""The C-ABI library loads and exports every entry point include/*.h declares;
host-side behaviour that needs no GPU."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(binder_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "binder_score_batch" in names and "binder_create" in names and len(names) > 25


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (binder_\w+)", out))
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, missing
    L = pkg.lib()
    for n in declared_symbols():
        assert getattr(L, n) is not None


def test_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "binder_gpu.h"\nint main(void){ binder_params p; binder_default_params(&p);'
                   ' return (int)sizeof(binder_gpu_atom) - 32; }\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-c", "-I", str(ROOT / "include"), str(src), "-o",
                    str(tmp_path / "t.o")], check=True)


def test_status_strings_and_abi_version(pkg):
    L = pkg.lib()
    assert L.binder_abi_version() == 2
    assert L.binder_status_string(0) == b"ok"
    assert b"sm_100" in L.binder_status_string(8)


def test_gpu_atom_layout(pkg):
    # gpu.rs:17-29: #[repr(C)] 8 x f32 = 32 bytes
    assert pkg.GPU_ATOM.itemsize == 32
    assert list(pkg.GPU_ATOM.names) == ["x", "y", "z", "q", "r_min_half", "epsilon", "hydrophobic", "_pad"]


def test_params_struct_matches_header(pkg):
    assert C.sizeof(pkg.Params) == 16 * 4 + 8


def test_try_init_without_device_returns_none(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert pkg.GpuContext.try_init() is None
    with pytest.raises(pkg.BinderError) as e:
        pkg.GpuContext.create()
    assert e.value.status == 8  # BINDER_ERR_NODEVICE: no CPU fallback


def test_atom_cloud_from_slots_matches_oracle_flatten(pkg, oracle):
    rng = np.random.default_rng(5)
    aa = rng.integers(0, 20, 30).astype(np.uint8)
    ca = rng.normal(size=(30, 3)).astype(np.float32) * 10
    pos, _ = oracle.build_residues(ca, aa)
    c = pkg.AtomCloud.from_slots(aa, pos)
    o = oracle.flatten(aa, pos)
    for a, b in [("x", "x"), ("y", "y"), ("z", "z"), ("charge", "q"), ("r_min_half", "rmh"), ("epsilon", "eps"),
                 ("hydrophobic", "hyd"), ("atom_type", "type"), ("residue_idx", "resi")]:
        assert np.array_equal(getattr(c, a), o[b]), a
