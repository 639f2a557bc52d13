"""binder_b200 — B200 (sm_100a) all-atom scoring + search for de novo antibody design.

Python host-side mirror of the reference engine's GPU interface (Rust crate
DilaDeniz/de-novo-antigen-binder): ``GpuContext.try_init`` / ``score_batch``
(gpu.rs:55,166), ``AtomCloud`` (allatom.rs:17), ``ResidueCloud`` (atom.rs:185),
``SpatialHashGrid`` (spatial.rs:12) and ``compute_forces_with_grid``
(energy.rs:322).  Every call goes through the C ABI of ``libbinder_b200.so``
(include/binder_gpu.h); there is no CPU fallback — importing the package
without the built library, or creating a context without an sm_100 device,
fails loudly.

The package directory name contains dashes, so it is imported under the name
``binder_b200`` by :func:`load` in the repository's entry points.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libbinder_b200.so"
SLOTS = 14
N_AA = 20

AMINO_ACIDS = ["Ala", "Arg", "Asn", "Asp", "Cys", "Gln", "Glu", "Gly", "His", "Ile",
               "Leu", "Lys", "Met", "Phe", "Pro", "Ser", "Thr", "Trp", "Tyr", "Val"]
ONE_LETTER = "ARNDCQEGHILKMFPSTWYV"

# GpuAtom (gpu.rs:17-29): 8 x f32
GPU_ATOM = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("q", "<f4"), ("r_min_half", "<f4"),
                     ("epsilon", "<f4"), ("hydrophobic", "<f4"), ("_pad", "<f4")])

STATUS = {0: "BINDER_OK", 1: "BINDER_ERR_ARG", 2: "BINDER_ERR_CUDA", 3: "BINDER_ERR_OOM", 4: "BINDER_ERR_TIMEOUT",
          5: "BINDER_ERR_NAN", 6: "BINDER_ERR_GRID", 7: "BINDER_ERR_STATE", 8: "BINDER_ERR_NODEVICE",
          9: "BINDER_ERR_CAPACITY"}
ACC_KAHAN, ACC_F32 = 0, 1


class BinderError(RuntimeError):
    def __init__(self, status, message=""):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{self.name}: {message}" if message else self.name)


class _AtomCloudC(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("charge", C.c_void_p),
                ("r_min_half", C.c_void_p), ("epsilon", C.c_void_p), ("hydrophobic", C.c_void_p),
                ("atom_type", C.c_void_p), ("residue_idx", C.c_void_p), ("n", C.c_size_t)]


class _ResidueCloudC(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("amino_acid", C.c_void_p),
                ("n", C.c_size_t)]


class Params(C.Structure):
    """binder_params (include/binder_gpu.h); defaults = reference constants."""
    _fields_ = [("step", C.c_float), ("noise_base", C.c_float), ("t_hot", C.c_float), ("t_cold", C.c_float),
                ("mutation_p", C.c_float), ("rotamer_move_p", C.c_float), ("backbone_move_p", C.c_float),
                ("max_torsion_deg", C.c_float), ("iface_cutoff_sq", C.c_float), ("shell_radius", C.c_float),
                ("max_disp", C.c_float), ("restraint_k", C.c_float), ("ca_cell", C.c_float),
                ("score_cell", C.c_float), ("accumulate", C.c_int32), ("flags", C.c_int32),
                ("seed", C.c_uint64)]

    @classmethod
    def defaults(cls, **kw):
        p = cls()
        lib().binder_default_params(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        return p


class LaunchCfg(C.Structure):
    """binder_launch_cfg (include/binder_gpu.h): launch shapes of the search block."""
    _fields_ = [("score_warps", C.c_int32), ("score_ctas_per_sm", C.c_int32), ("cg_warps", C.c_int32),
                ("cg_lanes", C.c_int32), ("cg_order", C.c_int32), ("score_order", C.c_int32),
                ("cg_queue", C.c_int32), ("cg_flat", C.c_int32)]

    def as_dict(self):
        return {"score_warps": self.score_warps, "score_ctas_per_sm": self.score_ctas_per_sm,
                "cg_warps": self.cg_warps, "cg_lanes": self.cg_lanes, "cg_order": self.cg_order,
                "score_order": self.score_order, "cg_queue": self.cg_queue, "cg_flat": self.cg_flat}


FLAG_GRAPH = 1
FLAG_AUTOTUNE = 2


class RunCfg(C.Structure):
    """binder_run_cfg (include/binder_gpu.h): the run_allatom schedule."""
    _fields_ = [("phase1_steps", C.c_int32), ("score_every", C.c_int32), ("survivors", C.c_int32),
                ("phase2_steps", C.c_int32), ("top_n", C.c_int32), ("phase1_mc", C.c_int32)]

    @classmethod
    def defaults(cls, **kw):
        c = cls()
        lib().binder_default_run_cfg(C.byref(c))
        for k, v in kw.items():
            setattr(c, k, v)
        return c


_LIB = None

_SIGS = {
    "binder_abi_version": (C.c_int, []),
    "binder_status_string": (C.c_char_p, [C.c_int]),
    "binder_default_params": (None, [C.c_void_p]),
    "binder_create": (C.c_void_p, [C.c_int, C.c_void_p, C.POINTER(C.c_int)]),
    "binder_destroy": (None, [C.c_void_p]),
    "binder_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "binder_last_error": (C.c_char_p, [C.c_void_p]),
    "binder_synchronize": (C.c_int, [C.c_void_p]),
    "binder_launch_count": (C.c_uint64, [C.c_void_p]),
    "binder_table_residue": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "binder_table_atom_type": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "binder_table_rotamers": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p]),
    "binder_table_residue_level": (C.c_int, [C.c_int, C.c_void_p]),
    "binder_score_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p,
                                     C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_score_batch_f64": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p,
                                         C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_score_batch_ragged": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                            C.c_void_p]),
    "binder_set_antigen_atoms": (C.c_int, [C.c_void_p, C.c_void_p]),
    "binder_last_pair_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "binder_grid_cells": (C.c_int, [C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                    C.c_void_p]),
    "binder_grid_neighbors": (C.c_int, [C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                        C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_compute_forces_with_grid": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_void_p]),
    "binder_forces_allatom": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                        C.c_void_p]),
    "binder_topk": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p]),
    "binder_topk_segmented": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p]),
    "binder_build_residues": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "binder_add_antigen": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
    "binder_clear_antigens": (C.c_int, [C.c_void_p]),
    "binder_state_upload": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]),
    "binder_state_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "binder_diffuse": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_int, C.c_int, C.c_void_p]),
    "binder_score_state": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "binder_block": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p]),
    "binder_stream": (C.c_void_p, [C.c_void_p]),
    "binder_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "binder_timing_summary": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
    "binder_block_fetch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "binder_block_io": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "binder_state_pair_counts": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "binder_fp32_peak": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "binder_mc_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "binder_state_select": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "binder_state_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p]),
    "binder_default_run_cfg": (None, [C.c_void_p]),
    "binder_run_allatom": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "binder_get_launch_cfg": (C.c_int, [C.c_void_p, C.c_void_p]),
    "binder_set_launch_cfg": (C.c_int, [C.c_void_p, C.c_void_p]),
    "binder_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "binder_mlp_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "binder_mlp_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "binder_mlp_features": (C.c_int, [C.c_void_p, C.c_int32, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]),
    "binder_mlp_forward": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "binder_mlp_loss_grad": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_float, C.POINTER(C.c_double), C.c_void_p]),
    "binder_mlp_set_tuples": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "binder_mlp_tuple_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "binder_mlp_get_tuples": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_mlp_train": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_uint64, C.c_void_p]),
    "binder_mc_log": (C.c_int, [C.c_void_p, C.c_size_t]),
    "binder_mc_log_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "binder_mc_log_fetch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_mlp_take_log": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "binder_set_proposal": (C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_float]),
    "binder_selftest_wait": (C.c_int, [C.c_void_p, C.c_uint32]),
    "binder_debug_fail_alloc": (C.c_int, [C.c_int64]),
    "binder_minimize": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "binder_validate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "binder_fv_upload": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int32, C.c_int32] + [C.c_void_p] * 8 +
                         [C.c_int32, C.c_void_p]),
    "binder_fv_run": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "binder_parse_pdb_text": (C.c_int, [C.c_char_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.POINTER(C.c_size_t)]),
    "binder_parse_pdb_file": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_parse_peptide": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_write_pdb_ca": (C.c_int, [C.c_size_t, C.c_void_p, C.c_void_p, C.c_char, C.c_void_p, C.c_size_t,
                                      C.POINTER(C.c_size_t)]),
    "binder_write_pdb_allatom": (C.c_int, [C.c_size_t, C.c_void_p, C.c_void_p, C.c_char, C.c_void_p, C.c_size_t,
                                           C.POINTER(C.c_size_t)]),
    "binder_write_pdb_multi": (C.c_int, [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_void_p,
                                         C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_write_fasta": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_write_json": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_write_csv": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "binder_affinity_maturation": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
}
PROPOSAL_UNIFORM, PROPOSAL_LEARNED = 0, 1

# learned proposal network (include/binder_gpu.h): sizes and the logged-tuple record
MLP_IN, MLP_OUT = 180, 25
MLP_NO_AA = 255  # amino-acid input of a mutation query (no one-hot)
MLP_K1, MLP_H, MLP_OUT_PAD = 192, 256, 32
MLP_OFF = {"w1": 0}
MLP_OFF["b1"] = MLP_OFF["w1"] + MLP_H * MLP_K1
MLP_OFF["w2"] = MLP_OFF["b1"] + MLP_H
MLP_OFF["b2"] = MLP_OFF["w2"] + MLP_H * MLP_H
MLP_OFF["w3"] = MLP_OFF["b2"] + MLP_H
MLP_OFF["b3"] = MLP_OFF["w3"] + MLP_OUT_PAD * MLP_H
MLP_N_PARAMS = MLP_OFF["b3"] + MLP_OUT_PAD  # 123424
MC_TUPLE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("delta_e", "<f4"), ("cand", "<i4"),
                     ("log_ratio", "<f4"), ("residue", "<i2"), ("aa", "u1"), ("action", "u1"), ("antigen", "u1"),
                     ("accepted", "u1"), ("_pad", "u1", (2,))])


def mlp_init_params(seed=0):
    """Initial parameters: uniform(+-1/sqrt(fan_in)) weights (PyTorch's Linear
    default), zero biases, zero padding rows / columns."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MLP_N_PARAMS, np.float32)
    w1 = rng.uniform(-1, 1, (MLP_H, MLP_IN)) / np.sqrt(MLP_IN)
    w2 = rng.uniform(-1, 1, (MLP_H, MLP_H)) / np.sqrt(MLP_H)
    w3 = rng.uniform(-1, 1, (MLP_OUT, MLP_H)) / np.sqrt(MLP_H)
    W1 = np.zeros((MLP_H, MLP_K1), np.float32)
    W1[:, :MLP_IN] = w1
    W3 = np.zeros((MLP_OUT_PAD, MLP_H), np.float32)
    W3[:MLP_OUT] = w3
    p[MLP_OFF["w1"]:MLP_OFF["b1"]] = W1.ravel()
    p[MLP_OFF["w2"]:MLP_OFF["b2"]] = w2.astype(np.float32).ravel()
    p[MLP_OFF["w3"]:MLP_OFF["b3"]] = W3.ravel()
    return p


def lib():
    """Load libbinder_b200.so and declare every entry point of include/binder_gpu.h."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = Path(os.environ.get("BINDER_B200_LIB", LIB_PATH))
    if not path.exists():
        raise ImportError(f"{path} is not built; run `python de-novo-antigen-binder_b200/build.py` "
                          "(or __graft_entry__.build())")
    L = C.CDLL(str(path))
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


# ---- tables ---------------------------------------------------------------------
class Tables:
    """The force-field tables compiled into the library (amber.rs / rotamer.rs / atom.rs)."""

    def __init__(self):
        L = lib()
        self.n_atoms = np.zeros(N_AA, np.int32)
        self.charge = np.zeros((N_AA, SLOTS), np.float32)
        self.atom_type = np.zeros((N_AA, SLOTS), np.uint8)
        self.hydrophobic = np.zeros((N_AA, SLOTS), np.uint8)
        for a in range(N_AA):
            n = C.c_int()
            L.binder_table_residue(a, C.byref(n), _ptr(self.charge[a]), _ptr(self.atom_type[a]),
                                   _ptr(self.hydrophobic[a]))
            self.n_atoms[a] = n.value
        self.r_min_half = np.zeros(16, np.float32)
        self.epsilon = np.zeros(16, np.float32)
        self.hbond = np.zeros(16, np.int32)
        self.eef1 = np.zeros((16, 3), np.float32)
        for t in range(16):
            r, e, h = C.c_float(), C.c_float(), C.c_int()
            L.binder_table_atom_type(t, C.byref(r), C.byref(e), C.byref(h), _ptr(self.eef1[t]))
            self.r_min_half[t], self.epsilon[t], self.hbond[t] = r.value, e.value, h.value
        self.n_rot = np.zeros(N_AA, np.int32)
        self.rot_chi = np.zeros((N_AA, 5, 4), np.float32)
        self.residue_level = np.zeros((N_AA, 4), np.float32)
        for a in range(N_AA):
            n = C.c_int()
            L.binder_table_rotamers(a, C.byref(n), _ptr(self.rot_chi[a]))
            self.n_rot[a] = n.value
            L.binder_table_residue_level(a, _ptr(self.residue_level[a]))


_TABLES = None


def tables() -> Tables:
    global _TABLES
    if _TABLES is None:
        _TABLES = Tables()
    return _TABLES


# ---- clouds -----------------------------------------------------------------------
class AtomCloud:
    """allatom.rs:17-31 AtomCloud: flat all-atom structure of arrays."""

    def __init__(self, x, y, z, charge, r_min_half, epsilon, hydrophobic, atom_type=None, residue_idx=None):
        self.x, self.y, self.z = _f32(x), _f32(y), _f32(z)
        self.charge, self.r_min_half, self.epsilon = _f32(charge), _f32(r_min_half), _f32(epsilon)
        self.hydrophobic = _u8(hydrophobic)
        self.atom_type = None if atom_type is None else _u8(atom_type)
        self.residue_idx = None if residue_idx is None else np.ascontiguousarray(residue_idx, np.uint32)

    def __len__(self):
        return len(self.x)

    @classmethod
    def from_slots(cls, aa, pos):
        """Flatten a slot-layout protein in push_residue order (allatom.rs:201-240)."""
        T = tables()
        aa = np.asarray(aa, np.uint8)
        pos = np.asarray(pos, np.float32).reshape(len(aa), SLOTS, 3)
        res_idx = np.repeat(np.arange(len(aa), dtype=np.uint32), T.n_atoms[aa])
        k = np.concatenate([np.arange(T.n_atoms[a]) for a in aa]) if len(aa) else np.zeros(0, int)
        xyz = pos[res_idx, k]
        types = T.atom_type[aa[res_idx], k]
        return cls(xyz[:, 0], xyz[:, 1], xyz[:, 2], T.charge[aa[res_idx], k], T.r_min_half[types],
                   T.epsilon[types], T.hydrophobic[aa[res_idx], k], types, res_idx)

    def to_gpu_atoms(self):
        """GpuAtom flattening of run_allatom (diffusion.rs:1029-1040)."""
        g = np.zeros(len(self), GPU_ATOM)
        g["x"], g["y"], g["z"] = self.x, self.y, self.z
        g["q"], g["r_min_half"], g["epsilon"] = self.charge, self.r_min_half, self.epsilon
        g["hydrophobic"] = self.hydrophobic.astype(np.float32)
        return g

    def _c(self):
        s = _AtomCloudC(_ptr(self.x), _ptr(self.y), _ptr(self.z), _ptr(self.charge), _ptr(self.r_min_half),
                        _ptr(self.epsilon), _ptr(self.hydrophobic), _ptr(self.atom_type), _ptr(self.residue_idx),
                        len(self.x))
        return s


class ResidueCloud:
    """atom.rs:185-195 ResidueCloud: Calpha positions + amino acid."""

    def __init__(self, x, y, z, amino_acid):
        self.x, self.y, self.z = _f32(x), _f32(y), _f32(z)
        self.amino_acid = _u8(amino_acid)

    def __len__(self):
        return len(self.x)

    def _c(self):
        return _ResidueCloudC(_ptr(self.x), _ptr(self.y), _ptr(self.z), _ptr(self.amino_acid), len(self.x))


# ---- context ----------------------------------------------------------------------
class GpuContext:
    """gpu.rs:46-268 GpuContext on a B200: one device, one stream."""

    def __init__(self, handle, params):
        self._h = handle
        self.params = params

    @classmethod
    def try_init(cls, device=0, params=None):
        """gpu.rs:55 try_init: None when no sm_100 device is usable."""
        try:
            return cls.create(device, params)
        except BinderError:
            return None

    @classmethod
    def create(cls, device=0, params=None):
        L = lib()
        params = params or Params.defaults()
        st = C.c_int(0)
        h = L.binder_create(device, C.byref(params), C.byref(st))
        if not h:
            raise BinderError(st.value, "binder_create failed")
        return cls(h, params)

    def close(self):
        if self._h:
            lib().binder_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, status):
        if status != 0:
            msg = lib().binder_last_error(self._h)
            raise BinderError(status, msg.decode() if msg else "")

    def set_params(self, params):
        self._check(lib().binder_set_params(self._h, C.byref(params)))
        self.params = params

    @property
    def launch_count(self):
        return int(lib().binder_launch_count(self._h))

    def synchronize(self):
        self._check(lib().binder_synchronize(self._h))

    # -- score_batch (gpu.rs:166-267) --
    def score_batch(self, antigen: AtomCloud, candidates, n_ab: int):
        cand = np.ascontiguousarray(candidates, GPU_ATOM)
        n_cand = len(cand) // n_ab if n_ab else 0
        out = np.zeros(n_cand, np.float32)
        got = C.c_size_t()
        ag = antigen._c()
        self._check(lib().binder_score_batch(self._h, C.byref(ag), _ptr(cand), len(cand), n_ab, _ptr(out), n_cand,
                                             C.byref(got)))
        return out

    def score_batch_f64(self, antigen: AtomCloud, candidates, n_ab: int, with_abs=False):
        cand = np.ascontiguousarray(candidates, GPU_ATOM)
        n_cand = len(cand) // n_ab if n_ab else 0
        out = np.zeros(n_cand, np.float64)
        ab = np.zeros(n_cand, np.float64) if with_abs else None
        got = C.c_size_t()
        ag = antigen._c()
        self._check(lib().binder_score_batch_f64(self._h, C.byref(ag), _ptr(cand), len(cand), n_ab, _ptr(out),
                                                 _ptr(ab), n_cand, C.byref(got)))
        return (out, ab) if with_abs else out

    def score_batch_ragged(self, antigen: AtomCloud, candidates, offsets, with_abs=False):
        cand = np.ascontiguousarray(candidates, GPU_ATOM)
        off = np.ascontiguousarray(offsets, np.int64)
        n_cand = len(off) - 1
        out = np.zeros(n_cand, np.float64)
        ab = np.zeros(n_cand, np.float64) if with_abs else None
        ag = antigen._c()
        self._check(lib().binder_score_batch_ragged(self._h, C.byref(ag), _ptr(cand), _ptr(off), n_cand, _ptr(out),
                                                    _ptr(ab)))
        return (out, ab) if with_abs else out

    def last_pair_count(self):
        n = C.c_int64()
        self._check(lib().binder_last_pair_count(self._h, C.byref(n)))
        return n.value

    # -- SpatialHashGrid (spatial.rs) --
    def grid_cells(self, cell, x, y, z):
        x, y, z = _f32(x), _f32(y), _f32(z)
        out = np.zeros((len(x), 3), np.int32)
        self._check(lib().binder_grid_cells(self._h, cell, _ptr(x), _ptr(y), _ptr(z), len(x), _ptr(out)))
        return out

    def grid_neighbors(self, cell, ax, ay, az, px, py, pz):
        """build + query_neighbors for each probe: (offsets int64[n_q+1], indices uint32)."""
        ax, ay, az, px, py, pz = (_f32(v) for v in (ax, ay, az, px, py, pz))
        off = np.zeros(len(px) + 1, np.int64)
        total = C.c_size_t(0)
        cap = max(1, len(px) * 32)
        idx = np.zeros(cap, np.uint32)
        st = lib().binder_grid_neighbors(self._h, cell, _ptr(ax), _ptr(ay), _ptr(az), len(ax), _ptr(px), _ptr(py),
                                         _ptr(pz), len(px), _ptr(off), _ptr(idx), cap, C.byref(total))
        if st == 9:
            cap = max(1, total.value)
            idx = np.zeros(cap, np.uint32)
            st = lib().binder_grid_neighbors(self._h, cell, _ptr(ax), _ptr(ay), _ptr(az), len(ax), _ptr(px),
                                             _ptr(py), _ptr(pz), len(px), _ptr(off), _ptr(idx), cap, C.byref(total))
        self._check(st)
        return off, idx[:total.value]

    # -- forces --
    def compute_forces_with_grid(self, antigen: ResidueCloud, cell: float, antibody: ResidueCloud):
        """energy.rs:322-398 on the GPU; returns (fx, fy, fz)."""
        n = len(antibody)
        fx, fy, fz = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32)
        ag, ab = antigen._c(), antibody._c()
        self._check(lib().binder_compute_forces_with_grid(self._h, C.byref(ag), cell, C.byref(ab), _ptr(fx),
                                                          _ptr(fy), _ptr(fz)))
        return fx, fy, fz

    def forces_allatom(self, antigen: AtomCloud, candidates, offsets):
        cand = np.ascontiguousarray(candidates, GPU_ATOM)
        off = np.ascontiguousarray(offsets, np.int64)
        n_cand = len(off) - 1
        f = np.zeros((len(cand), 3), np.float32)
        e = np.zeros(n_cand, np.float64)
        ag = antigen._c()
        self._check(lib().binder_forces_allatom(self._h, C.byref(ag), _ptr(cand), _ptr(off), n_cand, _ptr(f),
                                                _ptr(e)))
        return f, e

    # -- survivor selection --
    def topk(self, energies, k):
        e = np.ascontiguousarray(energies, np.float64)
        out = np.zeros(k, np.int32)
        self._check(lib().binder_topk(self._h, _ptr(e), len(e), k, _ptr(out)))
        return out

    def topk_segmented(self, energies, seg_offsets, k):
        e = np.ascontiguousarray(energies, np.float64)
        so = np.ascontiguousarray(seg_offsets, np.int64)
        out = np.zeros((len(so) - 1) * k, np.int32)
        self._check(lib().binder_topk_segmented(self._h, _ptr(e), _ptr(so), len(so) - 1, k, _ptr(out)))
        return out.reshape(len(so) - 1, k)

    # -- residue construction --
    def build_residues(self, ca_xyz, aa, chi=None):
        """protein_from_ca_trace (allatom.rs:523-541): (pos [n,14,3], chi [n,4])."""
        ca = _f32(ca_xyz).reshape(-1, 3)
        aa = _u8(aa)
        n = len(aa)
        pos = np.zeros((n, SLOTS, 3), np.float32)
        chi_out = np.zeros((n, 4), np.float32)
        chi_in = None if chi is None else _f32(chi).reshape(n, 4)
        self._check(lib().binder_build_residues(self._h, n, _ptr(ca), _ptr(aa), _ptr(chi_in), _ptr(pos),
                                                _ptr(chi_out)))
        return pos, chi_out

    # -- resident search state --
    def add_antigen(self, aa, pos):
        aa = _u8(aa)
        pos = _f32(pos)
        out = C.c_int32()
        self._check(lib().binder_add_antigen(self._h, len(aa), _ptr(aa), _ptr(pos), C.byref(out)))
        return out.value

    def clear_antigens(self):
        self._check(lib().binder_clear_antigens(self._h))

    def state_upload(self, aa, chi, pos, n_res=None, uniform_n_res=0, antigen_id=None, cand_id=None):
        aa, chi, pos = _u8(aa), _f32(chi), _f32(pos)
        nr = None if n_res is None else np.ascontiguousarray(n_res, np.int32)
        n_cand = len(nr) if nr is not None else len(aa) // max(1, uniform_n_res)
        agi = None if antigen_id is None else np.ascontiguousarray(antigen_id, np.int32)
        cid = None if cand_id is None else np.ascontiguousarray(cand_id, np.uint32)
        self._check(lib().binder_state_upload(self._h, n_cand, _ptr(nr), uniform_n_res, _ptr(agi), _ptr(cid),
                                              _ptr(aa), _ptr(chi), _ptr(pos)))
        self._state_res = len(aa)
        self._state_cand = n_cand

    def state_download(self, aa=None, chi=None, pos=None):
        """Device state -> host (optionally into caller-provided, e.g. pinned, arrays)."""
        n = self._state_res
        aa = np.zeros(n, np.uint8) if aa is None else aa
        chi = np.zeros((n, 4), np.float32) if chi is None else chi
        pos = np.zeros((n, SLOTS, 3), np.float32) if pos is None else pos
        self._check(lib().binder_state_download(self._h, _ptr(aa), _ptr(chi), _ptr(pos)))
        return aa, chi, pos

    def diffuse(self, n_steps, step0=0, with_noise=False, with_mc=False, temps=None):
        t = None if temps is None else _f32(temps)
        self._check(lib().binder_diffuse(self._h, n_steps, step0, int(with_noise), int(with_mc), _ptr(t)))

    def mc_stats(self, reset=False):
        """int64[n_cand, 4]: mutation/rotamer tried, accepted, backbone tried, accepted."""
        out = np.zeros((self._state_cand, 4), np.int64)
        self._check(lib().binder_mc_stats(self._h, _ptr(out), int(reset)))
        return out

    def state_select(self, idx):
        """Keep candidates idx (in that order) of the resident state."""
        idx = np.ascontiguousarray(idx, np.int32)
        self._check(lib().binder_state_select(self._h, _ptr(idx), len(idx)))
        self._sync_state_info()

    def _sync_state_info(self):
        n, t = C.c_int32(), C.c_int32()
        self._check(lib().binder_state_info(self._h, C.byref(n), C.byref(t), None))
        self._state_cand, self._state_res = n.value, t.value

    def state_info(self):
        """(n_cand, total_res, original upload index of each candidate)."""
        n, t = C.c_int32(), C.c_int32()
        self._check(lib().binder_state_info(self._h, C.byref(n), C.byref(t), None))
        orig = np.zeros(n.value, np.int32)
        self._check(lib().binder_state_info(self._h, C.byref(n), C.byref(t), _ptr(orig)))
        return n.value, t.value, orig

    def run_allatom(self, cfg=None, n_segments=1):
        """run_allatom (diffusion.rs:983-1107) on the resident state.  Returns
        (cand[n_segments, top_n], energy[n_segments, top_n]); the resident state then
        holds the ranked results."""
        cfg = RunCfg.defaults() if cfg is None else cfg
        cand = np.zeros(n_segments * cfg.top_n, np.int32)
        e = np.zeros(n_segments * cfg.top_n, np.float64)
        self._check(lib().binder_run_allatom(self._h, C.byref(cfg), _ptr(cand), _ptr(e)))
        self._sync_state_info()
        return cand.reshape(n_segments, -1), e.reshape(n_segments, -1)

    def minimize(self, steps=60):
        """minimize (diffusion.rs:854-916) of every resident candidate against its
        antigen, in place; returns the final energies."""
        out = np.zeros(self._state_cand, np.float64)
        self._check(lib().binder_minimize(self._h, int(steps), _ptr(out)))
        return out

    def affinity_maturation(self):
        """affinity_maturation_allatom (diffusion.rs:924-961) over every resident
        candidate's interface residues, in place; returns (final scores, mutations
        kept)."""
        out = np.zeros(self._state_cand, np.float64)
        kept = np.zeros(self._state_cand, np.int32)
        self._check(lib().binder_affinity_maturation(self._h, _ptr(out), _ptr(kept)))
        return out, kept

    def fv_upload(self, heavy, light, antigen_id=0, cand_id=None):
        """Upload an Fv population: heavy / light = (aa, chi, pos, cdr) stacked over the
        candidates (uniform chain lengths).  The state then interleaves heavy 2i and
        light 2i + 1."""
        (ha, hc, hp, hr), (la, lc, lp, lr) = heavy, light
        ha, la, hr, lr = _u8(ha), _u8(la), _u8(hr), _u8(lr)
        hc, hp, lc, lp = _f32(hc), _f32(hp), _f32(lc), _f32(lp)
        n = len(cand_id) if cand_id is not None else None
        if n is None:
            raise ValueError("cand_id (one per candidate) is required")
        n_h, n_l = len(ha) // n, len(la) // n
        cid = np.ascontiguousarray(cand_id, np.uint32)
        self._check(lib().binder_fv_upload(self._h, n, n_h, n_l, _ptr(ha), _ptr(hc), _ptr(hp), _ptr(hr), _ptr(la),
                                           _ptr(lc), _ptr(lp), _ptr(lr), antigen_id, _ptr(cid)))
        self._state_res = n * (n_h + n_l)
        self._state_cand = 2 * n
        self._fv = (n, n_h, n_l)

    def fv_run(self, iterations):
        """run_fv's iteration loop on the uploaded population; returns the best
        fv_energy per candidate (the state holds the best pairs)."""
        n = self._fv[0]
        out = np.zeros(n, np.float64)
        self._check(lib().binder_fv_run(self._h, int(iterations), _ptr(out)))
        return out

    def fv_download(self):
        """(heavy, light) = ((aa, chi, pos), (aa, chi, pos)) of the resident Fv pairs."""
        n, n_h, n_l = self._fv
        aa, chi, pos = self.state_download()
        per = n_h + n_l
        idx_h = (np.arange(n)[:, None] * per + np.arange(n_h)).ravel()
        idx_l = (np.arange(n)[:, None] * per + n_h + np.arange(n_l)).ravel()
        return (aa[idx_h], chi[idx_h], pos[idx_h]), (aa[idx_l], chi[idx_l], pos[idx_l])

    def validate(self):
        """ValidationReport::assess (validate.rs:24-132) of every resident candidate:
        (clashes, rama_outliers) int32 arrays."""
        cl = np.zeros(self._state_cand, np.int32)
        ra = np.zeros(self._state_cand, np.int32)
        self._check(lib().binder_validate(self._h, _ptr(cl), _ptr(ra)))
        return cl, ra

    def launch_cfg(self):
        c = LaunchCfg()
        self._check(lib().binder_get_launch_cfg(self._h, C.byref(c)))
        return c

    def set_launch_cfg(self, score_warps=8, score_ctas_per_sm=4, cg_warps=8, cg_lanes=8, cg_order=1, score_order=0,
                       cg_queue=1, cg_flat=0):
        c = LaunchCfg(score_warps, score_ctas_per_sm, cg_warps, cg_lanes, cg_order, score_order, cg_queue, cg_flat)
        self._check(lib().binder_set_launch_cfg(self._h, C.byref(c)))

    def autotune(self, reps=5):
        """Pick the fastest launch shapes for the resident state; returns them."""
        c = LaunchCfg()
        self._check(lib().binder_autotune(self._h, reps, C.byref(c)))
        return c

    def score_state(self, full=False):
        out = np.zeros(self._state_cand, np.float64)
        self._check(lib().binder_score_state(self._h, int(full), _ptr(out)))
        return out

    def mc_energy(self):
        """The Metropolis energy of every candidate (Calpha-level contributions + disulfide)."""
        out = np.zeros(self._state_cand, np.float64)
        self._check(lib().binder_score_state(self._h, 2, _ptr(out)))
        return out

    def block(self, n_steps, step0=0, k=64, n_segments=1, out_e=None, out_top=None):
        e = np.zeros(self._state_cand, np.float64) if out_e is None else out_e
        top = (np.zeros(n_segments * k, np.int32) if k else None) if out_top is None else out_top
        self._check(lib().binder_block(self._h, n_steps, step0, k, _ptr(e), _ptr(top)))
        return e, (top.reshape(n_segments, k) if k else None)

    def block_io(self, aa, chi, pos, n_steps, k=64, uniform_n_res=0, n_res=None, antigen_id=None, cand_id=None,
                 n_segments=1, out_e=None, out_top=None):
        """Upload the population (aa uint8[R], chi float32[R][4], pos float32[R][14][3]),
        run one block and write the moved residues back into the same arrays (they
        must be C-contiguous arrays of those types: pinned ones copy fastest);
        returns the energies and the top-k as block() does (n_segments = the number of
        resident antigens)."""
        for a, t in ((aa, np.uint8), (chi, np.float32), (pos, np.float32)):
            if not (isinstance(a, np.ndarray) and a.dtype == t and a.flags["C_CONTIGUOUS"] and a.flags["WRITEABLE"]):
                raise TypeError("block_io needs writable C-contiguous %s arrays" % np.dtype(t).name)
        nr = None if n_res is None else np.ascontiguousarray(n_res, np.int32)
        n_cand = len(nr) if nr is not None else len(aa) // max(1, uniform_n_res)
        agi = None if antigen_id is None else np.ascontiguousarray(antigen_id, np.int32)
        cid = None if cand_id is None else np.ascontiguousarray(cand_id, np.uint32)
        e = np.zeros(n_cand, np.float64) if out_e is None else out_e
        top = (np.zeros(n_segments * k, np.int32) if k else None) if out_top is None else out_top
        self._check(lib().binder_block_io(self._h, n_cand, _ptr(nr), uniform_n_res, _ptr(agi), _ptr(cid), _ptr(aa),
                                          _ptr(chi), _ptr(pos), n_steps, k, _ptr(e), _ptr(top)))
        self._state_res = len(aa)
        self._state_cand = n_cand
        return e, (top.reshape(n_segments, k) if k else None)

    def block_async(self, n_steps, step0=0, k=64):
        """Enqueue one block on the context stream; results stay on the device."""
        self._check(lib().binder_block(self._h, n_steps, step0, k, None, None))

    def block_fetch(self, k=64, n_segments=1, out_e=None, out_top=None):
        e = np.zeros(self._state_cand, np.float64) if out_e is None else out_e
        top = (np.zeros(n_segments * k, np.int32) if k else None) if out_top is None else out_top
        self._check(lib().binder_block_fetch(self._h, _ptr(e), _ptr(top)))
        return e, (top.reshape(n_segments, k) if k else None)

    # -- instrumentation --
    @property
    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        return int(lib().binder_stream(self._h) or 0)

    def set_timing(self, on=True):
        self._check(lib().binder_set_timing(self._h, int(on)))

    def timing_summary(self):
        """(summed [gradient, scoring, top-k] ms, number of blocks) since set_timing."""
        out = np.zeros(3, np.float64)
        n = C.c_int32()
        self._check(lib().binder_timing_summary(self._h, _ptr(out), C.byref(n)))
        return out, n.value

    def state_pair_counts(self, n_steps):
        a, b = C.c_int64(), C.c_int64()
        self._check(lib().binder_state_pair_counts(self._h, n_steps, C.byref(a), C.byref(b)))
        return a.value, b.value

    def fp32_peak(self):
        a, b = C.c_double(), C.c_double()
        self._check(lib().binder_fp32_peak(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # -- learned proposal network --
    def mlp_set_params(self, params):
        p = _f32(params)
        assert p.shape == (MLP_N_PARAMS,)
        self._check(lib().binder_mlp_set_params(self._h, _ptr(p)))

    def mlp_get_params(self):
        out = np.zeros(MLP_N_PARAMS, np.float32)
        self._check(lib().binder_mlp_get_params(self._h, _ptr(out)))
        return out

    def mlp_features(self, antigen_id, ca, aa):
        ca, aa = _f32(ca).reshape(-1, 3), _u8(aa)
        out = np.zeros((len(aa), MLP_IN), np.float32)
        self._check(lib().binder_mlp_features(self._h, antigen_id, len(aa), _ptr(ca), _ptr(aa), _ptr(out)))
        return out

    def mlp_forward(self, features):
        f = _f32(features).reshape(-1, MLP_IN)
        out = np.zeros((len(f), MLP_OUT), np.float32)
        self._check(lib().binder_mlp_forward(self._h, len(f), _ptr(f), _ptr(out)))
        return out

    def mlp_loss_grad(self, features, action, target, huber_delta=1.0, ref=None):
        """Mean Huber loss of y[action] - y[ref] (y[action] where ref is None or -1)
        against target, and the parameter gradient."""
        f = _f32(features).reshape(-1, MLP_IN)
        a = np.ascontiguousarray(action, np.int32)
        r = None if ref is None else np.ascontiguousarray(ref, np.int32)
        t = _f32(target)
        loss = C.c_double()
        g = np.zeros(MLP_N_PARAMS, np.float32)
        self._check(lib().binder_mlp_loss_grad(self._h, len(f), _ptr(f), _ptr(a), _ptr(r), _ptr(t), huber_delta,
                                               C.byref(loss), _ptr(g)))
        return loss.value, g

    def mlp_set_tuples(self, tuples):
        t = np.ascontiguousarray(tuples, MC_TUPLE)
        self._check(lib().binder_mlp_set_tuples(self._h, _ptr(t), len(t)))

    def mlp_get_tuples(self):
        n = C.c_size_t()
        self._check(lib().binder_mlp_tuple_count(self._h, C.byref(n)))
        out = np.zeros(n.value, MC_TUPLE)
        self._check(lib().binder_mlp_get_tuples(self._h, _ptr(out), len(out), C.byref(n)))
        return out

    def set_proposal(self, learned, t_prop_min=0.5, t_max=float("inf")):
        """Mutation / rotamer proposal of diffuse(): uniform (the reference) or the
        network (at steps with temperature <= t_max)."""
        self._check(lib().binder_set_proposal(self._h, PROPOSAL_LEARNED if learned else PROPOSAL_UNIFORM,
                                              t_prop_min, t_max))

    def mc_log(self, capacity):
        """Log the mutation / rotamer decisions of the following diffuse() calls (0 stops)."""
        self._check(lib().binder_mc_log(self._h, capacity))

    def mc_log_count(self):
        a, b = C.c_size_t(), C.c_size_t()
        self._check(lib().binder_mc_log_count(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def mc_log_fetch(self):
        n, _ = self.mc_log_count()
        out = np.zeros(n, MC_TUPLE)
        got = C.c_size_t()
        self._check(lib().binder_mc_log_fetch(self._h, _ptr(out), len(out), C.byref(got)))
        return out[:got.value]

    def mlp_take_log(self):
        """The logged tuples become the training set; returns their number."""
        n = C.c_size_t()
        self._check(lib().binder_mlp_take_log(self._h, C.byref(n)))
        return n.value

    def mlp_train(self, n_steps, batch=8192, lr=1e-3, huber_delta=1.0, seed=0):
        """n_steps Adam steps on minibatches of the training set; per-step losses."""
        out = np.zeros(max(0, n_steps), np.float64)
        self._check(lib().binder_mlp_train(self._h, n_steps, batch, lr, huber_delta, seed, _ptr(out)))
        return out


# ---- input and output formats (pdb.rs, report.rs): host code of the library ------------
class CandidateReport(C.Structure):
    """binder_candidate_report = CandidateReport (report.rs:8-20); light_sequence None
    for single-chain candidates, clashes / rama_outliers None when not assessed."""
    _fields_ = [("rank", C.c_int32), ("_sequence", C.c_char_p), ("_light", C.c_char_p), ("energy", C.c_float),
                ("entropy_penalty", C.c_float), ("dg_corrected", C.c_float), ("net_charge", C.c_int32),
                ("aggregation_risk", C.c_int32), ("n_interface", C.c_int32), ("_clashes", C.c_int32),
                ("_rama", C.c_int32)]

    @classmethod
    def make(cls, rank, sequence, energy, entropy_penalty=0.0, dg_corrected=0.0, net_charge=0,
             aggregation_risk=False, n_interface=0, clashes=None, rama_outliers=None, light_sequence=None):
        return cls(rank, sequence.encode(), None if light_sequence is None else light_sequence.encode(), energy,
                   entropy_penalty, dg_corrected, net_charge, int(aggregation_risk), n_interface,
                   -1 if clashes is None else clashes, -1 if rama_outliers is None else rama_outliers)


def _text(fn, *args):
    n = C.c_size_t(0)
    st = fn(*args, None, 0, C.byref(n))
    if st not in (0, 9):
        raise BinderError(st)
    buf = C.create_string_buffer(n.value + 1)
    st = fn(*args, buf, n.value + 1, C.byref(n))
    if st:
        raise BinderError(st)
    return buf.raw[: n.value].decode()


def _points(fn, *args):
    n = C.c_size_t(0)
    st = fn(*args, None, None, 0, C.byref(n))
    if st not in (0, 9):
        raise BinderError(st)
    xyz = np.zeros((n.value, 3), np.float32)
    aa = np.zeros(n.value, np.uint8)
    if n.value:
        st = fn(*args, _ptr(xyz), _ptr(aa), n.value, C.byref(n))
        if st:
            raise BinderError(st)
    return xyz, aa


def parse_pdb(text=None, path=None):
    """parse_pdb (pdb.rs:19-57): the CA records as (xyz float32[n, 3], amino acids)."""
    if path is not None:
        return _points(lib().binder_parse_pdb_file, str(path).encode())
    b = text.encode() if isinstance(text, str) else bytes(text)
    return _points(lib().binder_parse_pdb_text, b, len(b))


def parse_peptide(seq):
    """parse_peptide (pdb.rs:64-83): (xyz, amino acids) of an extended trace."""
    return _points(lib().binder_parse_peptide, seq.encode())


def write_pdb_ca(xyz, aa, chain="A"):
    xyz, aa = _f32(xyz), _u8(aa)
    return _text(lib().binder_write_pdb_ca, len(aa), _ptr(xyz), _ptr(aa), chain.encode())


def write_pdb_allatom(aa, pos, chain="A"):
    aa, pos = _u8(aa), _f32(pos)
    return _text(lib().binder_write_pdb_allatom, len(aa), _ptr(aa), _ptr(pos), chain.encode())


def write_pdb_multi(chains):
    """chains: [(aa, pos, chain_id), ...] -> one PDB text with TER records."""
    n_res = np.array([len(a) for a, _, _ in chains], np.uint64)
    aa = _u8(np.concatenate([a for a, _, _ in chains])) if chains else _u8([])
    pos = _f32(np.concatenate([p for _, p, _ in chains])) if chains else _f32([])
    ids = "".join(c for _, _, c in chains).encode()
    return _text(lib().binder_write_pdb_multi, len(chains), _ptr(n_res), _ptr(aa), _ptr(pos), ids)


def _reports(reports):
    arr = (CandidateReport * max(1, len(reports)))(*reports)
    return C.cast(arr, C.c_void_p), len(reports), arr


def write_fasta(reports):
    p, n, keep = _reports(reports)
    return _text(lib().binder_write_fasta, p, n)


def write_json(reports):
    p, n, keep = _reports(reports)
    return _text(lib().binder_write_json, p, n)


def write_csv(reports):
    p, n, keep = _reports(reports)
    return _text(lib().binder_write_csv, p, n)


def temperature(iteration, total, t_hot=3.0, t_cold=0.02):
    """diffusion.rs:102-104 in f32: T_HOT * (T_COLD/T_HOT)^(iter/total)."""
    t_hot, t_cold = np.float32(t_hot), np.float32(t_cold)
    return np.float32(t_hot * np.power(np.float32(t_cold / t_hot), np.float32(iteration) / np.float32(total)))


from . import workloads  # noqa: E402,F401  (seeded synthetic inputs)
from . import learned  # noqa: E402,F401  (learned-proposal workflow)
