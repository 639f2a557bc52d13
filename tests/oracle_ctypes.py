"""ctypes bindings of the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure only: the checker the CUDA library is compared against.
Builds the oracle with `make -C oracle` on first use when the .so is missing.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE = ROOT / "oracle"
LIB = ORACLE / "_build" / "liboracle.so"
SLOTS = 14
GPU_ATOM = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("q", "<f4"), ("r_min_half", "<f4"),
                     ("epsilon", "<f4"), ("hydrophobic", "<f4"), ("_pad", "<f4")])

_L = None


def lib():
    global _L
    if _L is None:
        if not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime
                                   for p in ORACLE.glob("oracle*")):
            subprocess.run(["make", "-s", "-C", str(ORACLE)], check=True)
        _L = C.CDLL(str(LIB))
        _L.orc_grid_neighbors.restype = C.c_int64
        _L.orc_count_pairs.restype = C.c_int64
        _L.orc_temperature.restype = C.c_float
        _L.orc_temperature.argtypes = [C.c_int, C.c_int]
        _L.orc_residue_contribution.restype = C.c_float
        _L.orc_residue_contribution64.restype = C.c_double
        _L.orc_disulfide.restype = C.c_float
        _L.orc_antigen_new.restype = C.c_void_p
        _L.orc_antigen_new.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_float]
        _L.orc_antigen_free.argtypes = [C.c_void_p]
        _L.orc_topology_size.restype = C.c_int
        _L.orc_fv_energy.restype = C.c_double
        for fn in ("orc_residue_contribution", "orc_residue_contribution64"):
            getattr(_L, fn).argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        _L.orc_disulfide.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        _L.orc_step.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_uint32, C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_int]
        _L.orc_score_slots64.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                         C.c_void_p, C.c_int]
        _L.orc_place_atom.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_void_p]
        _L.orc_grid_cell.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p]
    return _L


def P(a):
    # pointer-sized argument (ctypes would pass a bare Python int as a C int)
    return None if a is None else C.c_void_p(a.ctypes.data)


class OrcCloud(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("q", C.c_void_p), ("rmh", C.c_void_p),
                ("eps", C.c_void_p), ("hyd", C.c_void_p), ("type", C.c_void_p), ("n", C.c_int64)]


class OrcParams(C.Structure):
    _fields_ = [("step", C.c_float), ("noise_base", C.c_float), ("t_hot", C.c_float), ("t_cold", C.c_float),
                ("mutation_p", C.c_float), ("rotamer_move_p", C.c_float), ("backbone_move_p", C.c_float),
                ("max_torsion_deg", C.c_float), ("iface_cutoff_sq", C.c_float), ("shell_radius", C.c_float),
                ("max_disp", C.c_float), ("restraint_k", C.c_float), ("ca_cell", C.c_float),
                ("accumulate", C.c_int32), ("seed", C.c_uint64)]

    @classmethod
    def defaults(cls, **kw):
        p = cls()
        lib().orc_default_params(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        return p


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def u8(a):
    return np.ascontiguousarray(a, np.uint8)


# ---- tables ----
def topology(aa):
    L = lib()
    n = L.orc_topology_size(aa)
    out = []
    for k in range(n):
        q, t, h = C.c_float(), C.c_int(), C.c_int()
        L.orc_topology_atom(aa, k, C.byref(q), C.byref(t), C.byref(h))
        out.append((q.value, t.value, h.value))
    return out


def amber_nb(t):
    r, e = C.c_float(), C.c_float()
    lib().orc_amber_nb(t, C.byref(r), C.byref(e))
    return r.value, e.value


def rotamers(aa):
    L = lib()
    rows = []
    for i in range(L.orc_rotamer_count(aa)):
        chi = np.zeros(4, np.float32)
        p = C.c_float()
        L.orc_rotamer(aa, i, P(chi), C.byref(p))
        rows.append(list(chi) + [p.value])
    return rows


def residue_level(aa):
    q, e, s, h = C.c_float(), C.c_float(), C.c_float(), C.c_int()
    lib().orc_residue_level(aa, C.byref(q), C.byref(e), C.byref(s), C.byref(h))
    return q.value, e.value, s.value, h.value


# ---- geometry ----
def place_atom(a, b, c, bond, angle, dih):
    out = np.zeros(3, np.float32)
    a, b, c = f32(a), f32(b), f32(c)
    lib().orc_place_atom(P(a), P(b), P(c), bond, angle, dih, P(out))
    return out


def build_residues(ca, aa, chi=None):
    ca = f32(ca).reshape(-1, 3)
    aa = u8(aa)
    n = len(aa)
    pos = np.zeros((n, SLOTS, 3), np.float32)
    chi_out = np.zeros((n, 4), np.float32)
    chi_in = None if chi is None else f32(chi)
    lib().orc_build_residues(n, P(ca), P(aa), P(chi_in), P(pos), P(chi_out))
    return pos, chi_out


def flatten(aa, pos):
    """-> dict of AtomCloud arrays (push_residue order)."""
    aa = u8(aa)
    pos = f32(pos)
    n_at = sum(lib().orc_topology_size(int(a)) for a in aa)
    arrs = {k: np.zeros(n_at, np.float32) for k in ("x", "y", "z", "q", "rmh", "eps")}
    arrs["hyd"] = np.zeros(n_at, np.uint8)
    arrs["type"] = np.zeros(n_at, np.uint8)
    arrs["resi"] = np.zeros(n_at, np.uint32)
    lib().orc_flatten(len(aa), P(aa), P(pos), *(P(arrs[k]) for k in ("x", "y", "z", "q", "rmh", "eps", "hyd",
                                                                      "type", "resi")))
    return arrs


def gpu_atoms(cloud):
    g = np.zeros(len(cloud["x"]), GPU_ATOM)
    g["x"], g["y"], g["z"] = cloud["x"], cloud["y"], cloud["z"]
    g["q"], g["r_min_half"], g["epsilon"] = cloud["q"], cloud["rmh"], cloud["eps"]
    g["hydrophobic"] = cloud["hyd"].astype(np.float32)
    return g


def cloud_struct(c):
    return OrcCloud(P(c["x"]), P(c["y"]), P(c["z"]), P(c["q"]), P(c["rmh"]), P(c["eps"]), P(c["hyd"]),
                    P(c["type"]), len(c["x"]))


# ---- grid ----
def grid_cell(cell, x, y, z):
    out = np.zeros(3, np.int32)
    lib().orc_grid_cell(cell, x, y, z, P(out))
    return out


def grid_neighbors(cell, ax, ay, az, px, py, pz):
    ax, ay, az, px, py, pz = (f32(v) for v in (ax, ay, az, px, py, pz))
    off = np.zeros(len(px) + 1, np.int64)
    cap = max(1, len(px) * len(ax))
    idx = np.zeros(cap, np.uint32)
    m = lib().orc_grid_neighbors(C.c_float(cell), P(ax), P(ay), P(az), C.c_int64(len(ax)), P(px), P(py), P(pz),
                                 C.c_int64(len(px)), P(off), P(idx), C.c_int64(cap))
    assert m >= 0
    return off, idx[:m]


# ---- forces / energies ----
def forces_cg_grid(cell, ag_xyz, ag_aa, ab_xyz, ab_aa):
    ag_xyz, ab_xyz = f32(ag_xyz).reshape(-1, 3), f32(ab_xyz).reshape(-1, 3)
    ag_aa, ab_aa = u8(ag_aa), u8(ab_aa)
    ax, ay, az = (f32(ag_xyz[:, k]) for k in range(3))
    bx, by, bz = (f32(ab_xyz[:, k]) for k in range(3))
    n = len(bx)
    f = [np.zeros(n, np.float32) for _ in range(3)]
    lib().orc_forces_cg_grid(C.c_float(cell), P(ax), P(ay), P(az), P(ag_aa), len(ax), P(bx), P(by), P(bz),
                             P(ab_aa), n, *(P(v) for v in f))
    return f


def forces_cg_brute(ag_xyz, ag_aa, ab_xyz, ab_aa):
    ag_xyz, ab_xyz = f32(ag_xyz).reshape(-1, 3), f32(ab_xyz).reshape(-1, 3)
    ag_aa, ab_aa = u8(ag_aa), u8(ab_aa)
    ax, ay, az = (f32(ag_xyz[:, k]) for k in range(3))
    bx, by, bz = (f32(ab_xyz[:, k]) for k in range(3))
    n = len(bx)
    f = [np.zeros(n, np.float32) for _ in range(3)]
    lib().orc_forces_cg_brute(P(ax), P(ay), P(az), P(ag_aa), len(ax), P(bx), P(by), P(bz), P(ab_aa), n,
                              *(P(v) for v in f))
    return f


def forces_cg64(cell, use_grid, ag_xyz, ag_aa, ab_xyz, ab_aa):
    ag_xyz, ab_xyz = f32(ag_xyz).reshape(-1, 3), f32(ab_xyz).reshape(-1, 3)
    ag_aa, ab_aa = u8(ag_aa), u8(ab_aa)
    ax, ay, az = (f32(ag_xyz[:, k]) for k in range(3))
    bx, by, bz = (f32(ab_xyz[:, k]) for k in range(3))
    n = len(bx)
    f = [np.zeros(n, np.float64) for _ in range(3)]
    lib().orc_forces_cg64(C.c_float(cell), int(use_grid), P(ax), P(ay), P(az), P(ag_aa), len(ax), P(bx), P(by),
                          P(bz), P(ab_aa), n, *(P(v) for v in f))
    return f


def energy_atoms32(ag, ab):
    out = np.zeros(5, np.float32)
    a, b = cloud_struct(ag), cloud_struct(ab)
    lib().orc_energy_atoms32(C.byref(a), C.byref(b), P(out))
    return out


def energy_atoms64(ag, ab):
    out = np.zeros(5, np.float64)
    ab_ = np.zeros(5, np.float64)
    a, b = cloud_struct(ag), cloud_struct(ab)
    lib().orc_energy_atoms64(C.byref(a), C.byref(b), P(out), P(ab_))
    return out, ab_


def _ga(a):
    return np.ascontiguousarray(a, GPU_ATOM)


def score_batch32(ag_atoms, cands, offsets, threads=8):
    ag_atoms, cands = _ga(ag_atoms), _ga(cands)
    off = np.ascontiguousarray(offsets, np.int64)
    out = np.zeros(len(off) - 1, np.float32)
    lib().orc_score_batch32(P(ag_atoms), C.c_int64(len(ag_atoms)), P(cands), P(off), C.c_int64(len(off) - 1), P(out),
                            threads)
    return out


def score_batch64(ag_atoms, cands, offsets, threads=8, with_abs=False):
    ag_atoms, cands = _ga(ag_atoms), _ga(cands)
    off = np.ascontiguousarray(offsets, np.int64)
    out = np.zeros(len(off) - 1, np.float64)
    ab = np.zeros(len(off) - 1, np.float64)
    lib().orc_score_batch64(P(ag_atoms), C.c_int64(len(ag_atoms)), P(cands), P(off), C.c_int64(len(off) - 1), P(out),
                            P(ab), threads)
    return (out, ab) if with_abs else out


def forces_allatom64(ag_atoms, cands, offsets, threads=8):
    ag_atoms, cands = _ga(ag_atoms), _ga(cands)
    off = np.ascontiguousarray(offsets, np.int64)
    f = np.zeros((len(cands), 3), np.float64)
    e = np.zeros(len(off) - 1, np.float64)
    lib().orc_forces_allatom64(P(ag_atoms), C.c_int64(len(ag_atoms)), P(cands), P(off), C.c_int64(len(off) - 1),
                               P(f), P(e), threads)
    return f, e


def count_pairs(ag_atoms, cands, threads=8):
    ag_atoms, cands = _ga(ag_atoms), _ga(cands)
    return lib().orc_count_pairs(P(ag_atoms), C.c_int64(len(ag_atoms)), P(cands), C.c_int64(len(cands)), threads)


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox(P(c), P(k), P(out))
    return out


def temperature(i, total):
    return lib().orc_temperature(i, total)


def topk(e, k):
    e = np.ascontiguousarray(e, np.float64)
    out = np.zeros(k, np.int32)
    lib().orc_topk(P(e), C.c_int64(len(e)), C.c_int64(k), P(out))
    return out


class Antigen:
    def __init__(self, aa, pos, ca_cell=10.0):
        self.aa, self.pos = u8(aa), f32(pos)
        self.h = lib().orc_antigen_new(len(self.aa), P(self.aa), P(self.pos), ca_cell)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_antigen_free(self.h)
            self.h = None

    def center(self):
        out = np.zeros(3, np.float32)
        lib().orc_antigen_center(C.c_void_p(self.h), P(out))
        return out

    def residue_contribution(self, aa, pos, r, f64_sum=False):
        """residue_contribution_allatom: f32 sum (the reference), or the same f32
        terms summed in double"""
        aa, pos = u8(aa), f32(pos)
        fn = lib().orc_residue_contribution64 if f64_sum else lib().orc_residue_contribution
        return fn(self.h, len(aa), P(aa), P(pos), r)

    def step(self, params, aa, chi, pos, n_res, cand_id, step_id, temp, with_noise, with_mc, threads=8, stats=None):
        """in-place: aa [n_cand*n_res], chi [..,4], pos [..,14,3]"""
        n_cand = len(aa) // n_res
        cid = np.ascontiguousarray(cand_id, np.uint32)
        lib().orc_step(self.h, C.byref(params), n_cand, n_res, P(aa), P(chi), P(pos), P(cid), step_id, temp,
                       int(with_noise), int(with_mc), P(stats), threads)

    def minimize(self, aa, chi, pos, n_res, steps, acc64=True, threads=8, with_margin=False):
        """minimize (diffusion.rs:854-916) against this antigen, in place; final
        energies (and the smallest relative keep / restore margin per candidate)"""
        n_cand = len(aa) // n_res
        out = np.zeros(n_cand, np.float64)
        margin = np.zeros(n_cand, np.float64)
        lib().orc_minimize(C.c_void_p(self.h), n_cand, n_res, P(aa), P(chi), P(pos), steps, int(acc64), P(out),
                           P(margin), threads)
        return (out, margin) if with_margin else out

    def affinity_maturation(self, aa, chi, pos, n_res, acc64=True, threads=8, with_margin=False):
        """affinity_maturation_allatom over the interface residues, in place; (final
        scores, mutations kept[, smallest relative decision margin]) per candidate"""
        n_cand = len(aa) // n_res
        out = np.zeros(n_cand, np.float64)
        kept = np.zeros(n_cand, np.int32)
        margin = np.zeros(n_cand, np.float64)
        lib().orc_affinity_maturation(C.c_void_p(self.h), n_cand, n_res, P(aa), P(chi), P(pos), int(acc64), P(out),
                                      P(kept), P(margin), threads)
        return (out, kept, margin) if with_margin else (out, kept)

    def fv_run(self, params, heavy, light, iterations, target_radius, cand_id=None, acc64=True, threads=8):
        """The run_fv iteration loop (diffusion.rs:791-812); heavy / light = (aa, chi,
        pos, cdr) stacked over candidates, updated in place to the best pairs.
        Returns (best fv_energy, smallest relative keep / restore margin) per candidate."""
        (ha, hc, hp, hr), (la, lc, lp, lr) = heavy, light
        n_cand = len(cand_id)
        n_h, n_l = len(hr) // n_cand, len(lr) // n_cand
        out = np.zeros(n_cand, np.float64)
        margin = np.zeros(n_cand, np.float64)
        cid = np.ascontiguousarray(cand_id, np.uint32)
        lib().orc_fv_run(C.c_void_p(self.h), C.byref(params), n_cand, n_h, n_l, P(ha), P(hc), P(hp), P(u8(hr)),
                         P(la), P(lc), P(lp), P(u8(lr)), P(cid), iterations, C.c_float(target_radius), int(acc64),
                         P(out), P(margin), threads)
        return out, margin

    def fv_energy(self, h_aa, h_pos, l_aa, l_pos, acc64=True):
        """fv_energy (diffusion.rs:541-547) of one heavy / light pair"""
        h_aa, h_pos, l_aa, l_pos = u8(h_aa), f32(h_pos), u8(l_aa), f32(l_pos)
        return lib().orc_fv_energy(C.c_void_p(self.h), len(h_aa), P(h_aa), P(h_pos), len(l_aa), P(l_aa), P(l_pos),
                                   int(acc64))

    def score_slots64(self, aa, pos, n_res, full=False, threads=8, with_abs=False):
        """f64 energy per candidate; with_abs also the sum of |pair term| (the
        denominator of the norm-wise error of ill-conditioned candidates)"""
        aa, pos = u8(aa), f32(pos)
        n_cand = len(aa) // n_res
        out = np.zeros(n_cand, np.float64)
        ab = np.zeros(n_cand, np.float64) if with_abs else None
        lib().orc_score_slots64(self.h, n_cand, n_res, P(aa), P(pos), int(full), P(out), P(ab), threads)
        return (out, ab) if with_abs else out


def validate(aa, pos):
    """ValidationReport::assess (validate.rs:24-132): (clashes, rama_outliers)"""
    aa, pos = u8(aa), f32(pos)
    cl, ra = C.c_int32(), C.c_int32()
    lib().orc_validate(len(aa), P(aa), P(pos), C.byref(cl), C.byref(ra))
    return cl.value, ra.value


def disulfide(aa, pos):
    aa, pos = u8(aa), f32(pos)
    return lib().orc_disulfide(len(aa), P(aa), P(pos))
