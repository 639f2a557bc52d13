"""Seeded synthetic workloads (the reference measures on no public dataset).

Each generator returns Calpha traces + sequences; all-atom structures are then
built on the GPU by ``GpuContext.build_residues`` (protein_from_ca_trace,
allatom.rs:523-541) or by the CPU oracle in tests.  Seeds: 0xB200 + config id.

  config 0  16-residue peptide antigen as an extended trace (pdb.rs:64-83),
            64 antibodies x 12 residues, Calpha on a 12 A sphere around the
            antigen Calpha centre of mass.
  config 1  300-residue compact globule: self-avoiding Calpha walk, 3.8 A steps,
            non-bonded Calpha >= 4 A, confined to a 22 A sphere; 1024 antibodies
            x 20 residues with Calpha on the shell 4 A outside the globule.
  config 2  8 globules of 50..800 residues (radius 22 (n/300)^(1/3) keeps the
            config-1 density), 4096 antibodies of 10..30 residues round-robin.
  config 3  config-1 antigen + 1024 frozen all-atom poses whose atoms sit at
            log-uniform 2.5-12 A from random antigen atoms; 30 % of residues
            charged (K, R, D, E).
  config 4  learned proposal: training antigens (300-residue globules built as
            in config 1 from their own seeds) with 1024 x 20-residue antibodies
            each, and held-out 300-residue antigens of other seeds with 1024 x 20
            antibodies for the evaluation.
"""
from __future__ import annotations

import numpy as np

# GpuAtom (gpu.rs:17-29): 8 x f32
GPU_ATOM = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("q", "<f4"), ("r_min_half", "<f4"),
                     ("epsilon", "<f4"), ("hydrophobic", "<f4"), ("_pad", "<f4")])
SEED_BASE = 0xB200
CA_BOND = np.float32(3.8)
N_AA = 20
AA_INDEX = {c: i for i, c in enumerate("ARNDCQEGHILKMFPSTWYV")}
CHARGED = np.array([AA_INDEX["K"], AA_INDEX["R"], AA_INDEX["D"], AA_INDEX["E"]], np.uint8)


def rng_for(config_id: int, salt: int = 0):
    return np.random.default_rng(SEED_BASE + config_id + 1000003 * salt)


def random_sequence(n, rng):
    return rng.integers(0, N_AA, size=n).astype(np.uint8)


def peptide_trace(n):
    """parse_peptide (pdb.rs:64-83): x = (i - n*0.5) * 3.8 along x, centred, in f32."""
    i = np.arange(n, dtype=np.float32)
    x = (i - np.float32(n) * np.float32(0.5)) * CA_BOND
    return np.stack([x, np.zeros(n, np.float32), np.zeros(n, np.float32)], axis=1).astype(np.float32)


def globule_trace(n, radius, rng, step=3.8, min_sep=4.0, tries=128):
    """Self-avoiding Calpha random walk confined to a sphere (rejection sampling
    with backtracking).  Non-bonded Calpha pairs stay >= min_sep apart."""
    pts = np.zeros((n, 3))
    pts[0] = _ball_point(rng, 0.5 * radius)
    i = 1
    fails = np.zeros(n, int)
    while i < n:
        d = rng.normal(size=(tries, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        cand = pts[i - 1] + step * d
        ok = np.linalg.norm(cand, axis=1) <= radius
        if i >= 2 and ok.any():
            dd = np.linalg.norm(cand[:, None, :] - pts[None, : i - 1, :], axis=2)
            ok &= dd.min(axis=1) >= min_sep
        if ok.any():
            pts[i] = cand[np.argmax(ok)]
            i += 1
        else:
            fails[i] += 1
            back = min(i - 1, 1 + fails[i] // 4)
            i -= back
    return pts.astype(np.float32)


def _ball_point(rng, r):
    while True:
        p = rng.uniform(-r, r, size=3)
        if np.dot(p, p) <= r * r:
            return p


def sphere_points(n, radius, center, rng):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return (np.asarray(center, np.float64) + radius * d).astype(np.float32)


def ca_center(ca):
    """ca_center_of_mass (allatom.rs:183-195): sequential f32 sums / n."""
    s = np.zeros(3, np.float32)
    for p in np.asarray(ca, np.float32):
        s = (s + p).astype(np.float32)
    return (s / np.float32(len(ca))).astype(np.float32)


class Population:
    """Antibody Calpha traces + sequences for one workload."""

    def __init__(self, ca, aa, n_res, antigen_id):
        self.ca = ca                  # [total_res, 3] f32
        self.aa = aa                  # [total_res] u8
        self.n_res = n_res            # [n_cand] i32
        self.antigen_id = antigen_id  # [n_cand] i32

    @property
    def n_cand(self):
        return len(self.n_res)


def config0():
    rng = rng_for(0)
    ag_aa = random_sequence(16, rng)
    ag_ca = peptide_trace(16)
    c = ca_center(ag_ca)
    n_cand, n_res = 64, 12
    ca = sphere_points(n_cand * n_res, 12.0, c, rng)
    aa = random_sequence(n_cand * n_res, rng)
    pop = Population(ca, aa, np.full(n_cand, n_res, np.int32), np.zeros(n_cand, np.int32))
    return dict(name="config0", antigens=[(ag_aa, ag_ca)], shell=[20.0], pop=pop, gpu_steps=200, score_every=10,
                population=64, mc_steps=600)


def _globule_antigen(n_res, rng):
    radius = 22.0 * (n_res / 300.0) ** (1.0 / 3.0)
    ca = globule_trace(n_res, radius, rng)
    return random_sequence(n_res, rng), ca, radius


def config1(n_cand=1024, n_res=20, salt=0):
    """salt != 0 draws an independent antibody population against the same antigen."""
    rng = rng_for(1)
    ag_aa, ag_ca, radius = _globule_antigen(300, rng)
    shell = radius + 4.0
    c = ca_center(ag_ca)
    if salt:
        rng = rng_for(1, salt)
    ca = sphere_points(n_cand * n_res, shell, c, rng)
    aa = random_sequence(n_cand * n_res, rng)
    pop = Population(ca, aa, np.full(n_cand, n_res, np.int32), np.zeros(n_cand, np.int32))
    return dict(name="config1", antigens=[(ag_aa, ag_ca)], shell=[shell], pop=pop, gpu_steps=200, score_every=10,
                population=64, mc_steps=600)


def config2(n_cand=4096):
    rng = rng_for(2)
    sizes = [50, 100, 200, 300, 400, 500, 650, 800]
    antigens, shells = [], []
    for n in sizes:
        aa, ca, radius = _globule_antigen(n, rng)
        antigens.append((aa, ca))
        shells.append(radius + 4.0)
    n_res = rng.integers(10, 31, size=n_cand).astype(np.int32)
    ag_id = (np.arange(n_cand) % len(sizes)).astype(np.int32)
    cas, aas = [], []
    for c in range(n_cand):
        center = ca_center(antigens[ag_id[c]][1])
        cas.append(sphere_points(int(n_res[c]), shells[ag_id[c]], center, rng))
        aas.append(random_sequence(int(n_res[c]), rng))
    pop = Population(np.concatenate(cas), np.concatenate(aas), n_res, ag_id)
    return dict(name="config2", antigens=antigens, shell=shells, pop=pop, gpu_steps=200, score_every=10,
                population=64, mc_steps=600)


def config3_poses(ag_cloud_xyz, tables, n_cand=1024, n_res=20, charged_frac=0.3):
    """Frozen contact-skewed poses for the precision study.  Returns (GpuAtom
    structured array, offsets, aa) built from the topology tables."""
    rng = rng_for(3)
    aa = random_sequence(n_cand * n_res, rng)
    charged = rng.random(n_cand * n_res) < charged_frac
    aa[charged] = CHARGED[rng.integers(0, 4, size=int(charged.sum()))]
    n_at = tables.n_atoms[aa]
    total = int(n_at.sum())
    res_of_atom = np.repeat(np.arange(len(aa)), n_at)
    slot = np.concatenate([np.arange(k) for k in n_at])
    anchor = ag_cloud_xyz[rng.integers(0, len(ag_cloud_xyz), size=total)]
    r = np.exp(rng.uniform(np.log(2.5), np.log(12.0), size=total))
    d = rng.normal(size=(total, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    xyz = (anchor + r[:, None] * d).astype(np.float32)
    a_of = aa[res_of_atom]
    types = tables.atom_type[a_of, slot]
    g = np.zeros(total, GPU_ATOM)
    g["x"], g["y"], g["z"] = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    g["q"] = tables.charge[a_of, slot]
    g["r_min_half"] = tables.r_min_half[types]
    g["epsilon"] = tables.epsilon[types]
    g["hydrophobic"] = tables.hydrophobic[a_of, slot].astype(np.float32)
    per_cand = np.add.reduceat(n_at, np.arange(0, len(aa), n_res))
    off = np.concatenate([[0], np.cumsum(per_cand)]).astype(np.int64)
    return g, off, aa



def _config1_like(rng, n_cand, n_res):
    ag_aa, ag_ca, radius = _globule_antigen(300, rng)
    shell = radius + 4.0
    c = ca_center(ag_ca)
    ca = sphere_points(n_cand * n_res, shell, c, rng)
    aa = random_sequence(n_cand * n_res, rng)
    return (ag_aa, ag_ca), shell, Population(ca, aa, np.full(n_cand, n_res, np.int32), np.zeros(n_cand, np.int32))


def config4(n_train=4, n_eval=2, n_cand=1024, n_res=20):
    """Training antigens (seeds 1..n_train) and held-out antigens (seeds 1001..),
    each a config-1-style 300-residue globule with its own population."""
    train = [_config1_like(rng_for(4, salt=s), n_cand, n_res) for s in range(1, n_train + 1)]
    held = [_config1_like(rng_for(4, salt=1000 + s), n_cand, n_res) for s in range(1, n_eval + 1)]
    return dict(name="config4", train=train, eval=held)


def config3_slots(ag_cloud_xyz, tables, n_cand=1024, n_res=20, charged_frac=0.3):
    """The frozen contact-skewed poses of config3_poses in the slot layout of the
    resident state: returns (aa [n_cand * n_res], pos [n_cand * n_res, 14, 3]), the
    used slots of every residue holding the pose's atoms, the others zero."""
    g, _, aa = config3_poses(ag_cloud_xyz, tables, n_cand, n_res, charged_frac)
    n_at = tables.n_atoms[aa]
    res_of_atom = np.repeat(np.arange(len(aa)), n_at)
    slot = np.concatenate([np.arange(k) for k in n_at])
    pos = np.zeros((len(aa), 14, 3), np.float32)
    pos[res_of_atom, slot, 0] = g["x"]
    pos[res_of_atom, slot, 1] = g["y"]
    pos[res_of_atom, slot, 2] = g["z"]
    return aa, pos


# ---- Fv two-chain workload (diffusion.rs:477-827, germline.rs) -------------------------
# Germline framework scaffolds (germline.rs:42-61): FR1, CDR1 length, FR2, CDR2 length,
# FR3, CDR3 length, FR4; VH3-23-like heavy chain and IGKV1-39-like kappa light chain.
VH_FRAMEWORK = ("EVQLLESGGGLVQPGGSLRLSCAAS", 8, "WVRQAPGKGLEWVS", 8, "RFTISRDNSKNTLYLQMNSLRAEDTAVYYCAK", 12,
                "WGQGTLVTVSS")
VL_FRAMEWORK = ("DIQMTQSPSSLSASVGDRVTITC", 11, "WYQQKPGKAPKLLIY", 7, "GVPSRFSGSGSGTDFTLTISSLQPEDFATYYC", 9,
                "FGQGTKVEIK")
FV_LOCAL_RADIUS_SCALE = np.float32(1.3)   # diffusion.rs:54
FV_CHAIN_MARGIN = np.float32(6.0)         # diffusion.rs:58
INIT_RADIUS = np.float32(20.0)            # diffusion.rs:81


def fv_layout(fw, cdr3_len=None):
    fr1, c1, fr2, c2, fr3, c3, fr4 = fw
    return fr1, c1, fr2, c2, fr3, c3 if cdr3_len is None else max(1, cdr3_len), fr4


def assemble_chain(fw, cdr1, cdr2, cdr3):
    """assemble_chain (germline.rs:91-123): sequence (AminoAcid indices) and a CDR flag
    per residue (0 framework, 1/2/3 the CDR loop)."""
    fr1, _, fr2, _, fr3, _, fr4 = fw
    seq, region = [], []
    for part, reg in ((fr1, 0), (cdr1, 1), (fr2, 0), (cdr2, 2), (fr3, 0), (cdr3, 3), (fr4, 0)):
        codes = [AA_INDEX[c] for c in part] if isinstance(part, str) else list(part)
        seq += codes
        region += [reg] * len(codes)
    return np.array(seq, np.uint8), np.array(region, np.uint8)


def fib_sphere_offset(i, n, radius):
    """fib_sphere_offset (diffusion.rs:501-507), f32."""
    f = np.float32
    n_f = f(max(n, 1))
    y = f(1.0) - f(2.0) * (f(i) + f(0.5)) / n_f
    r_y = np.sqrt(np.maximum(f(1.0) - y * y, f(0.0)))
    theta = f(2.399963) * f(i)
    return np.array([np.cos(theta) * r_y * f(radius), y * f(radius), np.sin(theta) * r_y * f(radius)], np.float32)


def config_fv(antigen_ca, n_cand=8, h3_len=12, l3_len=9, seed=0xB200 + 5):
    """The initial population of run_fv (diffusion.rs:704-776): per candidate a random
    approach direction toward the antigen's Calpha centre, the heavy and light chains
    as two clusters beside it (CDRs uniform random, Calphas on Fibonacci spheres of
    1.3 sqrt(n) A plus uniform +-1.5 A noise).  The reference draws these from its
    per-candidate SmallRng; here from a seeded numpy generator (the chains are
    uploaded as they are).  Returns dict(heavy=(aa, ca, region) stacked over
    candidates, light=..., target_radius, center)."""
    rng = np.random.default_rng(seed)
    vh, vl = fv_layout(VH_FRAMEWORK, h3_len), fv_layout(VL_FRAMEWORK, l3_len)
    n_h = sum(len(p) if isinstance(p, str) else p for p in vh)
    n_l = sum(len(p) if isinstance(p, str) else p for p in vl)
    center = ca_center(antigen_ca)
    f = np.float32
    radius_h = FV_LOCAL_RADIUS_SCALE * np.sqrt(f(n_h))
    radius_l = FV_LOCAL_RADIUS_SCALE * np.sqrt(f(n_l))
    half_sep = (radius_h + radius_l + FV_CHAIN_MARGIN) * f(0.5)
    approach_radius = INIT_RADIUS + max(radius_h, radius_l) + f(5.0)
    target_radius = np.sqrt(approach_radius * approach_radius + half_sep * half_sep)
    chains = {"heavy": ([], [], []), "light": ([], [], [])}
    for _ in range(n_cand):
        theta = f(rng.uniform(0.0, 2 * np.pi))
        cos_phi = f(rng.uniform(-1.0, 1.0))
        sin_phi = np.sqrt(max(f(1.0) - cos_phi * cos_phi, f(0.0)))
        d = np.array([sin_phi * np.cos(theta), cos_phi, sin_phi * np.sin(theta)], np.float32)
        approach = center + d * approach_radius
        up = np.float32([0, 1, 0]) if abs(d[1]) < 0.9 else np.float32([1, 0, 0])
        perp = np.cross(d, up).astype(np.float32)
        perp = perp / max(np.float32(np.linalg.norm(perp)), np.float32(1e-8))
        for name, fw, sign in (("heavy", vh, 1.0), ("light", vl, -1.0)):
            cdr = [rng.integers(0, N_AA, size=fw[k]) for k in (1, 3, 5)]
            seq, region = assemble_chain(fw, *cdr)
            n = len(seq)
            local = FV_LOCAL_RADIUS_SCALE * np.sqrt(f(n))
            cc = approach + f(sign) * perp * half_sep
            ca = np.stack([cc + fib_sphere_offset(i, n, local) + rng.uniform(-1.5, 1.5, 3).astype(np.float32)
                           for i in range(n)]).astype(np.float32)
            chains[name][0].append(seq)
            chains[name][1].append(ca)
            chains[name][2].append(region)
    out = {k: tuple(np.concatenate(v) for v in chains[k]) for k in chains}
    out.update(n_heavy=n_h, n_light=n_l, target_radius=float(target_radius), center=center, n_cand=n_cand)
    return out
