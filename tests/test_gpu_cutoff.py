"""The pair set at its boundaries: candidate atoms placed at r^2 within a few ulps of
the cutoff (100), the hydrophobic cutoff (36) and the minimum distance (0.25) of an
antigen atom.  A pair belongs to the set when the reference's f32 rounding of
(dx*dx + dy*dy) + dz*dz (energy.rs:269-275, two roundings, never fused) is inside;
a fused multiply-add on any of the three steps moves about a third of these pairs
across the boundary.  GPU pair counts equal the oracle's exactly and energies agree
within 1e-5 of the sum of |pair terms| (a single flip changes a candidate's energy
by several kcal/mol).  Includes the pair found in a full-size run: r^2 = 100.000008
in the reference's rounding, 100.0 when fused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _r2_ref(a, b):
    d = (b - a).astype(np.float32)
    return (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]  # numpy f32: never fused


def _boundary_case(pkg, radius, n_ag=96, per=8, hyd=0.0, seed=5):
    """n_ag antigen atoms 40 A apart; candidate k = `per` atoms at `radius` (+- a few
    ulps) around antigen atom k, so that every pair of the set is a boundary pair."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(6), np.arange(4), np.arange(4), indexing="ij"), -1).reshape(-1, 3)[:n_ag]
    ag_xyz = (g * 40.0 + rng.uniform(-3, 3, size=(n_ag, 3))).astype(np.float32)
    q = rng.choice([-0.8, 0.8], size=n_ag).astype(np.float32)
    ag = pkg.AtomCloud(ag_xyz[:, 0].copy(), ag_xyz[:, 1].copy(), ag_xyz[:, 2].copy(), q,
                       np.full(n_ag, 1.9, np.float32), np.full(n_ag, 0.1, np.float32),
                       np.full(n_ag, hyd > 0, np.uint8))
    cands = np.zeros((n_ag * per, 8), np.float32)
    scale = (radius * (1 + rng.uniform(-3e-7, 3e-7, size=(n_ag * per, 1)))).astype(np.float32)
    cxyz = (np.repeat(ag_xyz, per, 0) + (_unit(rng, n_ag * per) * scale).astype(np.float32)).astype(np.float32)
    cands[:, :3] = cxyz
    cands[:, 3] = rng.choice([-0.9, 0.9], size=n_ag * per)
    cands[:, 4], cands[:, 5], cands[:, 6] = 1.7, 0.15, hyd
    off = np.arange(0, n_ag * per + 1, per, dtype=np.int64)
    return ag, _atoms(pkg, cands), off, ag_xyz, cxyz


def _atoms(pkg, rows):
    """(n, 8) float32 rows -> binder_gpu_atom records"""
    return np.ascontiguousarray(rows, np.float32).view(pkg.GPU_ATOM).reshape(-1)


def _check(ctx, oracle, ag, cands, off, lo, hi, ag_xyz, cxyz, per):
    r2 = _r2_ref(np.repeat(ag_xyz, per, 0), cxyz)
    inside = (r2 >= lo) & (r2 <= hi)
    assert 0.2 < inside.mean() < 0.8  # both sides of the boundary are populated
    e, eabs = ctx.score_batch_ragged(ag, cands, off, with_abs=True)
    assert ctx.last_pair_count() == oracle.count_pairs(ag.to_gpu_atoms(), cands)
    e64, abs64 = oracle.score_batch64(ag.to_gpu_atoms(), cands, off, with_abs=True)
    assert np.all(np.abs(e - e64) <= 1e-5 * np.maximum(abs64, 1e-3))


def test_pair_set_at_the_cutoff(ctx, oracle, pkg):
    ag, cands, off, ag_xyz, cxyz = _boundary_case(pkg, 10.0)
    inside = _r2_ref(np.repeat(ag_xyz, 8, 0), cxyz) <= 100.0
    assert inside.sum() == oracle.count_pairs(ag.to_gpu_atoms(), cands)
    _check(ctx, oracle, ag, cands, off, 0.25, 100.0, ag_xyz, cxyz, 8)


def test_pair_set_at_the_minimum_distance(ctx, oracle, pkg):
    ag, cands, off, ag_xyz, cxyz = _boundary_case(pkg, 0.5, seed=6)
    _check(ctx, oracle, ag, cands, off, 0.25, 100.0, ag_xyz, cxyz, 8)


def test_hydrophobic_term_at_its_cutoff(ctx, oracle, pkg):
    # r^2 < 36 decides the -0.5 bonus between hydrophobic atoms (energy.rs:293-299)
    ag, cands, off, ag_xyz, cxyz = _boundary_case(pkg, 6.0, hyd=1.0, seed=7)
    r2 = _r2_ref(np.repeat(ag_xyz, 8, 0), cxyz)
    assert 0.2 < (r2 < 36.0).mean() < 0.8
    e, eabs = ctx.score_batch_ragged(ag, cands, off, with_abs=True)
    e64, abs64 = oracle.score_batch64(ag.to_gpu_atoms(), cands, off, with_abs=True)
    assert np.all(np.abs(e - e64) <= 1e-5 * np.maximum(abs64, 1e-3))


def test_pair_from_a_full_size_run(ctx, oracle, pkg):
    """Antigen atom 1483 of the 300-residue globule against the first eight atoms of a
    Glu of candidate 303 after one block; atom 3 (OE1) sits at r^2 = 100.000008."""
    h = lambda *u: np.array(u, np.uint32).view(np.float32)  # noqa: E731
    a = h(0x40f40b70, 0xc12253c1, 0x414c4d66)  # 7.626396, -10.145448, 12.768896
    b3 = h(0x4187743c, 0xc11b41ad, 0x4112236f)  # 16.931755, -9.703534, 9.133651
    assert np.array_equal((b3 - a).view(np.uint32), [0x4114e2c0, 0x3ee24280, 0xc068a7dc])
    rng = np.random.default_rng(11)
    others = (a + _unit(rng, 7) * rng.uniform(6.5, 9.5, size=(7, 1))).astype(np.float32)
    xyz = np.concatenate([others[:3], b3[None], others[3:]]).astype(np.float32)
    assert _r2_ref(a[None], b3[None])[0] > 100.0
    ag = pkg.AtomCloud(a[0:1], a[1:2], a[2:3], np.float32([-0.4157]), np.float32([1.824]), np.float32([0.17]),
                       np.uint8([0]))
    cands = np.zeros((8, 8), np.float32)
    cands[:, :3] = xyz
    cands[:, 3], cands[:, 4], cands[:, 5] = -0.5819, 1.6612, 0.21
    off = np.array([0, 8], np.int64)
    cands = _atoms(pkg, cands)
    e = ctx.score_batch_ragged(ag, cands, off)
    assert ctx.last_pair_count() == 7
    e64 = oracle.score_batch64(ag.to_gpu_atoms(), cands, off)
    assert abs(e[0] - e64[0]) <= 1e-5 * max(abs(e64[0]), 1.0)
