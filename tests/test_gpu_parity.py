"""CUDA path vs the CPU oracle, through the C ABI.

Tolerances (stated per test): integer / index results bit-exact; grid cells and
neighbour lists bit-exact; the coarse-grained force, residue construction and
gradient-phase trajectories bit-exact (the kernels keep the reference's f32
operation order); per-candidate all-atom energies within 1e-5 relative of the
f64 oracle (norm-wise 1e-5 of the sum of |pair terms| for ill-conditioned
candidates); all-atom forces within 1e-4 relative (norm-wise, floor 1e-3 of
the largest force)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _population(oracle, wl, cfg, limit=None):
    pop = cfg["pop"]
    n_cand = pop.n_cand if limit is None else min(limit, pop.n_cand)
    off_res = np.concatenate([[0], np.cumsum(pop.n_res)])
    cands, offs = [], [0]
    for c in range(n_cand):
        aa = pop.aa[off_res[c]:off_res[c + 1]]
        pos, _ = oracle.build_residues(pop.ca[off_res[c]:off_res[c + 1]], aa)
        g = oracle.gpu_atoms(oracle.flatten(aa, pos))
        cands.append(g)
        offs.append(offs[-1] + len(g))
    return np.concatenate(cands), np.asarray(offs, np.int64)


def _antigen(oracle, pkg, cfg, i=0):
    aa, ca = cfg["antigens"][i]
    pos, _ = oracle.build_residues(ca, aa)
    return aa, pos, pkg.AtomCloud.from_slots(aa, pos)


def _check_energy(e_gpu, e64, eabs, tol=1e-5):
    rel = rel_err(e_gpu, e64)
    normwise = np.abs(e_gpu - e64) / np.maximum(eabs, 1e-6)
    cond = eabs / np.maximum(np.abs(e64), 1e-30)
    well = cond <= 10
    assert np.all(rel[well] < tol), (rel[well].max(), np.argmax(rel * well))
    assert np.all(normwise < tol), normwise.max()
    return rel, normwise


# ---- spatial grid (bit-exact) ---------------------------------------------------------
@pytest.mark.parametrize("cell", [10.0, 8.0, 3.3])
def test_grid_cells_bit_exact(ctx, oracle, cell):
    rng = np.random.default_rng(1)
    p = rng.uniform(-60, 60, size=(3000, 3)).astype(np.float32)
    # points on cell boundaries and their neighbours in float
    edges = (np.arange(-5, 6, dtype=np.float32) * np.float32(cell))
    p[:11, 0] = edges
    p[11:22, 1] = np.nextafter(edges, np.float32(-np.inf))
    p[22:33, 2] = np.nextafter(edges, np.float32(np.inf))
    got = ctx.grid_cells(cell, p[:, 0], p[:, 1], p[:, 2])
    exp = np.array([oracle.grid_cell(cell, *q) for q in p])
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("cell,n_ag,n_q", [(10.0, 300, 500), (8.0, 2500, 400), (4.0, 1000, 300), (10.0, 1, 5),
                                           (10.0, 0, 5)])
def test_grid_neighbors_bit_exact(ctx, oracle, cell, n_ag, n_q):
    rng = np.random.default_rng(n_ag + n_q)
    ag = rng.uniform(-25, 25, size=(n_ag, 3)).astype(np.float32)
    q = rng.uniform(-40, 40, size=(n_q, 3)).astype(np.float32)
    if n_ag:
        q[: min(n_q, n_ag)] = ag[: min(n_q, n_ag)]  # probes sitting on atoms
    go, gi = ctx.grid_neighbors(cell, ag[:, 0], ag[:, 1], ag[:, 2], q[:, 0], q[:, 1], q[:, 2])
    oo, oi = oracle.grid_neighbors(cell, ag[:, 0], ag[:, 1], ag[:, 2], q[:, 0], q[:, 1], q[:, 2])
    assert np.array_equal(go, oo) and np.array_equal(gi, oi)


def test_grid_far_probe_and_huge_box(ctx, oracle, pkg):
    ag = np.float32([[0, 0, 0], [1e5, 0, 0]])  # 1e8 cells of 1 mA > 2^24 cap
    with pytest.raises(pkg.BinderError) as e:
        ctx.grid_neighbors(0.001, ag[:, 0], ag[:, 1], ag[:, 2], [0.0], [0.0], [0.0])
    assert e.value.status == 6  # BINDER_ERR_GRID
    go, gi = ctx.grid_neighbors(10.0, ag[:, 0], ag[:, 1], ag[:, 2], [5000.0], [0.0], [0.0])
    assert go.tolist() == [0, 0] and len(gi) == 0


# ---- residue construction (bit-exact) ---------------------------------------------------
def test_build_residues_bit_exact(ctx, oracle):
    rng = np.random.default_rng(7)
    aa = np.tile(np.arange(20, dtype=np.uint8), 10)
    ca = rng.uniform(-30, 30, size=(len(aa), 3)).astype(np.float32)
    gp, gc = ctx.build_residues(ca, aa)
    op, oc = oracle.build_residues(ca, aa)
    assert np.array_equal(gp, op) and np.array_equal(gc, oc)
    chi = rng.uniform(-180, 180, size=(len(aa), 4)).astype(np.float32)
    gp, gc = ctx.build_residues(ca, aa, chi)
    op, oc = oracle.build_residues(ca, aa, chi)
    assert np.array_equal(gp, op) and np.array_equal(gc, oc)


# ---- score_batch --------------------------------------------------------------------------
def test_score_batch_config0(ctx, oracle, pkg):
    cfg = pkg.workloads.config0()
    _, _, ag = _antigen(oracle, pkg, cfg)
    cands, off = _population(oracle, pkg.workloads, cfg)
    e64, eabs = oracle.score_batch64(ag.to_gpu_atoms(), cands, off, with_abs=True)
    eg = ctx.score_batch_ragged(ag, cands, off)
    _check_energy(eg, e64, eabs)


def test_score_batch_config1_subset(ctx, oracle, pkg):
    cfg = pkg.workloads.config1(n_cand=128)
    _, _, ag = _antigen(oracle, pkg, cfg)
    cands, off = _population(oracle, pkg.workloads, cfg)
    e64, eabs = oracle.score_batch64(ag.to_gpu_atoms(), cands, off, with_abs=True)
    eg, gabs = ctx.score_batch_ragged(ag, cands, off, with_abs=True)
    _check_energy(eg, e64, eabs)
    assert np.all(rel_err(gabs, eabs) < 1e-4)
    assert ctx.last_pair_count() == oracle.count_pairs(ag.to_gpu_atoms(), cands)


def test_score_batch_uniform_dropin(ctx, oracle, pkg):
    cfg = pkg.workloads.config0()
    _, _, ag = _antigen(oracle, pkg, cfg)
    rng = np.random.default_rng(3)
    n_ab, n_cand = 40, 50
    g = np.zeros(n_ab * n_cand, pkg.GPU_ATOM)
    src = ag.to_gpu_atoms()
    pick = rng.integers(0, len(src), len(g))
    g[:] = src[pick]
    g["x"] += rng.normal(scale=4.0, size=len(g)).astype(np.float32)
    g["y"] += rng.normal(scale=4.0, size=len(g)).astype(np.float32)
    off = np.arange(0, len(g) + 1, n_ab, dtype=np.int64)
    e32 = ctx.score_batch(ag, g, n_ab)
    e64, eabs = oracle.score_batch64(src, g, off, with_abs=True)
    _check_energy(e32.astype(np.float64), e64, eabs, tol=2e-7 + 1e-5)
    assert e32.dtype == np.float32 and len(e32) == n_cand
    # n_ab = 0 -> no candidates (gpu.rs:172-174); trailing atoms ignored like the integer division
    assert len(ctx.score_batch(ag, g, 0)) == 0
    assert len(ctx.score_batch(ag, g[:-3], n_ab)) == n_cand - 1


def test_score_batch_rejects_nan(ctx, oracle, pkg):
    cfg = pkg.workloads.config0()
    _, _, ag = _antigen(oracle, pkg, cfg)
    g = ag.to_gpu_atoms()[:20].copy()
    g["x"][3] = np.nan
    with pytest.raises(pkg.BinderError) as e:
        ctx.score_batch(ag, g, 10)
    assert e.value.status == 5


def test_score_batch_plain_f32_accumulation_within_tolerance(ctx, oracle, pkg):
    cfg = pkg.workloads.config1(n_cand=64)
    _, _, ag = _antigen(oracle, pkg, cfg)
    cands, off = _population(oracle, pkg.workloads, cfg)
    e64, eabs = oracle.score_batch64(ag.to_gpu_atoms(), cands, off, with_abs=True)
    ek = ctx.score_batch_ragged(ag, cands, off)
    p = pkg.Params.defaults(accumulate=pkg.ACC_F32)
    c2 = pkg.GpuContext.create(0, p)
    ep = c2.score_batch_ragged(ag, cands, off)
    c2.close()
    # both accumulation modes meet the energy tolerance on this workload (the
    # per-term rounding dominates; the stress set of the precision study separates them)
    _check_energy(ek, e64, eabs)
    _check_energy(ep, e64, eabs)


# ---- forces ----------------------------------------------------------------------------------
def test_cg_forces_bit_exact_and_reference_tests(ctx, oracle, pkg):
    A = {c: i for i, c in enumerate("ARNDCQEGHILKMFPSTWYV")}
    # energy.rs:406-441 two-residue case through the GPU
    ag = pkg.ResidueCloud([0, 5], [0, 0], [0, 0], [A["K"], A["L"]])
    ab = pkg.ResidueCloud([3], [0], [0], [A["D"]])
    fx, fy, fz = ctx.compute_forces_with_grid(ag, 10.0, ab)
    bx, by, bz = oracle.forces_cg_brute([[0, 0, 0], [5, 0, 0]], [A["K"], A["L"]], [[3, 0, 0]], [A["D"]])
    assert abs(fx[0] - bx[0]) < 1e-4 and fx[0] < 0  # grid == brute (1e-4), attraction
    rng = np.random.default_rng(11)
    ag_xyz = rng.uniform(-22, 22, size=(300, 3)).astype(np.float32)
    ag_aa = rng.integers(0, 20, 300).astype(np.uint8)
    ab_xyz = rng.uniform(-30, 30, size=(2000, 3)).astype(np.float32)
    ab_aa = rng.integers(0, 20, 2000).astype(np.uint8)
    g = ctx.compute_forces_with_grid(pkg.ResidueCloud(*ag_xyz.T, ag_aa), 10.0, pkg.ResidueCloud(*ab_xyz.T, ab_aa))
    o = oracle.forces_cg_grid(10.0, ag_xyz, ag_aa, ab_xyz, ab_aa)
    for a, b in zip(g, o):
        assert np.array_equal(a, b)


def test_allatom_forces_vs_f64(ctx, oracle, pkg):
    cfg = pkg.workloads.config1(n_cand=16)
    _, _, ag = _antigen(oracle, pkg, cfg)
    cands, off = _population(oracle, pkg.workloads, cfg)
    f, e = ctx.forces_allatom(ag, cands, off)
    f64, e64 = oracle.forces_allatom64(ag.to_gpu_atoms(), cands, off)
    scale = np.maximum(np.linalg.norm(f64, axis=1), 1e-3 * np.abs(f64).max())
    err = np.linalg.norm(f - f64, axis=1) / scale
    assert err.max() < 1e-4, err.max()


# ---- survivor selection (bit-exact) ----------------------------------------------------------
def test_topk_matches_stable_sort(ctx, oracle):
    rng = np.random.default_rng(2)
    e = rng.normal(size=1024)
    e[100:110] = e[5]          # ties keep index order
    e[7] = np.nan              # NaN last
    e[9] = -0.0
    e[11] = 0.0
    for k in (1, 64, 1024):
        assert np.array_equal(ctx.topk(e, k), oracle.topk(e, k))
    big = rng.integers(-50, 50, size=20000).astype(np.float64)
    assert np.array_equal(ctx.topk(big, 700), oracle.topk(big, 700))


@pytest.mark.parametrize("n", [1, 31, 1024, 5000])
def test_topk_small_k_matches_stable_sort(ctx, oracle, n):
    """k <= 64 (warp sorts + merge tree): ties across warps and chunks, NaNs, -0/+0,
    fewer elements than k."""
    rng = np.random.default_rng(n)
    e = rng.integers(-20, 20, size=n).astype(np.float64)  # many ties
    e[rng.random(n) < 0.05] = np.nan
    if n > 9:
        e[3], e[9] = -0.0, 0.0
    for k in (1, 17, 33, 64):
        exp = oracle.topk(e, min(k, n))
        got = ctx.topk(e, min(k, n))
        assert np.array_equal(got, exp), (n, k)


def test_topk_segmented(ctx, oracle):
    rng = np.random.default_rng(4)
    e = rng.normal(size=3000)
    so = np.array([0, 512, 512, 1500, 3000], np.int64)
    got = ctx.topk_segmented(e, so, 64)
    for s in range(4):
        seg = e[so[s]:so[s + 1]]
        exp = oracle.topk(seg, min(64, len(seg))) + so[s]
        row = got[s]
        assert np.array_equal(row[:len(exp)], exp) and np.all(row[len(exp):] == -1)


# ---- gradient phase (bit-exact trajectories) --------------------------------------------------
def _setup_search(ctx, oracle, pkg, cfg, n_cand):
    ag_aa, ag_pos, _ = _antigen(oracle, pkg, cfg)
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=cfg["shell"][0], seed=1234))
    ctx.add_antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    n_res = int(pop.n_res[0])
    aa = pop.aa[: n_cand * n_res].copy()
    pos, chi = oracle.build_residues(pop.ca[: n_cand * n_res], aa)
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    return oracle.Antigen(ag_aa, ag_pos), aa, chi, pos, n_res


@pytest.mark.parametrize("with_noise", [False, True])
@pytest.mark.parametrize("flat,warps,n_steps", [(0, 8, 10), (8, 8, 10), (16, 4, 25), (32, 4, 10)])
def test_langevin_steps_bit_exact(ctx, oracle, pkg, with_noise, flat, warps, n_steps):
    """Gradient steps in the lane-group form (flat 0) and the flat form with 8, 16,
    32 residues per warp (25 steps: the recorded translations are applied twice
    mid-launch and once at the end)."""
    cfg = pkg.workloads.config1(n_cand=64)
    A, aa, chi, pos, n_res = _setup_search(ctx, oracle, pkg, cfg, 64)
    temps = np.array([oracle.temperature(i, 600) for i in range(n_steps)], np.float32)
    ctx.set_launch_cfg(cg_warps=warps, cg_flat=flat)
    try:
        ctx.diffuse(n_steps, step0=0, with_noise=with_noise, temps=temps)
    finally:
        ctx.set_launch_cfg()
    g_aa, g_chi, g_pos = ctx.state_download()
    prm = oracle.OrcParams.defaults(shell_radius=cfg["shell"][0], seed=1234)
    for s in range(n_steps):
        A.step(prm, aa, chi, pos, n_res, np.arange(64), s, temps[s], with_noise, False)
    assert np.array_equal(g_aa, aa) and np.array_equal(g_pos, pos)


@pytest.mark.parametrize("with_noise", [False, True])
def test_langevin_steps_bit_exact_mixed_antigens(ctx, oracle, pkg, with_noise):
    """Ragged candidates of 8 antigens interleaved, so that the warps of the
    gradient-step kernel hold residues of different antigens: every candidate's
    trajectory equals the oracle's against its own antigen, under the default
    schedule (candidate order, work queue) and the Calpha-cell order on a static grid."""
    cfg = pkg.workloads.config2(n_cand=48)
    pop = cfg["pop"]
    As = []
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=26.0, seed=1234))
    for ag_aa, ag_ca in cfg["antigens"]:
        ag_pos, _ = oracle.build_residues(ag_ca, ag_aa)
        ctx.add_antigen(ag_aa, ag_pos)
        As.append(oracle.Antigen(ag_aa, ag_pos))
    pos0, chi0 = oracle.build_residues(pop.ca, pop.aa)
    off = np.concatenate([[0], np.cumsum(pop.n_res)])
    n_steps = 10
    temps = np.array([oracle.temperature(i, 600) for i in range(n_steps)], np.float32)
    aa, chi, pos = pop.aa.copy(), chi0.copy(), pos0.copy()
    prm = oracle.OrcParams.defaults(shell_radius=26.0, seed=1234)
    for s in range(n_steps):
        for c in range(len(pop.n_res)):
            o0, o1 = off[c], off[c + 1]
            As[pop.antigen_id[c]].step(prm, aa[o0:o1], chi[o0:o1], pos[o0:o1], int(pop.n_res[c]), [c], s,
                                       temps[s], with_noise, False)
    for shape in ((8, 4, 8, 8, 1, 1, 1), (8, 4, 8, 8, 0, 0, 0), (8, 4, 8, 8, 1, 1, 1, 16), (8, 4, 4, 8, 0, 0, 0, 32),
                  (8, 4, 8, 8, 2, 1, 0, 8)):
        ctx.set_launch_cfg(*shape)
        ctx.state_upload(pop.aa, chi0, pos0, n_res=pop.n_res, antigen_id=pop.antigen_id)
        ctx.diffuse(n_steps, step0=0, with_noise=with_noise, temps=temps)
        g_aa, g_chi, g_pos = ctx.state_download()
        assert np.array_equal(g_aa, aa) and np.array_equal(g_pos, pos), shape
    ctx.set_launch_cfg()


def test_block_scores_and_survivors(ctx, oracle, pkg):
    cfg = pkg.workloads.config1(n_cand=256)
    A, aa, chi, pos, n_res = _setup_search(ctx, oracle, pkg, cfg, 256)
    e, top = ctx.block(10, 0, k=64)
    prm = oracle.OrcParams.defaults(shell_radius=cfg["shell"][0], seed=1234)
    for s in range(10):
        A.step(prm, aa, chi, pos, n_res, np.arange(256), s, 3.0, False, False)
    e64 = A.score_slots64(aa, pos, n_res)
    assert np.all(rel_err(e, e64) < 1e-5)
    exp = oracle.topk(e64, 64)
    # identical survivor sets when the 64/65 gap exceeds the error bound
    order = np.argsort(e64, kind="stable")
    gap = e64[order[64]] - e64[order[63]]
    if gap > 1e-5 * abs(e64[order[63]]):
        assert set(top[0].tolist()) == set(exp.tolist())
    assert np.array_equal(np.sort(top[0]), np.sort(oracle.topk(e, 64)))
