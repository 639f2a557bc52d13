"""Langevin + Metropolis steps (diffusion.rs:290-463) and run_allatom on the GPU
vs the CPU oracle, through the C ABI.

Tolerances: trajectories (amino acids, chi angles, every atom position) and the
move counts are compared bit for bit, in both accumulation modes: BINDER_ACC_F32
(the reference's f32 sums; the energies themselves are then bit-identical) and
the default (f32 pair terms summed in double; the oracle sums in a different
order, so energies differ in the last bits of a double and a decision could only
flip when u lands within ~1e-15 of exp(-dE/T)).  Final energies within 1e-5
relative of the f64 oracle."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

HOT = [0, 1, 2, 3, 4, 5]
COLD = [560, 561, 562, 563, 564, 565]


def _params(pkg, oracle, shell, acc, flags=None, **kw):
    g = pkg.Params.defaults(shell_radius=shell, seed=1234, accumulate=acc, **kw)
    if flags is not None:
        g.flags = flags
    o = oracle.OrcParams.defaults(shell_radius=shell, seed=1234, accumulate=acc, **kw)
    return g, o


def _antigen(oracle, cfg, i=0):
    aa, ca = cfg["antigens"][i]
    pos, _ = oracle.build_residues(ca, aa)
    return aa, pos


def _run_pair(ctx, oracle, A, gp, op, aa, chi, pos, n_res, cand_id, steps, temps, noise=True):
    """GPU and oracle over the same steps; returns the GPU state and stats, the
    oracle state (in place) and stats."""
    n_cand = len(aa) // n_res
    ctx.set_params(gp)
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res, cand_id=cand_id)
    ctx.diffuse(len(steps), step0=steps[0], with_noise=noise, with_mc=True, temps=temps)
    g = ctx.state_download()
    g_stats = ctx.mc_stats()
    o_stats = np.zeros((n_cand, 4), np.int64)
    for j, s in enumerate(steps):
        A.step(op, aa, chi, pos, n_res, cand_id, s, temps[j], noise, True, stats=o_stats)
    return g, g_stats, o_stats


@pytest.mark.parametrize("acc", [0, 1])
@pytest.mark.parametrize("sched", ["hot", "cold"])
def test_mc_steps_bit_exact(ctx, oracle, pkg, acc, sched):
    cfg = pkg.workloads.config1(n_cand=64)
    ag_aa, ag_pos = _antigen(oracle, cfg)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, cfg["shell"][0], acc, mutation_p=0.3, rotamer_move_p=0.5, backbone_move_p=0.2)
    ctx.set_params(gp)
    ctx.add_antigen(ag_aa, ag_pos)
    A = oracle.Antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    n_res = 20
    aa = pop.aa[:64 * n_res].copy()
    pos, chi = oracle.build_residues(pop.ca[:64 * n_res], aa)
    steps = HOT if sched == "hot" else COLD
    temps = np.array([oracle.temperature(s, 600) for s in steps], np.float32)
    cid = np.arange(64, dtype=np.uint32) * 7 + 3
    (g_aa, g_chi, g_pos), g_stats, o_stats = _run_pair(ctx, oracle, A, gp, op, aa, chi, pos, n_res, cid, steps,
                                                       temps)
    assert o_stats[:, 0].sum() > 1000 and o_stats[:, 2].sum() > 500
    assert (o_stats[:, 1] < o_stats[:, 0]).any() and (o_stats[:, 3] < o_stats[:, 2]).any()
    assert np.array_equal(g_stats, o_stats)
    assert np.array_equal(g_aa, aa)
    assert np.array_equal(g_chi, chi)
    assert np.array_equal(g_pos, pos)


@pytest.mark.parametrize("acc", [0, 1])
@pytest.mark.parametrize("sched", ["hot", "cold"])
def test_mc_long_candidates_bit_exact(ctx, oracle, pkg, acc, sched):
    """40-residue candidates: more residues than one Langevin pass holds, so the
    Langevin force walks the 27 neighbouring Calpha cells every step instead of
    reading Verlet lists from shared memory."""
    cfg = pkg.workloads.config1(n_cand=64)
    ag_aa, ag_pos = _antigen(oracle, cfg)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, cfg["shell"][0], acc, mutation_p=0.3, rotamer_move_p=0.5, backbone_move_p=0.2)
    ctx.set_params(gp)
    ctx.add_antigen(ag_aa, ag_pos)
    A = oracle.Antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    n_res, n_cand = 40, 32
    aa = pop.aa[:n_cand * n_res].copy()
    pos, chi = oracle.build_residues(pop.ca[:n_cand * n_res], aa)
    steps = HOT if sched == "hot" else COLD
    temps = np.array([oracle.temperature(s, 600) for s in steps], np.float32)
    cid = np.arange(n_cand, dtype=np.uint32) * 5 + 1
    (g_aa, g_chi, g_pos), g_stats, o_stats = _run_pair(ctx, oracle, A, gp, op, aa, chi, pos, n_res, cid, steps,
                                                       temps)
    assert o_stats[:, 0].sum() > 2000 and o_stats[:, 2].sum() > 1000
    assert (o_stats[:, 3] < o_stats[:, 2]).any()
    assert np.array_equal(g_stats, o_stats)
    assert np.array_equal(g_aa, aa)
    assert np.array_equal(g_chi, chi)
    assert np.array_equal(g_pos, pos)


@pytest.mark.parametrize("acc", [0, 1])
def test_mc_odd_antigen_bit_exact(ctx, oracle, pkg, acc):
    """An antigen of 299 residues: the Calpha-energy scan tests two antigen Calphas
    per lane and step, so an odd count leaves a padded entry in the last step."""
    cfg = pkg.workloads.config1(n_cand=64)
    ag_aa, ag_ca = cfg["antigens"][0]
    ag_aa, ag_ca = ag_aa[:299].copy(), ag_ca[:299].copy()
    ag_pos, _ = oracle.build_residues(ag_ca, ag_aa)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, cfg["shell"][0], acc, mutation_p=0.3, rotamer_move_p=0.5, backbone_move_p=0.2)
    ctx.set_params(gp)
    ctx.add_antigen(ag_aa, ag_pos)
    A = oracle.Antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    n_res, n_cand = 20, 32
    aa = pop.aa[:n_cand * n_res].copy()
    pos, chi = oracle.build_residues(pop.ca[:n_cand * n_res], aa)
    temps = np.array([oracle.temperature(s, 600) for s in COLD], np.float32)
    cid = np.arange(n_cand, dtype=np.uint32) * 3 + 2
    (g_aa, g_chi, g_pos), g_stats, o_stats = _run_pair(ctx, oracle, A, gp, op, aa, chi, pos, n_res, cid, COLD,
                                                       temps)
    assert o_stats[:, 0].sum() > 500
    assert np.array_equal(g_stats, o_stats)
    assert np.array_equal(g_aa, aa) and np.array_equal(g_chi, chi) and np.array_equal(g_pos, pos)


_LARGE = {}


def _large_antigen(W):
    """A seeded 1101-residue globule (built once: the self-avoiding walk takes seconds)."""
    if not _LARGE:
        rng = W.rng_for(7)
        _LARGE["ag"] = W._globule_antigen(1101, rng)
        _LARGE["rng_state"] = rng.bit_generator.state
    rng = np.random.default_rng()
    rng.bit_generator.state = _LARGE["rng_state"]
    return _LARGE["ag"], rng


@pytest.mark.parametrize("acc", [0, 1])
def test_mc_large_antigen_bit_exact(ctx, oracle, pkg, acc):
    """An antigen of 1101 residues, more than the Metropolis kernel stages in shared
    memory: its Calphas, CG grid and parameters are read from global memory."""
    W = pkg.workloads
    (ag_aa, ag_ca, radius), rng = _large_antigen(W)
    ag_pos, _ = oracle.build_residues(ag_ca, ag_aa)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, radius + 4.0, acc, mutation_p=0.3, rotamer_move_p=0.5, backbone_move_p=0.2)
    ctx.set_params(gp)
    ctx.add_antigen(ag_aa, ag_pos)
    A = oracle.Antigen(ag_aa, ag_pos)
    n_res, n_cand = 20, 16
    ca = W.sphere_points(n_cand * n_res, radius + 4.0, W.ca_center(ag_ca), rng)
    aa = W.random_sequence(n_cand * n_res, rng)
    pos, chi = oracle.build_residues(ca, aa)
    temps = np.array([oracle.temperature(s, 600) for s in HOT], np.float32)
    cid = np.arange(n_cand, dtype=np.uint32) * 11 + 5
    (g_aa, g_chi, g_pos), g_stats, o_stats = _run_pair(ctx, oracle, A, gp, op, aa, chi, pos, n_res, cid, HOT,
                                                       temps)
    assert o_stats[:, 0].sum() > 100
    assert np.array_equal(g_stats, o_stats)
    assert np.array_equal(g_aa, aa) and np.array_equal(g_chi, chi) and np.array_equal(g_pos, pos)


def _ball(rng, n, r_lo, r_hi):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (v * (r_lo + (r_hi - r_lo) * rng.random((n, 1)))).astype(np.float32)


@pytest.mark.parametrize("acc", [0, 1])
def test_mc_dense_antigen_bit_exact(ctx, oracle, pkg, acc):
    """120 antigen Calphas packed into a 9 A ball, candidates around it: up to ~90
    antigen Calphas within the cutoff of one residue, more than the Calpha-energy
    stage holds, so the scan computes and adds its staged terms mid-way."""
    W = pkg.workloads
    rng = np.random.default_rng(123)
    ag_ca = _ball(rng, 120, 0.0, 9.0)
    ag_aa = W.random_sequence(120, rng)
    ag_pos, _ = oracle.build_residues(ag_ca, ag_aa)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, 10.0, acc, mutation_p=0.3, rotamer_move_p=0.5, backbone_move_p=0.2)
    ctx.set_params(gp)
    ctx.add_antigen(ag_aa, ag_pos)
    A = oracle.Antigen(ag_aa, ag_pos)
    n_res, n_cand = 8, 16
    ca = _ball(rng, n_cand * n_res, 4.0, 12.0)
    aa = W.random_sequence(n_cand * n_res, rng)
    pos, chi = oracle.build_residues(ca, aa)
    d2 = ((ca[:, None, :] - ag_ca[None, :, :]) ** 2).sum(-1)
    assert (d2 <= 100.0).sum(1).max() > 64
    temps = np.array([oracle.temperature(s, 600) for s in HOT], np.float32)
    cid = np.arange(n_cand, dtype=np.uint32)
    (g_aa, g_chi, g_pos), g_stats, o_stats = _run_pair(ctx, oracle, A, gp, op, aa, chi, pos, n_res, cid, HOT,
                                                       temps)
    assert o_stats[:, 0].sum() > 300
    assert np.array_equal(g_stats, o_stats)
    assert np.array_equal(g_aa, aa) and np.array_equal(g_chi, chi) and np.array_equal(g_pos, pos)


def _cys_chains(oracle, center, n_cand, n_res, rng):
    """Straight Calpha chains (3.8 A steps) half made of Cys: every residue of the
    ideal backbone has the same orientation, so neighbouring SG atoms sit 3.8 A
    apart and the disulfide term is active from the start."""
    cas, aas = [], []
    for _ in range(n_cand):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        start = center + 9.0 * d
        cas.append(start + np.outer(np.arange(n_res) * 3.8, u))
        aa = rng.integers(0, 20, size=n_res)
        aa[rng.random(n_res) < 0.5] = 4  # CYS
        aas.append(aa)
    aa = np.concatenate(aas).astype(np.uint8)
    pos, chi = oracle.build_residues(np.concatenate(cas).astype(np.float32), aa)
    return aa, chi, pos


@pytest.mark.parametrize("acc", [0, 1])
def test_mc_cys_chains_bit_exact(ctx, oracle, pkg, acc):
    cfg = pkg.workloads.config0()
    ag_aa, ag_pos = _antigen(oracle, cfg)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, 12.0, acc, mutation_p=0.4, rotamer_move_p=0.6, backbone_move_p=0.25)
    ctx.set_params(gp)
    ctx.add_antigen(ag_aa, ag_pos)
    A = oracle.Antigen(ag_aa, ag_pos)
    rng = np.random.default_rng(7)
    n_cand, n_res = 48, 12
    aa, chi, pos = _cys_chains(oracle, A.center(), n_cand, n_res, rng)
    assert oracle.disulfide(aa[:n_res], pos[:n_res]) < 0.0
    steps = list(range(100, 108))
    temps = np.array([oracle.temperature(s, 200) for s in steps], np.float32)
    cid = np.arange(n_cand, dtype=np.uint32)
    (g_aa, g_chi, g_pos), g_stats, o_stats = _run_pair(ctx, oracle, A, gp, op, aa, chi, pos, n_res, cid, steps,
                                                       temps)
    assert np.array_equal(g_stats, o_stats)
    assert np.array_equal(g_aa, aa) and np.array_equal(g_chi, chi) and np.array_equal(g_pos, pos)


def test_mc_default_rates_long(ctx, oracle, pkg):
    """config0 sizes, the reference's move rates, 40 annealed steps in one launch."""
    cfg = pkg.workloads.config0()
    ag_aa, ag_pos = _antigen(oracle, cfg)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, cfg["shell"][0], 0)
    ctx.set_params(gp)
    ctx.add_antigen(ag_aa, ag_pos)
    A = oracle.Antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    n_res = 12
    aa = pop.aa.copy()
    pos, chi = oracle.build_residues(pop.ca, aa)
    steps = list(range(40))
    temps = np.array([oracle.temperature(s, 40) for s in steps], np.float32)
    cid = np.arange(64, dtype=np.uint32)
    (g_aa, g_chi, g_pos), g_stats, o_stats = _run_pair(ctx, oracle, A, gp, op, aa, chi, pos, n_res, cid, steps,
                                                       temps)
    assert np.array_equal(g_stats, o_stats)
    assert np.array_equal(g_aa, aa) and np.array_equal(g_chi, chi) and np.array_equal(g_pos, pos)


def test_mc_ragged_multi_antigen(ctx, oracle, pkg):
    """Uneven antibody lengths over several antigens in one launch."""
    cfg = pkg.workloads.config2(n_cand=48)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, 20.0, 0, mutation_p=0.3, backbone_move_p=0.15)
    ctx.set_params(gp)
    ants = []
    for i in range(len(cfg["antigens"])):
        a_aa, a_pos = _antigen(oracle, cfg, i)
        ctx.add_antigen(a_aa, a_pos)
        ants.append(oracle.Antigen(a_aa, a_pos))
    pop = cfg["pop"]
    aa = pop.aa.copy()
    pos, chi = oracle.build_residues(pop.ca, aa)
    steps = [10, 11, 12, 13]
    temps = np.array([oracle.temperature(s, 50) for s in steps], np.float32)
    ctx.state_upload(aa, chi, pos, n_res=pop.n_res, antigen_id=pop.antigen_id)
    ctx.diffuse(len(steps), step0=steps[0], with_noise=True, with_mc=True, temps=temps)
    g_aa, g_chi, g_pos = ctx.state_download()
    g_stats = ctx.mc_stats()
    off = np.concatenate([[0], np.cumsum(pop.n_res)])
    o_stats = np.zeros((len(pop.n_res), 4), np.int64)
    for c in range(len(pop.n_res)):
        sl = slice(off[c], off[c + 1])
        a, ch, p = aa[sl].copy(), chi[sl].copy(), pos[sl].copy()
        st = np.zeros((1, 4), np.int64)
        for j, s in enumerate(steps):
            ants[pop.antigen_id[c]].step(op, a, ch, p, int(pop.n_res[c]), [c], s, temps[j], True, True, stats=st)
        aa[sl], chi[sl], pos[sl] = a, ch, p
        o_stats[c] = st[0]
    assert np.array_equal(g_stats, o_stats)
    assert np.array_equal(g_aa, aa) and np.array_equal(g_chi, chi) and np.array_equal(g_pos, pos)


def test_state_select(ctx, oracle, pkg):
    cfg = pkg.workloads.config2(n_cand=24)
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=20.0, seed=9))
    for i in range(len(cfg["antigens"])):
        a_aa, a_pos = _antigen(oracle, cfg, i)
        ctx.add_antigen(a_aa, a_pos)
    pop = cfg["pop"]
    aa = pop.aa.copy()
    pos, chi = oracle.build_residues(pop.ca, aa)
    ctx.state_upload(aa, chi, pos, n_res=pop.n_res, antigen_id=pop.antigen_id)
    ctx.diffuse(3, step0=0, with_noise=True, with_mc=True)
    s_aa, s_chi, s_pos = ctx.state_download()
    stats = ctx.mc_stats()
    sel = np.array([5, 2, 2, 17, 0], np.int32)
    ctx.state_select(sel)
    n, total, orig = ctx.state_info()
    off = np.concatenate([[0], np.cumsum(pop.n_res)])
    idx = np.concatenate([np.arange(off[c], off[c + 1]) for c in sel])
    assert n == len(sel) and total == len(idx) and np.array_equal(orig, sel)
    g_aa, g_chi, g_pos = ctx.state_download()
    assert np.array_equal(g_aa, s_aa[idx]) and np.array_equal(g_chi, s_chi[idx]) and np.array_equal(g_pos, s_pos[idx])
    assert np.array_equal(ctx.mc_stats(), stats[sel])
    # scoring the selection = scoring those candidates
    e_sel = ctx.score_state()
    ctx.state_upload(s_aa, s_chi, s_pos, n_res=pop.n_res, antigen_id=pop.antigen_id)
    e_all = ctx.score_state()
    assert np.array_equal(e_sel, e_all[sel])


@pytest.mark.parametrize("flags", [1, 0])
def test_run_allatom_small(ctx, oracle, pkg, flags):
    """run_allatom on config0 sizes with a short schedule vs the oracle pipeline;
    phase 1 replayed from the search block's CUDA graph (flags 1) or issued
    launch by launch (0)."""
    cfg = pkg.workloads.config0()
    ag_aa, ag_pos = _antigen(oracle, cfg)
    ctx.clear_antigens()
    gp, op = _params(pkg, oracle, cfg["shell"][0], 0, flags=flags)
    ctx.set_params(gp)
    ctx.add_antigen(ag_aa, ag_pos)
    A = oracle.Antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    n_res, n_cand = 12, 64
    aa = pop.aa.copy()
    pos, chi = oracle.build_residues(pop.ca, aa)
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    n1, n2, surv, top_n = 20, 12, 16, 5
    rc = pkg.RunCfg.defaults(phase1_steps=n1, score_every=10, survivors=surv, phase2_steps=n2, top_n=top_n)
    g_cand, g_e = ctx.run_allatom(rc)
    g_aa, g_chi, g_pos = ctx.state_download()
    # oracle: phase 1 gradient steps, score, stable top-k
    cid = np.arange(n_cand, dtype=np.uint32)
    for s in range(n1):
        A.step(op, aa, chi, pos, n_res, cid, s, oracle.temperature(s, n1 + n2), False, False)
    e1 = A.score_slots64(aa, pos, n_res)
    order = np.argsort(e1, kind="stable")
    assert e1[order[surv]] - e1[order[surv - 1]] > 1e-5 * abs(e1[order[surv - 1]])
    keep = oracle.topk(e1, surv)
    rs = (keep[:, None] * n_res + np.arange(n_res)).ravel()
    aa2, chi2, pos2 = aa[rs].copy(), chi[rs].copy(), pos[rs].copy()
    for i in range(n2):
        A.step(op, aa2, chi2, pos2, n_res, keep.astype(np.uint32), n1 + i, oracle.temperature(i, n2), True, True)
    e2 = A.score_slots64(aa2, pos2, n_res, full=True)
    rank = oracle.topk(e2, top_n)
    o2 = np.argsort(e2, kind="stable")
    if e2[o2[top_n]] - e2[o2[top_n - 1]] > 1e-5 * abs(e2[o2[top_n - 1]]):
        assert np.array_equal(g_cand[0], keep[rank])
    assert np.all(rel_err(g_e[0], e2[rank]) < 1e-5)
    rs2 = (rank[:, None] * n_res + np.arange(n_res)).ravel()
    assert np.array_equal(g_aa, aa2[rs2]) and np.array_equal(g_chi, chi2[rs2]) and np.array_equal(g_pos, pos2[rs2])
