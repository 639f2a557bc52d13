"""Learned mutation / rotamer proposal inside the Metropolis kernel, and the
proposal log that trains it, through the C ABI.

  * A network with constant outputs proposes exactly as the uniform proposal:
    the learned path then reproduces the plain trajectory bit for bit.
  * Every mutation / rotamer decision is logged once; logged energy changes of
    mutations match the oracle's residue_contribution_allatom differences
    (diffusion.rs:425-463, the same f32 pair terms summed in double) within 1e-5
    relative (clash-range Calphas make f32 sums too coarse to compare with).
  * With a trained-size random network, the logged Hastings log-ratios match the
    oracle network evaluated at the logged environments (BF16 network: within
    0.05 absolute at proposal temperature 3): a mutation query carries no amino
    acid, so log q(reverse) - log q(move) = (y[new] - y[old]) / Tp.
  * The logged tuples train the network on the GPU (loss falls), and the trained
    network's proposals on a held-out antigen are better than uniform ones: higher
    acceptance and a far lower mean energy change of the proposed mutations."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


def _setup(ctx, pkg, n_cand=48, seed=77):
    cfg = pkg.workloads.config1(n_cand=n_cand)
    ag_aa, ag_ca = cfg["antigens"][0]
    ag_pos, _ = ctx.build_residues(ag_ca, ag_aa)
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=float(cfg["shell"][0]), seed=seed))
    ctx.add_antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    pos, chi = ctx.build_residues(pop.ca, pop.aa)
    # a few gradient steps bring the candidates into contact first
    ctx.state_upload(pop.aa, chi, pos, uniform_n_res=int(pop.n_res[0]))
    ctx.diffuse(30, 0, with_noise=False, with_mc=False)
    aa, chi, pos = ctx.state_download()
    return ag_aa, ag_pos, aa, chi, pos, int(pop.n_res[0])


def _run(ctx, aa, chi, pos, n_res, steps=40, step0=100, temps=None):
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    ctx.diffuse(steps, step0, with_noise=True, with_mc=True, temps=temps)
    return ctx.state_download(), ctx.mc_stats()


def test_constant_network_reproduces_uniform_proposal(ctx, pkg):
    ag_aa, ag_pos, aa, chi, pos, n_res = _setup(ctx, pkg)
    temps = np.array([pkg.temperature(i, 40) for i in range(40)], np.float32)
    ctx.set_proposal(False)
    (a0, c0, p0), s0 = _run(ctx, aa, chi, pos, n_res, temps=temps)
    p = np.zeros(pkg.MLP_N_PARAMS, np.float32)
    p[pkg.MLP_OFF["b1"]:pkg.MLP_OFF["b1"] + pkg.MLP_H] = 0.3  # hidden units active, output weights zero
    ctx.mlp_set_params(p)
    ctx.set_proposal(True, t_prop_min=0.5)
    (a1, c1, p1), s1 = _run(ctx, aa, chi, pos, n_res, temps=temps)
    ctx.set_proposal(False)
    assert s0[:, 0].sum() > 100  # moves were made
    assert np.array_equal(a0, a1) and np.array_equal(c0, c1) and np.array_equal(p0, p1)
    assert np.array_equal(s0, s1)


def test_log_records_every_decision_with_exact_energy_changes(ctx, pkg, oracle):
    ag_aa, ag_pos, aa, chi, pos, n_res = _setup(ctx, pkg, seed=78)
    ctx.set_proposal(False)
    ctx.mc_log(100000)
    _, st = _run(ctx, aa, chi, pos, n_res, steps=30)
    logged, proposed = ctx.mc_log_count()
    tup = ctx.mc_log_fetch()
    ctx.mc_log(0)
    assert proposed == logged == len(tup) == st[:, 0].sum()
    assert tup["accepted"].sum() == st[:, 1].sum()
    assert np.all(tup["log_ratio"] == 0.0)
    assert np.all(tup["action"] < 25) and np.all(tup["aa"] < 20)
    A = oracle.Antigen(ag_aa, ag_pos)
    mut = np.nonzero((tup["action"] < 20) & (tup["aa"] != 4) & (tup["action"] != 4))[0]  # no cysteine involved
    assert len(mut) > 50
    for i in mut[:200]:
        t = tup[i]
        p1 = np.zeros((1, 14, 3), np.float32)
        p1[0, 1] = (t["x"], t["y"], t["z"])
        e_old = A.residue_contribution(np.array([t["aa"]], np.uint8), p1, 0, f64_sum=True)
        e_new = A.residue_contribution(np.array([t["action"]], np.uint8), p1, 0, f64_sum=True)
        ref = np.float32(e_new - e_old)
        assert abs(t["delta_e"] - ref) <= 1e-5 * max(1.0, abs(ref)), (i, t["delta_e"], ref)
    # rotamer moves without cysteine change nothing in the energy
    rot = (tup["action"] >= 20) & (tup["aa"] != 4)
    assert np.all(tup["delta_e"][rot] == 0.0)


def test_learned_hastings_ratios_match_oracle_network(ctx, pkg):
    ag_aa, ag_pos, aa, chi, pos, n_res = _setup(ctx, pkg, seed=79)
    p = pkg.mlp_init_params(5)
    p[pkg.MLP_OFF["b3"]:pkg.MLP_OFF["b3"] + 20] = np.linspace(-1, 1, 20)
    ctx.mlp_set_params(p)
    ctx.set_proposal(True, t_prop_min=3.0)  # constant temperature T_HOT = 3: Tp = 3
    ctx.mc_log(100000)
    (a1, c1, p1), st = _run(ctx, aa, chi, pos, n_res, steps=20)
    tup = ctx.mc_log_fetch()
    ctx.mc_log(0)
    ctx.set_proposal(False)
    assert len(tup) == st[:, 0].sum() > 100
    mut = tup[tup["action"] < 20]
    assert len(mut) > 50
    ag_ca = ag_pos[:, 1, :]
    ca = np.stack([mut["x"], mut["y"], mut["z"]], 1)
    yf, _ = mo.forward(p, mo.features(ag_ca, ag_aa, ca, np.full(len(mut), mo.NO_AA)), bf16_path=True)
    tp = 3.0

    def logq(y, k):
        lg = -y[:, :20] / tp
        m = lg.max(1, keepdims=True)
        return lg[np.arange(len(y)), k] - (m[:, 0] + np.log(np.exp(lg - m).sum(1)))

    ref = logq(yf, mut["aa"].astype(int)) - logq(yf, mut["action"].astype(int))
    assert np.abs(mut["log_ratio"] - ref).max() < 0.05
    assert np.abs(ref).max() > 0.05  # the network is not flat
    # the network's proposals favour low predicted energy changes
    pred = yf[np.arange(len(mut)), mut["action"].astype(int)]
    assert pred.mean() < yf[:, :20].mean()


def test_learned_hastings_ratios_with_two_tiles_per_step(ctx, pkg):
    """More than 8 moves in a candidate-step: the network runs on a second 8-row
    tile in the same step; every logged ratio still matches the oracle network."""
    ag_aa, ag_pos, aa, chi, pos, n_res = _setup(ctx, pkg, n_cand=32, seed=81)
    p = pkg.mlp_init_params(6)
    p[pkg.MLP_OFF["b3"]:pkg.MLP_OFF["b3"] + 20] = np.linspace(-1, 1, 20)
    ctx.mlp_set_params(p)
    prm = ctx.params
    prm.mutation_p = 0.45  # x3 at the interface, x0.4 elsewhere: about 8-12 moves per step
    ctx.set_params(prm)
    ctx.set_proposal(True, t_prop_min=3.0)
    ctx.mc_log(100000)
    (a1, c1, p1), st = _run(ctx, aa, chi, pos, n_res, steps=8)
    tup = ctx.mc_log_fetch()
    ctx.mc_log(0)
    ctx.set_proposal(False)
    assert len(tup) == st[:, 0].sum()
    # some candidate averaged more than 8 moves per step: it had steps of two tiles
    assert st[:, 0].max() > 8 * 8 and st[:, 0].sum() > 32 * 8 * 4
    mut = tup[tup["action"] < 20]
    ca = np.stack([mut["x"], mut["y"], mut["z"]], 1)
    yf, _ = mo.forward(p, mo.features(ag_pos[:, 1, :], ag_aa, ca, np.full(len(mut), mo.NO_AA)), bf16_path=True)
    lg = -yf[:, :20] / 3.0
    ref = lg[np.arange(len(mut)), mut["aa"].astype(int)] - lg[np.arange(len(mut)), mut["action"].astype(int)]
    assert np.abs(mut["log_ratio"] - ref).max() < 0.05
    rot = tup[(tup["action"] >= 20) & (tup["log_ratio"] != 0.0)]
    assert len(rot) > 20  # rotamer moves from library rotamers are learned too


def test_logged_tuples_train_the_network(ctx, pkg):
    ag_aa, ag_pos, aa, chi, pos, n_res = _setup(ctx, pkg, n_cand=128, seed=80)
    ctx.set_proposal(False)
    ctx.mc_log(200000)
    _run(ctx, aa, chi, pos, n_res, steps=60)
    n = ctx.mlp_take_log()
    ctx.mc_log(0)
    assert n > 2000
    ctx.mlp_set_params(pkg.mlp_init_params(1))
    losses = ctx.mlp_train(300, batch=1024, lr=1e-3, huber_delta=1.0, seed=9)
    assert np.all(np.isfinite(losses))
    assert losses[-30:].mean() < 0.5 * losses[:5].mean(), (losses[:5], losses[-30:])


def test_trained_network_beats_uniform_proposals_on_held_out_antigen(ctx, pkg):
    L = pkg.learned
    cfg = pkg.workloads.config4(n_train=2, n_eval=1, n_cand=256)
    shell = float(cfg["train"][0][1])
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=shell, seed=5))
    ids = L.add_antigens(ctx, [t[0] for t in cfg["train"]])
    (eval_id,) = L.add_antigens(ctx, [cfg["eval"][0][0]])
    n = L.generate_tuples(ctx, [t[2] for t in cfg["train"]], ids, 20, gen_steps=200)
    assert n > 50000
    losses, _ = L.train(ctx, 400, batch=4096, lr=1e-3)
    assert losses[-20:].mean() < 0.2 * losses[:5].mean()
    agid = L.upload_populations(ctx, [cfg["eval"][0][2]], [eval_id], 20)
    ctx.diffuse(100, 0)
    s0 = ctx.state_download()
    stats = {}
    for learned in (False, True):
        ctx.mc_log(1_000_000)
        _, st = L.anneal_champions(ctx, s0, agid, 20, n_steps=200, chunk=50, learned=learned, t_prop_min=1.0)
        tup = ctx.mc_log_fetch()
        ctx.mc_log(0)
        mut = tup[tup["action"] < 20]
        stats[learned] = (st["mutation_rotamer_acceptance"], float(mut["delta_e"].mean()))
    (acc_u, de_u), (acc_l, de_l) = stats[False], stats[True]
    assert acc_l > acc_u + 0.05, stats
    assert de_l < de_u - 0.5, stats
