"""The learned proposal network: oracle self-checks on CPU, GPU kernels (features,
tcgen05 forward and backward GEMMs, Adam training) against the oracle.

Tolerances: features bit-exact.  Forward outputs: the GPU sums BF16 products in
FP32 and rounds hidden activations to BF16 from its own FP32 pre-activations, the
oracle sums the same BF16 operands exactly; a hidden activation whose FP32 and
exact pre-activations round to different BF16 values moves an output by about one
BF16 ulp of that activation times its weight, so outputs agree within 2e-2 of the
output scale.  Gradients: norm-wise within 3e-2 relative per parameter block.  The
oracle's own float64 gradient matches central differences within 1e-6."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle as mo  # noqa: E402

BLOCKS = [("w1", "b1"), ("b1", "w2"), ("w2", "b2"), ("b2", "w3"), ("w3", "b3"), ("b3", None)]


def _block(g, a, b):
    return g[mo.OFF[a]:(mo.OFF[b] if b else mo.N_PARAMS)]


def _random_features(rng, n):
    f = np.zeros((n, mo.MLP_IN), np.float32)
    f[np.arange(n), rng.integers(0, 20, n)] = 1.0
    counts = rng.poisson(0.6, size=(n, 160))
    f[:, 20:] = mo.LOG1P[counts]
    return mo.bf16(f)


def _params(pkg, seed=0, scale=1.0):
    p = pkg.mlp_init_params(seed)
    rng = np.random.default_rng(seed + 99)
    nz = np.zeros(mo.N_PARAMS, bool)
    for name in ("b1", "b2"):
        nz[mo.OFF[name]:mo.OFF[name] + mo.MLP_H] = True
    p[nz] = rng.uniform(-0.1, 0.1, nz.sum()).astype(np.float32)
    p[mo.OFF["b3"]:mo.OFF["b3"] + 25] = rng.uniform(-0.1, 0.1, 25).astype(np.float32)
    return (p * scale).astype(np.float32)


# ---- oracle self-checks (CPU) ------------------------------------------------------
@pytest.mark.parametrize("with_ref", [False, True])
def test_oracle_gradient_matches_finite_differences(pkg, with_ref):
    rng = np.random.default_rng(1)
    X = rng.normal(size=(12, mo.MLP_IN))
    a = rng.integers(0, 25, 12)
    t = rng.normal(scale=2.0, size=12)
    # reference outputs: mutation rows (y[action] - y[ref]), rotamer rows (-1), a no-op row
    ref = np.where(a < 20, rng.integers(0, 20, 12), -1) if with_ref else None
    if with_ref:
        ref[0], a[0] = 3, 3
    p = _params(pkg, 3).astype(np.float64)
    _, g = mo.loss_grad(p, X, a, t, delta=1.0, bf16_path=False, ref=ref)
    idx = np.concatenate([rng.integers(mo.OFF[a_], mo.OFF[b_] if b_ else mo.OFF["b3"] + 25, 8) for a_, b_ in BLOCKS])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_grad(pp, X, a, t, 1.0, False, ref)[0] - mo.loss_grad(pm, X, a, t, 1.0, False, ref)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_oracle_counts_match_distance_definition():
    rng = np.random.default_rng(2)
    ag = rng.uniform(-12, 12, size=(300, 3)).astype(np.float32)
    ag_aa = rng.integers(0, 20, 300)
    ca = rng.uniform(-14, 14, size=(40, 3)).astype(np.float32)
    cnt = mo.env_counts(ag, ag_aa, ca)
    for r in range(len(ca)):
        d = np.linalg.norm(ag.astype(np.float64) - ca[r], axis=1)
        ok = np.abs(d[:, None] - 1.25 * np.arange(1, 9)[None, :]).min(1) > 1e-4  # away from shell edges
        ref = np.zeros((8, 20), np.int64)
        for i in np.nonzero((d < 10) & ok)[0]:
            ref[int(d[i] // 1.25), ag_aa[i]] += 1
        amb = np.zeros((8, 20), bool)
        for i in np.nonzero(~ok)[0]:
            amb[:, ag_aa[i]] = True
        assert np.array_equal(cnt[r][~amb], ref[~amb])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125 + 2**-10, -3.14159, 0.0], np.float32)
    y = mo.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0 and y[2] == 1.0078125 and y[3] == 1.0078125
    assert abs(y[4] + 3.140625) < 1e-6 and y[5] == 0.0


# ---- GPU -----------------------------------------------------------------------------
def _antigen(ctx, pkg):
    cfg = pkg.workloads.config1(n_cand=16)
    ag_aa, ag_ca = cfg["antigens"][0]
    ag_pos, _ = ctx.build_residues(ag_ca, ag_aa)
    ctx.clear_antigens()
    ctx.add_antigen(ag_aa, ag_pos)
    return ag_aa, ag_pos[:, 1, :].copy()


@pytest.mark.gpu
def test_features_bit_exact(ctx, pkg):
    ag_aa, ag_ca = _antigen(ctx, pkg)
    rng = np.random.default_rng(5)
    anchor = ag_ca[rng.integers(0, len(ag_ca), 500)]
    d = rng.normal(size=(500, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ca = (anchor + d * rng.uniform(0.0, 14.0, (500, 1))).astype(np.float32)
    # points exactly on shell radii from an antigen Calpha
    ca[:8] = (ag_ca[0] + np.array([[1.25 * k, 0, 0] for k in range(1, 9)])).astype(np.float32)
    aa = rng.integers(0, 20, 500).astype(np.uint8)
    aa[::3] = pkg.MLP_NO_AA  # mutation queries: no one-hot
    got = ctx.mlp_features(0, ca, aa)
    ref = mo.features(ag_ca, ag_aa, ca, aa)
    assert got.dtype == np.float32 and got.shape == (500, 180)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert not got[::3, :20].any() and np.all(got[1::3, :20].sum(1) == 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 300])
def test_forward_matches_oracle(ctx, pkg, n):
    rng = np.random.default_rng(n)
    p = _params(pkg, 7)
    ctx.mlp_set_params(p)
    X = _random_features(rng, n)
    got = ctx.mlp_forward(X)
    ref, _ = mo.forward(p, X, bf16_path=True)
    scale = max(1.0, float(np.abs(ref).max()))
    assert np.abs(got - ref).max() <= 2e-2 * scale
    # the same rows in a larger batch give the same outputs (row independence)
    if n < 300:
        big = np.concatenate([X, _random_features(rng, 300)])
        assert np.array_equal(ctx.mlp_forward(big)[:n], got)


@pytest.mark.gpu
@pytest.mark.parametrize("n,with_ref", [(128, False), (1000, False), (1000, True)])
def test_loss_grad_matches_oracle(ctx, pkg, n, with_ref):
    rng = np.random.default_rng(11 + n)
    p = _params(pkg, 8)
    ctx.mlp_set_params(p)
    X = _random_features(rng, n)
    a = rng.integers(0, 25, n).astype(np.int32)
    t = rng.normal(scale=1.5, size=n).astype(np.float32)
    ref = None
    if with_ref:  # mutation rows against the amino acid before the move, some of them no-ops
        ref = np.where(a < 20, rng.integers(0, 20, n), -1).astype(np.int32)
        ref[:10] = a[:10] = 7
    loss, g = ctx.mlp_loss_grad(X, a, t, 1.0, ref=ref)
    rloss, rg = mo.loss_grad(p, X, a, t, 1.0, bf16_path=True, ref=ref)
    assert abs(loss - rloss) <= 1e-3 * max(1.0, abs(rloss))
    for a_, b_ in BLOCKS:
        gg, rr = _block(g, a_, b_).astype(np.float64), _block(rg, a_, b_)
        assert np.linalg.norm(gg - rr) <= 3e-2 * np.linalg.norm(rr) + 1e-7, (a_, np.linalg.norm(gg - rr),
                                                                             np.linalg.norm(rr))
    # padding stays exactly zero
    W1 = _block(g, "w1", "b1").reshape(mo.MLP_H, 192)
    assert not W1[:, 180:].any()
    assert not _block(g, "w3", "b3").reshape(32, mo.MLP_H)[25:].any()
    assert not g[mo.OFF["b3"] + 25:].any()
    assert np.array_equal(ctx.mlp_get_params(), p)  # no update


@pytest.mark.gpu
def test_training_fits_a_learnable_target(ctx, pkg):
    """Tuples whose energy change is a fixed function of the environment (a mutation
    old -> new: f_new(env) - f_old(env), as the network's mutation queries model it):
    Adam on the GPU drives the loss down by an order of magnitude."""
    ag_aa, ag_ca = _antigen(ctx, pkg)
    rng = np.random.default_rng(21)
    n = 20000
    anchor = ag_ca[rng.integers(0, len(ag_ca), n)]
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ca = (anchor + d * rng.uniform(3.0, 9.0, (n, 1))).astype(np.float32)
    aa = rng.integers(0, 20, n).astype(np.uint8)
    act = rng.integers(0, 20, n).astype(np.uint8)
    feats = mo.features(ag_ca, ag_aa, ca, aa)
    w = np.random.default_rng(3).normal(size=(160, 20)) * 0.3
    f_env = feats[:, 20:] @ w
    target = (f_env[np.arange(n), act] - f_env[np.arange(n), aa]) * 0.5
    tup = np.zeros(n, pkg.MC_TUPLE)
    tup["x"], tup["y"], tup["z"] = ca[:, 0], ca[:, 1], ca[:, 2]
    tup["delta_e"] = target.astype(np.float32)
    tup["aa"], tup["action"] = aa, act
    ctx.mlp_set_params(pkg.mlp_init_params(0))
    ctx.mlp_set_tuples(tup)
    back = ctx.mlp_get_tuples()
    assert np.array_equal(back["delta_e"], tup["delta_e"]) and np.array_equal(back["action"], act)
    losses = ctx.mlp_train(400, batch=2048, lr=2e-3, huber_delta=1.0, seed=4)
    assert np.all(np.isfinite(losses))
    assert losses[-20:].mean() < 0.1 * losses[:5].mean(), (losses[:5], losses[-20:])
    p = ctx.mlp_get_params()
    assert not p.reshape(-1)[mo.OFF["w1"]:mo.OFF["b1"]].reshape(mo.MLP_H, 192)[:, 180:].any()
