"""CPU oracle of the learned proposal network (test infrastructure only).

The network has no counterpart in the reference (the reference proposes mutations
and rotamers uniformly, diffusion.rs:354-399); this restatement is the checker of
the GPU kernels in de-novo-antigen-binder_b200/csrc/k_mlp.cu:

  * features(): the 180 environment features of a residue, bit for bit (f32
    squared distances with the reference's rounding, exact shell radii squared,
    log1p table rounded once to f32, BF16 round-to-nearest-even); a mutation
    query (amino acid NO_AA) carries no one-hot;
  * loss_grad(ref=...): mutation rows predict y[new] - y[old];
  * forward() / loss_grad(): the MLP 180 -> 256 -> 256 -> 25 with SiLU in float64.
    With bf16=True the BF16 roundings of the GPU path are applied (weights, input
    rows, hidden activations, output and hidden gradients) and only the sums are
    exact, so the GPU's FP32 sums are compared against exact sums of the same
    BF16 operands (the SiLU' factors the forward pass keeps are BF16 too); with
    bf16=False it is the plain float64 network whose analytic gradient is checked
    against central finite differences.

Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

MLP_IN, MLP_K1, MLP_H, MLP_OUT, MLP_OUT_PAD = 180, 192, 256, 25, 32
N_AA, SHELLS = 20, 8
OFF = {"w1": 0, "b1": MLP_H * MLP_K1}
OFF["w2"] = OFF["b1"] + MLP_H
OFF["b2"] = OFF["w2"] + MLP_H * MLP_H
OFF["w3"] = OFF["b2"] + MLP_H
OFF["b3"] = OFF["w3"] + MLP_OUT_PAD * MLP_H
N_PARAMS = OFF["b3"] + MLP_OUT_PAD
SHELL_R2 = np.array([1.5625, 6.25, 14.0625, 25.0, 39.0625, 56.25, 76.5625], np.float32)
LOG1P = np.array([np.float32(np.log1p(np.float64(n))) for n in range(256)], np.float32)


def bf16(x):
    """Round float32 values to BF16 (nearest, ties to even) and back to float32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    out = np.where(nan, a, out)
    return out.reshape(a.shape)


def env_counts(ag_ca, ag_aa, ca):
    """Counts [n][8][20] of antigen Calphas by shell and amino acid within r^2 < 100
    (r^2 = (dx*dx + dy*dy) + dz*dz in f32, dx = residue - antigen)."""
    ag_ca = np.asarray(ag_ca, np.float32)
    ca = np.asarray(ca, np.float32).reshape(-1, 3)
    n = len(ca)
    cnt = np.zeros((n, SHELLS, N_AA), np.int64)
    for r in range(n):
        d = (ca[r][None, :] - ag_ca).astype(np.float32)
        r2 = ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]).astype(np.float32) + d[:, 2] * d[:, 2]).astype(np.float32)
        inside = r2 < np.float32(100.0)
        shell = (r2[:, None] >= SHELL_R2[None, :]).sum(1)
        np.add.at(cnt[r], (shell[inside], np.asarray(ag_aa)[inside].astype(np.int64)), 1)
    return cnt


NO_AA = 255  # amino-acid input of a mutation query: no one-hot


def features(ag_ca, ag_aa, ca, aa):
    """float32 [n][180]: one-hot of aa (none for NO_AA), then log1p(count[shell][aa'])
    at 20 + 20*shell + aa'."""
    cnt = env_counts(ag_ca, ag_aa, ca)
    n = len(cnt)
    f = np.zeros((n, MLP_IN), np.float32)
    a = np.asarray(aa, np.int64)
    has = a < N_AA
    f[np.arange(n)[has], a[has]] = 1.0
    f[:, N_AA:] = LOG1P[np.minimum(cnt.reshape(n, -1), 255)]
    return bf16(f)


def unpack(p):
    p = np.asarray(p, np.float64)
    W1 = p[OFF["w1"]:OFF["b1"]].reshape(MLP_H, MLP_K1)[:, :MLP_IN]
    b1 = p[OFF["b1"]:OFF["w2"]]
    W2 = p[OFF["w2"]:OFF["b2"]].reshape(MLP_H, MLP_H)
    b2 = p[OFF["b2"]:OFF["w3"]]
    W3 = p[OFF["w3"]:OFF["b3"]].reshape(MLP_OUT_PAD, MLP_H)[:MLP_OUT]
    b3 = p[OFF["b3"]:][:MLP_OUT]
    return W1, b1, W2, b2, W3, b3


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def _b(x, on):
    return bf16(np.asarray(x, np.float32)).astype(np.float64) if on else np.asarray(x, np.float64)


def forward(params, X, bf16_path=True):
    """Outputs [n][25] and the intermediates (float64)."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    if bf16_path:
        W1, W2, W3 = _b(W1, 1), _b(W2, 1), _b(W3, 1)
    X = _b(X, bf16_path)
    Z1 = X @ W1.T + b1
    H1 = _b(Z1 * _sig(Z1), bf16_path)
    Z2 = H1 @ W2.T + b2
    H2 = _b(Z2 * _sig(Z2), bf16_path)
    Y = H2 @ W3.T + b3
    return Y, (X, Z1, H1, Z2, H2)


def loss_grad(params, X, action, target, delta=1.0, bf16_path=True, ref=None):
    """Mean Huber loss of Y[i, action[i]] - Y[i, ref[i]] (Y[i, action[i]] where ref is
    None or -1; rows with ref[i] == action[i] contribute zero) against target[i] and
    the gradient with respect to the flat parameter vector (float64, padding entries
    zero)."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    if bf16_path:
        W1, W2, W3 = _b(W1, 1), _b(W2, 1), _b(W3, 1)
    Y, (Xb, Z1, H1, Z2, H2) = forward(params, X, bf16_path)
    m = len(Y)
    a = np.asarray(action, np.int64)
    b = np.full(m, -1, np.int64) if ref is None else np.asarray(ref, np.int64)
    keep = b != a
    pred = Y[np.arange(m), a] - np.where(b >= 0, Y[np.arange(m), np.maximum(b, 0)], 0.0)
    d = np.where(keep, pred - np.asarray(target, np.float64), 0.0)
    ad = np.abs(d)
    loss = float(np.where(ad <= delta, 0.5 * d * d, delta * (ad - 0.5 * delta)).mean())
    g = np.clip(d, -delta, delta) / m
    dY = np.zeros_like(Y)
    rows = np.arange(m)
    dY[rows[keep], a[keep]] += g[keep]
    withb = keep & (b >= 0)
    dY[rows[withb], b[withb]] -= g[withb]
    dY = _b(dY, bf16_path)
    gW3 = dY.T @ H2
    gb3 = dY.sum(0)
    # the GPU keeps silu'(z) of the forward pass as BF16
    dZ2 = _b((dY @ W3) * _b(_sig(Z2) * (1 + Z2 * (1 - _sig(Z2))), bf16_path), bf16_path)
    gW2 = dZ2.T @ H1
    gb2 = dZ2.sum(0)
    dZ1 = _b((dZ2 @ W2) * _b(_sig(Z1) * (1 + Z1 * (1 - _sig(Z1))), bf16_path), bf16_path)
    gW1 = dZ1.T @ Xb
    gb1 = dZ1.sum(0)
    g = np.zeros(N_PARAMS, np.float64)
    G1 = np.zeros((MLP_H, MLP_K1))
    G1[:, :MLP_IN] = gW1
    G3 = np.zeros((MLP_OUT_PAD, MLP_H))
    G3[:MLP_OUT] = gW3
    g[OFF["w1"]:OFF["b1"]] = G1.ravel()
    g[OFF["b1"]:OFF["w2"]] = gb1
    g[OFF["w2"]:OFF["b2"]] = gW2.ravel()
    g[OFF["b2"]:OFF["w3"]] = gb2
    g[OFF["w3"]:OFF["b3"]] = G3.ravel()
    g[OFF["b3"]:OFF["b3"] + MLP_OUT] = gb3
    return loss, g
