"""CPU restatement of the learned CG initial guess (test infrastructure only).

The network has no counterpart in the reference (whose CG starts from zero,
VoxarMPS/VoxarMPS/functions.cu:2503, or from the previous pressure on its GPU
path, VoxarMPS/VoxarMPS/main.cu:1159-1261); this module is the oracle for the
CUDA kernels of voxarmps_b200/csrc/mps_gnn.cu.  It restates

    h0  = relu(We f + be)
    m_l = mean over the neighbour list of i of h_(l-1)
    h_l = h_(l-1) + relu(W_l [h_(l-1), m_l] + b_l)        l = 1..L
    y   = wd . h_L + bd

with the parameter layout of the CUDA code (We [64 x 8], be, then per layer
W_l [64 x 128] row-major and b_l, then wd [64] and bd).

`forward(..., bf16=True)` rounds weights and stored activations to BF16
(round to nearest even) at the same points as the kernels and sums in FP32
in the kernels' sequential order, so it reproduces the GPU forward pass.
`backward` returns the exact (FP64) gradient of the mean squared error of y
against a target over the masked rows, through the stored (rounded)
activations; with `bf16=False` and float64 inputs the pair is a plain FP64
network whose gradient tests/test_gnn_oracle.py checks by central
differences.
"""
from __future__ import annotations

import numpy as np

H = 64
F = 8


def layout(L: int) -> dict:
    o = 0
    lay = {"L": L}
    lay["We"] = o; o += H * F
    lay["be"] = o; o += H
    lay["W"], lay["b"] = [], []
    for _ in range(L):
        lay["W"].append(o); o += H * 2 * H
        lay["b"].append(o); o += H
    lay["wd"] = o; o += H
    lay["bd"] = o; o += 1
    lay["P"] = o
    return lay


def bf16(a) -> np.ndarray:
    """Round float32 values to BF16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def unpack(params, L: int, dtype=np.float32):
    lay = layout(L)
    p = np.asarray(params, dtype)
    We = p[lay["We"]:lay["We"] + H * F].reshape(H, F)
    be = p[lay["be"]:lay["be"] + H]
    W = [p[o:o + H * 2 * H].reshape(H, 2 * H) for o in lay["W"]]
    b = [p[o:o + H] for o in lay["b"]]
    wd = p[lay["wd"]:lay["wd"] + H]
    bd = p[lay["bd"]]
    return We, be, W, b, wd, bd


def _lists(nbr, length, cap):
    nbr = np.asarray(nbr).reshape(-1, cap)
    length = np.asarray(length)
    return nbr, length


def forward(params, feat, nbr, length, cap, L: int, bf16_round: bool = True):
    """Forward pass; returns dict(h=[h0..hL], m=[m1..mL], z=[z0..zL], y)."""
    dt = np.float32 if bf16_round else np.float64
    rnd = bf16 if bf16_round else (lambda a: np.asarray(a, np.float64))
    We, be, W, b, wd, bd = unpack(rnd(params) if bf16_round else params, L, dt)
    f = np.asarray(feat, dt).reshape(-1, F)
    n = f.shape[0]
    nb, ln = _lists(nbr, length, cap)
    a = np.broadcast_to(be, (n, H)).astype(dt)
    for k in range(F):  # sequential over inputs, as the kernel
        a = a + We[:, k][None, :] * f[:, k][:, None]
    z = [rnd(a)]
    h = [rnd(np.maximum(a, 0))]
    m = []
    for l in range(L):
        s = np.zeros((n, H), dt)
        for k in range(int(ln.max()) if n else 0):  # list order
            act = ln > k
            idx = np.where(act)[0]
            s[idx] = s[idx] + h[l][nb[idx, k]]
        with np.errstate(invalid="ignore", divide="ignore"):
            mean = np.where(ln[:, None] > 0, s / np.maximum(ln, 1)[:, None].astype(dt), s)
        m.append(rnd(mean))
        u = np.concatenate([h[l], m[l]], axis=1)
        a = np.broadcast_to(b[l], (n, H)).astype(dt)
        for k in range(2 * H):
            a = a + W[l][:, k][None, :] * u[:, k][:, None]
        z.append(rnd(a))
        h.append(rnd(h[l] + np.maximum(a, 0)))
    y = np.full(n, bd, dt)
    for c in range(H):
        y = y + wd[c] * h[L][:, c]
    return {"h": h, "m": m, "z": z, "y": y}


def loss_and_grad(params, feat, nbr, length, cap, L, target, mask, acts=None,
                  bf16_round: bool = True):
    """Mean squared error over mask rows and its gradient (float64) with
    respect to the parameters, through the stored activations of `acts`."""
    if acts is None:
        acts = forward(params, feat, nbr, length, cap, L, bf16_round)
    lay = layout(L)
    w = bf16(params) if bf16_round else np.asarray(params, np.float64)
    We, be, W, b, wd, bd = unpack(w, L, np.float64)
    h = [np.asarray(x, np.float64) for x in acts["h"]]
    m = [np.asarray(x, np.float64) for x in acts["m"]]
    z = [np.asarray(x, np.float64) for x in acts["z"]]
    y = np.asarray(acts["y"], np.float64)
    t = np.asarray(target, np.float64)
    mk = np.asarray(mask, bool)
    cnt = max(int(mk.sum()), 1)
    e = np.where(mk, y - t, 0.0)
    loss = float((e * e).sum() / cnt)
    dy = 2.0 * e / cnt
    g = np.zeros(lay["P"], np.float64)
    g[lay["wd"]:lay["wd"] + H] = h[L].T @ dy
    g[lay["bd"]] = dy.sum()
    nb, ln = _lists(nbr, length, cap)
    n = len(y)
    rows = np.repeat(np.arange(n), ln)
    cols = np.concatenate([nb[i, :ln[i]] for i in range(n)]) if n else np.zeros(0, int)
    dh = dy[:, None] * wd[None, :]
    for l in range(L - 1, -1, -1):
        dz = dh * (z[l + 1] > 0)
        u = np.concatenate([h[l], m[l]], axis=1)
        g[lay["W"][l]:lay["W"][l] + H * 2 * H] = (dz.T @ u).ravel()
        g[lay["b"][l]:lay["b"][l] + H] = dz.sum(axis=0)
        du = dz @ W[l]
        dm = du[:, H:]
        dprev = dh + du[:, :H]
        # transpose of the mean aggregation: m_i gathers h_j for j in list(i)
        contrib = dm[rows] / np.maximum(ln[rows], 1)[:, None]
        np.add.at(dprev, cols, contrib)
        dh = dprev
    dz0 = dh * (z[0] > 0)
    f = np.asarray(feat, np.float64).reshape(-1, F)
    g[lay["We"]:lay["We"] + H * F] = (dz0.T @ f).ravel()
    g[lay["be"]:lay["be"] + H] = dz0.sum(axis=0)
    return loss, g
