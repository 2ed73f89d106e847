"""The CPU restatement of the learned-guess network (oracle/gnn_oracle.py):
its backward pass is checked against central differences of its own FP64
forward pass on a random symmetric neighbour graph, so that it can serve as
the oracle for the CUDA training kernels."""
import numpy as np

import gnn_oracle as G


def random_graph(n=40, radius=0.23, cap=16, seed=3):
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    nbr = np.zeros((n, cap), np.int32)
    ln = np.zeros(n, np.int32)
    for i in range(n):
        d = np.sqrt(((pts - pts[i]) ** 2).sum(1))
        js = [j for j in np.argsort(d) if j != i and d[j] < radius][:cap]
        ln[i] = len(js)
        nbr[i, :len(js)] = js
    # symmetric by construction unless the cap cut a list
    for i in range(n):
        for j in nbr[i, :ln[i]]:
            assert i in nbr[j, :ln[j]]
    return nbr, ln, cap


def test_backward_matches_central_differences():
    rng = np.random.default_rng(0)
    L = 2
    lay = G.layout(L)
    nbr, ln, cap = random_graph()
    n = len(ln)
    feat = rng.normal(size=(n, G.F))
    params = rng.normal(size=lay["P"]) * 0.3
    target = rng.normal(size=n)
    mask = rng.random(n) < 0.7
    loss, g = G.loss_and_grad(params, feat, nbr, ln, cap, L, target, mask, bf16_round=False)

    def f(p):
        return G.loss_and_grad(p, feat, nbr, ln, cap, L, target, mask, bf16_round=False)[0]

    picks = np.concatenate([rng.choice(lay["P"], 60, replace=False),
                            [lay["bd"], lay["wd"], lay["be"], lay["b"][0], lay["W"][1]]])
    eps = 1e-6
    for k in picks:
        e = np.zeros_like(params)
        e[k] = eps
        fd = (f(params + e) - f(params - e)) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])
    assert loss > 0


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-39, 65504.0], np.float32)
    r = G.bf16(x)
    assert r[0] == 1.0 and r[3] == -2.5
    assert r[1] == 1.0            # halfway between 1 and 1+2^-7: ties to even
    assert r[2] == 1.0078125      # above halfway: rounds up
    # half an ulp: relative 2^-8 for normal values, 2^-134 absolute for subnormals
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8 + 2.0 ** -134)


def test_rounded_forward_close_to_fp64():
    rng = np.random.default_rng(1)
    L = 3
    nbr, ln, cap = random_graph(seed=5)
    n = len(ln)
    feat = rng.normal(size=(n, G.F)).astype(np.float32)
    params = (rng.normal(size=G.layout(L)["P"]) * 0.2).astype(np.float32)
    a = G.forward(params, feat, nbr, ln, cap, L, bf16_round=True)["y"]
    b = G.forward(params.astype(np.float64), feat.astype(np.float64), nbr, ln, cap, L,
                  bf16_round=False)["y"]
    assert np.abs(a - b).max() <= 0.05 * np.abs(b).max()
