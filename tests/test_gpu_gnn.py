"""Learned CG initial guess (mps_gnn_*): the CUDA forward pass against the
CPU restatement in oracle/gnn_oracle.py (same BF16 rounding points, same
FP32 summation order), the training kernels' gradient against the oracle's
FP64 gradient, training on the solver's own PPE snapshots, and the guess in
use: same answer (the PPE residual in the oracle's FP64 system), graph and
eager steps identical, and the iteration counts it gives."""
import numpy as np
import pytest

import gnn_oracle as G
import voxarmps_b200 as vm
from voxarmps_b200 import config
from gpu_util import gpu_cfg, oracle_relres

pytestmark = pytest.mark.gpu

L = 4
# forward: the layer products run on the tensor cores, which sum the 128
# products of a row in their own order (FP32); an activation rounded to BF16
# can then land one BF16 unit (2^-8 relative) away from the oracle's, and
# four layers carry that forward
Y_TOL = 1e-2
# gradient: FP32 sums in a different order than the FP64 oracle, on the
# tensor-core forward's activations
GRAD_TOL = 1e-2
# the trained guess must leave at most this fraction of the previous
# pressure's starting residual |b - A x0| / |b|
GAIN_R0 = 0.5


def _ctx(steps=2, seed=7, scale=0.1):
    cfg, case = config.baseline(0)
    s = vm.Solver(gpu_cfg(cfg), case)
    assert s.init() == 0
    s.gnn_create(L, seed)
    if scale:
        p = s.gnn_params()
        rng = np.random.default_rng(seed)
        s.gnn_params(set_to=(rng.normal(size=p.size) * scale).astype(np.float32))
    for _ in range(steps):
        assert s.step() == 0
    return s


def _graph(s):
    cap = int(s.gnn_get("cap")[0])
    return s.gnn_get("feat").reshape(-1, G.F), s.gnn_get("nbr"), s.gnn_get("len"), cap


def test_forward_matches_oracle():
    s = _ctx()
    p = s.gnn_params()
    s.gnn_forward()
    feat, nbr, ln, cap = _graph(s)
    y = s.gnn_get("y")
    ref = G.forward(p, feat, nbr, ln, cap, L)["y"]
    err = np.abs(y - ref).max() / max(np.abs(ref).max(), 1e-30)
    print(f"\nforward: max |y - y_oracle| / max |y_oracle| = {err:.3e}")
    assert err <= Y_TOL
    s.close()


def test_gradient_matches_oracle():
    s = _ctx()
    p = s.gnn_params()
    loss = s.gnn_train(1, 1e-3, grad_only=True, objective="increment")
    g = s.gnn_get("grad")
    feat, nbr, ln, cap = _graph(s)
    tgt = s.gnn_get("target")
    mask = s.gnn_get("bcon") == 0  # the PPE's unknowns
    acts = G.forward(p, feat, nbr, ln, cap, L)
    lref, gref = G.loss_and_grad(p, feat, nbr, ln, cap, L, tgt, mask, acts=acts)
    assert abs(loss - lref) <= 1e-4 * lref
    lay = G.layout(L)
    blocks = [("We", lay["We"], lay["be"] + G.H), ("wd", lay["wd"], lay["P"])]
    blocks += [(f"W{l}", lay["W"][l], lay["b"][l] + G.H) for l in range(L)]
    for name, a, b in blocks:
        err = np.linalg.norm(g[a:b] - gref[a:b]) / max(np.linalg.norm(gref[a:b]), 1e-30)
        print(f"gradient {name}: relative error {err:.3e}")
        assert err <= GRAD_TOL, (name, err)
    s.close()


def test_residual_objective_gradient_by_differences():
    """Objective 1 (|b - A x0|^2/|b|^2, gradient through A r): the kernels'
    derivative with respect to output-layer parameters against central
    differences of the same GPU loss (quadratic in those parameters)."""
    s = _ctx()
    p = s.gnn_params()
    s.gnn_train(1, 1e-3, grad_only=True, objective="residual")
    g = s.gnn_get("grad")
    lay = G.layout(L)
    for k in (lay["bd"], lay["wd"] + 3, lay["wd"] + 40):
        vals, used = [], []
        for sgn in (1, -1):
            q = p.copy()
            q[k] += sgn * 1e-2 * max(1.0, abs(float(p[k])))
            s.gnn_params(set_to=q)
            vals.append(s.gnn_train(1, 1e-3, grad_only=True, objective="residual"))
            used.append(float(G.bf16(q[k:k + 1])[0]))  # the kernels see BF16 weights
        fd = (vals[0] - vals[1]) / (used[0] - used[1])
        assert abs(fd - g[k]) <= 2e-2 * max(abs(fd), 1e-6), (k, fd, g[k])
    s.close()


def _train(s, steps, iters=2, lr=2e-3, objective="residual"):
    losses = []
    for _ in range(steps):
        assert s.step() == 0
        losses.append(s.gnn_train(iters, lr, objective=objective))
    return losses


def test_training_on_own_snapshots_reduces_loss():
    s = _ctx(steps=1, scale=0)
    losses = _train(s, 120, objective="increment")
    first, last = np.mean(losses[:10]), np.mean(losses[-10:])
    print(f"\nloss first 10 steps {first:.4g}, last 10 steps {last:.4g}")
    assert last < 0.5 * first
    s.close()


def test_learned_guess_keeps_the_answer_and_reports_iterations():
    cfg, case = config.baseline(0)
    # no clamp: the pressure is the raw CG solution of the system
    cfg = gpu_cfg(cfg, pmin=-1e30, pmax=1e30)
    base = vm.Solver(cfg, case)
    assert base.init() == 0
    s = vm.Solver(cfg, case)
    assert s.init() == 0
    s.gnn_create(L, 11)
    _train(s, 150)
    for _ in range(150):
        assert base.step() == 0
    s.gnn_use(True)
    its_b, its_g, r0_b, r0_g = [], [], [], []
    for _ in range(20):
        assert base.step() == 0
        assert s.step() == 0
        its_b.append(base.scalar("cg_iters"))
        its_g.append(s.scalar("cg_iters"))
        r0_b.append(base.scalar("cg_r0"))
        r0_g.append(s.scalar("cg_r0"))
        assert s.scalar("cg_relres") <= 1e-8
    assert oracle_relres(s, cfg) <= 1.5e-8
    print(f"\nprevious-pressure guess: |r0|/|b| {np.mean(r0_b):.3g}, CG iterations "
          f"{np.mean(its_b):.2f}; learned guess: |r0|/|b| {np.mean(r0_g):.3g}, "
          f"CG iterations {np.mean(its_g):.2f}")
    # what the trained network gains: a smaller starting residual than the
    # previous pressure leaves, and no more CG iterations
    assert np.mean(r0_g) <= GAIN_R0 * np.mean(r0_b)
    assert np.mean(its_g) <= np.mean(its_b)
    base.close()
    s.close()


def test_learned_guess_graph_matches_eager():
    out = []
    for graph in (False, True):
        s = _ctx(steps=1, seed=5)
        s.gnn_use(True)
        s.set_graph(graph)
        its = []
        for _ in range(4):
            assert s.step() == 0
            its.append(s.scalar("cg_iters"))
        out.append(({f: s.get(f) for f in ("x", "y", "p")}, its))
        s.close()
    for f in out[0][0]:
        assert np.array_equal(out[0][0][f], out[1][0][f]), f
    assert out[0][1] == out[1][1]


def test_training_state_moves_between_contexts():
    """mps_gnn_state carries weights, Adam moments and the step count: a
    network trained in one context and continued in another takes exactly
    the Adam steps it would have taken in the first (same snapshot, same
    state), and a state round trip is exact."""
    a, b = _ctx(steps=2), _ctx(steps=2)
    a.gnn_train(3, 1e-3)
    st = a.gnn_state()
    P = a.gnn_params().size
    assert st.size == 3 * P + 1 and st[3 * P] == 3.0
    assert np.any(st[P:2 * P] != 0) and np.any(st[2 * P:3 * P] != 0)
    b.gnn_state(set_to=st)
    assert np.array_equal(b.gnn_state(), st)
    assert np.array_equal(b.gnn_params(), a.gnn_params())
    # both contexts hold the same snapshot (same case, same steps): two more
    # Adam steps from the same state give the same weights
    a.gnn_train(2, 1e-3)
    b.gnn_train(2, 1e-3)
    assert np.array_equal(a.gnn_params(), b.gnn_params())
    assert a.gnn_state()[3 * P] == 5.0
    # setting the parameters alone restarts Adam
    b.gnn_params(set_to=a.gnn_params())
    assert b.gnn_state()[3 * P] == 0.0
    a.close()
    b.close()
