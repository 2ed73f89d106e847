"""Graph mode (mps_set_graph): every step captured once per reorder buffer
set and replayed, the CG loop as a conditional while node.  The replayed
steps must give bit-identical state and the same iteration counts as the
eager launches of the same stages."""
import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import cases, config
from gpu_util import gpu_cfg

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "u", "v", "w", "p", "pnew", "phat")


def _run(cfg, case, graph, steps, scenes=None):
    s = vm.Solver(cfg, case)
    if scenes is not None:
        s.set_scenes(*scenes)
    assert s.init() == 0
    if graph:
        s.set_graph(True)
    iters, launches = [], []
    for _ in range(steps):
        before = s.scalar("launches")
        assert s.step() == 0
        launches.append(s.scalar("launches") - before)
        iters.append(int(s.scalar("cg_iters")))
    out = {f: s.get(f) for f in FIELDS if cfg["dim"] == 3 or f not in ("z", "w")}
    rel = s.scalar("cg_relres")
    s.close()
    return out, iters, launches, rel


def _same(a, b):
    for f in a[0]:
        assert np.array_equal(a[0][f], b[0][f]), f
    assert a[1] == b[1]
    assert a[3] == b[3]


def test_graph_matches_eager_2d_dam():
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg)
    eager = _run(cfg, case, False, 7)
    graph = _run(cfg, case, True, 7)
    _same(eager, graph)
    assert min(graph[2]) > 0  # replays count the graph's kernels


def test_graph_matches_eager_weakly_compressible():
    dam = cases.dam_break(2, 0.01, (20, 30), (60, 40))
    cfg = config.with_box(config.reference_defaults(0.01, 2, compressible=True), dam)
    cfg.update(re_s=0.021, re_l=0.04)
    cfg = gpu_cfg(cfg)
    _same(_run(cfg, dam, False, 5), _run(cfg, dam, True, 5))


def test_graph_matches_eager_batched_scenes():
    l0 = 0.01
    scenes = [cases.dam_break(2, l0, (w, h), (100, 60)) for w, h in ((10, 20), (25, 50), (18, 33))]
    base = config.reference_defaults(l0, 2)
    base.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=1e-4, gy=-9.81)
    cfg, case, sid, boxes, pmax = config.batched(gpu_cfg(base), scenes)
    eager = _run(cfg, case, False, 5, (sid, boxes, pmax))
    graph = _run(cfg, case, True, 5, (sid, boxes, pmax))
    _same(eager, graph)


def test_graph_matches_eager_3d_extrapolated_guess():
    cfg, case = config.scaled_dam3d(1)
    cfg = gpu_cfg(cfg, warm_start=2)
    _same(_run(cfg, case, False, 4), _run(cfg, case, True, 4))


def test_graph_off_again_and_reinit():
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg)
    s = vm.Solver(cfg, case)
    assert s.init() == 0
    s.set_graph(True)
    for _ in range(3):
        assert s.step() == 0
    s.set_graph(False)
    assert s.step() == 0
    s.set_graph(True)
    assert s.step() == 0
    ref = vm.Solver(cfg, case)
    assert ref.init() == 0
    for _ in range(5):
        assert ref.step() == 0
    for f in ("x", "y", "u", "v", "p"):
        assert np.array_equal(s.get(f), ref.get(f)), f
    s.close()
    ref.close()


def test_cg_loop_equals_four_kernel_loop():
    """The 2D dam's 1,928-row system solves in one cooperative launch
    (k_cg_loop); profiled steps, which time every SpMV launch, run the four
    kernels per iteration over the same grid and partials instead.  Both
    give the same bits and iteration counts."""
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg)
    runs = []
    for profile in (False, True):
        s = vm.Solver(cfg, case)
        assert s.init() == 0
        s.set_profile(profile)
        iters = []
        for _ in range(5):
            assert s.step() == 0
            iters.append(int(s.scalar("cg_iters")))
        runs.append(({f: s.get(f) for f in ("x", "y", "u", "v", "p", "pnew")}, iters))
        s.close()
    for f in runs[0][0]:
        assert np.array_equal(runs[0][0][f].view(np.uint64), runs[1][0][f].view(np.uint64)), f
    assert runs[0][1] == runs[1][1]
