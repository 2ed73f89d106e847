"""Mixed-precision PPE (precision 1): FP32 inner CG on an FP32 copy of the
matrix, FP64 dot products, FP64 residual and refinement.  The pressure must
satisfy the same FP64 system to the same cg_tol as the FP64 path, checked in
the oracle's own FP64 assembly; the difference from the FP64 run is stated
as a tolerance below.  Precision 2 also runs PNUMSTAR and the pressure
gradient in FP32; its pressure still solves its own FP64 system to cg_tol,
and its difference from the FP64 run is measured and bounded below."""
import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import cases, config
from gpu_util import gpu_cfg, oracle_relres, rel_err

pytestmark = pytest.mark.gpu

# Both paths solved to relative residual 1e-12 (the FP64 refinement takes the
# mixed path there too): two solutions of one FP64 system differ by about
# cond(A) * 2e-12, so pressures agree to 1e-7 (as two FP64 CG runs with
# different dot orders do) and positions after 10 steps to 1e-10.  At the
# benchmark's 1e-8 the measured differences are reported by bench.py.
MIXED_VS_FP64_P = 1e-7
MIXED_VS_FP64_X = 1e-10


def test_mixed_pressure_solves_fp64_system():
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg, cg_tol=1e-8, pmin=-1e30, precision=1)
    g = vm.Solver(cfg, case)
    assert g.init() == 0
    for _ in range(3):
        assert g.step() == 0
    assert g.scalar("cg_relres") <= 1e-8
    assert g.scalar("cg_outer") >= 1
    assert oracle_relres(g, cfg) <= 1.5e-8
    g.close()


def test_mixed_3d_solves_fp64_system():
    cfg, case = config.scaled_dam3d(1)
    cfg = gpu_cfg(cfg, cg_tol=1e-8, pmin=-1e30, precision=1)
    g = vm.Solver(cfg, case)
    assert g.init() == 0
    for _ in range(2):
        assert g.step() == 0
    assert g.scalar("cg_relres") <= 1e-8
    assert oracle_relres(g, cfg) <= 1.5e-8
    g.close()


@pytest.mark.parametrize("which", ["dam2d", "dam3d"])
def test_mixed_against_fp64_run(which):
    if which == "dam2d":
        cfg, case = config.baseline(0)
    else:
        cfg, case = config.scaled_dam3d(1)
    runs = {}
    for prec in (0, 1):
        g = vm.Solver(gpu_cfg(cfg, precision=prec, cg_tol=1e-12), case)
        assert g.init() == 0
        p1 = None
        for k in range(10):
            assert g.step() == 0
            if k == 0:
                p1 = g.get("p")
        runs[prec] = (p1, {f: g.get(f) for f in ("x", "y", "z")})
        g.close()
    assert rel_err(runs[1][0], runs[0][0]) <= MIXED_VS_FP64_P
    for f in ("x", "y", "z"):
        assert rel_err(runs[1][1][f], runs[0][1][f]) <= MIXED_VS_FP64_X, f


def test_mixed_graph_matches_eager():
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg, precision=1)
    out = []
    for graph in (False, True):
        g = vm.Solver(cfg, case)
        assert g.init() == 0
        g.set_graph(graph)
        its = []
        for _ in range(5):
            assert g.step() == 0
            its.append((g.scalar("cg_iters"), g.scalar("cg_outer")))
        out.append(({f: g.get(f) for f in ("x", "y", "p")}, its))
        g.close()
    for f in out[0][0]:
        assert np.array_equal(out[0][0][f], out[1][0][f]), f
    assert out[0][1] == out[1][1]


def test_mixed_batched_scenes_each_converged():
    l0 = 0.01
    scenes = [cases.dam_break(2, l0, (w, h), (100, 60)) for w, h in ((10, 20), (25, 50), (18, 33))]
    base = config.reference_defaults(l0, 2)
    base.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=1e-4, gy=-9.81)
    cfg, case, sid, boxes, pmax = config.batched(gpu_cfg(base, precision=1), scenes)
    g = vm.Solver(cfg, case)
    g.set_scenes(sid, boxes, pmax)
    assert g.init() == 0
    for _ in range(3):
        assert g.step() == 0
    assert g.scalar("cg_relres") <= 1e-8  # the worst scene's relative residual
    g.close()


# precision 2 against the FP64 run after 10 steps (max-norm relative):
# measured p 1.4e-4 / 3.9e-5, u 7e-5 / 4e-5, x 1e-7 / 2e-7 on the 2D dam /
# the 12,608-particle 3D dam.  FP32 positions relative to the box carry
# about 1e-7 m of rounding, which n* turns into noise of a few 1e-6 of n0
# in the source (n* - n0)/n0; on the 1.6 M-particle dam, where the box is
# larger and the fluid starts at rest, that noise is as large as the first
# step's pressure (bench.py --config 2 --precision 2 reports it)
FP32_EXPLICIT_P = 1e-3
FP32_EXPLICIT_U = 1e-3
FP32_EXPLICIT_X = 1e-6


@pytest.mark.parametrize("which", ["dam2d", "dam3d"])
def test_fp32_pnd_and_gradient_against_fp64(which):
    if which == "dam2d":
        cfg, case = config.baseline(0)
    else:
        cfg, case = config.scaled_dam3d(1)
    runs = {}
    for prec in (0, 2):
        g = vm.Solver(gpu_cfg(cfg, precision=prec, cg_tol=1e-8, pmin=-1e30), case)
        assert g.init() == 0
        for _ in range(10):
            assert g.step() == 0
        assert g.scalar("cg_relres") <= 1e-8
        if prec == 2:
            assert oracle_relres(g, g.cfg) <= 1.5e-8  # its own FP64 system
        runs[prec] = {f: g.get(f) for f in ("p", "x", "y", "z", "u", "v", "w", "nstar")}
        g.close()
    errs = {f: rel_err(runs[2][f], runs[0][f]) for f in runs[0]}
    print(f"\nprecision 2 vs FP64 after 10 steps ({which}): " +
          ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    assert errs["p"] <= FP32_EXPLICIT_P
    for f in ("u", "v", "w"):
        assert errs[f] <= FP32_EXPLICIT_U, f
    for f in ("x", "y", "z"):
        assert errs[f] <= FP32_EXPLICIT_X, f


def test_full_size_mixed_error_at_benchmark_tolerance():
    """The 1.6 M-particle dam at the benchmark's own tolerance (1e-8): the
    mixed-precision run against the FP64 run after 10 steps, the figures
    bench.py --config 2 reports as error_vs_fp64 (measured: pressure 4.8e-7
    of its maximum, positions 1.1e-13, velocities 1.9e-7); the bounds leave
    a factor 10."""
    cfg, case = config.baseline(1)
    out = {}
    for prec in (0, 1):
        g = vm.Solver(gpu_cfg(cfg, precision=prec, cg_tol=1e-8), case)
        assert g.init() == 0
        g.set_graph(True)
        for _ in range(10):
            assert g.step() == 0
        out[prec] = {f: g.get(f) for f in ("x", "y", "z", "u", "v", "w", "p")}
        g.close()
    bounds = {"p": 5e-6, "x": 1e-12, "y": 1e-12, "z": 1e-12, "u": 2e-6, "v": 2e-6, "w": 2e-6}
    for f, b in bounds.items():
        assert rel_err(out[1][f], out[0][f]) <= b, f
