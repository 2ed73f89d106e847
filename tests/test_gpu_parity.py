"""CUDA path vs the oracle, through the C-ABI (needs a B200).

Integer work (cells, sort permutations, neighbour lists) must be bit-exact.
FP64 stages accumulate in the reference's list order without FMA
contraction, so they match the oracle to the last bits except where CUDA's
pow() differs from glibc's; the tolerances below are written per field.
"""
import numpy as np
import pytest

import pyoracle
from voxarmps_b200 import cases, config
from gpu_util import gpu_cfg, pair, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12      # FP64 stages: same terms, each within a few ulps of the oracle's
PPE_TOL = 1e-7        # pressure: two FP64 CG runs to cg_tol=1e-12 (different dot orders)


def small_3d():
    case = cases.dam_break(3, 0.005, (8, 12, 6), (24, 16, 8))
    cfg = config.reference_defaults(0.005, 3)
    cfg.update(re_s=2.1 * 0.005, re_l=4.0 * 0.005, dt=5e-5, gy=-9.81)
    return config.with_box(cfg, case), case


CASES = {
    "config0": lambda: config.baseline(0),
    "dam3d_small": small_3d,
    # the two-phase configuration at its full geometry (86,118 particles;
    # SPS-LES, Herschel-Bulkley second fluid)
    "config3": lambda: config.baseline(3),
}


@pytest.mark.parametrize("name", list(CASES))
def test_cells_permutation_lists_bit_exact(name):
    cfg, case = CASES[name]()
    g, o = pair(gpu_cfg(cfg), case)
    for which, sfx, re in ((0, "s", cfg["re_s"]), (1, "l", cfg["re_l"])):
        cell, perm, off, nbr = pyoracle.neighbor(cfg, re, case["x"], case["y"], case["z"])
        assert np.array_equal(g.get("cell_" + sfx), cell), f"cells {sfx}"
        assert np.array_equal(g.get("perm_" + sfx), perm), f"permutation {sfx}"
        goff, gnbr = g.lists(which)
        assert np.array_equal(goff, off), f"list lengths {sfx}"
        assert np.array_equal(gnbr, nbr), f"list entries {sfx}"
    # n0 is an FP64 sum whose terms use rsqrt instead of sqrt and divisions
    assert abs(g.scalar("n0_s") / o.scalar("n0_s") - 1) <= 1e-14
    assert abs(g.scalar("n0_l") / o.scalar("n0_l") - 1) <= 1e-14


@pytest.mark.parametrize("name", list(CASES))
def test_one_step_matches_oracle(name):
    cfg, case = CASES[name]()
    cfg = gpu_cfg(cfg, cg_tol=1e-12)
    g, o = pair(cfg, case)
    assert g.step() == 0
    assert o.step() == 0
    for f in ("xs", "ys", "zs", "us", "vs", "ws", "nstar", "C", "meu"):
        assert rel_err(g.get(f), o.get(f)) <= FP64_TOL, f
    assert np.array_equal(g.get("bcon"), o.get("bcon"))
    assert rel_err(g.get("source"), o.get("source")) <= FP64_TOL
    assert rel_err(g.get("pnew"), o.get("pnew")) <= PPE_TOL
    for f in ("x", "y", "z", "u", "v", "w", "p"):
        assert rel_err(g.get(f), o.get(f)) <= PPE_TOL, f
    goff, gnbr = g.lists(0)
    assert np.array_equal(goff, o.get("off_s")) and np.array_equal(gnbr, o.get("nbr_s"))


def test_pressure_solves_oracle_system():
    """The GPU pressure satisfies the oracle's own FP64 system to cg_tol
    (lower clamp disabled so that pnew is the raw CG solution)."""
    import ctypes as C
    import voxarmps_b200 as vm
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg, cg_tol=1e-8, pmin=-1e30)
    g = vm.Solver(cfg, case)
    g.init()
    for _ in range(3):
        assert g.step() == 0
    lib = pyoracle.oracle_lib()
    P = pyoracle.params_from(cfg)
    n = g.n
    goff, gnbr = g.lists(1)
    xs, ys, zs = g.get("xs"), g.get("ys"), g.get("zs")
    bcon, src, p = g.get("bcon"), g.get("source"), g.get("pnew")
    diag, val = np.zeros(n), np.zeros(max(len(gnbr), 1))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    lib.mo_matrix(C.byref(P), cfg["re_l"], lib.mo_lambda(cfg["ktype"], cfg["re_l"]),
                  g.scalar("n0_l"), n, ip(goff), ip(gnbr), dp(xs), dp(ys), dp(zs), ip(bcon),
                  dp(diag), dp(val))
    assert rel_err(diag, g.get("diag")) <= FP64_TOL
    rel = lib.mo_relres(n, ip(goff), ip(gnbr), ip(bcon), dp(diag), dp(val), dp(src), dp(p))
    assert rel <= 1.5e-8
    assert g.scalar("cg_relres") <= 1e-8
    assert g.scalar("cg_iters") >= 1


def test_trajectory_config0_20_steps():
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg, cg_tol=1e-12)
    g, o = pair(cfg, case)
    for s in range(20):
        assert g.step() == 0
        o.step()
    for f in ("x", "y"):
        assert rel_err(g.get(f), o.get(f)) <= 1e-9, f
    for f in ("u", "v", "p"):
        assert rel_err(g.get(f), o.get(f)) <= 1e-5, f


def test_deterministic_bitwise():
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg)
    runs = []
    for _ in range(2):
        g, _o = pair(cfg, case)
        for _s in range(5):
            g.step()
        runs.append([g.get(f) for f in ("x", "y", "u", "v", "p")])
    for a, b in zip(*runs):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_weakly_compressible_step():
    dam = cases.dam_break(2, 0.01, (20, 30), (60, 40))
    cfg = config.with_box(config.reference_defaults(0.01, 2, compressible=True), dam)
    cfg.update(re_s=0.021, re_l=0.04)
    cfg = gpu_cfg(cfg)
    g, o = pair(cfg, dam)
    for _ in range(5):
        g.step()
        o.step()
    assert rel_err(g.get("p"), o.get("p")) <= 1e-9
    assert rel_err(g.get("x"), o.get("x")) <= 1e-12


def test_two_phase_turbulence_hb():
    tp = cases.dam_break(2, 0.01, (20, 20), (60, 40), blocks=[(2, (0, 20), (15, 15))])
    cfg = config.with_box(config.reference_defaults(0.01, 2), tp)
    cfg.update(re_s=0.021, re_l=0.04, turb=1, fluid2_type=1, rho2=900.0, nu2=1e-4, n_pl=1.3,
               meu0=0.04, cohes=5.0, cs=0.12)
    cfg = gpu_cfg(cfg, cg_tol=1e-12)
    g, o = pair(cfg, tp)
    for _ in range(3):
        g.step()
        o.step()
    for f in ("neut", "t1", "t2", "meu", "C"):
        assert rel_err(g.get(f), o.get(f)) <= 1e-9, f
    assert rel_err(g.get("p"), o.get("p")) <= 1e-6


def test_matopt_srcopt():
    cfg, case = config.baseline(0)
    for kw in (dict(matopt=1), dict(srcopt=1)):
        c = gpu_cfg(cfg, cg_tol=1e-12, **kw)
        g, o = pair(c, case)
        g.step()
        o.step()
        assert rel_err(g.get("source"), o.get("source")) <= 1e-9, kw
        assert rel_err(g.get("p"), o.get("p")) <= 1e-6, kw


def test_extrapolated_initial_guess_matches_oracle():
    """warm_start = 2 (x0 = 2 p^n - p^(n-1)) on both sides, 6 steps."""
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg, cg_tol=1e-12, warm_start=2)
    g, o = pair(cfg, case)
    for _ in range(6):
        assert g.step() == 0
        o.step()
    for f in ("x", "y", "u", "v", "p"):
        assert rel_err(g.get(f), o.get(f)) <= 1e-6, f


@pytest.mark.parametrize("precision", [0, 1])
def test_zero_initial_guess_matches_oracle(precision):
    """warm_start = 0 (the reference CPU path's x0 = 0; the start kernels
    take r = b without a product) on both sides, 6 steps, FP64 and mixed."""
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg, cg_tol=1e-12, warm_start=0, precision=precision)
    g, o = pair(cfg, case)
    for _ in range(6):
        assert g.step() == 0
        o.step()
        assert g.scalar("cg_r0") == 1.0  # ||b - A 0|| / ||b||
    for f in ("x", "y", "u", "v", "p"):
        assert rel_err(g.get(f), o.get(f)) <= 1e-6, f
