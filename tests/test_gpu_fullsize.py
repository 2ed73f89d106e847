"""Cell numbers, sort permutations and both neighbour lists bit-exact against
the oracle's NEIGHBOR (functions.cu:2788-2929, pinned to the reference by
tests/test_oracle_pin.py) at the benchmark sizes (needs a B200):

* the 3D dam break of the headline workload, 1,595,308 particles;
* the two-phase scene, 86,118 particles;
* the 64 batched dam breaks in one context, 345 k particles;

each at the initial lattice and again after 20 GPU steps, when particles
have left the lattice: the lists are rebuilt at the GPU's own positions
(mps_neighbors) and the oracle bins the same positions.  Along long runs
too: the 2D dam over its whole 2000 steps and a small 3D dam over 600, at
the splashing states the collapse produces.  And one whole step of the
headline dam against the oracle's.
"""
import numpy as np
import pytest

import pyoracle
import voxarmps_b200 as vm
from voxarmps_b200 import config
from gpu_util import gpu_cfg, pair, rel_err

pytestmark = pytest.mark.gpu


def check_lists(g, cfg, what):
    x, y, z = g.get("x"), g.get("y"), g.get("z")
    for which, sfx, re in ((0, "s", cfg["re_s"]), (1, "l", cfg["re_l"])):
        cell, perm, off, nbr = pyoracle.neighbor(cfg, re, x, y, z)
        assert np.array_equal(g.get("cell_" + sfx), cell), f"{what}: cells {sfx}"
        assert np.array_equal(g.get("perm_" + sfx), perm), f"{what}: permutation {sfx}"
        goff, gnbr = g.lists(which)
        assert np.array_equal(goff, off), f"{what}: list lengths {sfx}"
        assert np.array_equal(gnbr, nbr), f"{what}: list entries {sfx}"
        del cell, perm, off, nbr, goff, gnbr


def run_case(cfg, case, scenes=None, steps=20):
    g = vm.Solver(cfg, case)
    if scenes is not None:
        g.set_scenes(*scenes)
    assert g.init() == 0
    check_lists(g, cfg, "initial lattice")
    g.set_graph(True)
    for _ in range(steps):
        assert g.step() == 0
    # lists at the positions the 20 steps left
    assert g.NEIGHBOR() == 0
    assert np.abs(g.get("y") - np.asarray(case["y"])).max() > 0  # off the lattice
    check_lists(g, cfg, f"after {steps} steps")
    g.close()


def test_dam3d_headline_size_lists_bit_exact():
    cfg, case = config.baseline(1)
    assert len(case["x"]) == 1595308
    run_case(gpu_cfg(cfg), case)


def test_two_phase_full_geometry_lists_bit_exact():
    cfg, case = config.baseline(3)
    run_case(gpu_cfg(cfg), case)


def test_batched_64_scenes_lists_bit_exact():
    base, scenes = config.baseline(4)
    cfg, case, sid, boxes, pmax = config.batched(gpu_cfg(base, precision=1), scenes)
    run_case(cfg, case, scenes=(sid, boxes, pmax))


def run_long(cfg, case, steps, every):
    """Lists against the oracle's NEIGHBOR along a long run, while the flow
    splashes and particles pack irregularly (the x-windows of the list
    passes see every spacing the run produces)."""
    g = vm.Solver(cfg, case)
    assert g.init() == 0
    g.set_graph(True)
    for k in range(1, steps + 1):
        assert g.step() == 0
        if k % every == 0:
            assert g.NEIGHBOR() == 0
            check_lists(g, cfg, f"after {k} steps")
    g.close()


def test_dam2d_whole_run_lists_bit_exact():
    cfg, case = config.baseline(0)
    run_long(gpu_cfg(cfg), case, 2000, 250)


def test_dam3d_small_long_run_lists_bit_exact():
    cfg, case = config.scaled_dam3d(1)
    run_long(gpu_cfg(cfg), case, 600, 100)


def test_dam3d_headline_one_step_matches_oracle():
    """One step of the 1,595,308-particle dam on the CUDA path and on the
    oracle: the FP64 stage outputs within a few ulps, the pressures (two
    FP64 CG runs to 1e-12, different dot orders) within 1e-7."""
    cfg, case = config.baseline(1)
    cfg = gpu_cfg(cfg, cg_tol=1e-12)
    g, o = pair(cfg, case)
    assert g.step() == 0
    assert o.step() == 0
    for f in ("xs", "ys", "zs", "us", "vs", "ws", "nstar"):
        assert rel_err(g.get(f), o.get(f)) <= 1e-12, f
    assert np.array_equal(g.get("bcon"), o.get("bcon"))
    assert rel_err(g.get("source"), o.get("source")) <= 1e-12
    for f in ("x", "y", "z", "u", "v", "w", "p"):
        assert rel_err(g.get(f), o.get(f)) <= 1e-7, f
    g.close()
