"""Error reporting of the CUDA path: each failure the reference prints (or
silently corrupts memory on) comes back as a status bit.  Failures are made
on the host side (bad inputs, tiny capacities); nothing faults the GPU."""
import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import config
from gpu_util import gpu_cfg

pytestmark = pytest.mark.gpu


def test_nan_input_flags_error1():
    cfg, case = config.baseline(0)
    case = dict(case)
    case["u"] = case["u"].copy()
    case["u"][-1] = np.nan
    g = vm.Solver(gpu_cfg(cfg), case)
    g.init()
    r = g.step()
    assert r & vm.MPS_ERR_NAN


def test_list_overflow_is_reported():
    cfg, case = config.baseline(0)
    g = vm.Solver(gpu_cfg(cfg, list_cap_l=8), case)
    r = g.init()
    assert r & vm.MPS_ERR_LIST_OVERFLOW


def test_cg_cap_reports_not_converged():
    cfg, case = config.baseline(0)
    g = vm.Solver(gpu_cfg(cfg, cg_max=1, warm_start=0), case)
    g.init()
    r = g.step()
    assert r & vm.MPS_ERR_NOT_CONVERGED


def test_particle_outside_grid_flags_cell_error():
    cfg, case = config.baseline(0)
    case = dict(case)
    case["x"] = case["x"].copy()
    g = vm.Solver(gpu_cfg(cfg), case)
    case["x"][-1] = cfg["xmax"] + 10.0   # outside the grown box set in cfg
    g.upload(case)
    r = g.init()
    assert r & vm.MPS_ERR_CELL


def test_stage_calls_before_init_rejected():
    cfg, case = config.baseline(0)
    g = vm.Solver(gpu_cfg(cfg), case)
    with pytest.raises(vm.MpsError):
        g.step()


@pytest.mark.parametrize("which", ["dam2d", "dam3d"])
def test_nonfinite_position_keeps_the_sort_a_permutation(which):
    """A particle whose position is NaN (and one at infinity) lands in cell 1
    with MPS_ERR_CELL; the in-cell order by (x, id) still gives every slot
    exactly once (x's order key places NaN and infinities at the ends), so
    the permutations stay permutations and further steps run and report."""
    cfg, case = config.baseline(0) if which == "dam2d" else config.scaled_dam3d(1)
    case = dict(case)
    case["x"] = case["x"].copy()
    fluid = np.flatnonzero(np.asarray(case["ptype"]) > 0)
    case["x"][fluid[-1]] = np.nan
    case["x"][fluid[-2]] = np.inf
    g = vm.Solver(gpu_cfg(cfg), case)
    r = g.init()
    assert r & vm.MPS_ERR_CELL
    n = len(case["x"])
    for sfx in ("l", "s"):
        perm = g.get("perm_" + sfx)
        assert np.array_equal(np.sort(perm), np.arange(n)), sfx
    for _ in range(2):
        r = g.step()
        assert r & (vm.MPS_ERR_CELL | vm.MPS_ERR_NAN | vm.MPS_ERR_BOX)
    for sfx in ("l", "s"):
        perm = g.get("perm_" + sfx)
        assert np.array_equal(np.sort(perm), np.arange(n)), sfx
    g.close()
