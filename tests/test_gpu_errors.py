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
