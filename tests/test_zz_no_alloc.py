"""mps_cell_order_noalloc: the allocation-free binning entry point.

It serves programs that may not allocate device memory -- an application
whose own pool already owns the device heap, or a loop that forbids
allocation after start-up -- and works only on the caller's buffers plus a
fixed static scratch area.  This test checks, through the C-ABI, that two
consecutive calls give exactly the cell numbers and cell order that the
context path (mps_init + mps_download) computes for the same particles.
The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import cases, config

pytestmark = pytest.mark.gpu


def _cfg_struct(cfg):
    return vm.MpsConfig(**{k: cfg[k] for k, _ in config.FIELDS})


def _scenes():
    c2, case2 = config.baseline(0)
    case3 = cases.dam_break(3, 0.005, (8, 12, 6), (24, 16, 8))
    c3 = config.reference_defaults(0.005, 3)
    c3.update(re_s=2.1 * 0.005, re_l=4.0 * 0.005, dt=5e-5, gy=-9.81)
    c3 = config.with_box(c3, case3)
    return [(config.solver_semantics(c2), case2), (config.solver_semantics(c3), case3)]


@pytest.mark.parametrize("k", [0, 1])
def test_noalloc_matches_context_path(k):
    import torch
    cfg, case = _scenes()[k]
    lib = vm.load_library()
    ref = vm.Solver(cfg, case)
    ref.init()
    n = ref.n
    dev = lambda a: torch.tensor(np.asarray(a, np.float64), device="cuda")
    x, y, z = dev(case["x"]), dev(case["y"]), dev(case["z"])
    cs = _cfg_struct(ref.cfg)
    for which, re in (("s", cfg["re_s"]), ("l", cfg["re_l"])):
        want_cell, want_perm = ref.get("cell_" + which), ref.get("perm_" + which)
        for _ in range(2):  # the second call must not see the first call's counters
            cell = torch.full((n,), -7, dtype=torch.int32, device="cuda")
            perm = torch.full((n,), -7, dtype=torch.int32, device="cuda")
            bad = torch.ones(1, dtype=torch.int32, device="cuda")
            r = lib.mps_cell_order_noalloc(C.byref(cs), re, n, x.data_ptr(), y.data_ptr(),
                                           z.data_ptr(), cell.data_ptr(), perm.data_ptr(),
                                           bad.data_ptr(), None)
            torch.cuda.synchronize()
            assert r == vm.MPS_OK
            assert int(bad.item()) == 0
            assert np.array_equal(cell.cpu().numpy(), want_cell)
            assert np.array_equal(perm.cpu().numpy(), want_perm)


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    cfg, case = _scenes()[0]
    lib = vm.load_library()
    cs = _cfg_struct(config.with_box(cfg, case))
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(8, dtype=torch.int32, device="cuda")
    r = lib.mps_cell_order_noalloc(C.byref(cs), cfg["re_s"], (1 << 18) + 1, buf.data_ptr(),
                                   buf.data_ptr(), buf.data_ptr(), out.data_ptr(),
                                   out.data_ptr(), out.data_ptr(), None)
    assert r == vm.MPS_ERR_ARG


def test_noalloc_rejects_grids_beyond_its_limit():
    """A support radius so small that the cell count along each axis, and
    their product, overflow 32 bits is refused before anything is launched."""
    import torch
    cfg, case = _scenes()[1]
    lib = vm.load_library()
    cs = _cfg_struct(cfg)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(8, dtype=torch.int32, device="cuda")
    for re in (1e-7, 1e-12):
        r = lib.mps_cell_order_noalloc(C.byref(cs), re, 8, buf.data_ptr(), buf.data_ptr(),
                                       buf.data_ptr(), out.data_ptr(), out.data_ptr(),
                                       out.data_ptr(), None)
        assert r == vm.MPS_ERR_ARG
