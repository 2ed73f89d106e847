"""Shared helpers for the GPU parity tests: run the CUDA path (through the
C-ABI) and the oracle on the same inputs and parameters."""
import numpy as np

import pyoracle
import voxarmps_b200 as vm
from voxarmps_b200 import config

STATE = ["x", "y", "z", "u", "v", "w", "p", "pnew", "phat", "un", "vn", "wn", "xs", "ys", "zs",
         "us", "vs", "ws", "nstar", "C", "meu", "neut", "t1", "t2", "t3", "bcon", "source"]


def gpu_cfg(cfg, **kw):
    c = config.solver_semantics(cfg)
    c.update(kw)
    return c


def pair(cfg, case):
    """(gpu Solver, oracle) initialised on the same case."""
    g = vm.Solver(cfg, case)
    g.init()
    o = pyoracle.Oracle(cfg, case)
    assert o.init() == 0
    return g, o


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def lists_equal(g_off, g_nbr, o_off, o_nbr):
    return np.array_equal(g_off, o_off) and np.array_equal(g_nbr, o_nbr)


def oracle_relres(g, cfg):
    """||b - A x|| / ||b|| of the GPU's pressure in the oracle's own FP64
    system, assembled by the oracle from the GPU's lists and positions."""
    import ctypes as C
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
    return lib.mo_relres(n, ip(goff), ip(gnbr), ip(bcon), dp(diag), dp(val), dp(src), dp(p))
