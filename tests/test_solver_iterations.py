"""Iteration counts of the reference's ICCG (IC(0) factor of INCDECOM,
functions.cu:1139-1258, in CGM's iteration, functions.cu:506-716) against the
Jacobi-PCG the CUDA path runs, both stopped at the same relative residual
1e-8 on the same PPE system: the oracle's system after 20 steps of the 2D
dam break.  IC(0) needs about a third of the iterations, but each of them
costs two sequential triangular solves and its factorisation costs O(k^3)
per row; on the GPU the Jacobi iteration is one SpMV.  The comparison is
recorded, not a target."""
import numpy as np

import pyoracle
from voxarmps_b200 import config
from gpu_util import gpu_cfg


def test_iccg_against_jacobi_iterations():
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg)
    o = pyoracle.Oracle(cfg, case)
    assert o.init() == 0
    prev = None
    for _ in range(20):
        prev = o.get("p")
        assert o.step() == 0
    off, nbr, bcon, diag, val, b, _p = pyoracle.ppe_system(cfg, o)
    for x0 in (np.zeros(len(b)), prev):
        it = pyoracle.solver_iterations(off, nbr, bcon, diag, val, b, x0)
        for k in ("iccg", "jacobi", "plain"):
            assert it[k + "_relres"] <= 1e-8, k
        assert it["iccg"] < it["jacobi"] <= it["plain"] + 1
        print(it)
