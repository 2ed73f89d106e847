"""The reference's own scenarios (built by voxarmps_b200/gen.py exactly as
its case generator writes them) through the CUDA path against the oracle:
both neighbour lists bit-exact and the state within the PPE tolerance after
a few steps, with the reference's default constants for each spacing."""
import numpy as np
import pytest

from voxarmps_b200 import config, gen
from gpu_util import gpu_cfg, pair, rel_err

pytestmark = pytest.mark.gpu

PPE_TOL = 1e-7  # two FP64 CG runs to cg_tol = 1e-12 (different dot orders)


@pytest.mark.parametrize("name,dl,mult", [("shear_cavity_2d", 0.01, 1),
                                          ("rt_instability_2d", 0.01, 1),
                                          ("dam_break_2d", 0.01, 1),
                                          ("dam_break_3d", 0.02, 1)])
def test_reference_scenario_steps(name, dl, mult):
    case = gen.GENERATORS[name](dl, mult)
    cfg = config.with_box(config.reference_defaults(dl, case["dim"]), case)
    cfg = gpu_cfg(cfg, cg_tol=1e-12)
    g, o = pair(cfg, case)
    for _ in range(3):
        assert g.step() == 0
        o.step()
    for which, key in ((0, "_s"), (1, "_l")):
        off, nbr = g.lists(which)
        assert np.array_equal(off, o.get("off" + key)) and np.array_equal(nbr, o.get("nbr" + key))
    fields = ("x", "y", "u", "v", "p") + (("z", "w") if case["dim"] == 3 else ())
    for f in fields:
        assert rel_err(g.get(f), o.get(f)) <= PPE_TOL, f
    g.close()
