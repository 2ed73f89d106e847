"""Launch-shape autotuning (mps_autotune / mps_set_tuning): every candidate
shape gives the same lists and, within rounding, the same state; the tuner
returns a valid choice and steps keep their results under it."""
import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import config
from gpu_util import gpu_cfg, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", [0, "dam3d"])
def test_every_shape_same_result(which):
    if which == 0:
        cfg, case = config.baseline(0)
        base = 4
    else:
        cfg, case = config.scaled_dam3d(1)
        base = 4
    cfg = gpu_cfg(cfg, cg_tol=1e-12)
    ref = None
    for lanes in (base, 2 * base):
        for bps in (1, 8):
            s = vm.Solver(cfg, case)
            assert s.init() == 0
            s.set_tuning(lanes, bps)
            for _ in range(3):
                assert s.step() == 0
            out = {f: s.get(f) for f in ("x", "y", "u", "v", "p")}
            off, nbr = s.lists(0)
            s.close()
            if ref is None:
                ref = (out, off, nbr)
                continue
            assert np.array_equal(off, ref[1]) and np.array_equal(nbr, ref[2])
            for f in out:
                assert rel_err(out[f], ref[0][f]) <= 1e-7, (lanes, bps, f)


def test_autotune_picks_valid_shape():
    cfg, case = config.baseline(0)
    s = vm.Solver(gpu_cfg(cfg), case)
    assert s.init() == 0
    t = s.autotune(2)
    assert t["small_lanes"] in (4, 8) and t["cg_blocks_per_sm"] in (1, 2, 4, 8)
    assert s.get_tuning() == t
    s.set_graph(True)
    for _ in range(3):
        assert s.step() == 0
    with pytest.raises(vm.MpsError):
        s.set_tuning(16, 1)
    s.close()
