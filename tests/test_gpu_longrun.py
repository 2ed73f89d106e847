"""Config 0 over the reference's whole run (2000 steps, 0.2 s of the dam
collapse) on the CUDA path and on the oracle: the flow's integral
quantities agree along the way.  Particle-level states drift apart slowly
(sums in different orders, discrete collision and free-surface decisions),
so the comparison is on the front position, the fluid's centroid and its
kinetic energy, every 200 steps.

The yardstick is the flow's own sensitivity, measured in the test on an
ensemble of equally valid oracle runs: the oracle at cg_tol 1e-12 instead
of 1e-8, and the oracle with every fluid particle's initial x, or y, moved
by one unit in the last place.  The collapse is chaotic: a one-ulp change
grows about a hundredfold every 200 steps and reaches 1.5% (front), 0.07%
(centroid) and 4% (kinetic energy) by step 2000.  So:

* up to step 600, while the ensemble's spread is still small, the CUDA
  path (whose sums differ from the oracle's by roundings every step) must
  stay at least as close to the oracle as every ensemble member, at every
  checkpoint (on B200 it is 1e2-1e4 times closer);
* over the whole run it must stay within fixed ceilings of the oracle
  (10% front, 1% centroid, 10% kinetic energy), the chaotic regime's
  physical agreement."""
import numpy as np
import pytest

import pyoracle
from voxarmps_b200 import config
from gpu_util import gpu_cfg, pair

pytestmark = pytest.mark.gpu

CEILING = (1e-1, 1e-2, 1e-1)   # whole run (front, centroid, KE)
STEPS, EVERY = 2000, 200
STRICT_UNTIL = 600             # checkpoints compared with the ensemble one by one


def _integrals(get, ptype):
    f = ptype > 0
    x, y, u, v = get("x")[f], get("y")[f], get("u")[f], get("v")[f]
    return np.array([x.max(), y.mean(), 0.5 * (u * u + v * v).sum()])


def _ulp(case, field, ptype):
    c = dict(case)
    a = np.array(case[field], dtype=np.float64)
    m = ptype > 0
    a[m] = np.nextafter(a[m], np.inf)
    c[field] = a
    return c


def test_config0_whole_run_integrals():
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg)
    pt = np.asarray(case["ptype"])
    g, o = pair(cfg, case)
    ensemble = [pyoracle.Oracle(gpu_cfg(cfg, cg_tol=1e-12), case),
                pyoracle.Oracle(cfg, _ulp(case, "x", pt)),
                pyoracle.Oracle(cfg, _ulp(case, "y", pt))]
    for e in ensemble:
        assert e.init() == 0
    gpu_dev, self_dev = [], []
    for k in range(STEPS):
        assert g.step() == 0
        o.step()
        for e in ensemble:
            e.step()
        if k % EVERY == EVERY - 1:
            b = _integrals(o.get, pt)
            gpu_dev.append(np.abs(_integrals(g.get, pt) - b) / np.abs(b))
            self_dev.append(np.max([np.abs(_integrals(e.get, pt) - b) / np.abs(b)
                                    for e in ensemble], axis=0))
    gpu_dev, self_dev = np.array(gpu_dev), np.array(self_dev)
    print("\nper checkpoint (front, centroid, kinetic energy):")
    for k in range(len(gpu_dev)):
        print(f"  step {(k + 1) * EVERY:5d}: CUDA vs oracle {gpu_dev[k]}, ensemble {self_dev[k]}")
    print(f"over {STEPS} steps: CUDA vs oracle {gpu_dev.max(0)}, ensemble {self_dev.max(0)}, "
          f"ceiling {CEILING}")
    early = STRICT_UNTIL // EVERY
    assert np.all(gpu_dev[:early] <= self_dev[:early]), (gpu_dev[:early], self_dev[:early])
    assert np.all(gpu_dev.max(0) <= CEILING), (gpu_dev.max(0), CEILING)
    g.close()
