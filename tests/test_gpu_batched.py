"""Batched independent scenes (mps_set_scenes) against one oracle run per
scene: every scene advanced in the shared context must match the same scene
simulated alone."""
import numpy as np
import pytest

import pyoracle
import voxarmps_b200 as vm
from voxarmps_b200 import cases, config
from gpu_util import gpu_cfg, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_four_scenes_match_separate_runs(precision):
    """In FP64 and in mixed precision (each scene's CG to its own residual)."""
    l0 = 0.01
    scenes = [cases.dam_break(2, l0, (w, h), (100, 60)) for w, h in ((10, 20), (25, 50), (18, 33),
                                                                     (40, 25))]
    base = config.reference_defaults(l0, 2)
    base.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=1e-4, gy=-9.81)
    base = gpu_cfg(base, cg_tol=1e-12)
    cfg, case, sid, boxes, pmax = config.batched(dict(base, precision=precision), scenes)
    g = vm.Solver(cfg, case)
    g.set_scenes(sid, boxes, pmax)
    assert g.init() == 0
    orc = []
    for sc in scenes:
        oc = config.with_box(base, sc)
        o = pyoracle.Oracle(oc, sc)
        assert o.init() == 0
        orc.append(o)
    for _ in range(4):
        assert g.step() == 0
        for o in orc:
            o.step()
    assert g.scalar("cg_relres") <= 1e-12
    for f in ("x", "y", "u", "v", "p"):
        a = g.get(f)
        for k, o in enumerate(orc):
            part = a[sid == k]
            ref = o.get(f)
            if f == "y":
                part = part - (case["y"][sid == k].min() - scenes[k]["y"].min())
            assert rel_err(part, ref) <= 1e-7, (f, k)


def test_config4_batch_matches_separate_runs():
    """The batched configuration itself: 64 scenes of 800 to 9,600 fluid
    particles in one context, mixed-precision PPE, two steps, against one
    FP64 oracle run per scene.  Both solve each scene's PPE to 1e-8; the
    bounds are the mixed mode's measured error against FP64 with margin."""
    base, scenes = config.baseline(4)
    base = gpu_cfg(base, cg_tol=1e-8, precision=1)
    cfg, case, sid, boxes, pmax = config.batched(base, scenes)
    g = vm.Solver(cfg, case)
    g.set_scenes(sid, boxes, pmax)
    assert g.init() == 0
    for _ in range(2):
        assert g.step() == 0
    assert g.scalar("cg_relres") <= 1e-8
    tol = {"x": 1e-9, "y": 1e-9, "u": 1e-5, "v": 1e-5, "p": 1e-5}
    got = {f: g.get(f) for f in tol}
    for k, sc in enumerate(scenes):
        o = pyoracle.Oracle(config.with_box(dict(base, precision=0), sc), sc)
        assert o.init() == 0
        for _ in range(2):
            o.step()
        for f, t in tol.items():
            part = got[f][sid == k]
            if f == "y":
                part = part - (case["y"][sid == k].min() - sc["y"].min())
            assert rel_err(part, o.get(f)) <= t, (f, k)
