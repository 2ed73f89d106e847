"""One scene split between contexts (voxarmps_b200/slab.py) against the
same scene in one context (needs a B200).

The ranks are emulated as independent contexts on the one GPU, each driven
by its own host thread through LocalComm: every exchange (ghost particles,
ghost rows of the CG vectors, the dot-product sums) is a host step between
two launches, and no kernel waits on another context.  The split run's PPE
sums its dot products per rank first, so it differs from the single
context in rounding only: both reach cg_tol = 1e-12, and positions agree to
1e-10, velocities and pressures to 1e-6 after 5 steps; the CG iteration
counts are equal."""
import threading

import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import config, slab
from gpu_util import gpu_cfg, rel_err

pytestmark = pytest.mark.gpu

STEPS = 5


def run_split(cfg, case, size, steps):
    world = slab.LocalComm.World(size)
    n = len(case["x"])
    res, errs = [None] * size, []

    def rank_main(r):
        try:
            mine = np.arange(r, n, size)  # any initial split: the first step redistributes
            fields = {k: np.asarray(case[k], np.float64)[mine] for k in ("x", "y", "z", "u", "v", "w", "p")}
            fields["pnew"] = fields["p"].copy()
            fields["pold"] = fields["p"].copy()
            fields["phat"] = np.zeros(len(mine))
            for k in ("un", "vn", "wn"):
                fields[k] = np.zeros(len(mine))
            rk = slab.SlabRank(slab.LocalComm(world, r), cfg, mine, np.asarray(case["ptype"])[mine],
                               fields)
            its = []
            for _ in range(steps):
                st = rk.step()
                assert st == 0, st
                its.append(rk.last["cg_iters"])
            out = {k: rk.gather(k) for k in ("x", "y", "u", "v", "p")}
            rk.close()
            res[r] = (out, its)
        except Exception as e:
            errs.append(repr(e))
            world.barrier.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(size)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errs, errs
    glob = {}
    for k in ("x", "y", "u", "v", "p"):
        a = np.empty(n)
        seen = np.zeros(n, bool)
        for out, _its in res:
            gid, val = out[k]
            assert not seen[gid].any()  # every particle owned once
            seen[gid] = True
            a[gid] = val
        assert seen.all()
        glob[k] = a
    return glob, res[0][1]


@pytest.mark.parametrize("size", [2, 3])
def test_split_scene_matches_one_context(size):
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg, cg_tol=1e-12)
    one = vm.Solver(cfg, case)
    assert one.init() == 0
    its = []
    for _ in range(STEPS):
        assert one.step() == 0
        its.append(one.scalar("cg_iters"))
    ref = {k: one.get(k) for k in ("x", "y", "u", "v", "p")}
    one.close()
    got, split_its = run_split(cfg, case, size, STEPS)
    print(f"\n{size} ranks: CG iterations {split_its} (one context {its}); " +
          ", ".join(f"{k} {rel_err(got[k], ref[k]):.1e}" for k in ref))
    for k in ("x", "y"):
        assert rel_err(got[k], ref[k]) <= 1e-10, k
    for k in ("u", "v", "p"):
        assert rel_err(got[k], ref[k]) <= 1e-6, k
    assert [int(i) for i in split_its] == [int(i) for i in its]
