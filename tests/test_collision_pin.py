"""COLLISION2 (functions.cu:1523-1678) pinned to the reference on constructed
states where collisions fire (tests/golden/ref_collision*.npz, made by
tests/golden/make_golden.py from the reference's own NEIGHBOR and
COLLISION2): fluid-fluid pairs along every axis and fluid particles pushed
into the bottom and side walls, 0.4 l0 apart with coll = 0.5 l0.

* the oracle's sequential restatement (mo_collision) equals the reference
  bit for bit;
* the order-independent pair replay (mo_collision_gather, the form the CUDA
  kernel computes) equals it bit for bit whenever colliding pairs do not
  share a particle -- walls included, where the reference pushes a pair
  twice;
* with three particles within coll of one another the replay stays within
  rounding of the sum of its pairs (the sequential result then depends on
  the visiting order, so it is not the target).
"""
import json
import os

import numpy as np
import pytest

import pyoracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DISJOINT = ["collision2d", "collision3d"]
CLUSTER = ["collision2d_cluster", "collision3d_cluster"]


def load(name):
    d = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    return json.loads(str(d["cfg"])), d


def run(cfg, d, gather):
    return pyoracle.collision(cfg, d["off"], d["nbr"], d["in_ptype"], d["in_un"], d["in_vn"],
                              d["in_wn"], d["in_x"], d["in_y"], d["in_z"], gather=gather)


def bits(a):
    return np.asarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("name", DISJOINT + CLUSTER)
def test_oracle_lists_match_reference(name):
    cfg, d = load(name)
    _cell, _perm, off, nbr = pyoracle.neighbor(cfg, cfg["re_s"], d["in_x"], d["in_y"], d["in_z"])
    assert np.array_equal(off, d["off"]) and np.array_equal(nbr, d["nbr"])


@pytest.mark.parametrize("name", DISJOINT + CLUSTER)
def test_sequential_collision_bit_exact(name):
    cfg, d = load(name)
    out = run(cfg, d, gather=False)
    for k, a in zip(("un", "vn", "wn", "x", "y", "z"), out):
        assert np.array_equal(bits(a), bits(d["out_" + k])), k


@pytest.mark.parametrize("name", DISJOINT)
def test_pair_replay_equals_reference_bit_exact(name):
    cfg, d = load(name)
    out = run(cfg, d, gather=True)
    for k, a in zip(("un", "vn", "wn", "x", "y", "z"), out):
        assert np.array_equal(bits(a), bits(d["out_" + k])), k
    # collisions fired: every pushed fluid particle changed velocity
    changed = (d["out_un"] != d["in_un"]) | (d["out_vn"] != d["in_vn"])
    assert changed.sum() >= 10
    # and a wall pair was pushed twice: the replay of one visit alone differs
    pt = d["in_ptype"]
    assert np.any(changed & (pt > 0))


@pytest.mark.parametrize("name", CLUSTER)
def test_pair_replay_cluster_within_rounding(name):
    cfg, d = load(name)
    g = run(cfg, d, gather=True)
    s = run(cfg, d, gather=False)
    for k, a, b in zip(("un", "vn", "wn", "x", "y", "z"), g, s):
        if k in ("un", "vn", "wn"):
            # the three-particle cluster: the replay sums pair impulses where the
            # sequential form applies them one after another
            assert np.abs(a - b).max() <= 2.0, k
        else:
            assert np.abs(a - b).max() <= 1e-2 * cfg["l0"], k
