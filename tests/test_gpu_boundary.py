"""The drop-in boundary, exercised the way the reference's caller uses it
(needs a B200).

* The per-stage entries (functions.cuh:44-111), called one by one in
  main.cu's loop order (main.cu:1036-1337), give mps_step's result bit for
  bit and follow the oracle.
* COLLISION2 on constructed states where collisions fire, against the
  reference's own result (tests/golden/ref_collision*.npz): bit for bit
  where colliding pairs do not share a particle.
* mps_load_grd on the reference's own input files (main.cu:496-684), kept
  byte for byte in tests/golden/ref_inputs_grd.npz.
"""
import json
import os

import numpy as np
import pytest

import pyoracle
import voxarmps_b200 as vm
from voxarmps_b200 import cases, config
from gpu_util import gpu_cfg, pair, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ["x", "y", "z", "u", "v", "w", "p", "pnew", "phat", "un", "vn", "wn", "xs", "ys", "zs",
          "us", "vs", "ws", "nstar", "C", "meu", "neut", "t1", "t2", "t3", "source", "diag"]


def two_phase():
    tp = cases.dam_break(2, 0.01, (20, 20), (60, 40), blocks=[(2, (0, 20), (15, 15))])
    cfg = config.with_box(config.reference_defaults(0.01, 2), tp)
    cfg.update(re_s=0.021, re_l=0.04, turb=1, fluid2_type=1, rho2=900.0, nu2=1e-4, n_pl=1.3,
               meu0=0.04, cohes=5.0, cs=0.12)
    return cfg, tp


def small_3d():
    case = cases.dam_break(3, 0.005, (8, 12, 6), (24, 16, 8))
    cfg = config.reference_defaults(0.005, 3)
    cfg.update(re_s=2.1 * 0.005, re_l=4.0 * 0.005, dt=5e-5, gy=-9.81)
    return config.with_box(cfg, case), case


STAGE_CASES = {"config0": lambda: config.baseline(0), "two_phase_turb_hb": two_phase,
               "dam3d_small": small_3d}


def stage_by_stage(g, cfg):
    """One loop iteration of main.cu:1036-1337 through the per-stage entries."""
    if cfg["method"] != 3:
        assert g.PNUM() == 0
    assert g.NEIGHBOR() == 0
    if cfg["turb"]:
        assert g.SPS() == 0
    assert g.V_FRACTION() == 0
    assert g.VISCOSITY() == 0
    assert g.PREDICTION() == 0
    assert g.PNUMSTAR() == 0
    if cfg["method"] != 3:
        assert g.BCON() == 0
    iters, relres = g.PRESSURECALC()
    assert cfg["method"] == 3 or (iters >= 1 and relres <= cfg["cg_tol"])
    assert g.PHATCALC() == 0
    assert g.PRESSGRAD() == 0
    assert g.EULERINTEGRATION() == 0
    assert g.COLLISION2() == 0
    assert g.PREPDATA() == 0


@pytest.mark.parametrize("name", list(STAGE_CASES))
def test_stage_entries_equal_step_bit_for_bit(name):
    cfg, case = STAGE_CASES[name]()
    cfg = gpu_cfg(cfg, cg_tol=1e-10)
    a = vm.Solver(cfg, case)
    b = vm.Solver(cfg, case)
    assert a.init() == 0 and b.init() == 0
    o = pyoracle.Oracle(cfg, case)
    assert o.init() == 0
    for _ in range(3):
        stage_by_stage(a, cfg)
        assert b.step() == 0
        o.step()
    for f in FIELDS + ["bcon", "cell_s", "cell_l", "perm_s", "perm_l"]:
        x, y = a.get(f), b.get(f)
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f
    for which in (0, 1):
        oa, na = a.lists(which)
        ob, nb = b.lists(which)
        assert np.array_equal(oa, ob) and np.array_equal(na, nb)
    # and the staged run follows the oracle as mps_step does
    for f in ("x", "y", "z"):
        assert rel_err(a.get(f), o.get(f)) <= 1e-9, f
    for f in ("u", "v", "p"):
        assert rel_err(a.get(f), o.get(f)) <= 1e-5, f


def _collision_fixture(name):
    d = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    cfg = gpu_cfg(json.loads(str(d["cfg"])))
    case = {"dim": int(d["in_dim"]), "x": d["in_x"], "y": d["in_y"], "z": d["in_z"],
            "ptype": d["in_ptype"], "u": np.zeros(len(d["in_x"])), "v": np.zeros(len(d["in_x"])),
            "w": np.zeros(len(d["in_x"])), "p": np.zeros(len(d["in_x"]))}
    return cfg, case, d


def _gpu_collision(cfg, case, d):
    g = vm.Solver(cfg, case)
    assert g.init() == 0
    for k in ("un", "vn") + (("wn",) if case["dim"] == 3 else ()):
        g.set(k, d["in_" + k])
    assert g.COLLISION2() == 0
    return g


@pytest.mark.parametrize("name", ["collision2d", "collision3d"])
def test_collision_stage_equals_reference_bit_for_bit(name):
    cfg, case, d = _collision_fixture(name)
    g = _gpu_collision(cfg, case, d)
    keys = ("x", "y", "un", "vn") + (("z", "wn") if case["dim"] == 3 else ())
    for k in keys:
        got = g.get(k)
        assert np.array_equal(got.view(np.uint64), d["out_" + k].view(np.uint64)), k
    # the collisions fired on the GPU too
    assert np.sum(g.get("un") != d["in_un"]) >= 10


@pytest.mark.parametrize("name", ["collision2d_cluster", "collision3d_cluster"])
def test_collision_stage_cluster_matches_pair_replay(name):
    """Three particles within coll of one another: the kernel sums the pair
    replays in its own lane order, the oracle in list order."""
    cfg, case, d = _collision_fixture(name)
    g = _gpu_collision(cfg, case, d)
    want = pyoracle.collision(cfg, d["off"], d["nbr"], d["in_ptype"], d["in_un"], d["in_vn"],
                              d["in_wn"], d["in_x"], d["in_y"], d["in_z"], gather=True)
    for k, w in zip(("un", "vn", "wn", "x", "y", "z"), want):
        if case["dim"] == 2 and k in ("wn", "z"):
            continue
        got = g.get(k)
        assert np.abs(got - w).max() <= 1e-14 * max(np.abs(w).max(), 1.0), k


@pytest.mark.parametrize("name,dim", [("input_dam_grd", 2), ("input_dam3d_grd", 3)])
def test_load_grd_reads_reference_inputs(tmp_path, name, dim):
    raw = np.load(os.path.join(GOLDEN, "ref_inputs_grd.npz"))[name]
    path = tmp_path / (name + ".grd")
    path.write_bytes(raw.tobytes())
    want = cases.read_grd(str(path), dim)
    l0 = 0.01
    cfg = gpu_cfg(config.reference_defaults(l0, dim))  # box grown from the file (main.cu:692-715)
    g = vm.Solver(cfg)
    g.load_grd(str(path))
    assert g.n == len(want["x"])
    assert np.array_equal(g.get("ptype"), want["ptype"])
    keys = ("x", "y", "u", "v", "p") + (("z", "w") if dim == 3 else ())
    for k in keys:
        assert np.array_equal(g.get(k), want[k]), k
    # the grown box and PMAX of main.cu:548, 692-715
    box = config.with_box(cfg, want)
    for k in ("xmin", "xmax", "ymin", "ymax") + (("zmin", "zmax") if dim == 3 else ()):
        assert g.scalar(k) == box[k], k
    assert g.scalar("pmax") == box["pmax"]
    assert g.init() == 0
    assert g.step() == 0


def test_grid_larger_than_limit_is_rejected():
    """A support radius so small that the cell count overflows 32 bits is an
    argument error, not a wrapped allocation."""
    cfg, case = config.baseline(1)
    cfg = gpu_cfg(cfg, re_s=1e-7, re_l=1e-7)
    with pytest.raises(vm.MpsError) as e:
        vm.Solver(cfg, case)
    assert e.value.code & vm.MPS_ERR_ARG
