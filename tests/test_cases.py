"""Case generator, .grd round trip and the benchmark geometries."""
import os

import numpy as np

from voxarmps_b200 import cases, config


def test_config0_geometry():
    cfg, case = config.baseline(0)
    c = cases.counts(case)
    assert c["FP"] == 1250
    assert c["TP"] == 1928
    assert cases.check_order(case)
    assert cfg["xmin"] == -0.01 and abs(cfg["xmax"] - 1.06) < 1e-12
    assert cfg["re_s"] == 2.1 * 0.01 and cfg["re_l"] == 4.0 * 0.01


def test_config1_counts_without_building_full_arrays():
    # 80 x 160 x 80 fluid, 320 x 200 x 80 interior, 3 boundary layers
    fp = 80 * 160 * 80
    solid = (326 * 203 * 86) - (320 * 200 * 80)
    assert fp == 1_024_000
    assert fp + solid == 1_595_308


def test_small_3d_case_layers():
    case = cases.dam_break(3, 0.005, (4, 6, 4), (10, 8, 6))
    c = cases.counts(case)
    assert c["FP"] == 96
    assert cases.check_order(case)
    pt = case["ptype"]
    # every wall particle touches the interior, dummies lie outside walls
    assert (pt == 0).sum() > 0 and (pt == -1).sum() > (pt == 0).sum()


def test_grd_round_trip(tmp_path):
    _, case = config.baseline(0)
    p = os.path.join(tmp_path, "c0.grd")
    cases.write_grd(p, case)
    back = cases.read_grd(p, 2)
    for k in ("x", "y", "u", "v", "p"):
        assert np.array_equal(back[k], case[k])
    assert np.array_equal(back["ptype"], case["ptype"])


def test_lattice_neighbour_counts():
    assert cases.lattice_neighbours(2, 2.1) == 12
    assert cases.lattice_neighbours(2, 4.0) == 44
    assert cases.lattice_neighbours(3, 2.1) == 32
    assert cases.lattice_neighbours(3, 4.0) == 250


def test_batched_scenes_deterministic():
    a = cases.batched_dam_scenes(4, seed=0)
    b = cases.batched_dam_scenes(4, seed=0)
    assert [len(s["x"]) for s in a] == [len(s["x"]) for s in b]
    fl = [cases.counts(s)["FP"] for s in cases.batched_dam_scenes(64, seed=0)]
    assert min(fl) >= 800 and max(fl) <= 9600
