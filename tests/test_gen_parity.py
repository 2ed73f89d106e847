"""The reference's scenario generators (generateSimulationCases), restated in
voxarmps_b200/gen.py, against the reference's own generator compiled from
its sources (oracle/Makefile target `gen`, run here where the sources are):
same particle count, order, kinds, velocities and coordinates (the
reference's 6-decimal "%lf" values, exactly)."""
import os
import subprocess

import numpy as np
import pytest

import pyoracle
from voxarmps_b200 import gen

ORACLE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")
GEN_EXE = os.path.join(ORACLE, "_ref", "gen")
REF_SRC = pyoracle.reference_path("generateSimulationCases", "generateSimulationCases")


@pytest.fixture(scope="module")
def ref_gen():
    if not os.path.isdir(REF_SRC):
        pytest.skip("reference generator sources not present")
    subprocess.run(["make", "-s", "-C", ORACLE, f"REFERENCE={pyoracle.REFERENCE_ROOT}", "gen"],
                   check=True)
    return GEN_EXE


def _read(path, dim):
    with open(path) as f:
        lines = f.read().split("\n")
    header = lines[0].split()[0]
    rows = [ln.split() for ln in lines[1:] if ln.strip()]
    a = np.array(rows, dtype=np.float64)
    return header, a


CASES = [("dam_break_2d", 0.01, 1), ("dam_break_2d", 0.004, 2), ("rt_instability_2d", 0.01, 1),
         ("shear_cavity_2d", 0.01, 1), ("shear_cavity_2d", 0.005, 2), ("water_drop_2d", 0.01, 1),
         ("water_drop_2d", 0.01, 2), ("poiseuille_2d", 0.001, 1), ("oil_spill_2d", 0.004, 1),
         ("dam_break_3d", 0.02, 1), ("dam_break_3d", 0.01, 2), ("dam_break_3d_offset", 0.02, 1)]


@pytest.mark.parametrize("name,dl,mult", CASES)
def test_generator_matches_reference(ref_gen, tmp_path, name, dl, mult):
    out = tmp_path / f"{name}.grd"
    subprocess.run([ref_gen, name, repr(dl), str(mult), str(out)], check=True,
                   capture_output=True, cwd=tmp_path)
    c = gen.GENERATORS[name](dl, mult)
    dim = c["dim"]
    header, a = _read(out, dim)
    n = len(c["x"])
    assert a.shape == (n, 8 if dim == 3 else 6)
    if name != "oil_spill_2d":  # the reference prints a double with %d there
        assert int(header) == c["header"]
    if dim == 3:
        cols = {"x": 0, "y": 1, "z": 2, "ptype": 3, "u": 4, "v": 5, "w": 6, "p": 7}
    else:
        cols = {"x": 0, "y": 1, "ptype": 2, "u": 3, "v": 4, "p": 5}
    for f, k in cols.items():
        want = a[:, k]
        got = np.asarray(c[f], np.float64)
        if name == "poiseuille_2d" and f == "y":
            mp = int(140 * mult)
            want, got = want[mp:], got[mp:]  # the reference's first row has no y
        assert np.array_equal(got, want), f
