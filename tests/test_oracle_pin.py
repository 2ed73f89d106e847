"""The C restatement (oracle/mps_oracle.c) against golden outputs of the
reference's own CPU functions (tests/golden/make_golden.py).

Every floating-point field must match bit for bit: the restatement keeps the
reference's operation order, so any difference is a restatement error.
"""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# whole-step runs; the collision and .grd-input fixtures have their own tests
FILES = sorted(f for f in glob.glob(os.path.join(GOLDEN, "ref_*.npz"))
               if "snaps" in np.load(f).files)


def _digest(off, nbr):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off, np.int32).tobytes())
    h.update(np.ascontiguousarray(nbr, np.int32).tobytes())
    return h.hexdigest()


def _bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        return bool(np.array_equal(a.view(np.uint64), b.view(np.uint64)))
    return bool(np.array_equal(a, b))


def test_golden_fixtures_present():
    assert len(FILES) >= 8


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[4:-4] for f in FILES])
def test_oracle_matches_reference_bit_exact(path, oracle_mod):
    g = np.load(path)
    cfg = json.loads(str(g["cfg"]))
    case = {k: g["in_" + k] for k in ("x", "y", "z", "u", "v", "w", "p", "ptype")}
    case["dim"] = int(g["in_dim"])
    o = oracle_mod.Oracle(cfg, case)
    assert o.init() == 0
    assert o.scalar("n0_s") == float(g["n0"])
    off, nbr = o.get("off_s"), o.get("nbr_s")
    assert _bits_equal(off, g["init_off"])
    assert _digest(off, nbr) == str(g["init_digest"])
    if "init_nbr" in g:
        assert _bits_equal(nbr, g["init_nbr"])
    step = 0
    for s in g["snaps"]:
        while step < s:
            o.step()
            step += 1
        for key in g.files:
            if not key.startswith(f"s{s}_"):
                continue
            f = key[len(f"s{s}_"):]
            if f == "digest":
                assert _digest(o.get("off_s"), o.get("nbr_s")) == str(g[key]), f"lists @ step {s}"
                continue
            assert _bits_equal(o.get(f), g[key]), f"{f} differs at step {s}"
