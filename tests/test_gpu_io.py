"""Checkpoint/resume and the binary VTU snapshot on the GPU: a run resumed
from a checkpoint continues bit for bit; the asynchronous binary snapshot
holds the state of the step it was taken at (while later steps ran) and
agrees with the ASCII writer."""
import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import cases, config, files
from gpu_util import gpu_cfg

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "u", "v", "w", "p", "pnew", "phat", "rho", "n", "pold")


def _state(s):
    return {f: s.get(f) for f in FIELDS}


@pytest.mark.parametrize("which", ["dam2d", "dam3d", "batched"])
def test_resume_is_bit_exact(tmp_path, which):
    scenes = None
    if which == "dam2d":
        cfg, case = config.baseline(0)
    elif which == "dam3d":
        cfg, case = config.scaled_dam3d(1)
    else:
        l0 = 0.01
        sc = [cases.dam_break(2, l0, (w, h), (100, 60)) for w, h in ((10, 20), (25, 50))]
        base = config.reference_defaults(l0, 2)
        base.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=1e-4, gy=-9.81)
        cfg, case, sid, boxes, pmax = config.batched(base, sc)
        scenes = (sid, boxes, pmax)
    cfg = gpu_cfg(cfg, warm_start=2)
    a = vm.Solver(cfg, case)
    if scenes:
        a.set_scenes(*scenes)
    assert a.init() == 0
    for _ in range(4):
        assert a.step() == 0
    ck = tmp_path / "state.ck"
    a.save_checkpoint(str(ck))
    parsed = files.read_checkpoint(str(ck))
    assert parsed["steps"] == 4 and parsed["n"] == a.n
    assert np.array_equal(parsed["x"], a.get("x"))
    for _ in range(5):
        assert a.step() == 0
    b = vm.Solver(cfg)
    b.load_checkpoint(str(ck))
    assert b.scalar("steps") == 4
    assert b.scalar("n0_s") == a.scalar("n0_s") and b.scalar("n0_l") == a.scalar("n0_l")
    for _ in range(5):
        assert b.step() == 0
    sa, sb = _state(a), _state(b)
    for f in FIELDS:
        assert np.array_equal(sa[f], sb[f]), f
    a.close()
    b.close()


def test_checkpoint_rejects_corruption(tmp_path):
    cfg, case = config.baseline(0)
    a = vm.Solver(gpu_cfg(cfg), case)
    assert a.init() == 0
    ck = tmp_path / "c.ck"
    a.save_checkpoint(str(ck))
    raw = bytearray(open(ck, "rb").read())
    raw[len(raw) // 2] ^= 0x40
    open(ck, "wb").write(bytes(raw))
    b = vm.Solver(gpu_cfg(cfg))
    with pytest.raises(vm.MpsError):
        b.load_checkpoint(str(ck))
    a.close()
    b.close()


def _fnv1a64(data: bytes) -> int:
    h = 14695981039346656037
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_checkpoint_rejects_trailing_bytes(tmp_path):
    """Extra bytes between the payload and the checksum are refused even when
    the checksum is recomputed over them."""
    cfg, case = config.baseline(0)
    a = vm.Solver(gpu_cfg(cfg), case)
    assert a.init() == 0
    ck = tmp_path / "c.ck"
    a.save_checkpoint(str(ck))
    raw = open(ck, "rb").read()
    payload = raw[:-8] + b"\0" * 16
    assert _fnv1a64(raw[:-8]) == int.from_bytes(raw[-8:], "little")  # the format's checksum
    open(ck, "wb").write(payload + _fnv1a64(payload).to_bytes(8, "little"))
    b = vm.Solver(gpu_cfg(cfg))
    with pytest.raises(vm.MpsError) as e:
        b.load_checkpoint(str(ck))
    assert e.value.code & vm.MPS_ERR_IO
    a.close()
    b.close()


@pytest.mark.parametrize("which", ["dam2d", "dam3d"])
def test_binary_snapshot_matches_state_and_ascii(tmp_path, which):
    cfg, case = config.baseline(0) if which == "dam2d" else config.scaled_dam3d(1)
    s = vm.Solver(gpu_cfg(cfg), case)
    assert s.init() == 0
    s.set_graph(True)
    for _ in range(3):
        assert s.step() == 0
    want = {f: s.get(f) for f in ("x", "y", "z", "u", "v", "w", "p")}
    pt = s.get("ptype")
    s.snapshot_vtu(str(tmp_path / "snap.vtu"))
    s.write_vtu(str(tmp_path / "ascii.vtu"))
    for _ in range(3):  # the write overlaps these steps
        assert s.step() == 0
    assert s.wait_io() == 0
    got = files.read_vtu_binary(str(tmp_path / "snap.vtu"))
    asc = files.read_vtu_ascii(str(tmp_path / "ascii.vtu"))
    three = cfg["dim"] == 3
    pos = np.stack([want["x"], want["y"], want["z"] if three else 0 * want["x"]], 1)
    vel = np.stack([want["u"], want["v"], want["w"] if three else 0 * want["u"]], 1)
    assert np.array_equal(got["Position"], pos.astype(np.float32))
    assert np.array_equal(got["Velocity"], vel.astype(np.float32))
    assert np.array_equal(got["Pressure"], want["p"].astype(np.float32))
    assert np.array_equal(got["partType"], pt)
    assert np.array_equal(got["connectivity"], np.arange(len(pt)))
    assert np.allclose(asc["Position"], got["Position"], rtol=1e-7, atol=0)
    assert np.array_equal(asc["partType"], got["partType"])
    s.close()


@pytest.mark.parametrize("which", ["dam2d", "dam3d"])
def test_state_round_trip(which):
    """mps_get_state / mps_set_state (the calls of a caller that keeps the
    state on the host between steps): the state comes back in caller order
    as the per-field downloads give it; a modified state goes in, comes back
    unchanged, p also becomes CG's next guess (pnew), and stepping from it
    equals stepping from the same values set field by field."""
    cfg, case = config.baseline(0) if which == "dam2d" else config.scaled_dam3d(1)
    names = ("x", "y", "z", "u", "v", "w", "p")
    a, b = vm.Solver(gpu_cfg(cfg), case), vm.Solver(gpu_cfg(cfg), case)
    assert a.init() == 0 and b.init() == 0
    for _ in range(3):
        assert a.step() == 0 and b.step() == 0
    n = len(case["x"])
    host = {k: np.zeros(n) for k in names}
    a.get_state(*[host[k].ctypes.data for k in names])
    for k in names:
        if which == "dam2d" and k in ("z", "w"):
            continue
        assert np.array_equal(host[k], a.get(k)), k
    host["u"] += 1e-3
    host["p"] *= 0.5
    a.set_state(*[host[k].ctypes.data for k in names])
    back = {k: np.zeros(n) for k in names}
    a.get_state(*[back[k].ctypes.data for k in names])
    for k in names:
        if which == "dam2d" and k in ("z", "w"):
            continue
        assert np.array_equal(back[k], host[k]), k
    assert np.array_equal(a.get("pnew"), host["p"])
    for k in names:
        if which == "dam2d" and k in ("z", "w"):
            continue
        b.set(k, host[k])
    b.set("pnew", host["p"])
    assert a.step() == 0 and b.step() == 0
    for k in names:
        assert np.array_equal(a.get(k), b.get(k)), k
    a.close()
    b.close()


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("which", ["dam2d", "dam3d"])
def test_step_io_equals_set_step_get(which, graph):
    """mps_step_io (state in host arrays, velocities and pressure copied
    beside the neighbour search) equals mps_set_state + mps_step +
    mps_get_state bit for bit, with the host state changed between steps
    (so that the copied values, not the device's own, are the ones used),
    and with the pressure left out of one step's input."""
    cfg, case = config.baseline(0) if which == "dam2d" else config.scaled_dam3d(1)
    names = ("x", "y", "z", "u", "v", "w", "p")
    a, b = vm.Solver(gpu_cfg(cfg), case), vm.Solver(gpu_cfg(cfg), case)
    assert a.init() == 0 and b.init() == 0
    a.set_graph(graph)
    b.set_graph(graph)
    n = len(case["x"])
    ha = {k: np.zeros(n) for k in names}
    hb = {k: np.zeros(n) for k in names}
    a.get_state(*[ha[k].ctypes.data for k in names])
    b.get_state(*[hb[k].ctypes.data for k in names])
    for step in range(6):
        for h in (ha, hb):
            h["u"] += 1e-4
            h["p"] *= 0.9
        ins_a = [ha[k].ctypes.data for k in names]
        ins_b = [hb[k].ctypes.data for k in names]
        if step == 3:  # the pressure stays the device's own
            ins_a[6] = ins_b[6] = 0
        assert a.set_state(*ins_a) == 0
        ra = a.step()
        assert a.get_state(*[ha[k].ctypes.data for k in names]) == 0
        rb = b.step_io(ins_b, [hb[k].ctypes.data for k in names])
        assert ra == rb == 0
        for k in names:
            assert np.array_equal(ha[k].view(np.uint64), hb[k].view(np.uint64)), (step, k)
    assert np.array_equal(a.get("pnew"), b.get("pnew"))
    a.close()
    b.close()
