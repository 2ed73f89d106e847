"""Checkpoint layout and reader (CPU): a file assembled byte by byte from the
documented layout parses back, and corruption is detected."""
import ctypes as C
import struct

import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import config, files


def _write(path, n=5, ns=2, steps=42):
    cfg = vm.MpsConfig()
    for f, _ in config.FIELDS:
        setattr(cfg, f, 1 if f == "dim" else 0)
    cfg.dim = 2
    body = b"VXMPSCK1" + struct.pack("<II", 1, C.sizeof(cfg)) + bytes(cfg)
    body += struct.pack("<iiqdd", n, ns, steps, 35.6, 6.5)
    fields = {}
    for k, f in enumerate(files.CK_FIELDS):
        fields[f] = np.arange(n, dtype=np.float64) + 10 * k
        body += fields[f].tobytes()
    pt = np.array([-1, 0, 1, 1, 2], np.int32)[:n]
    sc = (np.arange(n) % ns).astype(np.int32)
    body += pt.tobytes() + sc.tobytes()
    boxes = np.arange(6 * ns, dtype=np.float64)
    pmax = np.full(ns, 99.0)
    body += boxes.tobytes() + pmax.tobytes()
    body += struct.pack("<Q", files.fnv1a64(body))
    open(path, "wb").write(body)
    return fields, pt, sc


def test_checkpoint_reader_roundtrip(tmp_path):
    p = tmp_path / "a.ck"
    fields, pt, sc = _write(p)
    ck = files.read_checkpoint(str(p))
    assert ck["n"] == 5 and ck["nscenes"] == 2 and ck["steps"] == 42
    assert ck["n0_s"] == 35.6 and ck["config"]["dim"] == 2
    for f in files.CK_FIELDS:
        assert np.array_equal(ck[f], fields[f])
    assert np.array_equal(ck["ptype"], pt) and np.array_equal(ck["scene"], sc)
    assert ck["boxes"].shape == (2, 6) and ck["pmax"][1] == 99.0


def test_checkpoint_corruption_detected(tmp_path):
    p = tmp_path / "b.ck"
    _write(p)
    raw = bytearray(open(p, "rb").read())
    raw[100] ^= 0x01
    open(p, "wb").write(bytes(raw))
    with pytest.raises(ValueError, match="checksum"):
        files.read_checkpoint(str(p))


def test_fnv1a64_known_answers():
    # published FNV-1a 64-bit test vectors
    assert files.fnv1a64(b"") == 0xCBF29CE484222325
    assert files.fnv1a64(b"a") == 0xAF63DC4C8601EC8C
    assert files.fnv1a64(b"foobar") == 0x85944171F73967E8
