"""Readers for the solver's binary outputs (checkpoint and appended-binary
VTU; layouts documented in include/voxarmps.h and mps_context.cu).  They
serve tests and inspection: the checkpoint hash is checked byte by byte in
Python, which takes seconds per hundred megabytes."""
from __future__ import annotations

import re
import struct

import numpy as np

from . import config

# per-particle fields in file order (the PND field "n" is returned as "pnd")
CK_FIELDS = ["x", "y", "z", "u", "v", "w", "p", "pnew", "phat", "un", "vn", "wn", "rho", "pnd",
             "pold"]


def fnv1a64(data: bytes) -> int:
    """64-bit FNV-1a (Fowler, Noll, Vo) of a byte string."""
    h = 14695981039346656037
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def read_checkpoint(path: str) -> dict:
    """Parse a checkpoint; raises ValueError on a bad magic, version, layout
    or checksum."""
    from . import MpsConfig
    raw = open(path, "rb").read()
    if len(raw) < 16:
        raise ValueError("truncated")
    (want,) = struct.unpack_from("<Q", raw, len(raw) - 8)
    if fnv1a64(raw[:-8]) != want:
        raise ValueError("checksum mismatch")
    if raw[:8] != b"VXMPSCK1":
        raise ValueError("not a checkpoint")
    version, cb = struct.unpack_from("<II", raw, 8)
    if version != 1:
        raise ValueError("unsupported version")
    import ctypes as C
    if cb != C.sizeof(MpsConfig):
        raise ValueError("configuration layout differs")
    o = 16
    cfg_s = MpsConfig.from_buffer_copy(raw[o:o + cb])
    o += cb
    n, ns, steps = struct.unpack_from("<iiq", raw, o)
    o += 16
    n0_s, n0_l = struct.unpack_from("<dd", raw, o)
    o += 16
    out = {"config": {f: getattr(cfg_s, f) for f, _ in config.FIELDS}, "n": n, "nscenes": ns,
           "steps": steps, "n0_s": n0_s, "n0_l": n0_l}
    for f in CK_FIELDS:
        out[f] = np.frombuffer(raw, np.float64, n, o).copy()
        o += 8 * n
    for f in ("ptype", "scene"):
        out[f] = np.frombuffer(raw, np.int32, n, o).copy()
        o += 4 * n
    if ns > 1:
        out["boxes"] = np.frombuffer(raw, np.float64, 6 * ns, o).reshape(ns, 6).copy()
        o += 48 * ns
        out["pmax"] = np.frombuffer(raw, np.float64, ns, o).copy()
        o += 8 * ns
    if o != len(raw) - 8:
        raise ValueError("size mismatch")
    return out


_TYPES = {"Float32": np.float32, "Int32": np.int32, "UInt8": np.uint8}


def read_vtu_binary(path: str) -> dict:
    """Arrays of a VTU file with raw appended data and UInt64 headers."""
    raw = open(path, "rb").read()
    start = raw.index(b"<AppendedData")
    base = raw.index(b"_", start) + 1
    head = raw[:start].decode()
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: NumberOfComponents="(\d+)")? '
                         r'Name="(\w+)" format="appended" offset="(\d+)"/>', head):
        typ, comp, name, off = m.group(1), int(m.group(2) or 1), m.group(3), int(m.group(4))
        (nbytes,) = struct.unpack_from("<Q", raw, base + off)
        a = np.frombuffer(raw, _TYPES[typ], nbytes // np.dtype(_TYPES[typ]).itemsize,
                          base + off + 8).copy()
        out[name] = a.reshape(-1, comp) if comp > 1 else a
    return out


def read_vtu_ascii(path: str) -> dict:
    """Arrays of the ASCII VTU written by mps_write_vtu."""
    txt = open(path).read()
    out = {}
    for m in re.finditer(r"<DataArray NumberOfComponents='(\d+)' type='(\w+)' Name='(\w+)' "
                         r"format='ascii'>\n(.*?)\n", txt, re.S):
        comp, typ, name, body = int(m.group(1)), m.group(2), m.group(3), m.group(4)
        a = np.array(body.split(), dtype=np.float64 if typ == "Float32" else np.int64)
        out[name] = a.reshape(-1, comp) if comp > 1 else a
    return out
