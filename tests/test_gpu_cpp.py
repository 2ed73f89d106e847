"""The reference's loop written in C++ against include/voxarmps.h
(tests/cpp/main_loop.cpp: mps_create, mps_load_grd, mps_init, then mps_step
or the fourteen per-stage entries in main.cu's order, mps_get_state into
1-based arrays), compiled with g++, linked to the library and run on the
GPU: its state equals the Python binding's bit for bit (needs a B200)."""
import os
import subprocess

import numpy as np
import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import cases, config
from gpu_util import gpu_cfg

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "voxarmps_b200")


def build_driver(tmp_path):
    exe = str(tmp_path / "main_loop")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "main_loop.cpp"), "-L", LIBDIR,
                    "-lvoxarmps_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def read_out(path):
    with open(path, "rb") as f:
        n = int(np.frombuffer(f.read(4), np.int32)[0])
        a = np.frombuffer(f.read(), np.float64).reshape(7, n)
    return dict(zip(("x", "y", "z", "u", "v", "w", "p"), a))


@pytest.mark.parametrize("mode", ["step", "stages"])
def test_cpp_loop_equals_python_binding(tmp_path, mode):
    exe = build_driver(tmp_path)
    cfg, case = config.baseline(0)
    cfg = gpu_cfg(cfg)
    grd = str(tmp_path / "dam.grd")
    cases.write_grd(grd, case)
    blob = tmp_path / "config.bin"
    blob.write_bytes(bytes(vm.MpsConfig(**{k: cfg[k] for k, _ in config.FIELDS})))
    out = str(tmp_path / "out.bin")
    steps = 10
    r = subprocess.run([exe, str(blob), grd, str(steps), mode, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = read_out(out)
    g = vm.Solver(cfg, case)
    assert g.init() == 0
    for _ in range(steps):
        assert g.step() == 0
    for k in ("x", "y", "u", "v", "p"):
        assert np.array_equal(got[k].view(np.uint64), g.get(k).view(np.uint64)), k
