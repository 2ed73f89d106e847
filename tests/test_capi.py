"""The C-ABI library: loads, exports every symbol include/voxarmps.h declares,
and the ctypes mirror of mps_config has the C layout.  No GPU needed."""
import os
import re
import subprocess
import ctypes as C

import pytest

import voxarmps_b200 as vm
from voxarmps_b200 import build, config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "voxarmps.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void\*|const char\*)\s+(mps_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return vm.load_library()


def test_library_exports_all_declared(lib):
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    assert sorted(vm.EXPORTS) == sorted(names)


def test_config_layout_matches_c(tmp_path):
    src = tmp_path / "lay.c"
    fields = [n for n, _ in config.FIELDS]
    body = "\n".join(f'printf("%s %zu\\n", "{f}", offsetof(mps_config, {f}));' for f in fields)
    src.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "{HEADER}"\n'
                   f'int main(void){{ {body} printf("SIZE %zu\\n", sizeof(mps_config)); return 0; }}\n')
    exe = tmp_path / "lay"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split() for line in out if line.strip())
    for f in fields:
        assert int(got[f]) == getattr(vm.MpsConfig, f).offset, f
    assert int(got["SIZE"]) == C.sizeof(vm.MpsConfig)


def test_tuning_layout_matches_c(tmp_path):
    src = tmp_path / "tun.c"
    fields = [n for n, _ in vm.MpsTuning._fields_]
    body = "\n".join(f'printf("%s %zu\\n", "{f}", offsetof(mps_tuning, {f}));' for f in fields)
    src.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "{HEADER}"\n'
                   f'int main(void){{ {body} printf("SIZE %zu\\n", sizeof(mps_tuning)); return 0; }}\n')
    exe = tmp_path / "tun"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split() for line in out if line.strip())
    for f in fields:
        assert int(got[f]) == getattr(vm.MpsTuning, f).offset, f
    assert int(got["SIZE"]) == C.sizeof(vm.MpsTuning)


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError):
        vm._LIB_SAVE = vm._LIB
        try:
            vm._LIB = None
            vm.load_library(str(tmp_path / "nope.so"))
        finally:
            vm._LIB = vm._LIB_SAVE


def test_invalid_config_rejected_without_gpu(lib):
    cfg = config.reference_defaults(0.01, 2)
    cfg.update(dim=4, solver=1)
    c = vm.MpsConfig(**{k: cfg[k] for k, _ in config.FIELDS})
    h = C.c_void_p()
    assert lib.mps_create(C.byref(c), 0, C.byref(h)) == vm.MPS_ERR_ARG


def test_status_codes_match_header():
    """Every MPS_OK / MPS_ERR_* bit the header defines has the same value in
    the Python layer, and the bits are distinct powers of two."""
    text = open(HEADER).read()
    codes = {k: int(v) for k, v in re.findall(r"#define\s+(MPS_(?:OK|ERR_\w+))\s+(\d+)", text)}
    assert codes["MPS_OK"] == 0 and len(codes) >= 9
    for name, value in codes.items():
        assert getattr(vm, name) == value, name
    bits = [v for k, v in codes.items() if k != "MPS_OK"]
    assert len(set(bits)) == len(bits)
    assert all(b > 0 and b & (b - 1) == 0 for b in bits)
    assert vm.FATAL == codes["MPS_ERR_ARG"] | codes["MPS_ERR_CUDA"] | codes["MPS_ERR_IO"]


def test_cpp_driver_compiles_and_links(tmp_path):
    """tests/cpp/main_loop.cpp (the reference's loop in C++ against the
    header) compiles and links against the library; it runs in
    tests/test_gpu_cpp.py."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "voxarmps_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I",
                    os.path.join(root, "include"), os.path.join(root, "tests", "cpp", "main_loop.cpp"),
                    "-L", libdir, "-lvoxarmps_b200", "-o", str(tmp_path / "main_loop")], check=True)
