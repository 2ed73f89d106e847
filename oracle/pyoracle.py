"""ctypes bindings for the oracle libraries (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm import this module.  The product package never does.

* ``Oracle``  -- the C restatement in ``oracle/liboracle.so`` (mps_oracle.c).
* ``RefHarness`` -- the reference's own CPU functions in
  ``oracle/_ref/libref.so`` (sequential) or ``libref_omp.so`` (OpenMP),
  driven in main.cu's loop order by ``oracle/ref_harness.cpp``.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libref.so")
LIB_REF_OMP = os.path.join(HERE, "_ref", "libref_omp.so")

# Where the reference's sources lie: the environment variable
# VOXARMPS_REFERENCE, by default /root/reference.  Only the recipes that
# compile the reference (oracle/Makefile) and the scripts that read its
# inputs (tests/golden/make_golden.py, the generator parity test) use it.
REFERENCE_ROOT = os.environ.get("VOXARMPS_REFERENCE", "/root/reference")


def reference_path(*parts: str) -> str:
    """A path under the reference's source tree."""
    return os.path.join(REFERENCE_ROOT, *parts)


class MoParams(C.Structure):
    """Mirror of ``mo_params`` in mps_oracle.h (field order matters)."""

    _fields_ = [
        ("dim", C.c_int), ("ktype", C.c_int), ("method", C.c_int),
        ("l0", C.c_double), ("re_s", C.c_double), ("re_l", C.c_double),
        ("delta", C.c_double), ("dt", C.c_double),
        ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
        ("rho1", C.c_double), ("rho2", C.c_double), ("nu1", C.c_double), ("nu2", C.c_double),
        ("beta_fs", C.c_double), ("dirichlet", C.c_double), ("relaxp", C.c_double),
        ("kh", C.c_int), ("vmax", C.c_double), ("coll", C.c_double), ("cc", C.c_double),
        ("velcor", C.c_double), ("ncorrection", C.c_double),
        ("pmin", C.c_double), ("pmax", C.c_double), ("c01", C.c_double), ("c02", C.c_double),
        ("turb", C.c_int), ("cs", C.c_double), ("fluid2_type", C.c_int),
        ("n_pl", C.c_double), ("meu0", C.c_double), ("phi", C.c_double), ("cohes", C.c_double),
        ("matopt", C.c_int), ("srcopt", C.c_int), ("fraction_method", C.c_int),
        ("ppe_at_predicted", C.c_int), ("warm_start", C.c_int), ("solver", C.c_int),
        ("cg_tol", C.c_double), ("cg_max", C.c_int), ("imin", C.c_int), ("imax", C.c_int),
        ("eps", C.c_double), ("collision_gather", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
    ]


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and the reference libraries when ``ref``)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE, f"REFERENCE={REFERENCE_ROOT}"] + targets,
                   check=True)


def params_from(cfg: dict) -> MoParams:
    """Fill MoParams from a solver-config dict (voxarmps_b200.config keys)."""
    P = MoParams()
    for name, _ in MoParams._fields_:
        if name in cfg:
            setattr(P, name, cfg[name])
    return P


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
INT_FIELDS = {"ptype", "bcon", "cell_s", "perm_s", "cell_l", "perm_l", "off_s", "off_l",
              "nbr_s", "nbr_l", "off", "nbr"}


def _load_oracle():
    if not os.path.exists(LIB_ORACLE):
        build()
    lib = C.CDLL(LIB_ORACLE)
    lib.mo_create.restype = C.c_void_p
    lib.mo_create.argtypes = [C.POINTER(MoParams), C.c_int, _DP, _DP, _DP, _IP, _DP, _DP, _DP, _DP]
    lib.mo_destroy.argtypes = [C.c_void_p]
    lib.mo_init.argtypes = [C.c_void_p]
    lib.mo_step.argtypes = [C.c_void_p]
    lib.mo_get.restype = C.c_long
    lib.mo_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
    lib.mo_set.restype = C.c_long
    lib.mo_set.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
    lib.mo_scalar.restype = C.c_double
    lib.mo_scalar.argtypes = [C.c_void_p, C.c_char_p]
    lib.mo_W.restype = C.c_double
    lib.mo_W.argtypes = [C.c_double, C.c_int, C.c_int, C.c_double]
    lib.mo_neighbor.restype = C.c_int
    lib.mo_neighbor.argtypes = [C.POINTER(MoParams), C.c_double, C.c_int, _DP, _DP, _DP, _IP,
                                _IP, _IP, _IP, C.c_int]
    lib.mo_grid.restype = C.c_int
    lib.mo_grid.argtypes = [C.POINTER(MoParams), C.c_double, _IP, _IP, _IP]
    lib.mo_cg.restype = C.c_int
    lib.mo_cg.argtypes = [C.c_int, _IP, _IP, _IP, _DP, _DP, _DP, _DP, C.c_double, C.c_int,
                          C.c_int, _DP]
    lib.mo_relres.restype = C.c_double
    lib.mo_relres.argtypes = [C.c_int, _IP, _IP, _IP, _DP, _DP, _DP, _DP]
    lib.mo_matrix.argtypes = [C.POINTER(MoParams), C.c_double, C.c_double, C.c_double, C.c_int,
                              _IP, _IP, _DP, _DP, _DP, _IP, _DP, _DP]
    lib.mo_lambda.restype = C.c_double
    lib.mo_lambda.argtypes = [C.c_int, C.c_double]
    lib.mo_incdecom.argtypes = [C.c_int, _IP, _IP, _IP, _DP, _DP, _DP, _DP]
    lib.mo_iccg.restype = C.c_int
    lib.mo_iccg.argtypes = [C.c_int, _IP, _IP, _IP, _DP, _DP, _DP, _DP, _DP, _DP, C.c_double,
                            C.c_int, _DP]
    for name in ("mo_collision", "mo_collision_gather"):
        getattr(lib, name).argtypes = [C.POINTER(MoParams), C.c_int, _IP, _IP, _IP, _DP, _DP,
                                       _DP, _DP, _DP, _DP]
    return lib


_ORACLE = None


def oracle_lib():
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = _load_oracle()
    return _ORACLE


class _StateBase:
    h = None

    def _arrays(self, case):
        n = len(case["x"])
        f = lambda k: np.ascontiguousarray(case[k], dtype=np.float64) if k in case else np.zeros(n)
        self._keep = [f("x"), f("y"), f("z"), np.ascontiguousarray(case["ptype"], dtype=np.int32),
                      f("u"), f("v"), f("w"), f("p")]
        return n, self._keep


class Oracle(_StateBase):
    """The C restatement, stepped like main.cu's loop."""

    def __init__(self, cfg: dict, case: dict):
        self.lib = oracle_lib()
        self.P = params_from(cfg)
        n, (x, y, z, pt, u, v, w, p) = self._arrays(case)
        self.n = n
        self.h = self.lib.mo_create(C.byref(self.P), n, _dp(x), _dp(y), _dp(z), _ip(pt), _dp(u),
                                    _dp(v), _dp(w), _dp(p))

    def init(self):
        return self.lib.mo_init(self.h)

    def step(self):
        return self.lib.mo_step(self.h)

    def get(self, name):
        cnt = self.lib.mo_get(self.h, name.encode(), None)
        if cnt < 0:
            raise KeyError(name)
        out = np.empty(cnt, dtype=np.int32 if name in INT_FIELDS else np.float64)
        self.lib.mo_get(self.h, name.encode(), out.ctypes.data_as(C.c_void_p))
        return out

    def set(self, name, arr):
        arr = np.ascontiguousarray(arr, dtype=np.int32 if name in INT_FIELDS else np.float64)
        if self.lib.mo_set(self.h, name.encode(), arr.ctypes.data_as(C.c_void_p)) < 0:
            raise KeyError(name)

    def scalar(self, name):
        return self.lib.mo_scalar(self.h, name.encode())

    def close(self):
        if self.h:
            self.lib.mo_destroy(self.h)
            self.h = None

    __del__ = close


_REF = {}


def ref_available(omp: bool = False) -> bool:
    return os.path.exists(LIB_REF_OMP if omp else LIB_REF)


def _load_ref(omp: bool):
    path = LIB_REF_OMP if omp else LIB_REF
    if path not in _REF:
        lib = C.CDLL(path)
        lib.rh_create.restype = C.c_void_p
        lib.rh_create.argtypes = [C.POINTER(MoParams), C.c_int, _DP, _DP, _DP, _IP, _DP, _DP, _DP,
                                  _DP, C.c_int]
        lib.rh_init.argtypes = [C.c_void_p]
        lib.rh_step.argtypes = [C.c_void_p]
        lib.rh_get.restype = C.c_long
        lib.rh_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        lib.rh_scalar.restype = C.c_double
        lib.rh_scalar.argtypes = [C.c_void_p, C.c_char_p]
        lib.rh_destroy.argtypes = [C.c_void_p]
        lib.rh_set.restype = C.c_long
        lib.rh_set.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        lib.rh_stage.argtypes = [C.c_void_p, C.c_char_p]
        _REF[path] = lib
    return _REF[path]


class RefHarness(_StateBase):
    """The reference's own CPU functions (single support radius re_s)."""

    def __init__(self, cfg: dict, case: dict, nthreads: int = 1):
        self.lib = _load_ref(nthreads > 1)
        self.P = params_from(cfg)
        n, (x, y, z, pt, u, v, w, p) = self._arrays(case)
        self.n = n
        self.h = self.lib.rh_create(C.byref(self.P), n, _dp(x), _dp(y), _dp(z), _ip(pt), _dp(u),
                                    _dp(v), _dp(w), _dp(p), nthreads)

    def init(self):
        return self.lib.rh_init(self.h)

    def step(self):
        return self.lib.rh_step(self.h)

    def get(self, name):
        cnt = self.lib.rh_get(self.h, name.encode(), None)
        if cnt < 0:
            raise KeyError(name)
        out = np.empty(cnt, dtype=np.int32 if name in INT_FIELDS else np.float64)
        self.lib.rh_get(self.h, name.encode(), out.ctypes.data_as(C.c_void_p))
        return out

    def scalar(self, name):
        return self.lib.rh_scalar(self.h, name.encode())

    def set(self, name, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        if self.lib.rh_set(self.h, name.encode(), arr.ctypes.data_as(C.c_void_p)) < 0:
            raise KeyError(name)

    def stage(self, name):
        """One reference routine by its name ("NEIGHBOR", "COLLISION2")."""
        if self.lib.rh_stage(self.h, name.encode()) != 0:
            raise KeyError(name)

    def close(self):
        if self.h:
            self.lib.rh_destroy(self.h)
            self.h = None

    __del__ = close


def collision(cfg: dict, off, nbr, ptype, un, vn, wn, x, y, z, gather: bool = False):
    """COLLISION2 on copies of the inputs: the sequential in-place form
    (mo_collision) or the order-independent gather (mo_collision_gather).
    Returns (un, vn, wn, x, y, z)."""
    lib = oracle_lib()
    P = params_from(cfg)
    a = [np.array(v, np.float64) for v in (un, vn, wn, x, y, z)]
    fn = lib.mo_collision_gather if gather else lib.mo_collision
    fn(C.byref(P), len(a[0]), _ip(np.ascontiguousarray(off, np.int32)),
       _ip(np.ascontiguousarray(nbr, np.int32)), _ip(np.ascontiguousarray(ptype, np.int32)),
       *[_dp(v) for v in a])
    return tuple(a)


def ppe_system(cfg: dict, o: "Oracle"):
    """The PPE system of the oracle's last step: (off, nbr, bcon, diag, val, b,
    p) with A assembled at the predicted positions on the Laplacian list, as
    the step solved it (functions.cu:869-1133)."""
    lib = oracle_lib()
    P = params_from(cfg)
    n = o.n
    off, nbr = o.get("off_l"), o.get("nbr_l")
    xs, ys, zs = o.get("xs"), o.get("ys"), o.get("zs")
    bcon, b, p = o.get("bcon"), o.get("source"), o.get("pnew")
    diag, val = np.zeros(n), np.zeros(max(len(nbr), 1))
    lib.mo_matrix(C.byref(P), cfg["re_l"], lib.mo_lambda(cfg["ktype"], cfg["re_l"]),
                  o.scalar("n0_l"), n, _ip(off), _ip(nbr), _dp(xs), _dp(ys), _dp(zs), _ip(bcon),
                  _dp(diag), _dp(val))
    return off, nbr, bcon, diag, val, b, p


def solver_iterations(off, nbr, bcon, diag, val, b, x0, tol=1e-8, maxit=5000):
    """Iterations to ||b-Ax||/||b|| <= tol from x0: the reference's ICCG
    (IC(0) preconditioner) against Jacobi-PCG and plain CG."""
    lib = oracle_lib()
    n = len(diag)
    out = {}
    icd, icv = np.zeros(n), np.zeros(max(len(nbr), 1))
    lib.mo_incdecom(n, _ip(off), _ip(nbr), _ip(bcon), _dp(diag), _dp(val), _dp(icd), _dp(icv))
    rr = C.c_double()
    x = np.array(x0, np.float64)
    out["iccg"] = lib.mo_iccg(n, _ip(off), _ip(nbr), _ip(bcon), _dp(diag), _dp(val), _dp(icd),
                              _dp(icv), _dp(b), _dp(x), tol, maxit, C.byref(rr))
    out["iccg_relres"] = rr.value
    for name, pre in (("jacobi", 1), ("plain", 0)):
        x = np.array(x0, np.float64)
        out[name] = lib.mo_cg(n, _ip(off), _ip(nbr), _ip(bcon), _dp(diag), _dp(val), _dp(b),
                              _dp(x), tol, maxit, pre, C.byref(rr))
        out[name + "_relres"] = rr.value
    return out


def W(r, ktype, dim, re):
    return oracle_lib().mo_W(r, ktype, dim, re)


def neighbor(cfg: dict, re: float, x, y, z=None):
    """Cells (1-based Cnum), permutation and CSR lists per NEIGHBOR."""
    lib = oracle_lib()
    P = params_from(cfg)
    n = len(x)
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    z = np.ascontiguousarray(z if z is not None else np.zeros(n), np.float64)
    cell = np.zeros(n, np.int32)
    perm = np.zeros(n, np.int32)
    off = np.zeros(n + 1, np.int32)
    cap = max(64 * n, 1)
    while True:
        nbr = np.zeros(cap, np.int32)
        r = lib.mo_neighbor(C.byref(P), re, n, _dp(x), _dp(y), _dp(z), _ip(cell), _ip(perm),
                            _ip(off), _ip(nbr), cap)
        if r == -2147483647:
            raise ValueError("particle outside the cell grid")
        if r >= 0:
            return cell, perm, off, nbr[:r].copy()
        cap = -r + 16


def grid(cfg: dict, re: float):
    P = params_from(cfg)
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    tnc = oracle_lib().mo_grid(C.byref(P), re, C.byref(a), C.byref(b), C.byref(c))
    return tnc, a.value, b.value, c.value
