"""voxarmps_b200 -- Blackwell-native (sm_100a) MPS solver core.

Python host-side mirror of the C-ABI in include/voxarmps.h.  ``Solver``
exposes one method per reference stage (NEIGHBOR, PNUM, ... PREPDATA of
VoxarMPS/VoxarMPS/functions.cuh) plus ``step()`` for main.cu's whole loop
body.  The CUDA library is required: there is no CPU path, and importing
``Solver`` on a machine without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import cases, config  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvoxarmps_b200.so")

MPS_OK = 0
MPS_ERR_ARG = 1
MPS_ERR_CUDA = 2
MPS_ERR_NAN = 4
MPS_ERR_BOX = 8
MPS_ERR_CELL = 16
MPS_ERR_LIST_OVERFLOW = 32
MPS_ERR_NOT_CONVERGED = 64
MPS_ERR_IO = 128
FATAL = MPS_ERR_ARG | MPS_ERR_CUDA | MPS_ERR_IO

_CT = {"i": C.c_int, "d": C.c_double}


class MpsConfig(C.Structure):
    """ctypes mirror of ``mps_config``."""
    _fields_ = [(name, _CT[t]) for name, t in config.FIELDS]


EXPORTS = [
    "mps_create", "mps_destroy", "mps_upload", "mps_load_grd", "mps_init", "mps_pnd",
    "mps_neighbors", "mps_sps", "mps_vfraction", "mps_viscosity", "mps_predict",
    "mps_pnd_star", "mps_bcon", "mps_pressure", "mps_phat", "mps_pressure_gradient",
    "mps_integrate", "mps_collision", "mps_commit", "mps_step", "mps_run", "mps_download",
    "mps_download_lists", "mps_get_scalar", "mps_get_error", "mps_last_message",
    "mps_write_vtu", "mps_stream", "mps_set_state", "mps_get_state", "mps_step_io",
    "mps_set_field",
    "mps_set_profile",
    "mps_cell_order_noalloc", "mps_set_scenes", "mps_set_graph",
    "mps_gnn_create", "mps_gnn_use", "mps_gnn_train", "mps_gnn_params", "mps_gnn_state",
    "mps_gnn_features",
    "mps_gnn_forward", "mps_gnn_download", "mps_get_tuning", "mps_set_tuning", "mps_autotune",
    "mps_snapshot_vtu", "mps_wait_io", "mps_save_checkpoint", "mps_load_checkpoint",
    "mps_set_owned", "mps_set_n0", "mps_get_rows", "mps_set_rows", "mps_ppe_assemble",
    "mps_dcg_start", "mps_dcg_spmv", "mps_dcg_update", "mps_dcg_direction", "mps_dcg_finish",
]

_LIB = None


class MpsTuning(C.Structure):
    """ctypes mirror of mps_tuning (include/voxarmps.h)."""
    _fields_ = [("small_lanes", C.c_int), ("cg_blocks_per_sm", C.c_int)]


class MpsError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"voxarmps error {code}: {msg}")
        self.code = code


def load_library(path: str = LIB_PATH):
    """Load the CUDA library (fails loudly when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with python -m voxarmps_b200.build")
    lib = C.CDLL(path)
    P = C.c_void_p
    DP = C.POINTER(C.c_double)
    IP = C.POINTER(C.c_int)
    lib.mps_create.argtypes = [C.POINTER(MpsConfig), C.c_int, C.POINTER(P)]
    lib.mps_destroy.argtypes = [P]
    lib.mps_upload.argtypes = [P, C.c_int, DP, DP, DP, IP, DP, DP, DP, DP]
    lib.mps_load_grd.argtypes = [P, C.c_char_p]
    for name in ("mps_init", "mps_pnd", "mps_neighbors", "mps_sps", "mps_vfraction",
                 "mps_viscosity", "mps_predict", "mps_pnd_star", "mps_bcon", "mps_phat",
                 "mps_pressure_gradient", "mps_integrate", "mps_collision", "mps_commit",
                 "mps_step", "mps_get_error"):
        getattr(lib, name).argtypes = [P]
    lib.mps_pressure.argtypes = [P, IP, DP]
    lib.mps_run.argtypes = [P, C.c_int]
    lib.mps_download.argtypes = [P, C.c_char_p, P, C.POINTER(C.c_long)]
    lib.mps_download_lists.argtypes = [P, C.c_int, IP, IP, C.POINTER(C.c_long)]
    lib.mps_get_scalar.argtypes = [P, C.c_char_p, DP]
    lib.mps_last_message.argtypes = [P]
    lib.mps_last_message.restype = C.c_char_p
    lib.mps_write_vtu.argtypes = [P, C.c_char_p, C.c_int]
    lib.mps_stream.argtypes = [P]
    lib.mps_stream.restype = P
    lib.mps_set_state.argtypes = [P, P, P, P, P, P, P, P]
    lib.mps_get_state.argtypes = [P, P, P, P, P, P, P, P]
    lib.mps_step_io.argtypes = [P, C.POINTER(P), C.POINTER(P)]
    lib.mps_set_field.argtypes = [P, C.c_char_p, DP]
    lib.mps_set_profile.argtypes = [P, C.c_int]
    lib.mps_set_graph.argtypes = [P, C.c_int]
    FP = C.POINTER(C.c_float)
    lib.mps_snapshot_vtu.argtypes = [P, C.c_char_p, C.c_int]
    lib.mps_wait_io.argtypes = [P]
    lib.mps_save_checkpoint.argtypes = [P, C.c_char_p]
    lib.mps_load_checkpoint.argtypes = [P, C.c_char_p]
    lib.mps_get_tuning.argtypes = [P, C.POINTER(MpsTuning)]
    lib.mps_set_tuning.argtypes = [P, C.POINTER(MpsTuning)]
    lib.mps_autotune.argtypes = [P, C.c_int, C.POINTER(MpsTuning)]
    lib.mps_gnn_create.argtypes = [P, C.c_int, C.c_ulonglong]
    lib.mps_gnn_use.argtypes = [P, C.c_int]
    lib.mps_gnn_train.argtypes = [P, C.c_int, C.c_float, C.c_int, C.c_int, FP]
    lib.mps_gnn_params.argtypes = [P, FP, FP, C.POINTER(C.c_int)]
    lib.mps_gnn_state.argtypes = [P, FP, FP, C.POINTER(C.c_int)]
    lib.mps_gnn_features.argtypes = [P]
    lib.mps_gnn_forward.argtypes = [P]
    lib.mps_gnn_download.argtypes = [P, C.c_char_p, P, C.POINTER(C.c_long)]
    lib.mps_set_scenes.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double)]
    lib.mps_cell_order_noalloc.argtypes = [C.POINTER(MpsConfig), C.c_double, C.c_int, P, P, P,
                                           P, P, P, P]
    lib.mps_set_owned.argtypes = [P, IP]
    lib.mps_set_n0.argtypes = [P, C.c_double, C.c_double]
    lib.mps_get_rows.argtypes = [P, C.c_char_p, C.c_int, IP, DP]
    lib.mps_set_rows.argtypes = [P, C.c_char_p, C.c_int, IP, DP]
    lib.mps_ppe_assemble.argtypes = [P]
    lib.mps_dcg_start.argtypes = [P, DP]
    lib.mps_dcg_spmv.argtypes = [P, DP]
    lib.mps_dcg_update.argtypes = [P, C.c_double, DP]
    lib.mps_dcg_direction.argtypes = [P, C.c_double]
    lib.mps_dcg_finish.argtypes = [P, C.c_int, C.c_double, C.c_double]
    _LIB = lib
    return lib


INT_FIELDS = {"ptype", "bcon", "cell_s", "cell_l", "perm_s", "perm_l"}


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


class Solver:
    """One simulation on one GPU (a context of the C-ABI)."""

    def __init__(self, cfg: dict, case: dict | None = None, device: int = 0):
        self.lib = load_library()
        self.cfg = dict(config.reference_defaults(cfg.get("l0", 0.01), cfg.get("dim", 2)))
        self.cfg.update(cfg)
        self._c = MpsConfig(**{k: self.cfg[k] for k, _ in config.FIELDS})
        self.h = C.c_void_p()
        self._chk(self.lib.mps_create(C.byref(self._c), device, C.byref(self.h)), "create")
        if case is not None:
            self.upload(case)

    def _chk(self, r, what=""):
        if r & FATAL:
            msg = self.lib.mps_last_message(self.h).decode() if self.h else ""
            raise MpsError(r, f"{what}: {msg}")
        return r

    def upload(self, case: dict):
        n = len(case["x"])
        f64 = lambda k: np.ascontiguousarray(case[k], np.float64) if k in case else None
        self._keep = [f64(k) for k in ("x", "y", "z", "u", "v", "w", "p")]
        pt = np.ascontiguousarray(case["ptype"], np.int32)
        x, y, z, u, v, w, p = self._keep
        self._chk(self.lib.mps_upload(self.h, n, _dp(x), _dp(y), _dp(z),
                                      pt.ctypes.data_as(C.POINTER(C.c_int)), _dp(u), _dp(v),
                                      _dp(w), _dp(p)), "upload")
        self.n = n
        return self

    def set_scenes(self, scene, boxes, pmax):
        """Batched independent scenes (after upload, before init)."""
        sc = np.ascontiguousarray(scene, np.int32)
        bx = np.ascontiguousarray(boxes, np.float64).reshape(-1)
        pm = np.ascontiguousarray(pmax, np.float64)
        self._scenes = (sc, bx, pm)
        self._chk(self.lib.mps_set_scenes(self.h, len(pm), sc.ctypes.data_as(C.POINTER(C.c_int)),
                                          bx.ctypes.data_as(C.POINTER(C.c_double)),
                                          pm.ctypes.data_as(C.POINTER(C.c_double))), "scenes")
        return self

    def load_grd(self, path: str):
        self._chk(self.lib.mps_load_grd(self.h, path.encode()), "load_grd")
        self.n = int(self.scalar("n"))
        return self

    # ---- stages, one per reference routine (functions.cuh:56-111) ----
    def init(self):
        return self._chk(self.lib.mps_init(self.h), "init")

    def neighbors(self):
        return self._chk(self.lib.mps_neighbors(self.h), "neighbors")

    def pnd(self):
        return self._chk(self.lib.mps_pnd(self.h), "pnd")

    def sps(self):
        return self._chk(self.lib.mps_sps(self.h), "sps")

    def vfraction(self):
        return self._chk(self.lib.mps_vfraction(self.h), "vfraction")

    def viscosity(self):
        return self._chk(self.lib.mps_viscosity(self.h), "viscosity")

    def predict(self):
        return self._chk(self.lib.mps_predict(self.h), "predict")

    def pnd_star(self):
        return self._chk(self.lib.mps_pnd_star(self.h), "pnd_star")

    def bcon(self):
        return self._chk(self.lib.mps_bcon(self.h), "bcon")

    def pressure(self):
        it, rr = C.c_int(), C.c_double()
        self._chk(self.lib.mps_pressure(self.h, C.byref(it), C.byref(rr)), "pressure")
        return it.value, rr.value

    def phat(self):
        return self._chk(self.lib.mps_phat(self.h), "phat")

    def pressure_gradient(self):
        return self._chk(self.lib.mps_pressure_gradient(self.h), "pressure_gradient")

    def integrate(self):
        return self._chk(self.lib.mps_integrate(self.h), "integrate")

    def collision(self):
        return self._chk(self.lib.mps_collision(self.h), "collision")

    def commit(self):
        return self._chk(self.lib.mps_commit(self.h), "commit")

    # the reference's routine names
    NEIGHBOR, PNUM, SPS, V_FRACTION, VISCOSITY = neighbors, pnd, sps, vfraction, viscosity
    PREDICTION, PNUMSTAR, BCON, PRESSURECALC = predict, pnd_star, bcon, pressure
    PHATCALC, PRESSGRAD, EULERINTEGRATION, COLLISION2, PREPDATA = (
        phat, pressure_gradient, integrate, collision, commit)

    def step(self):
        """One time step (main.cu:1027-1349); returns the MPS_ERR_* bits."""
        return self._chk(self.lib.mps_step(self.h), "step")

    def run(self, steps: int):
        return self._chk(self.lib.mps_run(self.h, steps), "run")

    # ---- data out ----
    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.n, np.int32 if name in INT_FIELDS else np.float64)
        self._chk(self.lib.mps_download(self.h, name.encode(), out.ctypes.data_as(C.c_void_p),
                                        None), f"download {name}")
        return out

    def lists(self, which: int):
        """(off, nbr) CSR in particle-id space; which 0 = PND radius, 1 = Laplacian."""
        tot = C.c_long()
        self._chk(self.lib.mps_download_lists(self.h, which, None, None, C.byref(tot)), "lists")
        off = np.empty(self.n + 1, np.int32)
        nbr = np.empty(max(tot.value, 1), np.int32)
        IP = C.POINTER(C.c_int)
        self._chk(self.lib.mps_download_lists(self.h, which, off.ctypes.data_as(IP),
                                              nbr.ctypes.data_as(IP), C.byref(tot)), "lists")
        return off, nbr[: tot.value]

    def set_state(self, *ptrs):
        """Host pointers (ints) for x, y, z, u, v, w, p in caller order; 0 skips."""
        return self._chk(self.lib.mps_set_state(self.h, *[p or None for p in ptrs]), "set_state")

    def step_io(self, ins, outs):
        """One step with the state in host arrays: ``ins`` and ``outs`` are 7
        host pointers (ints; 0 skips) for x, y, z, u, v, w, p in caller order."""
        a = (C.c_void_p * 7)(*[p or None for p in ins])
        b = (C.c_void_p * 7)(*[p or None for p in outs])
        return self._chk(self.lib.mps_step_io(self.h, a, b), "step_io")

    def set(self, name: str, values):
        """Overwrite one state array (caller order) between stage calls."""
        a = np.ascontiguousarray(values, np.float64)
        if a.shape != (self.n,):
            raise ValueError(f"{name}: expected {self.n} values")
        return self._chk(self.lib.mps_set_field(self.h, name.encode(), _dp(a)), f"set {name}")

    # ---- one scene split between contexts (voxarmps_b200/slab.py) -------
    def set_owned(self, owned):
        o = np.ascontiguousarray(owned, np.int32)
        return self._chk(self.lib.mps_set_owned(self.h, o.ctypes.data_as(C.POINTER(C.c_int))),
                         "set_owned")

    def set_n0(self, n0_s: float, n0_l: float):
        return self._chk(self.lib.mps_set_n0(self.h, n0_s, n0_l), "set_n0")

    def get_rows(self, name: str, ids) -> np.ndarray:
        i = np.ascontiguousarray(ids, np.int32)
        out = np.empty(len(i), np.float64)
        self._chk(self.lib.mps_get_rows(self.h, name.encode(), len(i),
                                        i.ctypes.data_as(C.POINTER(C.c_int)), _dp(out)),
                  f"get_rows {name}")
        return out

    def set_rows(self, name: str, ids, values):
        i = np.ascontiguousarray(ids, np.int32)
        v = np.ascontiguousarray(values, np.float64)
        if len(v) != len(i):
            raise ValueError("one value per index")
        return self._chk(self.lib.mps_set_rows(self.h, name.encode(), len(i),
                                               i.ctypes.data_as(C.POINTER(C.c_int)), _dp(v)),
                         f"set_rows {name}")

    def ppe_assemble(self):
        return self._chk(self.lib.mps_ppe_assemble(self.h), "ppe_assemble")

    def dcg_start(self) -> np.ndarray:
        out = np.zeros(3)
        self._chk(self.lib.mps_dcg_start(self.h, _dp(out)), "dcg_start")
        return out

    def dcg_spmv(self) -> float:
        out = np.zeros(1)
        self._chk(self.lib.mps_dcg_spmv(self.h, _dp(out)), "dcg_spmv")
        return float(out[0])

    def dcg_update(self, alpha: float) -> np.ndarray:
        out = np.zeros(2)
        self._chk(self.lib.mps_dcg_update(self.h, alpha, _dp(out)), "dcg_update")
        return out

    def dcg_direction(self, beta: float):
        return self._chk(self.lib.mps_dcg_direction(self.h, beta), "dcg_direction")

    def dcg_finish(self, iters: int, relres: float, bb: float):
        return self._chk(self.lib.mps_dcg_finish(self.h, iters, relres, bb), "dcg_finish")

    def get_state(self, *ptrs):
        return self._chk(self.lib.mps_get_state(self.h, *[p or None for p in ptrs]), "get_state")

    def set_profile(self, on: bool = True):
        return self._chk(self.lib.mps_set_profile(self.h, int(on)), "profile")

    # ---- output and checkpoints ----------------------------------------
    def snapshot_vtu(self, path: str, fluid_only: bool = False):
        """Binary VTU written asynchronously (see wait_io)."""
        return self._chk(self.lib.mps_snapshot_vtu(self.h, str(path).encode(), int(fluid_only)),
                         "snapshot_vtu")

    def wait_io(self):
        return self._chk(self.lib.mps_wait_io(self.h), "wait_io")

    def save_checkpoint(self, path: str):
        return self._chk(self.lib.mps_save_checkpoint(self.h, str(path).encode()), "checkpoint")

    def load_checkpoint(self, path: str):
        r = self._chk(self.lib.mps_load_checkpoint(self.h, str(path).encode()), "checkpoint")
        self.n = int(self.scalar("n"))
        return r

    # ---- launch-shape tuning -------------------------------------------
    def get_tuning(self) -> dict:
        t = MpsTuning()
        self._chk(self.lib.mps_get_tuning(self.h, C.byref(t)), "get_tuning")
        return {"small_lanes": t.small_lanes, "cg_blocks_per_sm": t.cg_blocks_per_sm}

    def set_tuning(self, small_lanes: int, cg_blocks_per_sm: int):
        t = MpsTuning(small_lanes, cg_blocks_per_sm)
        return self._chk(self.lib.mps_set_tuning(self.h, C.byref(t)), "set_tuning")

    def autotune(self, steps: int = 3) -> dict:
        """Time the candidate launch shapes on real steps; keep the fastest."""
        t = MpsTuning()
        self._chk(self.lib.mps_autotune(self.h, steps, C.byref(t)), "autotune")
        return {"small_lanes": t.small_lanes, "cg_blocks_per_sm": t.cg_blocks_per_sm}

    # ---- learned CG initial guess -------------------------------------
    def gnn_create(self, layers: int = 4, seed: int = 0):
        return self._chk(self.lib.mps_gnn_create(self.h, layers, seed), "gnn_create")

    def gnn_use(self, on: bool = True):
        return self._chk(self.lib.mps_gnn_use(self.h, int(on)), "gnn_use")

    def gnn_train(self, iters: int = 1, lr: float = 1e-3, grad_only: bool = False,
                  objective: str = "residual") -> float:
        """Adam steps on the last PPE; objective "residual" (|b - A x0|^2/|b|^2)
        or "increment" (squared error of the scaled pressure increment)."""
        obj = {"increment": 0, "residual": 1}[objective]
        loss = C.c_float()
        self._chk(self.lib.mps_gnn_train(self.h, iters, lr, obj, int(grad_only), C.byref(loss)),
                  "gnn_train")
        return loss.value

    def gnn_params(self, set_to=None) -> np.ndarray:
        cnt = C.c_int()
        self._chk(self.lib.mps_gnn_params(self.h, None, None, C.byref(cnt)), "gnn_params")
        out = np.zeros(cnt.value, np.float32)
        src = None
        if set_to is not None:
            src = np.ascontiguousarray(set_to, np.float32)
            assert src.size == cnt.value
            src = src.ctypes.data_as(C.POINTER(C.c_float))
        self._chk(self.lib.mps_gnn_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), src,
                                          None), "gnn_params")
        return out

    def gnn_state(self, set_to=None) -> np.ndarray:
        """The training state (parameters, Adam moments, Adam step count);
        with set_to, load one taken from another context first."""
        cnt = C.c_int()
        self._chk(self.lib.mps_gnn_state(self.h, None, None, C.byref(cnt)), "gnn_state")
        out = np.zeros(cnt.value, np.float32)
        src = None
        if set_to is not None:
            src = np.ascontiguousarray(set_to, np.float32)
            assert src.size == cnt.value
            src = src.ctypes.data_as(C.POINTER(C.c_float))
        self._chk(self.lib.mps_gnn_state(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), src,
                                         None), "gnn_state")
        return out

    def gnn_features(self):
        return self._chk(self.lib.mps_gnn_features(self.h), "gnn_features")

    def gnn_forward(self):
        return self._chk(self.lib.mps_gnn_forward(self.h), "gnn_forward")

    def gnn_get(self, what: str) -> np.ndarray:
        cnt = C.c_long()
        self._chk(self.lib.mps_gnn_download(self.h, what.encode(), None, C.byref(cnt)), what)
        dt = np.int32 if what in ("nbr", "len", "cap", "bcon", "ptype") else np.float32
        out = np.zeros(max(cnt.value, 1), dt)
        self._chk(self.lib.mps_gnn_download(self.h, what.encode(), out.ctypes.data_as(C.c_void_p),
                                            None), what)
        return out[:cnt.value]

    def set_graph(self, on: bool = True):
        """Replay each step as one CUDA graph (CG loop as a while node)."""
        return self._chk(self.lib.mps_set_graph(self.h, int(on)), "graph")

    def scalar(self, name: str) -> float:
        v = C.c_double()
        self._chk(self.lib.mps_get_scalar(self.h, name.encode(), C.byref(v)), f"scalar {name}")
        return v.value

    def error(self) -> int:
        return self.lib.mps_get_error(self.h)

    def write_vtu(self, path: str, fluid_only: bool = False):
        return self._chk(self.lib.mps_write_vtu(self.h, path.encode(), int(fluid_only)), "vtu")

    def stream(self) -> int:
        return self.lib.mps_stream(self.h) or 0

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.mps_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
