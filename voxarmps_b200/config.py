"""Solver parameters.

Every constant that the reference hard-codes in main.cu:211-394 is a field
here, with the reference's value as the default.  The same field names are
used by the C-ABI ``mps_config`` (include/voxarmps.h) and by the oracle.
"""
from __future__ import annotations

import math

import numpy as np

from . import cases

# fields shared with include/voxarmps.h::mps_config (order is the C layout)
FIELDS = [
    ("dim", "i"), ("ktype", "i"), ("method", "i"),
    ("l0", "d"), ("re_s", "d"), ("re_l", "d"), ("delta", "d"), ("dt", "d"),
    ("gx", "d"), ("gy", "d"), ("gz", "d"),
    ("rho1", "d"), ("rho2", "d"), ("nu1", "d"), ("nu2", "d"),
    ("beta_fs", "d"), ("dirichlet", "d"), ("relaxp", "d"),
    ("kh", "i"), ("vmax", "d"), ("coll", "d"), ("cc", "d"), ("velcor", "d"),
    ("ncorrection", "d"), ("pmin", "d"), ("pmax", "d"), ("c01", "d"), ("c02", "d"),
    ("turb", "i"), ("cs", "d"), ("fluid2_type", "i"),
    ("n_pl", "d"), ("meu0", "d"), ("phi", "d"), ("cohes", "d"),
    ("matopt", "i"), ("srcopt", "i"), ("fraction_method", "i"),
    ("ppe_at_predicted", "i"), ("warm_start", "i"), ("solver", "i"),
    ("cg_tol", "d"), ("cg_max", "i"), ("imin", "i"), ("imax", "i"), ("eps", "d"),
    ("collision_gather", "i"),
    ("xmin", "d"), ("xmax", "d"), ("ymin", "d"), ("ymax", "d"), ("zmin", "d"), ("zmax", "d"),
    ("precision", "i"), ("list_cap_s", "i"), ("list_cap_l", "i"),
]


def reference_defaults(dl: float, dim: int, compressible: bool = False) -> dict:
    """The reference's constants for spacing ``dl`` (main.cu:211-394)."""
    re = (3.2 if dim == 3 else 4.0) * dl  # main.cu:252-260
    cfg = dict(
        dim=dim, ktype=6 if compressible else 2, method=3 if compressible else 1,
        l0=dl, re_s=re, re_l=re, delta=dl / 5.0,
        dt=1.0 * dl / 20.0,  # DTcalculation: COURANT*DL/max(c01,c02), functions.cu:1684
        gx=0.0, gy=-9.8, gz=0.0,
        rho1=1000.0, rho2=1000.0, nu1=1e-6, nu2=1e-6,
        beta_fs=0.92, dirichlet=0.97, relaxp=0.5 if compressible else 0.2,
        kh=1, vmax=2.5, coll=math.sqrt(dl * dl * 0.5 * 0.5),
        cc=0.5 if compressible else 0.20, velcor=1.0, ncorrection=0.99,
        pmin=0.0, pmax=10000.0, c01=20.0, c02=20.0,
        turb=0, cs=0.18, fluid2_type=0, n_pl=0.0, meu0=0.0, phi=0.0, cohes=0.0,
        matopt=0, srcopt=0, fraction_method=2,
        ppe_at_predicted=0, warm_start=0, solver=0, cg_tol=1e-8, cg_max=2000,
        imin=10, imax=50, eps=1.0e-9, collision_gather=0,
        xmin=0.0, xmax=0.0, ymin=0.0, ymax=0.0, zmin=0.0, zmax=0.0,
        precision=0, list_cap_s=0, list_cap_l=0,
    )
    return cfg


def with_box(cfg: dict, case: dict) -> dict:
    """Bounding box grown by DL (main.cu:625-715) and PMAX = TP*4.5 (main.cu:548)."""
    c = dict(cfg)
    dl = c["l0"]
    x, y = np.asarray(case["x"]), np.asarray(case["y"])
    c["xmin"] = float(x.min()) - dl
    c["xmax"] = float(x.max()) + dl
    c["ymin"] = float(y.min()) - dl
    c["ymax"] = float(y.max()) + dl
    if c["dim"] == 3:
        z = np.asarray(case["z"])
        c["zmin"] = float(z.min()) - dl
        c["zmax"] = float(z.max()) + dl
    else:
        # the reference leaves Zmin/Zmax at +-99999999 in 2D (main.cu:615-620)
        c["zmin"], c["zmax"] = 99999999.0, -99999999.0
    c.setdefault("pmax", 0.0)
    c["pmax"] = float(len(x)) * 4.50
    return c


def solver_semantics(cfg: dict, precision: str = "fp64") -> dict:
    """Semantics of the CUDA path: A at x*, b from n*, warm start, Jacobi CG to
    a relative residual of cg_tol, order-independent collision."""
    c = dict(cfg)
    c.update(ppe_at_predicted=1, warm_start=1, solver=1, collision_gather=1)
    return c


def baseline(idx: int):
    """(cfg, case) for the five benchmark configurations.

    0: 2D dam, l0=0.01, 25x50 fluid, 1.0 x 0.6 m tank, dt=1e-4, re 2.1/4.0 l0.
    1: 3D dam, l0=0.005, 80x160x80 fluid, 1.6 x 1.0 x 0.4 m tank, dt=5e-5.
    2: config 1 (the precision mode differs, not the inputs).
    3: 2D two-phase + SPS, l0=0.002, water 600x100, HB block 150x150.
    4: 64 batched 2D dams (see cases.batched_dam_scenes), returns the list.
    """
    if idx == 0:
        l0 = 0.01
        case = cases.dam_break(2, l0, (25, 50), (100, 60))
        cfg = reference_defaults(l0, 2)
        cfg.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=1e-4, gy=-9.81)
    elif idx in (1, 2):
        l0 = 0.005
        case = cases.dam_break(3, l0, (80, 160, 80), (320, 200, 80))
        cfg = reference_defaults(l0, 3)
        cfg.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=5e-5, gy=-9.81)
    elif idx == 3:
        l0 = 0.002
        case = cases.dam_break(2, l0, (600, 100), (600, 300),
                               blocks=[(cases.FLUID2, (0, 100), (150, 150))])
        cfg = reference_defaults(l0, 2)
        cfg.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=1e-4, gy=-9.81, turb=1, cs=0.12,
                   rho2=900.0, nu2=1e-4, fluid2_type=1, n_pl=1.0, meu0=1e-4 * 900.0,
                   cohes=5.0, phi=0.0)
    elif idx == 4:
        l0 = 0.005
        scenes = cases.batched_dam_scenes(64, 0, l0)
        cfg = reference_defaults(l0, 2)
        cfg.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=1e-4, gy=-9.81)
        return cfg, scenes
    else:
        raise ValueError(idx)
    return with_box(cfg, case), case


def partition_scenes(sizes, ws: int):
    """Split independent scenes over ws ranks by particle count (largest
    first, each to the least-loaded rank; ties to the lower rank): a list of
    ws lists of scene indices, each in increasing order.  Deterministic, so
    every rank computes the same split without exchanging anything."""
    if ws < 1:
        raise ValueError("ws must be >= 1")
    load = [0] * ws
    parts = [[] for _ in range(ws)]
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    for k in order:
        r = min(range(ws), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += int(sizes[k])
    return [sorted(p) for p in parts]


def batched(cfg: dict, scenes, gap_radii: float = 4.0):
    """(cfg, stacked case, scene ids, boxes, pmax) for scenes advanced in one
    context; the gap between scenes is gap_radii Laplacian radii."""
    case, sid, boxes, pmax = cases.stack_scenes(scenes, gap_radii * cfg["re_l"])
    c = dict(cfg)
    c["xmin"], c["xmax"] = float(boxes[:, 0].min()), float(boxes[:, 1].max())
    c["ymin"], c["ymax"] = float(boxes[:, 2].min()), float(boxes[:, 3].max())
    if c["dim"] == 3:
        c["zmin"], c["zmax"] = float(boxes[:, 4].min()), float(boxes[:, 5].max())
    else:
        c["zmin"], c["zmax"] = 99999999.0, -99999999.0
    c["pmax"] = float(pmax.max())
    return c, case, sid, boxes, pmax



def scaled_dam3d(scale: int, l0: float = 0.005):
    """3D dam with the config-1 spacing and radii and a 10s x 20s x 10s column in
    a proportionally smaller tank (the bounded CPU sample)."""
    case = cases.dam_break(3, l0, (10 * scale, 20 * scale, 10 * scale),
                           (40 * scale, 25 * scale, 10 * scale))
    cfg = reference_defaults(l0, 3)
    cfg.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=5e-5, gy=-9.81)
    return with_box(cfg, case), case
