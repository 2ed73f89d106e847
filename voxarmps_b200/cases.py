"""Particle-lattice case generation and the .grd text format.

The reference generates its inputs with a separate tool
(generateSimulationCases/genParticlesFunctions.cpp:124-219 for the 2D dam,
:455-558 for the 3D dam) and reads them in main.cu:496-684.  This module is
config-driven instead of hard-coding one lattice per function, and keeps the
reference's conventions:

* particles are ordered dummies (PTYPE -1), then walls (PTYPE 0), then fluid
  (PTYPE 1, second fluid PTYPE 2) -- the solver's fluid loops rely on it
  (main.cu:666-668, functions.cu:2701);
* y is the vertical axis, z the depth in 3D (gravity is gy);
* a .grd file holds ``TP`` then one particle per line:
  ``x y [z] PTYPE u v [w] p`` (main.cu:629-661).
"""
from __future__ import annotations

import math

import numpy as np

DUMMY, WALL, FLUID1, FLUID2 = -1, 0, 1, 2


def _lattice(ranges):
    axes = [np.arange(a, b, dtype=np.int64) for a, b in ranges]
    mesh = np.meshgrid(*axes, indexing="ij")
    return np.stack([m.ravel() for m in mesh], axis=1)


def dam_break(dim: int, l0: float, fluid_cells, tank_cells, wall_layers: int = 1,
              dummy_layers: int = 2, blocks=()):
    """Dam-break lattice: a fluid column in the left (x = 0) corner of a tank.

    ``fluid_cells``: (nx, ny) or (nx, ny, nz) fluid particles, y vertical.
    ``tank_cells``: interior size of the tank in lattice steps, same axes.
    ``blocks``: extra fluid blocks ``(ptype, origin_cells, size_cells)``.
    Walls cover the bottom and the sides (no lid); ``wall_layers`` PTYPE 0
    layers sit next to the interior and ``dummy_layers`` PTYPE -1 layers
    outside them.  Node (i, j[, k]) sits at i*l0, j*l0[, k*l0].
    """
    B = wall_layers + dummy_layers
    if dim == 2:
        tx, ty = tank_cells
        nodes = _lattice([(0, tx + 2 * B), (0, ty + B)])
        ix, iy = nodes[:, 0], nodes[:, 1]
        interior = (ix >= B) & (ix < B + tx) & (iy >= B)
        depth = np.minimum.reduce([B - 1 - ix, ix - (B + tx), B - 1 - iy])
        # layer index outward from the interior: 0 = wall next to fluid
        layer = np.maximum.reduce([B - 1 - ix, ix - (B + tx), B - 1 - iy])
        del depth
    else:
        tx, ty, tz = tank_cells
        nodes = _lattice([(0, tx + 2 * B), (0, ty + B), (0, tz + 2 * B)])
        ix, iy, iz = nodes[:, 0], nodes[:, 1], nodes[:, 2]
        interior = (ix >= B) & (ix < B + tx) & (iy >= B) & (iz >= B) & (iz < B + tz)
        layer = np.maximum.reduce([B - 1 - ix, ix - (B + tx), B - 1 - iy, B - 1 - iz,
                                   iz - (B + tz)])
    solid = ~interior
    wall = solid & (layer < wall_layers)
    dummy = solid & ~wall
    fluid_sets = [(FLUID1, (0,) * dim, tuple(fluid_cells))] + list(blocks)
    fl_nodes, fl_type = [], []
    for ptype, origin, size in fluid_sets:
        rng = [(B + o, B + o + s) for o, s in zip(origin, size)]
        nd = _lattice(rng)
        fl_nodes.append(nd)
        fl_type.append(np.full(len(nd), ptype, np.int32))
    fl_nodes = np.concatenate(fl_nodes)
    fl_type = np.concatenate(fl_type)
    allnodes = np.concatenate([nodes[dummy], nodes[wall], fl_nodes])
    ptype = np.concatenate([np.full(int(dummy.sum()), DUMMY, np.int32),
                            np.full(int(wall.sum()), WALL, np.int32), fl_type])
    n = len(allnodes)
    case = {
        "dim": dim, "l0": l0,
        "x": allnodes[:, 0] * l0, "y": allnodes[:, 1] * l0,
        "z": (allnodes[:, 2] * l0) if dim == 3 else np.zeros(n),
        "ptype": ptype,
        "u": np.zeros(n), "v": np.zeros(n), "w": np.zeros(n), "p": np.zeros(n),
    }
    return case


def counts(case):
    pt = np.asarray(case["ptype"])
    return {"TP": int(len(pt)), "GP": int((pt < 0).sum()), "WP": int((pt == 0).sum()),
            "FP": int((pt > 0).sum())}


def check_order(case) -> bool:
    """True when particles are ordered dummies, walls, fluid (main.cu:666-668)."""
    pt = np.asarray(case["ptype"])
    cls = np.where(pt < 0, 0, np.where(pt == 0, 1, 2))
    return bool(np.all(np.diff(cls) >= 0))


def write_grd(path: str, case: dict) -> None:
    """Write a .grd file (main.cu:629-661 column order), doubles round-trip exact."""
    dim = case["dim"]
    n = len(case["x"])
    cols = [case["x"], case["y"]] + ([case["z"]] if dim == 3 else [])
    with open(path, "w") as f:
        f.write(f"{n}\n")
        for i in range(n):
            pos = " ".join(repr(float(c[i])) for c in cols)
            vel = [case["u"][i], case["v"][i]] + ([case["w"][i]] if dim == 3 else [])
            f.write(f"{pos} {int(case['ptype'][i])} " + " ".join(repr(float(v)) for v in vel)
                    + f" {repr(float(case['p'][i]))}\n")


def read_grd(path: str, dim: int) -> dict:
    """Read a .grd file exactly as main.cu:623-661 does (whitespace separated)."""
    with open(path) as f:
        tok = f.read().split()
    n = int(tok[0])
    per = 8 if dim == 3 else 6
    a = np.array(tok[1:1 + n * per], dtype=np.float64).reshape(n, per)
    case = {"dim": dim, "x": a[:, 0].copy(), "y": a[:, 1].copy()}
    if dim == 3:
        case.update(z=a[:, 2].copy(), ptype=a[:, 3].astype(np.int32), u=a[:, 4].copy(),
                    v=a[:, 5].copy(), w=a[:, 6].copy(), p=a[:, 7].copy())
    else:
        case.update(z=np.zeros(n), ptype=a[:, 2].astype(np.int32), u=a[:, 3].copy(),
                    v=a[:, 4].copy(), w=np.zeros(n), p=a[:, 5].copy())
    return case


def splitmix64(seed: int):
    """Deterministic PRNG stream (Steele et al., SplitMix64) for scene batches."""
    state = seed & 0xFFFFFFFFFFFFFFFF
    while True:
        state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        yield (z ^ (z >> 31)) / 2.0 ** 64


def batched_dam_scenes(count: int = 64, seed: int = 0, l0: float = 0.005):
    """Independent 2D dam breaks, column width U[0.1,0.4] m, height U[0.2,0.6] m,
    in 1.0 x 0.6 m tanks with 1 wall + 2 dummy layers."""
    rng = splitmix64(seed)
    scenes = []
    for _ in range(count):
        wdt = 0.1 + 0.3 * next(rng)
        hgt = 0.2 + 0.4 * next(rng)
        nx, ny = max(1, int(round(wdt / l0))), max(1, int(round(hgt / l0)))
        scenes.append(dam_break(2, l0, (nx, ny), (int(round(1.0 / l0)), int(round(0.6 / l0)))))
    return scenes


def stack_scenes(scenes, gap: float):
    """Independent scenes in one domain, stacked along y with ``gap`` metres
    of empty space between neighbouring scenes (gap > the largest support
    radius keeps every neighbour list inside its scene, and each scene then
    occupies whole cell rows, i.e. a contiguous range of the cell order).

    Returns (case, scene_of_particle, boxes, pmax): boxes holds each scene's
    grown box (main.cu:692-715) after the shift, pmax = TP*4.5 per scene
    (main.cu:548)."""
    dim = scenes[0]["dim"]
    dl = scenes[0]["l0"]
    parts = {k: [] for k in ("x", "y", "z", "u", "v", "w", "p", "ptype")}
    scene_id, boxes, pmax = [], [], []
    y0 = 0.0
    for k, sc in enumerate(scenes):
        ys = np.asarray(sc["y"])
        shift = y0 - ys.min()
        for key in parts:
            a = np.asarray(sc[key])
            parts[key].append(a + shift if key == "y" else a)
        scene_id.append(np.full(len(ys), k, np.int32))
        x = np.asarray(sc["x"])
        z = np.asarray(sc["z"])
        box = [x.min() - dl, x.max() + dl, ys.min() + shift - dl, ys.max() + shift + dl]
        box += [z.min() - dl, z.max() + dl] if dim == 3 else [99999999.0, -99999999.0]
        boxes.append(box)
        pmax.append(len(ys) * 4.50)
        y0 = ys.max() + shift + gap
    case = {key: np.concatenate(v) for key, v in parts.items()}
    case["ptype"] = case["ptype"].astype(np.int32)
    case["dim"], case["l0"] = dim, dl
    return (case, np.concatenate(scene_id), np.asarray(boxes, np.float64),
            np.asarray(pmax, np.float64))


def lattice_neighbours(dim: int, ratio: float, inclusive: bool = False) -> int:
    """Number of lattice nodes within ratio*l0 of a node (self excluded)."""
    r = int(math.ceil(ratio)) + 1
    ax = np.arange(-r, r + 1)
    g = np.stack(np.meshgrid(*([ax] * dim), indexing="ij"), -1).reshape(-1, dim)
    d2 = (g ** 2).sum(1)
    lim = ratio * ratio
    m = (d2 <= lim) if inclusive else (d2 < lim)
    return int(m.sum()) - 1
