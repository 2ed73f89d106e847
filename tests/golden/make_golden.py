"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference's own CPU stage functions (oracle/_ref/libref.so, built by
``make -C oracle ref`` from the reference's sources, found under
$VOXARMPS_REFERENCE, by default /root/reference) through
oracle/ref_harness.cpp and stores inputs, parameters and outputs as .npz.
The reference ships no tests or golden data; these fixtures are how the C
restatement (oracle/mps_oracle.c) is pinned on machines without the
reference sources.

Usage: python tests/golden/make_golden.py [--collision]   (needs the reference's sources)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle as po  # noqa: E402
from voxarmps_b200 import cases, config  # noqa: E402

REF_INPUTS = po.reference_path("inputs")
FIELDS = ["x", "y", "z", "u", "v", "w", "p", "pnew", "phat", "un", "vn", "wn", "xs", "ys", "zs",
          "us", "vs", "ws", "n", "nstar", "C", "meu", "neut", "t1", "t2", "t3", "source", "bcon"]


def list_digest(off, nbr):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off, np.int32).tobytes())
    h.update(np.ascontiguousarray(nbr, np.int32).tobytes())
    return h.hexdigest()


def run_case(name, cfg, case, snap_steps, full_lists=True, fields=FIELDS):
    r = po.RefHarness(cfg, case)
    r.init()
    out = {"cfg": json.dumps(cfg), "n0": r.scalar("n0")}
    for k in ("x", "y", "z", "u", "v", "w", "p"):
        out["in_" + k] = np.asarray(case[k], np.float64)
    out["in_ptype"] = np.asarray(case["ptype"], np.int32)
    out["in_dim"] = case["dim"]
    off, nbr = r.get("off"), r.get("nbr")
    out["init_off"] = off
    out["init_digest"] = list_digest(off, nbr)
    if full_lists:
        out["init_nbr"] = nbr
    else:
        out["init_nbr_head"] = nbr[: off[min(200, len(off) - 1)]]
    step = 0
    for s in snap_steps:
        while step < s:
            r.step()
            step += 1
        for f in fields:
            out[f"s{s}_{f}"] = r.get(f)
        off, nbr = r.get("off"), r.get("nbr")
        out[f"s{s}_digest"] = list_digest(off, nbr)
    out["snaps"] = np.asarray(snap_steps, np.int32)
    path = os.path.join(HERE, f"ref_{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: TP={len(case['x'])} -> {os.path.getsize(path) / 1024:.0f} KiB")


def collision_case(dim: int, cluster: bool = False, seed: int = 7):
    """A fluid block with pairs of particles pushed closer than the collision
    distance (0.4 l0 < coll = 0.5 l0): fluid-fluid pairs along every axis and
    fluid particles pushed toward the bottom and side walls, all pairs far
    from one another, with random velocities (some pairs approach, some
    separate).  ``cluster`` adds three particles within coll of one another."""
    rng = np.random.default_rng(seed + dim + (10 if cluster else 0))
    l0 = 0.01
    nf = 12 if dim == 2 else 8
    fluid = (nf,) * dim
    tank = (20, 16) if dim == 2 else (14, 12, 10)
    case = cases.dam_break(dim, l0, fluid, tank)
    n = len(case["x"])
    first = n - nf ** dim  # fluid particles come last, lattice order (x outermost)

    def fid(*ijk):
        f = 0
        for c in ijk:
            f = f * nf + c
        return first + f

    pos = {"x": case["x"], "y": case["y"], "z": case["z"]}
    axes = ["x", "y", "z"][:dim]
    moves = []  # (particle, axis, shift in l0)
    if dim == 2:
        for a in (0, 3, 6, 9):
            for b in (1, 4, 7, 10):
                moves += [(fid(a, b), "x", 0.3), (fid(a + 1, b), "x", -0.3)]
        for b in (2, 8):
            moves.append((fid(0, b), "x", -0.6))        # toward the left wall
        for a in (2, 5, 8):
            moves.append((fid(a, 0), "y", -0.6))        # toward the bottom wall
    else:
        for a in (0, 4):
            for b in (1, 5):
                for c in (1, 5):
                    moves += [(fid(a, b, c), "x", 0.3), (fid(a + 1, b, c), "x", -0.3)]
        for a in (2, 6):
            moves += [(fid(a, 2, 3), "y", 0.3), (fid(a, 3, 3), "y", -0.3)]
            moves += [(fid(a, 6, 6), "z", 0.3), (fid(a, 6, 7), "z", -0.3)]
        for a in (3, 7):
            moves.append((fid(a, 0, 3), "y", -0.6))     # toward the bottom wall
            moves.append((fid(a, 4, 0), "z", -0.6))     # toward the side wall
    if cluster:
        c = fid(*((nf // 2,) * dim)) if dim == 2 else fid(3, 6, 2)
        nb = c + (nf if dim == 2 else nf * nf)          # the next particle along x
        moves += [(c, "x", 0.25), (nb, "x", -0.25)]
        third = c + 1                                   # the next particle along the last axis
        moves.append((third, axes[-1], -0.6))
        if dim == 2:
            moves.append((third, "x", 0.5))
        else:
            moves.append((third, "x", 0.5))
    for i, ax, sh in moves:
        pos[ax][i] += sh * l0
    for k in ("x", "y", "z"):
        case[k] = pos[k]
    vel = rng.normal(0.0, 0.4, (3, n))
    vel[:, : first] = 0.0                                # walls and dummies at rest
    if dim == 2:
        vel[2] = 0.0
    cfg = config.with_box(config.reference_defaults(l0, dim), case)
    cfg.update(re_s=2.1 * l0, re_l=4.0 * l0, dt=1e-3)
    return cfg, case, vel


def run_collision(name, dim, cluster=False):
    """NEIGHBOR then COLLISION2 of the reference on a constructed state."""
    cfg, case, vel = collision_case(dim, cluster)
    r = po.RefHarness(cfg, case)
    for k, v in zip(("un", "vn", "wn"), vel):
        r.set(k, v)
    r.stage("NEIGHBOR")
    out = {"cfg": json.dumps(cfg), "in_dim": dim}
    for k in ("x", "y", "z"):
        out["in_" + k] = np.asarray(case[k], np.float64)
    out["in_ptype"] = np.asarray(case["ptype"], np.int32)
    for k, v in zip(("un", "vn", "wn"), vel):
        out["in_" + k] = np.asarray(v, np.float64)
    out["off"], out["nbr"] = r.get("off"), r.get("nbr")
    r.stage("COLLISION2")
    for k in ("x", "y", "z", "un", "vn", "wn"):
        out["out_" + k] = r.get(k)
    path = os.path.join(HERE, f"ref_{name}.npz")
    np.savez_compressed(path, **out)
    moved = int(np.sum((out["out_un"] != out["in_un"]) | (out["out_vn"] != out["in_vn"])))
    print(f"{name}: TP={len(case['x'])}, {moved} particles changed -> "
          f"{os.path.getsize(path) / 1024:.0f} KiB")


def save_inputs():
    """The reference's own .grd inputs, byte for byte (the .grd reader's
    fixtures on machines without the reference)."""
    out = {}
    for name in ("input-dam.grd", "input-dam3d.grd"):
        with open(os.path.join(REF_INPUTS, name), "rb") as f:
            out[name.replace("-", "_").replace(".", "_")] = np.frombuffer(f.read(), np.uint8)
    path = os.path.join(HERE, "ref_inputs_grd.npz")
    np.savez_compressed(path, **out)
    print(f"inputs: {os.path.getsize(path) / 1024:.0f} KiB")


def main_collision():
    po.build(ref=True)
    run_collision("collision2d", 2)
    run_collision("collision3d", 3)
    run_collision("collision2d_cluster", 2, cluster=True)
    run_collision("collision3d_cluster", 3, cluster=True)
    save_inputs()


def main():
    po.build(ref=True)
    dam2 = cases.read_grd(os.path.join(REF_INPUTS, "input-dam.grd"), 2)
    dam3 = cases.read_grd(os.path.join(REF_INPUTS, "input-dam3d.grd"), 3)
    # 1. the reference's own 2D dam input, its own constants (dt = COURANT*DL/c0)
    cfg = config.with_box(config.reference_defaults(0.01, 2), dam2)
    run_case("dam2d", cfg, dam2, [1, 5, 20])
    # 2. the reference's own 3D dam input (re = 3.2 DL)
    cfg = config.with_box(config.reference_defaults(0.01, 3), dam3)
    run_case("dam3d", cfg, dam3, [1, 2], full_lists=False,
             fields=["x", "y", "z", "u", "v", "w", "p", "pnew", "n", "nstar", "bcon", "source"])
    # 3. weakly compressible (Method 3, kernel 6) on the 2D dam
    cfg = config.with_box(config.reference_defaults(0.01, 2, compressible=True), dam2)
    cfg["re_s"] = cfg["re_l"] = 0.04
    run_case("dam2d_wc", cfg, dam2, [1, 10])
    # 4. HL Laplacian (matopt) and HS+ECS source (srcopt)
    cfg = config.with_box(config.reference_defaults(0.01, 2), dam2)
    cfg["matopt"] = 1
    run_case("dam2d_matopt", cfg, dam2, [5])
    cfg = config.with_box(config.reference_defaults(0.01, 2), dam2)
    cfg["srcopt"] = 1
    run_case("dam2d_srcopt", cfg, dam2, [5])
    # 5. two-phase with SPS turbulence and a Herschel-Bulkley second fluid
    tp = cases.dam_break(2, 0.01, (20, 20), (60, 40), blocks=[(2, (0, 20), (15, 15))])
    cfg = config.with_box(config.reference_defaults(0.01, 2), tp)
    cfg.update(turb=1, fluid2_type=1, rho2=900.0, nu2=1e-4, n_pl=1.3, meu0=0.04, cohes=5.0)
    run_case("twophase_turb_hb", cfg, tp, [1, 8])
    # 6. the config-0 dam geometry at a single radius (re = 4.0 l0, dt = 1e-4)
    c0cfg, c0case = config.baseline(0)
    cfg = dict(c0cfg)
    cfg["re_s"] = cfg["re_l"] = 4.0 * cfg["l0"]
    run_case("config0_single_radius", cfg, c0case, [1, 10])
    # 7. a small 3D dam at the config-1 spacing and radius 4.0*l0, SPS on
    g3 = cases.dam_break(3, 0.005, (6, 10, 6), (20, 14, 8))
    cfg = config.with_box(config.reference_defaults(0.005, 3), g3)
    cfg.update(re_s=4.0 * 0.005, re_l=4.0 * 0.005, dt=5e-5, gy=-9.81, turb=1)
    run_case("gen3d_turb", cfg, g3, [1, 3], full_lists=False)


if __name__ == "__main__":
    # --collision: only the collision and .grd-input fixtures
    if "--collision" in sys.argv:
        main_collision()
    else:
        main()
        main_collision()
