"""The reference's scenario lattices (generateSimulationCases).

Each function here builds the particle set that the reference's case
generator writes for the same spacing DL and size multiplier mult
(generateSimulationCases/genParticlesFunctions.cpp), in the same particle
order and with its coordinates rounded to the 6 decimals of its "%lf"
output, so that a case built here is the .grd file the reference would have
produced.  The layouts are the reference's and are kept alike on purpose:
its users' scenarios must run unchanged.  Returned dicts have the format of
voxarmps_b200.cases (x, y, z, ptype, u, v, w, p, dim, l0) plus "header",
the particle count the reference writes on the file's first line.

Two reference defects are not reproduced: the oil-spill header passes a
double to "%d" (the count on its first line is undefined; here it is the
number of particles), and the first Poiseuille wall row passes one value to
"%lf %lf" (its y is undefined; here it is 0).
"""
from __future__ import annotations

import math

import numpy as np


class _Lattice:
    def __init__(self, dim: int, l0: float, round6: bool):
        self.dim, self.l0, self.round6 = dim, l0, round6
        self.rows = []

    def add(self, x, y, z, ptype, u=0.0, v=0.0, w=0.0):
        self.rows.append((x, y, z, ptype, u, v, w))

    def case(self, header):
        a = np.array([r[:3] for r in self.rows], np.float64).reshape(-1, 3)
        if self.round6:  # the reference prints "%lf"
            a = np.array([[float(f"{c:f}") for c in row] for row in a], np.float64).reshape(-1, 3)
        vel = np.array([r[4:] for r in self.rows], np.float64).reshape(-1, 3)
        n = len(self.rows)
        return {"dim": self.dim, "l0": self.l0, "x": a[:, 0].copy(), "y": a[:, 1].copy(),
                "z": a[:, 2].copy() if self.dim == 3 else np.zeros(n),
                "ptype": np.array([r[3] for r in self.rows], np.int32),
                "u": vel[:, 0].copy(), "v": vel[:, 1].copy(),
                "w": vel[:, 2].copy() if self.dim == 3 else np.zeros(n), "p": np.zeros(n),
                "header": int(header) if header is not None else n}


def _box2d(L, dx, dy, xl, mp, left_right):
    """Bottom and side walls of the 2D tanks: two dummy-free layer sets
    (PTYPE -1 outermost, then two PTYPE 0 layers), as the dam, RT and oil
    cases lay them out.  left_right = (dummy left, dummy right) counts; the
    wall layers have one and two fewer."""
    nl, nr = left_right
    for i in range(2 * mp + 5):
        L.add(i * dx, 0.0, 0.0, -1)
    for i in range(nl):
        L.add(0.0, i * dy + dy, 0.0, -1)
    for i in range(nr):
        L.add(2 * xl + 5 * dx, i * dy, 0.0, -1)
    for i in range(2 * mp + 3):
        L.add(i * dx + dx, dy, 0.0, 0)
    for i in range(nl - 1):
        L.add(dx, i * dy + 2 * dy, 0.0, 0)
    for i in range(nr - 1):
        L.add(2 * xl + 4 * dx, i * dy + dy, 0.0, 0)
    for i in range(2 * mp + 1):
        L.add(i * dx + 2 * dx, 2 * dy, 0.0, 0)
    for i in range(nl - 2):
        L.add(2 * dx, i * dy + 3 * dy, 0.0, 0)
    for i in range(nr - 2):
        L.add(2 * xl + 3 * dx, i * dy + 2 * dy, 0.0, 0)


def dam_break_2d(DL: float, mult: float, round6: bool = True) -> dict:
    """createParticlesDamBreak2D (genParticlesFunctions.cpp:124-219)."""
    mp = int(36 * mult)
    np_ = int(36 * mult)
    xl, yl = mp * DL, np_ * DL
    dx, dy = xl / mp, yl / np_
    L = _Lattice(2, DL, round6)
    _box2d(L, dx, dy, xl, mp, (mp + 6, mp + 7))
    for i in range(mp // 2):
        for j in range(np_):
            L.add(i * dx + 3 * dx, j * dy + 3 * dy, 0.0, 1)
    header = (mp // 2) * np_ + (4 * mp + 3 * 1 + 7) + (4 * mp + 3 * 3 + 5) + (4 * mp + 3 * 5 + 3)
    return L.case(header)


def rt_instability_2d(DL: float, mult: float, round6: bool = True) -> dict:
    """createParticlesRTinstability (genParticlesFunctions.cpp:329-405): the
    dam tank filled with a heavy fluid (PTYPE 1) above a light one (PTYPE 2)."""
    mp = int(36 * mult)
    np_ = int(36 * mult)
    xl, yl = mp * DL, np_ * DL
    dx, dy = xl / mp, yl / np_
    L = _Lattice(2, DL, round6)
    _box2d(L, dx, dy, xl, mp, (mp + 6, mp + 7))
    for i in range(2 * mp):
        for j in range(np_ // 2):
            L.add(i * dx + 3 * dx, j * dy + 3 * dy, 0.0, 2)
    for i in range(2 * mp):
        for j in range(np_ // 2, np_):
            L.add(i * dx + 3 * dx, j * dy + 3 * dy, 0.0, 1)
    header = 2 * mp * np_ + (4 * mp + 3 * 1 + 7) + (4 * mp + 3 * 3 + 5) + (4 * mp + 3 * 5 + 3)
    return L.case(header)


def oil_spill_2d(DL: float, mult: float, round6: bool = True) -> dict:
    """createParticlesOilSpill2D (genParticlesFunctions.cpp:3-122): a long
    tank with a water layer (PTYPE 1), an oil block (PTYPE 2) and a
    three-particle-thick barrier with a gap."""
    mp = int(mult * 200)
    np_ = int(mult * 25)
    xl = mp * DL
    yl = mp * DL
    dx, dy = xl / mp, yl / mp
    mp2 = float(mp)
    offset_wall = xl * 2 - 28 * dx * mult
    size_water = int(mp2 * 465 * dx)
    L = _Lattice(2, DL, round6)
    _box2d(L, dx, dy, xl, mp, (mp // 4 + 25, mp // 4 + 26))
    for i in range(3):
        for j in range(mp // 20):
            L.add(i * dx + 2 * dx + offset_wall, j * dy + 3 * dy, 0.0, 0)
    top = (mp // 20 + 3) + (mp // 10) * 3 - 20 * (mult - 1)
    for i in range(3):
        j = mp // 20 + 3
        while j < top:
            L.add(i * dx + 2 * dx + offset_wall, j * dy + 3 * dy, 0.0, 0)
            j += 1
    for i in range(size_water - 1):
        for j in range(np_):
            L.add(i * dx + 3 * dx, j * dy + 3 * dy, 0.0, 1)
    i = size_water + 2
    while i < size_water + 28 * mult:
        for j in range(2 * np_ + 13):
            L.add(i * dx + 3 * dx, j * dy + 3 * dy, 0.0, 2)
        i += 1
    return L.case(None)


def shear_cavity_2d(DL: float, mult: float, round6: bool = True) -> dict:
    """createParticlesShearCavity2D (genParticlesFunctions.cpp:221-296): a
    closed square cavity whose two top wall layers move with u = 1."""
    mp = int(36 * mult)
    np_ = int(36 * mult)
    xl, yl = mp * DL, np_ * DL
    dx, dy = xl / mp, yl / np_
    L = _Lattice(2, DL, round6)
    for i in range(mp):
        L.add(i * dx, 0.0, 0.0, 0)
    for i in range(np_):
        L.add(0.0 * dx, i * dy + dy, 0.0, 0)
    for i in range(np_):
        L.add(xl, i * dy, 0.0, 0)
    for i in range(mp):
        L.add(i * dx + dx, yl, 0.0, 0)
    for i in range(mp - 2):
        L.add(i * dx + dx, dy, 0.0, 0)
    for i in range(np_ - 2):
        L.add(dx, i * dy + 2 * dy, 0.0, 0)
    for i in range(np_ - 2):
        L.add(xl - dx, i * dy + dy, 0.0, 0)
    for i in range(mp - 2):
        L.add(i * dx + 2 * dx, yl - dy, 0.0, 0, u=1.0)
    for i in range(mp - 4):
        L.add(i * dx + 2 * dx, 2 * dy, 0.0, 0)
    for i in range(np_ - 4):
        L.add(2 * dx, i * dy + 3 * dy, 0.0, 0)
    for i in range(np_ - 4):
        L.add(xl - 2 * dx, i * dy + 2 * dy, 0.0, 0)
    for i in range(mp - 4):
        L.add(i * dx + 3 * dx, yl - 2 * dy, 0.0, 0, u=1.0)
    for i in range(mp - 7):
        for j in range(np_ - 6):
            L.add(i * dx + 4 * dx, 4 * dy + dy * j, 0.0, 1)
    header = ((mp - 7) * (np_ - 6) + 2 * (mp - 4) + 2 * (np_ - 4) + 2 * (mp - 2) + 2 * (np_ - 2)
              + 4 * mp)
    return L.case(header)


def water_drop_2d(DL: float, mult: float, round6: bool = True) -> dict:
    """createParticlesWaterDrop2D (genParticlesFunctions.cpp:298-327): a free
    circular drop of radius 18 mult particles (the reference writes the
    count of mult = 1, 1005, whatever mult is)."""
    mp = int(18 * mult)
    xl = mp * DL
    dx = xl / mp
    L = _Lattice(2, DL, round6)
    for i in range(-mp, mp):
        for j in range(-mp, mp):
            if i * i + j * j < mp * mp:
                L.add(i * dx + 2 * mp * dx, j * dx + 2 * mp * dx, 0.0, 1)
    return L.case(1005)


def poiseuille_2d(DL: float, mult: float, round6: bool = True) -> dict:
    """createParticlesPoiseuilleFlow2D (genParticlesFunctions.cpp:407-453): a
    channel between two moving walls (u = -0.1) with the fluid at u = 0.5."""
    mp = int(140 * mult)
    np_ = int(70 * mult)
    xl, yl = mp * DL, np_ * DL
    dx, dy = xl / mp, yl / np_
    L = _Lattice(2, DL, round6)
    for i in range(mp):
        L.add(i * dx, 0.0, 0.0, -1)  # reference: y undefined (one argument for two)
    for i in range(mp):
        L.add(i * dx, dy * np_, 0.0, -1)
    for j in (1, 2):
        for i in range(mp):
            L.add(i * dx, dy * j, 0.0, 0, u=-0.1)
        for i in range(mp):
            L.add(i * dx, dy * (np_ - j), 0.0, 0, u=-0.1)
    for j in range(3, np_ - 2):
        for i in range(1, mp - 1):
            L.add(i * dx, dy * j, 0.0, 1, u=0.5)
    header = (np_ - 5) * (mp - 2) + 2 * mp + 2 * mp + 2 * mp
    return L.case(header)


def _walls3d(L, mp, op, dx, dy, dz, xl, off, inner_face):
    """The 3D tanks' dummy and wall layers (dam_break_3d and its offset
    variant differ only in the inner faces' extents, inner_face)."""
    ox, oy, oz = off
    for k in range(op + 6):
        for i in range(2 * mp + 6):
            L.add(i * dx + ox, 0.0 + oy, dz * k - 3 * dz + oz, -1)
        for i in range(mp + 6):
            L.add(0.0 + ox, i * dy + dy + oy, dz * k - 3 * dz + oz, -1)
        for i in range(mp + 6):
            L.add(2 * xl + 5 * dx + ox, i * dy + dy + oy, dz * k - 3 * dz + oz, -1)
    for zf in (-3 * dz, (op + 2) * dz):
        for i in range(2 * mp + 4):
            for j in range(mp + 6):
                L.add(i * dx + dx + ox, j * dy + dy + oy, zf + oz, -1)
    for k in range(op + 4):
        for i in range(2 * mp + 4):
            L.add(i * dx + dx + ox, dy + oy, dz * k - 2 * dz + oz, 0)
        for i in range(mp + 5):
            L.add(dx + ox, i * dy + 2 * dy + oy, dz * k - 2 * dz + oz, 0)
        for i in range(mp + 5):
            L.add(2 * xl + 4 * dx + ox, i * dy + 2 * dy + oy, dz * k - 2 * dz + oz, 0)
    for zf in (-2 * dz, (op + 1) * dz):
        for i in range(2 * mp + 2):
            for j in range(mp + 5):
                L.add(i * dx + 2 * dx + ox, 2 * dy + j * dy + oy, zf + oz, 0)
    for k in range(op):
        for i in range(2 * mp + 1):
            L.add(i * dx + 2 * dx + ox, 2 * dy + oy, dz * k + oz, 0)
        for i in range(mp + 4):
            L.add(2 * dx + ox, i * dy + 3 * dy + oy, dz * k + oz, 0)
        for i in range(mp + 5):
            L.add(2 * xl + 3 * dx + ox, i * dy + 2 * dy + oy, dz * k + oz, 0)
    ni, nj = inner_face
    for zf in (-dz, op * dz):
        for i in range(ni):
            for j in range(nj):
                L.add(i * dx + 2 * dx + ox, 2 * dy + j * dy + oy, zf + oz, 0)


def dam_break_3d(DL: float, mult: float, round6: bool = True) -> dict:
    """createParticlesDamBreak3D (genParticlesFunctions.cpp:455-558)."""
    mp, np_, op = int(16 * mult), int(8 * mult), int(8 * mult)
    xl, yl, zl = mp * DL, np_ * DL, op * DL
    dx, dy, dz = xl / mp, yl / np_, zl / op
    L = _Lattice(3, DL, round6)
    _walls3d(L, mp, op, dx, dy, dz, xl, (0.0, 0.0, 0.0), (2 * mp + 2, mp + 5))
    for k in range(op):
        for i in range(mp // 2):
            for j in range(2 * np_):
                L.add(i * dx + 3 * dx, j * dy + 3 * dy, dz * k, 1)
    header = (op * (mp * np_) + op * (4 * mp + 10) + (4 * mp + 4) * (mp + 5)
              + (op + 4) * (4 * mp + 14) + (4 * mp + 4) * (mp + 5)
              + (op + 6) * (4 * mp + 18) + (4 * mp + 8) * (mp + 6))
    return L.case(header)


def dam_break_3d_offset(DL: float, mult: float, round6: bool = True) -> dict:
    """createParticlesDamBreak3D_offset_nozero (genParticlesFunctions.cpp:560-673)."""
    mp, np_, op = int(10 * mult), int(5 * mult), int(5 * mult)
    xl, yl, zl = mp * DL, np_ * DL, op * DL
    dx, dy, dz = xl / mp, yl / np_, zl / op
    off = (0 * dx, 0 * dx, 0 * dx)
    L = _Lattice(3, DL, round6)
    _walls3d(L, mp, op, dx, dy, dz, xl, off, (2 * mp, mp + 4))
    for k in range(op):
        for i in range(mp // 2):
            for j in range(np_):
                L.add(i * dx + 3 * dx + off[0], j * dy + 3 * dy + off[1], dz * k + off[2], 1)
    header = (op * (mp * np_ // 2) + op * (4 * mp + 10) + (4 * mp) * (mp + 4)
              + (op + 4) * (4 * mp + 14) + (4 * mp + 4) * (mp + 5)
              + (op + 6) * (4 * mp + 18) + (4 * mp + 8) * (mp + 6))
    return L.case(header)


GENERATORS = {
    "dam_break_2d": dam_break_2d, "rt_instability_2d": rt_instability_2d,
    "oil_spill_2d": oil_spill_2d, "shear_cavity_2d": shear_cavity_2d,
    "water_drop_2d": water_drop_2d, "poiseuille_2d": poiseuille_2d,
    "dam_break_3d": dam_break_3d, "dam_break_3d_offset": dam_break_3d_offset,
}
