"""Seeded synthetic geometries for the workloads the engine is measured on.

No public dataset is involved; these generators produce inputs of the sizes
and value distributions of the five workloads:

* ``benzene()``            12-atom planar C6H6 ring (C-C 1.39 A, C-H 1.09 A,
                           ring in the xz-plane, H radially outward), Hirshfeld
                           ratio 0.806 (C) / 0.602 (H), isolated.
* ``cluster(N, seed)``     isolated {H,C,N,O} cluster, species weights
                           0.45/0.35/0.10/0.10, random sequential packing in a
                           sphere at 0.1 atoms/A^3 with minimum pair distance
                           0.95 A, Hirshfeld ratio ~ U(0.6, 1.0).
* ``graphene_sheet()``     hexagonal carbon, a = 2.46 A, 2-atom cell tiled 8x8
                           (128 atoms), 20 A along z with vacuum axis z,
                           Hirshfeld ratio 0.77; cut-offs 120/100/25 A.
* ``cluster_batch()``      256 clusters with N ~ U{20..600}.
* ``periodic_box(N, seed)`` cubic periodic box at 0.1 atoms/A^3 packed as the
                           clusters, cut-offs 120/100/25 A.
"""
from __future__ import annotations

import math

import numpy as np

from .io import Geometry, Settings

SPECIES = ("H", "C", "N", "O")
WEIGHTS = (0.45, 0.35, 0.10, 0.10)
DENSITY = 0.1          # atoms / A^3
MIN_DIST = 0.95        # A


def benzene() -> tuple[Geometry, Settings]:
    cc, ch = 1.39, 1.09
    names, xyz, hv = [], [], []
    for k in range(6):
        t = 2.0 * math.pi * k / 6.0
        names.append("C")
        xyz.append([cc * math.cos(t), 0.0, cc * math.sin(t)])
        hv.append(0.806)
    for k in range(6):
        t = 2.0 * math.pi * k / 6.0
        names.append("H")
        xyz.append([(cc + ch) * math.cos(t), 0.0, (cc + ch) * math.sin(t)])
        hv.append(0.602)
    return Geometry(names, np.array(xyz), np.array(hv)), Settings(xc=1)


def _pack(n: int, rng: np.random.Generator, inside, sample, min_dist: float, periodic_box=None):
    pts = np.zeros((n, 3))
    placed = 0
    tries = 0
    while placed < n:
        tries += 1
        if tries > 200 * n + 10000:
            raise RuntimeError("random sequential packing did not converge")
        p = sample()
        if not inside(p):
            continue
        if placed:
            d = pts[:placed] - p
            if periodic_box is not None:
                d -= periodic_box * np.round(d / periodic_box)
            if np.min(np.einsum("ij,ij->i", d, d)) < min_dist * min_dist:
                continue
        pts[placed] = p
        placed += 1
    return pts


def _species(n: int, rng: np.random.Generator):
    idx = rng.choice(len(SPECIES), size=n, p=np.array(WEIGHTS))
    return [SPECIES[i] for i in idx]


def cluster(n: int, seed: int = 0) -> tuple[Geometry, Settings]:
    rng = np.random.default_rng(seed)
    radius = (3.0 * n / (4.0 * math.pi * DENSITY)) ** (1.0 / 3.0)
    pts = _pack(n, rng, lambda p: float(p @ p) <= radius * radius,
                lambda: rng.uniform(-radius, radius, 3), MIN_DIST)
    names = _species(n, rng)
    hv = rng.uniform(0.6, 1.0, n)
    return Geometry(names, pts, hv), Settings(xc=1)


def graphene_sheet(reps: int = 8, a: float = 2.46, c: float = 20.0) -> tuple[Geometry, Settings]:
    a1 = np.array([a, 0.0, 0.0])
    a2 = np.array([0.5 * a, 0.5 * math.sqrt(3.0) * a, 0.0])
    basis = [np.zeros(3), (a1 + a2) / 3.0]
    xyz = []
    for i in range(reps):
        for j in range(reps):
            for b in basis:
                xyz.append(i * a1 + j * a2 + b)
    n = len(xyz)
    lat = np.array([reps * a1, reps * a2, [0.0, 0.0, c]])
    geo = Geometry(["C"] * n, np.array(xyz), np.full(n, 0.77), lat, 3)
    st = Settings(xc=1, mbd_supercell_cutoff=25.0, mbd_cfdm_dip_cutoff=100.0, mbd_scs_dip_cutoff=120.0,
                  mbd_scs_vacuum_axis=(False, False, True))
    return geo, st


def cluster_batch(count: int = 256, nmin: int = 20, nmax: int = 600, seed: int = 0):
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nmin, nmax + 1, size=count)
    return [cluster(int(n), seed=1000 + k) for k, n in enumerate(sizes)]


def periodic_box(n: int, seed: int = 0, scs_cut=120.0, cfdm_cut=100.0, sc_cut=25.0) -> tuple[Geometry, Settings]:
    rng = np.random.default_rng(seed)
    side = (n / DENSITY) ** (1.0 / 3.0)
    box = np.array([side, side, side])
    pts = _pack(n, rng, lambda p: True, lambda: rng.uniform(0.0, side, 3), MIN_DIST, periodic_box=box)
    names = _species(n, rng)
    hv = rng.uniform(0.6, 1.0, n)
    geo = Geometry(names, pts, hv, np.diag(box), 3)
    st = Settings(xc=1, mbd_supercell_cutoff=sc_cut, mbd_cfdm_dip_cutoff=cfdm_cut, mbd_scs_dip_cutoff=scs_cut)
    return geo, st
