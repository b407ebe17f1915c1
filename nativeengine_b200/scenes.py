"""Seeded synthetic scenes: the benchmark configurations and small test worlds.

All randomness comes from numpy's PCG64 with fixed seeds.  A scene is a
``(params, BodyArrays)`` pair that both the device path and the oracle take.

Benchmark configurations (shapes, sizes and distributions as specified):
  gas_1000        periodic elastic gas: 1,000 spheres r=0.5, m=1, L=25,
                  uniform centres with overlap rejection, v ~ N(0,1), e=1,
                  mu=0, g=0, dt=1/60
  box_pile_4096   open boundary: static ground box (50,1,50) + 4,096 boxes with
                  half extents U[0.25,0.75]^3, density 1, random unit
                  quaternions, 16^3 lattice at spacing 1.6 from y=2; mu=0.5,
                  e=0.2, g=-9.81, dt=1/60
  granular_mix    periodic mix of spheres / capsules / cylinders / 12-point
                  hulls at a target packing fraction, v ~ N(0,0.5), mu=0.3,
                  e=0.5, g=0
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from . import _ffi
from .bodies import (Body, BodyArrays, default_params, make_box, make_capsule, make_convex, make_cylinder,
                     make_plane, make_sphere, make_static, normalized_quat, PI)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def random_quat(rng) -> tuple:
    return normalized_quat(rng.normal(0.0, 1.0, 4))


def gas(n: int = 1000, half: float = 12.5, radius: float = 0.5, mass: float = 1.0, seed: int = 1,
        sigma_v: float = 1.0, dt: float = 1.0 / 60.0):
    """Periodic elastic sphere gas with min-image overlap rejection."""
    rng = _rng(seed)
    L = 2.0 * half
    density = mass / ((4.0 / 3.0) * PI * radius * radius * radius)
    pts = np.empty((0, 3))
    bodies: List[Body] = []
    dmin2 = (2.0 * radius) ** 2
    attempts = 0
    while len(bodies) < n:
        attempts += 1
        if attempts > 1000 * n:
            raise RuntimeError("gas placement did not converge")
        c = rng.uniform(-half, half, 3)
        if len(pts):
            d = pts - c
            d -= L * np.floor(d / L + 0.5)
            if np.min(np.einsum("ij,ij->i", d, d)) < dmin2:
                continue
        pts = np.vstack([pts, c])
        b = make_sphere(tuple(c), radius, density)
        b.v = tuple(rng.normal(0.0, sigma_v, 3))
        bodies.append(b)
    params = default_params(half=half, periodic=1, dt=dt, restitution=1.0, friction=0.0, gravity=(0, 0, 0))
    return params, BodyArrays(bodies)


def box_pile(nx: int = 16, ny: int = 16, nz: int = 16, seed: int = 2, spacing: float = 1.6, y0: float = 2.0,
             dt: float = 1.0 / 60.0):
    """Boxes dropped from a lattice onto a static ground box (open boundary)."""
    rng = _rng(seed)
    bodies: List[Body] = [make_static(make_box((0.0, -1.0, 0.0), (1.0, 0.0, 0.0, 0.0), (50.0, 1.0, 50.0), 1.0))]
    cx, cz = (nx - 1) / 2.0, (nz - 1) / 2.0
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                he = tuple(rng.uniform(0.25, 0.75, 3))
                q = random_quat(rng)
                x = ((i - cx) * spacing, y0 + j * spacing, (k - cz) * spacing)
                bodies.append(make_box(x, q, he, 1.0))
    params = default_params(open_boundary=1, gravity=(0.0, -9.81, 0.0), dt=dt, friction=0.5, restitution=0.2)
    return params, BodyArrays(bodies)


def _hull_points(rng, npts=12, scale=0.5):
    pts = []
    while len(pts) < npts:
        p = rng.uniform(-1.0, 1.0, 3)
        if p @ p <= 1.0:
            pts.append(tuple(p * scale))
    return pts


def granular_mix(n: int = 65536, phi: float = 0.3, seed: int = 3, max_attempts: int = 60,
                 dt: float = 1.0 / 60.0):
    """Periodic granular mix, placed by random sequential addition with
    bounding-sphere rejection.  The box edge is chosen for the target packing
    fraction of the true shape volumes and grown until every body places."""
    rng = _rng(seed)
    protos = []
    vols = []
    for idx in range(n):
        t = idx % 4
        if t == 0:
            r = rng.uniform(0.3, 0.6)
            protos.append(("s", r))
            vols.append(4.0 / 3.0 * math.pi * r ** 3)
        elif t == 1:
            hh = rng.uniform(0.2, 0.6)
            protos.append(("c", 0.25, hh))
            vols.append(math.pi * 0.25 ** 2 * 2 * hh + 4.0 / 3.0 * math.pi * 0.25 ** 3)
        elif t == 2:
            protos.append(("y", 0.3, 0.8))
            vols.append(math.pi * 0.09 * 0.8)
        else:
            pts = _hull_points(rng)
            protos.append(("h", pts))
            vols.append(_hull_volume(np.array(pts)))
    bound = []
    for p in protos:
        if p[0] == "s":
            bound.append(p[1])
        elif p[0] == "c":
            bound.append(p[1] + p[2])
        elif p[0] == "y":
            bound.append(math.sqrt(0.4 * 0.4 + 0.3 * 0.3))
        else:
            bound.append(max(math.sqrt(x * x + y * y + z * z) for x, y, z in p[1]))
    bound = np.array(bound)
    L = (sum(vols) / phi) ** (1.0 / 3.0)
    while True:
        centres = _rsa_periodic(bound, L, rng, max_attempts)
        if centres is not None:
            break
        L *= 1.03
    half = L / 2.0
    bodies: List[Body] = []
    for idx, (p, c) in enumerate(zip(protos, centres)):
        q = random_quat(rng)
        if p[0] == "s":
            b = make_sphere(tuple(c), p[1], 1.0)
        elif p[0] == "c":
            b = make_capsule(tuple(c), q, p[1], p[2], 1.0)
        elif p[0] == "y":
            b = make_cylinder(tuple(c), q, p[1], p[2], 1.0)
        else:
            b = make_convex(tuple(c), q, p[1], 1.0)
        b.v = tuple(rng.normal(0.0, 0.5, 3))
        bodies.append(b)
    params = default_params(half=half, periodic=1, dt=dt, friction=0.3, restitution=0.5, gravity=(0, 0, 0))
    ba = BodyArrays(bodies)
    ba.packing_fraction = float(sum(vols) / L ** 3)
    return params, ba


def _hull_volume(pts: np.ndarray) -> float:
    try:
        from scipy.spatial import ConvexHull
        return float(ConvexHull(pts).volume)
    except Exception:
        ext = pts.max(0) - pts.min(0)
        return float(np.prod(ext)) * 0.3


def _rsa_periodic(bound: np.ndarray, L: float, rng, max_attempts: int):
    """Sequential placement with a cell list; None if some body never fits."""
    n = len(bound)
    cell = 2.0 * float(bound.max())
    nc = max(1, int(math.floor(L / cell)))
    cs = L / nc
    grid = {}
    centres = np.empty((n, 3))
    for i in range(n):
        ri = bound[i]
        ok = False
        for _ in range(max_attempts):
            c = rng.uniform(-L / 2, L / 2, 3)
            g = tuple(int(math.floor((c[a] + L / 2) / cs)) % nc for a in range(3))
            clash = False
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        key = ((g[0] + dx) % nc, (g[1] + dy) % nc, (g[2] + dz) % nc)
                        for j in grid.get(key, ()):
                            d = centres[j] - c
                            d -= L * np.floor(d / L + 0.5)
                            rr = ri + bound[j]
                            if d @ d < rr * rr:
                                clash = True
                                break
                        if clash:
                            break
                    if clash:
                        break
                if clash:
                    break
            if not clash:
                ok = True
                break
        if not ok:
            return None
        centres[i] = c
        grid.setdefault(g, []).append(i)
    return centres


# ---- small worlds for parity tests -----------------------------------------

def small_gas(n=50, half=8.0, periodic=True, seed=999, dt=5e-3, spin=True):
    """Random overlapping sphere gas in the style of the reference's makeGas."""
    rng = _rng(seed)
    bodies = []
    for _ in range(n):
        b = make_sphere(tuple(rng.uniform(-6.0, 6.0, 3)), 1.0, 1.0)
        b.v = tuple(rng.uniform(-2.0, 2.0, 3))
        if spin:
            b.w = tuple(rng.uniform(-2.0, 2.0, 3))
        bodies.append(b)
    params = default_params(half=half, periodic=1 if periodic else 0, dt=dt, restitution=1.0)
    return params, BodyArrays(bodies)


def mixed_shapes(n=96, half=6.0, periodic=True, seed=7, dt=1.0 / 60.0, friction=0.3, restitution=0.5,
                 with_plane=False, gravity=(0.0, 0.0, 0.0)):
    """Dense random mix of every supported convex shape (overlapping starts)."""
    rng = _rng(seed)
    bodies = []
    if with_plane:
        bodies.append(make_plane((0.0, -half + 0.5, 0.0), (0.0, 1.0, 0.0)))
    for idx in range(n):
        t = idx % 5
        c = tuple(rng.uniform(-half * 0.9, half * 0.9, 3))
        q = random_quat(rng)
        if t == 0:
            b = make_sphere(c, rng.uniform(0.3, 0.7), 1.0)
        elif t == 1:
            b = make_box(c, q, tuple(rng.uniform(0.25, 0.7, 3)), 1.0)
        elif t == 2:
            b = make_capsule(c, q, 0.25, rng.uniform(0.2, 0.6), 1.0)
        elif t == 3:
            b = make_cylinder(c, q, 0.3, 0.8, 1.0)
        else:
            b = make_convex(c, q, _hull_points(rng), 1.0)
        b.v = tuple(rng.normal(0.0, 1.0, 3))
        b.w = tuple(rng.normal(0.0, 0.5, 3))
        bodies.append(b)
    params = default_params(half=half, periodic=1 if periodic else 0, dt=dt, friction=friction,
                            restitution=restitution, gravity=gravity)
    return params, BodyArrays(bodies)


def box_stack(levels=6, friction=0.6, dt=1.0 / 240.0):
    """A tall stack of unit boxes on a static floor (warm-start settling)."""
    bodies = [make_static(make_box((0.0, -1.0, 0.0), (1, 0, 0, 0), (20.0, 1.0, 20.0), 1.0))]
    for i in range(levels):
        bodies.append(make_box((0.0, 1.0 + i * 2.0, 0.0), (1, 0, 0, 0), (1.0, 1.0, 1.0), 1.0))
    params = default_params(half=1000.0, dt=dt, gravity=(0.0, -10.0, 0.0), restitution=0.0, friction=friction)
    return params, BodyArrays(bodies)
