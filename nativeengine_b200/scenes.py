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


def granular_mix(n: int = 65536, phi: float = 0.3, seed: int = 3, max_attempts: int = 400,
                 dt: float = 1.0 / 60.0, grow: float = 1.02):
    """Periodic granular mix (types by index mod 4: sphere r U[0.3,0.6], capsule
    r 0.25 half-height U[0.2,0.6], cylinder r 0.3 height 0.8, convex hull of 12
    points uniform in the unit ball scaled by 0.5), random orientations,
    v ~ N(0, 0.5) per axis, mu 0.3, e 0.5, g 0.  Bodies are placed by random
    sequential addition with exact (GJK) overlap rejection; the box edge starts
    at the target packing fraction of the true shape volumes and grows by
    `grow` until every body places.  The achieved fraction is stored as
    ``packing_fraction`` on the returned BodyArrays."""
    import ctypes as C
    rng = _rng(seed)
    bodies: List[Body] = []
    vols = []
    for idx in range(n):
        t = idx % 4
        q = random_quat(rng)
        if t == 0:
            r = rng.uniform(0.3, 0.6)
            b = make_sphere((0.0, 0.0, 0.0), r, 1.0)
            vols.append(4.0 / 3.0 * math.pi * r ** 3)
        elif t == 1:
            hh = rng.uniform(0.2, 0.6)
            b = make_capsule((0.0, 0.0, 0.0), q, 0.25, hh, 1.0)
            vols.append(math.pi * 0.25 ** 2 * 2 * hh + 4.0 / 3.0 * math.pi * 0.25 ** 3)
        elif t == 2:
            b = make_cylinder((0.0, 0.0, 0.0), q, 0.3, 0.8, 1.0)
            vols.append(math.pi * 0.09 * 0.8)
        else:
            pts = _hull_points(rng)
            b = make_convex((0.0, 0.0, 0.0), q, pts, 1.0)
            vols.append(_hull_volume(np.array(pts)))
        b.v = tuple(rng.normal(0.0, 0.5, 3))
        bodies.append(b)
    ba = BodyArrays(bodies)
    lib = _host_lib()
    L = (sum(vols) / phi) ** (1.0 / 3.0)
    xs = np.zeros((n, 3))
    dp = lambda a: a.ctypes.data_as(C.c_void_p)
    while True:
        placed = lib.ne_scene_place_periodic(n, dp(ba.shape), dp(ba.radius), dp(ba.half_height), dp(ba.half_extents),
                                             dp(ba.q), dp(ba.vert_offset), dp(ba.vert_count), dp(ba.verts), L,
                                             seed, max_attempts, dp(xs))
        if placed == n:
            break
        L *= grow
    ba.x[:] = xs
    params = default_params(half=L / 2.0, periodic=1, dt=dt, friction=0.3, restitution=0.5, gravity=(0, 0, 0))
    ba.packing_fraction = float(sum(vols) / L ** 3)
    return params, ba


_HOST = None


def _host_lib():
    """libne_host.so (scene placement lives there; it is host code)."""
    global _HOST
    if _HOST is None:
        import ctypes as C
        import os
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libne_host.so")
        lib = C.CDLL(path)
        fn = lib.ne_scene_place_periodic
        fn.restype = C.c_uint32
        fn.argtypes = [C.c_uint32] + [C.c_void_p] * 8 + [C.c_double, C.c_uint64, C.c_uint32, C.c_void_p]
        _HOST = lib
    return _HOST


def _hull_volume(pts: np.ndarray) -> float:
    try:
        from scipy.spatial import ConvexHull
        return float(ConvexHull(pts).volume)
    except Exception:
        ext = pts.max(0) - pts.min(0)
        return float(np.prod(ext)) * 0.3


def batch_mix(nworlds: int = 2048, lo: int = 16, hi: int = 2048, seed: int = 4, dt: float = 1.0 / 60.0):
    """Independent worlds for the batched form: body counts log-uniform in
    [lo, hi]; each world is (by a seeded coin) a box pile -- static ground box
    plus ceil(n^(1/3))^3 lattice truncated to n boxes -- or a periodic sphere
    gas at the gas_1000 density (edge 25*(n/1000)^(1/3)).  Returns
    (params_list, BodyArrays, world_begin, kinds)."""
    from .bodies import concat
    rng = _rng(seed)
    params, parts, kinds = [], [], []
    for w in range(nworlds):
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        wseed = int(rng.integers(1, 2**31 - 1))
        if rng.integers(0, 2) == 0:
            side = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
            p, b = _pile_truncated(side, n, wseed, dt)
            kinds.append("box_pile")
        else:
            half = 12.5 * (n / 1000.0) ** (1.0 / 3.0)
            p, b = gas(n=n, half=half, seed=wseed, dt=dt)
            kinds.append("gas")
        params.append(p)
        parts.append(b)
    bodies, begin = concat(parts)
    return params, bodies, begin, kinds


def _pile_truncated(side, n, seed, dt):
    rng = _rng(seed)
    bodies: List[Body] = [make_static(make_box((0.0, -1.0, 0.0), (1.0, 0.0, 0.0, 0.0), (50.0, 1.0, 50.0), 1.0))]
    c = (side - 1) / 2.0
    for i in range(side):
        for j in range(side):
            for k in range(side):
                if len(bodies) > n:
                    break
                he = tuple(rng.uniform(0.25, 0.75, 3))
                bodies.append(make_box(((i - c) * 1.6, 2.0 + j * 1.6, (k - c) * 1.6), random_quat(rng), he, 1.0))
    params = default_params(open_boundary=1, gravity=(0.0, -9.81, 0.0), dt=dt, friction=0.5, restitution=0.2)
    return params, BodyArrays(bodies)


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


# ---- triangle meshes and compounds -------------------------------------------

def heightfield_mesh(origin, spacing, rows, cols, heights) -> "MeshData":
    """A rows x cols height grid (row-major heights, spacing in x/z) as a
    triangle mesh, two triangles per cell, with its BVH."""
    from .bodies import MeshData
    verts = [(origin[0] + c * spacing, origin[1] + heights[r * cols + c], origin[2] + r * spacing)
             for r in range(rows) for c in range(cols)]
    tris = []
    for r in range(rows - 1):
        for c in range(cols - 1):
            a, b, d, e = r * cols + c, r * cols + c + 1, (r + 1) * cols + c, (r + 1) * cols + c + 1
            tris += [(a, d, b), (b, d, e)]
    return MeshData(verts, tris).build()


def mesh_floor(dt=1.0 / 240.0):
    """A sphere and a box dropped on a two-triangle floor mesh (the setting of
    the reference's mesh self-test)."""
    from .bodies import MeshData, make_mesh
    floor = MeshData([(-10, 0, -10), (10, 0, -10), (10, 0, 10), (-10, 0, 10)], [(0, 1, 2), (0, 2, 3)]).build()
    bodies = [make_mesh((0.0, 0.0, 0.0), (1, 0, 0, 0), floor),
              make_sphere((1.0, 5.0, 1.0), 0.5, 1.0),
              make_box((-3.0, 5.0, -2.0), (1, 0, 0, 0), (0.5, 0.5, 0.5), 1.0)]
    params = default_params(half=1000.0, dt=dt, gravity=(0.0, -10.0, 0.0), restitution=0.0, friction=0.5)
    return params, BodyArrays(bodies)


def terrain_drop(n=24, rows=9, cols=9, seed=12, dt=1.0 / 120.0):
    """Spheres, boxes, capsules and hulls dropped on a bumpy height-field mesh
    placed off the origin and turned (contacts against many triangles)."""
    from .bodies import make_mesh
    rng = _rng(seed)
    h = [0.6 * math.sin(0.9 * c) * math.cos(0.7 * r) for r in range(rows) for c in range(cols)]
    terrain = heightfield_mesh((-8.0, 0.0, -8.0), 2.0, rows, cols, h)
    bodies = [make_mesh((0.5, -0.2, 0.3), normalized_quat((1.0, 0.0, 0.08, 0.0)), terrain)]
    for k in range(n):
        x = (float(rng.uniform(-5, 5)), float(2.0 + 1.3 * k), float(rng.uniform(-5, 5)))
        kind = k % 4
        if kind == 0:
            bodies.append(make_sphere(x, float(rng.uniform(0.3, 0.6)), 1.0))
        elif kind == 1:
            bodies.append(make_box(x, random_quat(rng), tuple(rng.uniform(0.25, 0.6, 3)), 1.0))
        elif kind == 2:
            bodies.append(make_capsule(x, random_quat(rng), 0.3, float(rng.uniform(0.2, 0.5)), 1.0))
        else:
            bodies.append(make_convex(x, random_quat(rng), _hull_points(rng), 1.0))
    params = default_params(half=1000.0, open_boundary=1, dt=dt, gravity=(0.0, -9.81, 0.0), restitution=0.2,
                            friction=0.5)
    return params, BodyArrays(bodies)


def compound_pile(n=12, seed=21, dt=1.0 / 120.0, with_mesh=False):
    """Compounds of mixed children (dumbbells, tables, capsule crosses) and
    boxes dropped on a static floor box, or on a floor mesh: compound-box,
    compound-compound and (with_mesh) compound-mesh contacts."""
    from .bodies import (MeshData, child_box, child_capsule, child_cylinder, child_sphere, make_compound,
                         make_mesh)
    rng = _rng(seed)
    if with_mesh:
        floor = MeshData([(-12, 0, -12), (12, 0, -12), (12, 0, 12), (-12, 0, 12)], [(0, 1, 2), (0, 2, 3)]).build()
        bodies = [make_mesh((0.0, 0.0, 0.0), (1, 0, 0, 0), floor)]
    else:
        bodies = [make_static(make_box((0.0, -1.0, 0.0), (1, 0, 0, 0), (20.0, 1.0, 20.0), 1.0))]
    for k in range(n):
        x = (float(rng.uniform(-3, 3)), float(2.0 + 1.6 * k), float(rng.uniform(-3, 3)))
        q = random_quat(rng)
        kind = k % 4
        if kind == 0:
            kids = [child_sphere((-0.8, 0.0, 0.0), 0.4), child_sphere((0.8, 0.0, 0.0), 0.4),
                    child_cylinder((0.0, 0.0, 0.0), normalized_quat((1.0, 0.0, 0.0, 1.0)), 0.15, 0.6)]
            bodies.append(make_compound(x, q, kids, 1.0))
        elif kind == 1:
            kids = [child_box((0.0, 0.3, 0.0), (1, 0, 0, 0), (0.8, 0.1, 0.5))] + [
                child_box((sx * 0.6, -0.1, sz * 0.35), (1, 0, 0, 0), (0.08, 0.3, 0.08))
                for sx in (-1, 1) for sz in (-1, 1)]
            bodies.append(make_compound(x, q, kids, 1.0))
        elif kind == 2:
            kids = [child_capsule((0.0, 0.0, 0.0), (1, 0, 0, 0), 0.2, 0.6),
                    child_capsule((0.0, 0.0, 0.0), normalized_quat((1.0, 0.0, 0.0, 1.0)), 0.2, 0.6)]
            bodies.append(make_compound(x, q, kids, 1.0))
        else:
            bodies.append(make_box(x, q, tuple(rng.uniform(0.3, 0.6, 3)), 1.0))
    params = default_params(half=1000.0, open_boundary=1, dt=dt, gravity=(0.0, -9.81, 0.0), restitution=0.1,
                            friction=0.6)
    return params, BodyArrays(bodies)


# ---- adjoint workload --------------------------------------------------------

def sliding_boxes(grid: int = 8, spacing: float = 1.5, mu: float = 0.5, e: float = 0.25, seed: int = 5,
                  vsigma: float = 2.0, dt: float = 1.0 / 60.0):
    """One world of the adjoint workload: a ground plane through the origin
    (normal +y) and grid x grid boxes of half extent 0.5, density 1, resting at
    y = 0.5 on a square grid, with horizontal initial velocities N(0, vsigma^2);
    open boundary, g = -9.81, world friction mu and restitution e (the bodies
    inherit both)."""
    rng = _rng(seed)
    bodies = [make_plane((0.0, 0.0, 0.0), (0.0, 1.0, 0.0))]
    c = (grid - 1) / 2.0
    for i in range(grid):
        for k in range(grid):
            b = make_box(((i - c) * spacing, 0.5, (k - c) * spacing), (1.0, 0.0, 0.0, 0.0), (0.5, 0.5, 0.5), 1.0)
            vx, vz = rng.normal(0.0, vsigma, 2)
            b.v = (float(vx), 0.0, float(vz))
            bodies.append(b)
    params = default_params(open_boundary=1, gravity=(0.0, -9.81, 0.0), dt=dt, friction=mu, restitution=e)
    return params, BodyArrays(bodies)


def adjoint_batch(nworlds: int = 512, grid: int = 8, seed: int = 6):
    """The adjoint workload: nworlds sliding_boxes worlds with per-world
    friction U[0.2, 0.8] and restitution U[0, 0.5], and loss targets
    U[-5, 5]^3 per box.  Returns (params_list, BodyArrays, world_begin,
    targets[n, 3]) (the plane's target row is unused)."""
    from .bodies import concat
    rng = _rng(seed)
    params, parts = [], []
    for w in range(nworlds):
        mu = float(rng.uniform(0.2, 0.8))
        e = float(rng.uniform(0.0, 0.5))
        p, b = sliding_boxes(grid=grid, mu=mu, e=e, seed=int(rng.integers(1, 2**31 - 1)))
        params.append(p)
        parts.append(b)
    bodies, begin = concat(parts)
    targets = rng.uniform(-5.0, 5.0, (bodies.n, 3))
    return params, bodies, begin, targets
