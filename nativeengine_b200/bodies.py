"""Host-side body sets: the shape factories of the reference and their packing
into the structure-of-arrays layout of the C-ABI (``NeBodyArrays``).

The factories reproduce the reference's mass and inertia formulas operation
for operation (``makeSphere`` ... ``makePlane``, src/body.hpp:206-345), so a
body built here carries the same IEEE-754 doubles the reference would compute.
``make_static`` / ``make_kinematic`` mirror ``PhysicsWorld::makeStatic`` /
``makeKinematic`` (src/physics_world.hpp:119-144).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _ffi

PI = 3.14159265358979323846


def _normalized3(v):
    x, y, z = float(v[0]), float(v[1]), float(v[2])
    n = math.sqrt(x * x + y * y + z * z)
    return (x / n, y / n, z / n) if n > 1e-300 else (0.0, 0.0, 0.0)


def normalized_quat(q):
    """Q::normalized (src/vmath.hpp:64-67)."""
    w, x, y, z = (float(c) for c in q)
    n = math.sqrt(w * w + x * x + y * y + z * z)
    return (w / n, x / n, y / n, z / n) if n > 1e-300 else (1.0, 0.0, 0.0, 0.0)


def _inv(v):
    return 1.0 / v if v > 0 else 0.0


def sphere_mass(radius, density):
    m = density * (4.0 / 3.0) * PI * radius * radius * radius
    I = (2.0 / 5.0) * m * radius * radius
    return _inv(m), (_inv(I), _inv(I), _inv(I))


def cylinder_mass(radius, height, density):
    m = density * PI * radius * radius * height
    Iyy = 0.5 * m * radius * radius
    Ixx = (1.0 / 12.0) * m * (3.0 * radius * radius + height * height)
    return _inv(m), (_inv(Ixx), _inv(Iyy), _inv(Ixx))


def box_mass(he, density):
    hx, hy, hz = (float(c) for c in he)
    m = density * 8.0 * hx * hy * hz
    Ix = (1.0 / 3.0) * m * (hy * hy + hz * hz)
    Iy = (1.0 / 3.0) * m * (hx * hx + hz * hz)
    Iz = (1.0 / 3.0) * m * (hx * hx + hy * hy)
    return _inv(m), (_inv(Ix), _inv(Iy), _inv(Iz))


def capsule_mass(radius, half_height, density):
    r, L = radius, 2.0 * half_height
    mc = density * PI * r * r * L
    mh = density * (4.0 / 3.0) * PI * r * r * r
    m = mc + mh
    Iyy = 0.5 * mc * r * r + 0.4 * mh * r * r
    Ixx = mc * (0.25 * r * r + L * L / 12.0) + mh * (0.4 * r * r + 0.25 * L * L)
    return _inv(m), (_inv(Ixx), _inv(Iyy), _inv(Ixx))


def convex_mass(verts, density):
    lo = [1e30, 1e30, 1e30]
    hi = [-1e30, -1e30, -1e30]
    for v in verts:
        for a in range(3):
            c = float(v[a])
            lo[a] = c if c < lo[a] else lo[a]
            hi[a] = c if hi[a] < c else hi[a]
    he = [(hi[a] - lo[a]) * 0.5 for a in range(3)]
    hx, hy, hz = (1e-4 if h < 1e-4 else h for h in he)
    m = density * 8.0 * hx * hy * hz
    Ix = (1.0 / 3.0) * m * (hy * hy + hz * hz)
    Iy = (1.0 / 3.0) * m * (hx * hx + hz * hz)
    Iz = (1.0 / 3.0) * m * (hx * hx + hy * hy)
    return _inv(m), (_inv(Ix), _inv(Iy), _inv(Iz))


@dataclass
class Body:
    shape: int
    x: tuple = (0.0, 0.0, 0.0)
    q: tuple = (1.0, 0.0, 0.0, 0.0)
    v: tuple = (0.0, 0.0, 0.0)
    w: tuple = (0.0, 0.0, 0.0)
    force: tuple = (0.0, 0.0, 0.0)
    torque: tuple = (0.0, 0.0, 0.0)
    inv_mass: float = 0.0
    inv_inertia: tuple = (0.0, 0.0, 0.0)
    radius: float = 1.0
    half_height: float = 0.0
    half_extents: tuple = (0.0, 0.0, 0.0)
    verts: Optional[list] = None
    friction: float = -1.0
    restitution: float = -1.0
    linear_damping: float = 0.0
    angular_damping: float = 0.0
    gravity_scale: float = 1.0
    layer: int = 0
    mask: int = 0xFFFFFFFF
    flags: int = _ffi.DYNAMIC
    nocollide: List[int] = field(default_factory=list)


def make_sphere(x, radius, density) -> Body:
    im, ii = sphere_mass(radius, density)
    return Body(_ffi.SPHERE, x=tuple(map(float, x)), radius=float(radius), inv_mass=im, inv_inertia=ii)


def make_cylinder(x, q, radius, height, density) -> Body:
    im, ii = cylinder_mass(radius, height, density)
    return Body(_ffi.CYLINDER, x=tuple(map(float, x)), q=tuple(map(float, q)), radius=float(radius),
                half_height=0.5 * height, inv_mass=im, inv_inertia=ii)


def make_box(x, q, he, density) -> Body:
    im, ii = box_mass(he, density)
    return Body(_ffi.BOX, x=tuple(map(float, x)), q=tuple(map(float, q)), half_extents=tuple(map(float, he)),
                inv_mass=im, inv_inertia=ii)


def make_capsule(x, q, radius, half_height, density) -> Body:
    im, ii = capsule_mass(radius, half_height, density)
    return Body(_ffi.CAPSULE, x=tuple(map(float, x)), q=tuple(map(float, q)), radius=float(radius),
                half_height=float(half_height), inv_mass=im, inv_inertia=ii)


def make_convex(x, q, verts, density) -> Body:
    vs = [tuple(map(float, v)) for v in verts]
    im, ii = convex_mass(vs, density)
    return Body(_ffi.CONVEX, x=tuple(map(float, x)), q=tuple(map(float, q)), verts=vs, inv_mass=im, inv_inertia=ii)


def make_plane(point, normal) -> Body:
    return Body(_ffi.PLANE, x=tuple(map(float, point)), half_extents=_normalized3(normal), inv_mass=0.0,
                inv_inertia=(0.0, 0.0, 0.0), flags=0)


def make_static(b: Body) -> Body:
    b.inv_mass = 0.0
    b.inv_inertia = (0.0, 0.0, 0.0)
    b.v = (0.0, 0.0, 0.0)
    b.w = (0.0, 0.0, 0.0)
    b.flags &= ~(_ffi.DYNAMIC | _ffi.KINEMATIC)
    return b


def make_kinematic(b: Body) -> Body:
    b.inv_mass = 0.0
    b.inv_inertia = (0.0, 0.0, 0.0)
    b.flags = (b.flags & ~(_ffi.DYNAMIC | _ffi.SLEEPING)) | _ffi.KINEMATIC
    return b


class BodyArrays:
    """Structure-of-arrays image of a body list, plus its NeBodyArrays view.

    The numpy arrays are owned here; ``.c`` points into them, so keep this
    object alive while the C struct is in use.
    """

    STATE = ("x", "q", "v", "w")

    def __init__(self, bodies: Sequence[Body]):
        n = len(bodies)
        self.n = n
        f64 = np.float64
        self.x = np.array([b.x for b in bodies], dtype=f64).reshape(n, 3)
        self.q = np.array([b.q for b in bodies], dtype=f64).reshape(n, 4)
        self.v = np.array([b.v for b in bodies], dtype=f64).reshape(n, 3)
        self.w = np.array([b.w for b in bodies], dtype=f64).reshape(n, 3)
        self.force = np.array([b.force for b in bodies], dtype=f64).reshape(n, 3)
        self.torque = np.array([b.torque for b in bodies], dtype=f64).reshape(n, 3)
        self.inv_mass = np.array([b.inv_mass for b in bodies], dtype=f64)
        self.inv_inertia = np.array([b.inv_inertia for b in bodies], dtype=f64).reshape(n, 3)
        self.shape = np.array([b.shape for b in bodies], dtype=np.int32)
        self.radius = np.array([b.radius for b in bodies], dtype=f64)
        self.half_height = np.array([b.half_height for b in bodies], dtype=f64)
        self.half_extents = np.array([b.half_extents for b in bodies], dtype=f64).reshape(n, 3)
        vo, vc, vl = [], [], []
        for b in bodies:
            vo.append(len(vl))
            vs = b.verts or []
            vc.append(len(vs))
            vl.extend(vs)
        self.vert_offset = np.array(vo, dtype=np.uint32)
        self.vert_count = np.array(vc, dtype=np.uint32)
        self.verts = np.array(vl if vl else [(0.0, 0.0, 0.0)], dtype=f64).reshape(-1, 3)
        self.n_verts = len(vl)
        self.friction = np.array([b.friction for b in bodies], dtype=f64)
        self.restitution = np.array([b.restitution for b in bodies], dtype=f64)
        self.linear_damping = np.array([b.linear_damping for b in bodies], dtype=f64)
        self.angular_damping = np.array([b.angular_damping for b in bodies], dtype=f64)
        self.gravity_scale = np.array([b.gravity_scale for b in bodies], dtype=f64)
        self.layer = np.array([b.layer for b in bodies], dtype=np.uint32)
        self.mask = np.array([b.mask & 0xFFFFFFFF for b in bodies], dtype=np.uint32)
        self.flags = np.array([b.flags for b in bodies], dtype=np.uint32)
        no, nc, nl = [], [], []
        for b in bodies:
            no.append(len(nl))
            nc.append(len(b.nocollide))
            nl.extend(b.nocollide)
        self.nocollide_offset = np.array(no, dtype=np.uint32)
        self.nocollide_count = np.array(nc, dtype=np.uint32)
        self.nocollide = np.array(nl if nl else [0], dtype=np.uint32)
        self.n_nocollide = len(nl)
        self._c = None

    def copy(self) -> "BodyArrays":
        other = BodyArrays.__new__(BodyArrays)
        for k, v in self.__dict__.items():
            other.__dict__[k] = v.copy() if isinstance(v, np.ndarray) else v
        other._c = None
        return other

    def state(self):
        return {k: getattr(self, k).copy() for k in self.STATE}

    @property
    def c(self) -> _ffi.NeBodyArrays:
        """NeBodyArrays view over the numpy buffers (rebuilt on access)."""
        for k in ("x", "q", "v", "w", "force", "torque", "inv_inertia", "half_extents", "verts"):
            a = getattr(self, k)
            if not a.flags["C_CONTIGUOUS"] or a.dtype != np.float64:
                setattr(self, k, np.ascontiguousarray(a, dtype=np.float64))

        def dp(a):
            return a.ctypes.data_as(C.POINTER(C.c_double))

        def up(a):
            return a.ctypes.data_as(C.POINTER(C.c_uint32))

        s = _ffi.NeBodyArrays()
        s.n = self.n
        s.x, s.q, s.v, s.w = dp(self.x), dp(self.q), dp(self.v), dp(self.w)
        s.force, s.torque = dp(self.force), dp(self.torque)
        s.inv_mass, s.inv_inertia = dp(self.inv_mass), dp(self.inv_inertia)
        s.shape = self.shape.ctypes.data_as(C.POINTER(C.c_int32))
        s.radius, s.half_height, s.half_extents = dp(self.radius), dp(self.half_height), dp(self.half_extents)
        s.vert_offset, s.vert_count, s.verts = up(self.vert_offset), up(self.vert_count), dp(self.verts)
        s.n_verts = self.n_verts
        s.friction, s.restitution = dp(self.friction), dp(self.restitution)
        s.linear_damping, s.angular_damping = dp(self.linear_damping), dp(self.angular_damping)
        s.gravity_scale = dp(self.gravity_scale)
        s.layer, s.mask, s.flags = up(self.layer), up(self.mask), up(self.flags)
        s.nocollide_offset, s.nocollide_count, s.nocollide = (
            up(self.nocollide_offset), up(self.nocollide_count), up(self.nocollide))
        s.n_nocollide = self.n_nocollide
        self._c = s
        return s


def default_params(**kw) -> _ffi.NeWorldParams:
    """ne::World defaults (src/world.hpp:75-126), with keyword overrides.

    ``gravity`` takes a 3-sequence; every other key is a NeWorldParams field.
    """
    p = _ffi.NeWorldParams()
    p.half = 12.0
    p.periodic = 0
    p.open_boundary = 0
    p.dt = 1.0 / 120.0
    p.restitution = 1.0
    p.friction = 0.0
    p.contact_beta = 0.2
    p.restitution_combine = _ffi.MAX
    p.friction_combine = _ffi.GEOMETRIC_MEAN
    p.warm_start = 1
    p.force_brute_force = 0
    p.capture_contacts = 0
    p.sleep_enabled = 0
    p.sleep_lin_vel = 0.05
    p.sleep_ang_vel = 0.05
    p.sleep_time = 0.5
    p.wake_vel = 0.5
    for k, v in kw.items():
        if k == "gravity":
            p.gravity[0], p.gravity[1], p.gravity[2] = (float(c) for c in v)
        else:
            setattr(p, k, v)
    return p


def params_dict(p: _ffi.NeWorldParams) -> dict:
    d = {name: getattr(p, name) for name, _ in p._fields_}
    d["gravity"] = tuple(p.gravity)
    return d


def concat(parts):
    """Concatenate BodyArrays into one batch; returns (BodyArrays, world_begin).
    Convex vertex offsets and noCollide indices are rebased onto the batch."""
    out = BodyArrays.__new__(BodyArrays)
    begin = [0]
    for b in parts:
        begin.append(begin[-1] + b.n)
    out.n = begin[-1]
    per_body = ("x", "q", "v", "w", "force", "torque", "inv_mass", "inv_inertia", "shape", "radius",
                "half_height", "half_extents", "friction", "restitution", "linear_damping", "angular_damping",
                "gravity_scale", "layer", "mask", "flags", "vert_count", "nocollide_count")
    for k in per_body:
        setattr(out, k, np.ascontiguousarray(np.concatenate([getattr(b, k) for b in parts])))
    vo, nco, verts, ncl = [], [], [], []
    vbase = nbase = 0
    for b, b0 in zip(parts, begin):
        vo.append(b.vert_offset.astype(np.int64) + vbase)
        verts.append(b.verts[: b.n_verts])
        vbase += b.n_verts
        nco.append(b.nocollide_offset.astype(np.int64) + nbase)
        ncl.append(b.nocollide[: b.n_nocollide].astype(np.int64) + b0)
        nbase += b.n_nocollide
    out.vert_offset = np.concatenate(vo).astype(np.uint32)
    out.n_verts = vbase
    v = np.concatenate(verts) if vbase else np.zeros((1, 3))
    out.verts = np.ascontiguousarray(v.reshape(-1, 3), dtype=np.float64)
    out.nocollide_offset = np.concatenate(nco).astype(np.uint32)
    out.n_nocollide = nbase
    nc = np.concatenate(ncl) if nbase else np.zeros(1)
    out.nocollide = np.ascontiguousarray(nc, dtype=np.uint32)
    out._c = None
    return out, np.array(begin, dtype=np.uint32)


def take_range(bodies: BodyArrays, b0: int, b1: int) -> BodyArrays:
    """Bodies [b0, b1) as a BodyArrays of their own.  Convex vertex offsets are
    rebased onto the copied vertices and noCollide partners onto b0 (partners
    must lie inside the range, as they do for whole worlds of a batch)."""
    out = BodyArrays.__new__(BodyArrays)
    out.n = b1 - b0
    per_body = ("x", "q", "v", "w", "force", "torque", "inv_mass", "inv_inertia", "shape", "radius",
                "half_height", "half_extents", "friction", "restitution", "linear_damping", "angular_damping",
                "gravity_scale", "layer", "mask", "flags", "vert_count", "nocollide_count")
    for k in per_body:
        setattr(out, k, np.ascontiguousarray(getattr(bodies, k)[b0:b1]))
    vo, verts, vbase = [], [], 0
    no, ncl, nbase = [], [], 0
    for i in range(b0, b1):
        c = int(bodies.vert_count[i])
        o = int(bodies.vert_offset[i])
        vo.append(vbase if c else 0)
        if c:
            verts.append(bodies.verts[o:o + c])
            vbase += c
        k = int(bodies.nocollide_count[i])
        s = int(bodies.nocollide_offset[i])
        no.append(nbase)
        if k:
            part = bodies.nocollide[s:s + k].astype(np.int64) - b0
            if np.any(part < 0) or np.any(part >= out.n):
                raise ValueError("a noCollide partner lies outside the range")
            ncl.append(part)
            nbase += k
    out.vert_offset = np.array(vo, dtype=np.uint32)
    out.n_verts = vbase
    out.verts = np.ascontiguousarray(np.concatenate(verts) if vbase else np.zeros((1, 3)), dtype=np.float64)
    out.nocollide_offset = np.array(no, dtype=np.uint32)
    out.n_nocollide = nbase
    out.nocollide = np.ascontiguousarray(np.concatenate(ncl) if nbase else np.zeros(1), dtype=np.uint32)
    out._c = None
    return out
