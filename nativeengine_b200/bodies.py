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


class MeshData:
    """A static triangle mesh and its AABB BVH in the layout of ne::MeshData
    (src/mesh.hpp:14-26): vertices, triangles, BVH-sorted triangle order and
    nodes (lo, hi, left, right, start, count; leaves of at most 4 triangles).

    ``build()`` makes a BVH of its own (median split of the centroids along the
    longest axis, stable order); any valid BVH gives the same set of contacts,
    and the order of a mesh pair's contacts follows the BVH walk.  For contacts
    in the reference's order, pass the arrays of the reference's own
    MeshData::build() via ``from_arrays``."""

    def __init__(self, verts, tris):
        self.verts = np.ascontiguousarray(np.asarray(verts, dtype=np.float64).reshape(-1, 3))
        self.tris = np.ascontiguousarray(np.asarray(tris, dtype=np.int32).reshape(-1, 3))
        self.order = np.zeros(0, np.int32)
        self.node_lo = self.node_hi = np.zeros((0, 3))
        self.node_left = self.node_right = self.node_start = self.node_count = np.zeros(0, np.int32)

    @classmethod
    def from_arrays(cls, verts, tris, order, node_lo, node_hi, node_left, node_right, node_start, node_count):
        m = cls(verts, tris)
        m.order = np.ascontiguousarray(order, dtype=np.int32)
        m.node_lo = np.ascontiguousarray(np.asarray(node_lo, np.float64).reshape(-1, 3))
        m.node_hi = np.ascontiguousarray(np.asarray(node_hi, np.float64).reshape(-1, 3))
        m.node_left, m.node_right, m.node_start, m.node_count = (
            np.ascontiguousarray(a, dtype=np.int32) for a in (node_left, node_right, node_start, node_count))
        return m

    def build(self) -> "MeshData":
        tv = self.verts[self.tris]                       # [m, 3, 3]
        lo_t, hi_t = tv.min(axis=1), tv.max(axis=1)
        cen = lo_t + hi_t
        order = list(range(len(self.tris)))
        lo_l, hi_l, left, right, start, count = [], [], [], [], [], []

        def node(s, c):
            idx = len(lo_l)
            ids = order[s:s + c]
            lo, hi = lo_t[ids].min(axis=0), hi_t[ids].max(axis=0)
            lo_l.append(lo); hi_l.append(hi)
            left.append(-1); right.append(-1); start.append(0); count.append(0)
            if c <= 4:
                start[idx], count[idx] = s, c
                return idx
            ext = hi - lo
            axis = 0 if (ext[0] > ext[1] and ext[0] > ext[2]) else (1 if ext[1] > ext[2] else 2)
            order[s:s + c] = sorted(ids, key=lambda t: cen[t, axis])
            mid = c // 2
            left[idx] = node(s, mid)
            right[idx] = node(s + mid, c - mid)
            return idx
        if len(self.tris):
            node(0, len(self.tris))
        self.order = np.array(order, dtype=np.int32)
        self.node_lo = np.array(lo_l, dtype=np.float64).reshape(-1, 3)
        self.node_hi = np.array(hi_l, dtype=np.float64).reshape(-1, 3)
        self.node_left, self.node_right, self.node_start, self.node_count = (
            np.array(a, dtype=np.int32) for a in (left, right, start, count))
        return self

    def c(self) -> _ffi.NeMeshData:
        def dp(a):
            return a.ctypes.data_as(C.POINTER(C.c_double))

        def ip(a):
            return a.ctypes.data_as(C.POINTER(C.c_int32))
        m = _ffi.NeMeshData()
        m.n_verts, m.verts = len(self.verts), dp(self.verts)
        m.n_tris, m.tris, m.order = len(self.tris), ip(self.tris), ip(self.order)
        m.n_nodes = len(self.node_left)
        m.node_lo, m.node_hi = dp(self.node_lo), dp(self.node_hi)
        m.node_left, m.node_right = ip(self.node_left), ip(self.node_right)
        m.node_start, m.node_count = ip(self.node_start), ip(self.node_count)
        return m


@dataclass
class Child:
    """ne::ChildShape (src/body.hpp:28-39): a primitive at a local transform."""
    shape: int
    pos: tuple = (0.0, 0.0, 0.0)
    rot: tuple = (1.0, 0.0, 0.0, 0.0)
    radius: float = 1.0
    half_height: float = 0.0
    half_extents: tuple = (0.0, 0.0, 0.0)


def child_sphere(pos, r) -> Child:
    return Child(_ffi.SPHERE, pos=tuple(map(float, pos)), radius=float(r))


def child_box(pos, q, he) -> Child:
    return Child(_ffi.BOX, pos=tuple(map(float, pos)), rot=tuple(map(float, q)), half_extents=tuple(map(float, he)))


def child_cylinder(pos, q, r, hh) -> Child:
    return Child(_ffi.CYLINDER, pos=tuple(map(float, pos)), rot=tuple(map(float, q)), radius=float(r),
                 half_height=float(hh))


def child_capsule(pos, q, r, hh) -> Child:
    return Child(_ffi.CAPSULE, pos=tuple(map(float, pos)), rot=tuple(map(float, q)), radius=float(r),
                 half_height=float(hh))


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
    children: Optional[List[Child]] = None
    mesh: Optional[MeshData] = None


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


def _child_mass(ch: Child, density):
    if ch.shape == _ffi.BOX:
        return box_mass(ch.half_extents, density)
    if ch.shape == _ffi.CYLINDER:
        return cylinder_mass(ch.radius, 2.0 * ch.half_height, density)
    if ch.shape == _ffi.CAPSULE:
        return capsule_mass(ch.radius, ch.half_height, density)
    return sphere_mass(ch.radius, density)


def make_compound(x, q, children: Sequence[Child], density) -> Body:
    """makeCompound (src/body.hpp:372-400): mass sums the children; the inertia
    is the diagonal of the summed tensor by the parallel-axis theorem."""
    M = 0.0
    Ix = Iy = Iz = 0.0
    for ch in children:
        im, ii = _child_mass(ch, density)
        mc = 1.0 / im if im > 0 else 0.0
        icx = 1.0 / ii[0] if ii[0] > 0 else 0.0
        icy = 1.0 / ii[1] if ii[1] > 0 else 0.0
        icz = 1.0 / ii[2] if ii[2] > 0 else 0.0
        ox, oy, oz = ch.pos
        M += mc
        Ix += icx + mc * (oy * oy + oz * oz)
        Iy += icy + mc * (ox * ox + oz * oz)
        Iz += icz + mc * (ox * ox + oy * oy)
    return Body(_ffi.COMPOUND, x=tuple(map(float, x)), q=tuple(map(float, q)), children=list(children),
                inv_mass=_inv(M), inv_inertia=(_inv(Ix), _inv(Iy), _inv(Iz)))


def make_mesh(x, q, mesh: MeshData) -> Body:
    """makeMesh (src/body.hpp:319-331): static, placed by (x, q)."""
    return Body(_ffi.MESH, x=tuple(map(float, x)), q=tuple(map(float, q)), mesh=mesh, inv_mass=0.0,
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
        co, cc, cl = [], [], []
        for b in bodies:
            co.append(len(cl))
            ch = b.children or []
            cc.append(len(ch))
            cl.extend(ch)
        self.child_offset = np.array(co, dtype=np.uint32)
        self.child_count = np.array(cc, dtype=np.uint32)
        self.n_children = len(cl)
        cl = cl or [Child(_ffi.SPHERE)]
        self.child_shape = np.array([c.shape for c in cl], dtype=np.int32)
        self.child_pos = np.array([c.pos for c in cl], dtype=f64).reshape(-1, 3)
        self.child_rot = np.array([c.rot for c in cl], dtype=f64).reshape(-1, 4)
        self.child_radius = np.array([c.radius for c in cl], dtype=f64)
        self.child_half_height = np.array([c.half_height for c in cl], dtype=f64)
        self.child_half_extents = np.array([c.half_extents for c in cl], dtype=f64).reshape(-1, 3)
        self.meshes = []
        mi = []
        for b in bodies:
            if b.mesh is not None:
                mi.append(len(self.meshes))
                self.meshes.append(b.mesh)
            else:
                mi.append(0)
        self.mesh_index = np.array(mi, dtype=np.uint32)
        self._c = None

    def copy(self) -> "BodyArrays":
        other = BodyArrays.__new__(BodyArrays)
        for k, v in self.__dict__.items():
            other.__dict__[k] = v.copy() if isinstance(v, np.ndarray) else (list(v) if isinstance(v, list) else v)
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
        if getattr(self, "n_children", 0):
            s.child_offset, s.child_count = up(self.child_offset), up(self.child_count)
            s.n_children = self.n_children
            s.child_shape = self.child_shape.ctypes.data_as(C.POINTER(C.c_int32))
            s.child_pos, s.child_rot = dp(self.child_pos), dp(self.child_rot)
            s.child_radius, s.child_half_height = dp(self.child_radius), dp(self.child_half_height)
            s.child_half_extents = dp(self.child_half_extents)
        if getattr(self, "meshes", None):
            self._mesh_c = (_ffi.NeMeshData * len(self.meshes))(*[m.c() for m in self.meshes])
            s.mesh_index = up(self.mesh_index)
            s.n_meshes = len(self.meshes)
            s.meshes = self._mesh_c
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


def _set_child_arrays(out, ranges, total):
    """Child-shape arrays of `out` from child rows [c0, c1) of each source."""
    names = ("child_shape", "child_pos", "child_rot", "child_radius", "child_half_height", "child_half_extents")
    out.n_children = total
    for k in names:
        rows = [getattr(b, k)[c0:c1] for b, c0, c1 in ranges]
        if total:
            setattr(out, k, np.ascontiguousarray(np.concatenate(rows)))
        else:
            setattr(out, k, np.ascontiguousarray(getattr(ranges[0][0], k)[:1]) if ranges else None)


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
    co, cparts, mi, meshes = [], [], [], []
    cbase = 0
    for b in parts:
        co.append(b.child_offset.astype(np.int64) + cbase)
        cparts.append(b)
        cbase += b.n_children
        mi.append(b.mesh_index.astype(np.int64) + len(meshes))
        meshes.extend(b.meshes)
    out.child_offset = np.concatenate(co).astype(np.uint32)
    out.child_count = np.ascontiguousarray(np.concatenate([b.child_count for b in parts]))
    _set_child_arrays(out, [(b, 0, b.n_children) for b in parts], cbase)
    out.mesh_index = np.concatenate(mi).astype(np.uint32)
    out.meshes = meshes
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
    c0 = int(bodies.child_offset[b0]) if b1 > b0 else 0
    c1 = int(bodies.child_offset[b1 - 1] + bodies.child_count[b1 - 1]) if b1 > b0 else 0
    out.child_offset = (bodies.child_offset[b0:b1].astype(np.int64) - c0).astype(np.uint32)
    out.child_count = np.ascontiguousarray(bodies.child_count[b0:b1])
    _set_child_arrays(out, [(bodies, c0, c1)], c1 - c0)
    out.mesh_index = np.ascontiguousarray(bodies.mesh_index[b0:b1])
    out.meshes = list(bodies.meshes)
    out._c = None
    return out
