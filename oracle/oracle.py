"""Oracle loaders -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker or the timed CPU baseline.  The
product path (nativeengine_b200) never imports it.

Two oracles share one interface:
  * ``RefOracle``  -- the reference NativeEngine compiled unmodified from its
    own sources (oracle/_ref/libneref.so, built by oracle/Makefile);
  * ``PortOracle`` -- the C restatement in oracle/ne_oracle.c
    (oracle/_build/libne_oracle.so), pinned bit-for-bit to RefOracle by the
    CPU test suite.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libneref.so")
PORT_LIB = os.path.join(HERE, "_build", "libne_oracle.so")


def _import_ffi():
    import sys
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    from nativeengine_b200 import _ffi  # struct layouts only (pure ctypes)
    return _ffi


_ffi = _import_ffi()


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def port_available() -> bool:
    return os.path.exists(PORT_LIB)


class _Oracle:
    PREFIX = ""
    PATH = ""
    _lib_cache = {}

    @classmethod
    def lib(cls):
        if cls.PATH not in cls._lib_cache:
            lib = C.CDLL(cls.PATH)
            p = cls.PREFIX
            vp = C.c_void_p
            getattr(lib, p + "create").restype = vp
            getattr(lib, p + "create").argtypes = [C.POINTER(_ffi.NeWorldParams), C.POINTER(_ffi.NeBodyArrays)]
            getattr(lib, p + "destroy").argtypes = [vp]
            getattr(lib, p + "step").argtypes = [vp, C.c_uint32]
            getattr(lib, p + "set_params").argtypes = [vp, C.POINTER(_ffi.NeWorldParams)]
            getattr(lib, p + "reset_warm_cache").argtypes = [vp]
            getattr(lib, p + "get_state").argtypes = [vp, C.POINTER(_ffi.NeBodyArrays)]
            getattr(lib, p + "pairs").restype = C.c_uint64
            getattr(lib, p + "pairs").argtypes = [vp, vp, vp, C.c_uint64]
            getattr(lib, p + "contacts").restype = C.c_uint64
            getattr(lib, p + "contacts").argtypes = [vp, C.POINTER(_ffi.NeContactArrays), C.c_uint64]
            getattr(lib, p + "islands").argtypes = [vp, vp, C.c_uint32]
            if hasattr(lib, p + "step_plain"):
                getattr(lib, p + "step_plain").argtypes = [vp, C.c_uint32]
            cls._lib_cache[cls.PATH] = lib
        return cls._lib_cache[cls.PATH]

    def __init__(self, params, bodies):
        self._l = self.lib()
        self._bodies = bodies
        self.n = bodies.n
        self._h = getattr(self._l, self.PREFIX + "create")(C.byref(params), C.byref(bodies.c))

    def close(self):
        if self._h:
            getattr(self._l, self.PREFIX + "destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, nsteps: int = 1):
        getattr(self._l, self.PREFIX + "step")(self._h, int(nsteps))

    def step_plain(self, nsteps: int = 1):
        fn = getattr(self._l, self.PREFIX + "step_plain", None) or getattr(self._l, self.PREFIX + "step")
        fn(self._h, int(nsteps))

    def set_params(self, params):
        getattr(self._l, self.PREFIX + "set_params")(self._h, C.byref(params))

    def reset_warm_cache(self):
        getattr(self._l, self.PREFIX + "reset_warm_cache")(self._h)

    def state(self) -> Dict[str, np.ndarray]:
        n = self.n
        out = {"x": np.empty((n, 3)), "q": np.empty((n, 4)), "v": np.empty((n, 3)), "w": np.empty((n, 3))}
        s = _ffi.NeBodyArrays()
        s.n = n
        for k, a in out.items():
            setattr(s, k, a.ctypes.data_as(C.POINTER(C.c_double)))
        getattr(self._l, self.PREFIX + "get_state")(self._h, C.byref(s))
        return out

    def pairs(self) -> np.ndarray:
        fn = getattr(self._l, self.PREFIX + "pairs")
        P = fn(self._h, None, None, 0)
        pi = np.empty(P, np.uint32)
        pj = np.empty(P, np.uint32)
        fn(self._h, pi.ctypes.data_as(C.c_void_p), pj.ctypes.data_as(C.c_void_p), P)
        return np.stack([pi, pj], axis=1)

    def contacts(self) -> Dict[str, np.ndarray]:
        fn = getattr(self._l, self.PREFIX + "contacts")
        empty = _ffi.NeContactArrays()
        m = fn(self._h, C.byref(empty), 0)
        out = {
            "i": np.empty(m, np.uint32), "j": np.empty(m, np.uint32), "slot": np.empty(m, np.uint32),
            "point": np.empty((m, 3)), "normal": np.empty((m, 3)), "depth": np.empty(m),
            "n_imp": np.empty(m), "t_imp": np.empty(m),
        }
        s = _ffi.NeContactArrays()
        for k in ("i", "j", "slot"):
            setattr(s, k, out[k].ctypes.data_as(C.POINTER(C.c_uint32)))
        for k in ("point", "normal", "depth", "n_imp", "t_imp"):
            setattr(s, k, out[k].ctypes.data_as(C.POINTER(C.c_double)))
        fn(self._h, C.byref(s), m)
        return out

    def islands(self) -> np.ndarray:
        lab = np.empty(self.n, np.uint32)
        getattr(self._l, self.PREFIX + "islands")(self._h, lab.ctypes.data_as(C.c_void_p), self.n)
        return lab


class RefOracle(_Oracle):
    PREFIX = "neref_"
    PATH = REF_LIB

    def pair_contacts(self, ia: int, ib: int):
        lib = self._l
        fn = lib.neref_pair_contacts
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        pt = np.zeros((4, 3))
        nr = np.zeros((4, 3))
        dp = np.zeros(4)
        k = fn(self._h, ia, ib, pt.ctypes.data_as(C.c_void_p), nr.ctypes.data_as(C.c_void_p),
               dp.ctypes.data_as(C.c_void_p))
        return pt[:k], nr[:k], dp[:k]


class PortOracle(_Oracle):
    PREFIX = "neport_"
    PATH = PORT_LIB

    def __init__(self, params, bodies):
        if np.any((bodies.shape == _ffi.MESH) | (bodies.shape == _ffi.COMPOUND)):
            raise NotImplementedError("the C restatement has no triangle meshes or compounds; use RefOracle")
        super().__init__(params, bodies)


def ref_mesh(verts, tris):
    """A triangle mesh with the reference's own BVH (MeshData::build()), as a
    nativeengine_b200.bodies.MeshData."""
    from nativeengine_b200.bodies import MeshData
    lib = RefOracle.lib()
    fn = lib.neref_mesh_build
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32] + [C.c_void_p] * 6
    v = np.ascontiguousarray(np.asarray(verts, np.float64).reshape(-1, 3))
    t = np.ascontiguousarray(np.asarray(tris, np.int32).reshape(-1, 3))
    cap = 2 * len(t) + 1
    order = np.zeros(len(t), np.int32)
    lo, hi = np.zeros((cap, 3)), np.zeros((cap, 3))
    ints = [np.zeros(cap, np.int32) for _ in range(4)]
    k = fn(v.ctypes.data_as(C.c_void_p), len(v), t.ctypes.data_as(C.c_void_p), len(t),
           order.ctypes.data_as(C.c_void_p), cap, lo.ctypes.data_as(C.c_void_p), hi.ctypes.data_as(C.c_void_p),
           *[a.ctypes.data_as(C.c_void_p) for a in ints])
    assert k >= 0
    return MeshData.from_arrays(v, t, order, lo[:k], hi[:k], *[a[:k] for a in ints])


def ref_readme_example() -> float:
    lib = RefOracle.lib()
    lib.neref_readme_example.restype = C.c_double
    return lib.neref_readme_example()


def ref_mass_props(kind: int, params, verts=None, density=1.0):
    lib = RefOracle.lib()
    fn = lib.neref_mass_props
    fn.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_void_p, C.c_void_p]
    p = np.asarray(params, dtype=np.float64).ravel()
    if p.size == 0:
        p = np.zeros(1)
    v = np.asarray(verts if verts is not None else [[0.0, 0.0, 0.0]], dtype=np.float64).reshape(-1, 3)
    nv = 0 if verts is None else v.shape[0]
    im = np.zeros(1)
    ii = np.zeros(3)
    fn(kind, p.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p), nv, density,
       im.ctypes.data_as(C.c_void_p), ii.ctypes.data_as(C.c_void_p))
    return float(im[0]), tuple(ii)
