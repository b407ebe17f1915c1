"""Python handle on one device world, over the C-ABI of libne_cuda.so.

This is test and benchmark plumbing around ``include/ne_cuda.h``; the C++17
facade (``host/include/ne/world.hpp``) is the reference-compatible API.  Every
call goes to the CUDA path -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np

from . import _ffi
from .bodies import BodyArrays, default_params


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class DeviceWorld:
    def __init__(self, params: Optional[_ffi.NeWorldParams] = None, bodies: Optional[BodyArrays] = None,
                 record: bool = True, precision: str = "f64"):
        """record=True keeps the reference-rule pair list of every step for
        pairs() (the parity tests need it); benchmarks pass record=False.
        precision: "f64" (bit-exact with the reference) or "f32" (the batched
        FP32 form)."""
        self._lib = _ffi.load()
        self.params = params if params is not None else default_params()
        h = C.c_void_p()
        _ffi.check(self._lib.ne_world_create(C.byref(self.params), C.byref(h)), "ne_world_create")
        self._h = h
        self.n = 0
        if record:
            _ffi.check(self._lib.ne_world_set_record(self._h, _ffi.RECORD_PAIRS), "ne_world_set_record")
        self.set_precision(precision)
        if bodies is not None:
            self.upload(bodies)

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.ne_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_params(self, params: _ffi.NeWorldParams):
        self.params = params
        _ffi.check(self._lib.ne_world_set_params(self._h, C.byref(params)), "ne_world_set_params")

    def upload(self, bodies: BodyArrays):
        self._bodies = bodies
        self.n = bodies.n
        self._wb = None
        _ffi.check(self._lib.ne_world_upload(self._h, C.byref(bodies.c)), "ne_world_upload")

    def upload_batch(self, params_list, bodies: BodyArrays, world_begin):
        """Upload a batch: world k owns bodies [world_begin[k], world_begin[k+1])."""
        self._bodies = bodies
        self.n = bodies.n
        nw = len(params_list)
        arr = (_ffi.NeWorldParams * nw)(*params_list)
        self._batch_params = arr
        wb = np.ascontiguousarray(world_begin, dtype=np.uint32)
        assert wb.shape == (nw + 1,)
        self._wb = wb
        _ffi.check(self._lib.ne_world_upload_batch(self._h, arr, nw, _ptr(wb), C.byref(bodies.c)),
                   "ne_world_upload_batch")

    def upload_state(self, x=None, q=None, v=None, w=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (x, q, v, w)]
        _ffi.check(self._lib.ne_world_upload_state(self._h, *[_ptr(a) for a in arrs]), "ne_world_upload_state")

    # -- stepping ------------------------------------------------------------
    def step(self, nsteps: int = 1) -> int:
        rc = self._lib.ne_world_step(self._h, int(nsteps))
        if rc not in (_ffi.NE_OK, _ffi.NE_ERR_NUMERIC):
            _ffi.check(rc, "ne_world_step")
        return rc

    def reset_warm_cache(self):
        _ffi.check(self._lib.ne_world_reset_warm_cache(self._h), "ne_world_reset_warm_cache")

    # -- readback ------------------------------------------------------------
    def state(self, with_forces: bool = False, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        """Download x, q, v, w (and force, torque).  `out` reuses caller-owned
        C-contiguous float64 arrays of the right shapes (no allocation)."""
        n = self.n
        if out is None:
            out = {"x": np.empty((n, 3)), "q": np.empty((n, 4)), "v": np.empty((n, 3)), "w": np.empty((n, 3))}
            if with_forces:
                out["force"] = np.empty((n, 3))
                out["torque"] = np.empty((n, 3))
        for k, a in out.items():
            if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"] or a.shape[0] != n:
                raise ValueError(f"out[{k!r}] must be a C-contiguous float64 array with {n} rows")
        s = _ffi.NeBodyArrays()
        s.n = n
        for k, a in out.items():
            setattr(s, k, a.ctypes.data_as(C.POINTER(C.c_double)))
        _ffi.check(self._lib.ne_world_download(self._h, C.byref(s)), "ne_world_download")
        return out

    def stats(self) -> Dict[str, int]:
        st = _ffi.NeStepStats()
        _ffi.check(self._lib.ne_world_stats(self._h, C.byref(st)), "ne_world_stats")
        return {name: int(getattr(st, name)) for name, _ in st._fields_}

    def pairs(self) -> np.ndarray:
        cnt = C.c_uint64()
        _ffi.check(self._lib.ne_world_pairs(self._h, None, None, 0, C.byref(cnt)), "ne_world_pairs")
        P = cnt.value
        pi = np.empty(P, dtype=np.uint32)
        pj = np.empty(P, dtype=np.uint32)
        _ffi.check(self._lib.ne_world_pairs(self._h, _ptr(pi), _ptr(pj), P, C.byref(cnt)), "ne_world_pairs")
        return np.stack([pi, pj], axis=1)

    def contacts(self) -> Dict[str, np.ndarray]:
        cnt = C.c_uint64()
        empty = _ffi.NeContactArrays()
        _ffi.check(self._lib.ne_world_contacts(self._h, C.byref(empty), 0, C.byref(cnt)), "ne_world_contacts")
        m = cnt.value
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
        _ffi.check(self._lib.ne_world_contacts(self._h, C.byref(s), m, C.byref(cnt)), "ne_world_contacts")
        return out

    def islands(self) -> np.ndarray:
        lab = np.empty(self.n, dtype=np.uint32)
        _ffi.check(self._lib.ne_world_islands(self._h, _ptr(lab), self.n), "ne_world_islands")
        return lab

    def set_precision(self, precision: str):
        code = {"f64": _ffi.PRECISION_F64, "f32": _ffi.PRECISION_F32}[precision]
        _ffi.check(self._lib.ne_world_set_precision(self._h, code), "ne_world_set_precision")
        self.precision = precision

    def solver_shape(self):
        s = _ffi.NeSolverShape()
        _ffi.check(self._lib.ne_world_get_solver_shape(self._h, C.byref(s)), "ne_world_get_solver_shape")
        return int(s.threads), int(s.ctas_per_sm), int(s.team_max)

    def set_solver_shape(self, threads: int, ctas_per_sm: int = 1, team_max: int = 1):
        s = _ffi.NeSolverShape(threads, ctas_per_sm, team_max)
        _ffi.check(self._lib.ne_world_set_solver_shape(self._h, C.byref(s)), "ne_world_set_solver_shape")

    def autotune(self, steps: int = 5):
        """Time the big-island solver's launch shapes from the current state,
        keep the fastest; the state is left as it was."""
        s = _ffi.NeSolverShape()
        _ffi.check(self._lib.ne_world_autotune(self._h, steps, C.byref(s)), "ne_world_autotune")
        return int(s.threads), int(s.ctas_per_sm), int(s.team_max)

    def step_backward(self, nsteps: int, checkpoint_every: int = 0, xbar=None, vbar=None) -> Dict[str, np.ndarray]:
        """Gradients through the next `nsteps` steps from the current state
        (the state is not changed), given dL/dx and dL/dv after them ([n, 3]
        each, None = 0).  Returns x, q, v, w (initial state), mass, inv_mass,
        inv_inertia (per body) and friction, restitution (per world)."""
        n = self.n
        nw = len(self._wb) - 1 if getattr(self, "_wb", None) is not None else 1
        out = {"x": np.zeros((n, 3)), "q": np.zeros((n, 4)), "v": np.zeros((n, 3)), "w": np.zeros((n, 3)),
               "mass": np.zeros(n), "inv_mass": np.zeros(n), "inv_inertia": np.zeros((n, 3)),
               "friction": np.zeros(nw), "restitution": np.zeros(nw)}
        keep = []

        def dp(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))
        fin = _ffi.NeStateGrad(dp(xbar), dp(vbar))
        pg = _ffi.NeParamGrad(*[out[k].ctypes.data_as(C.POINTER(C.c_double)) for k in
                                ("x", "q", "v", "w", "mass", "inv_mass", "inv_inertia", "friction", "restitution")])
        _ffi.check(self._lib.ne_world_step_backward(self._h, int(nsteps), int(checkpoint_every), C.byref(fin),
                                                    C.byref(pg)), "ne_world_step_backward")
        return out

    def checkpoint(self) -> "Checkpoint":
        """Device copy of the state and the warm cache (see restore())."""
        h = C.c_void_p()
        _ffi.check(self._lib.ne_world_checkpoint(self._h, C.byref(h)), "ne_world_checkpoint")
        return Checkpoint(self._lib, h)

    def restore(self, ck: "Checkpoint"):
        _ffi.check(self._lib.ne_world_restore(self._h, ck._h), "ne_world_restore")

    def profile(self, enable: bool = True):
        _ffi.check(self._lib.ne_world_profile(self._h, 1 if enable else 0), "ne_world_profile")

    def stage_times(self) -> Dict[str, float]:
        ms = (C.c_double * _ffi.NUM_STAGES)()
        steps = C.c_uint64()
        _ffi.check(self._lib.ne_world_stage_times(self._h, ms, C.byref(steps)), "ne_world_stage_times")
        out = {self._lib.ne_stage_name(k).decode(): ms[k] for k in range(_ffi.NUM_STAGES)}
        out["steps"] = int(steps.value)
        return out

    def stream_handle(self) -> int:
        s = C.c_void_p()
        _ffi.check(self._lib.ne_world_stream(self._h, C.byref(s)), "ne_world_stream")
        return s.value or 0

    def set_graph(self, enable: bool) -> None:
        """Steps by replaying a captured CUDA graph of one step (default on)."""
        _ffi.check(self._lib.ne_world_set_graph(self._h, 1 if enable else 0), "ne_world_set_graph")

    def launch_count(self) -> int:
        v = C.c_uint64()
        _ffi.check(self._lib.ne_world_launch_count(self._h, C.byref(v)), "ne_world_launch_count")
        return int(v.value)


class Checkpoint:
    """Owned handle of an NeCheckpoint; destroy it before its world."""

    def __init__(self, lib, h):
        self._lib = lib
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ne_checkpoint_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
