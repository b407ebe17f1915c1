"""The allocation-free broadphase entry point against the world step's own.

ne_broadphase_pairs_noalloc serves callers that may not allocate GPU memory
where they call it (an engine that hands out device memory only from its own
pool, a frame loop that forbids cudaMalloc/cudaFree).  It keeps all of its
device working memory in one array the library reserves at load time, so this
test checks that it returns exactly the pair list ne_world_pairs reports for a
step over the same positions -- twice in a row with different scenes, so that
contents left in the shared array by the first call cannot leak into the
second.  Collected last on purpose: it runs after every other test, and also
passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from nativeengine_b200 import DeviceWorld, _ffi, scenes


def _still(params, bodies):
    """The scene at rest with gravity off, so one step's broadphase sees the
    bodies exactly where they were uploaded (x + 0*dt == x)."""
    b = bodies.copy()
    b.v[:] = 0.0
    b.w[:] = 0.0
    params.gravity[0] = params.gravity[1] = params.gravity[2] = 0.0
    return params, b


def _world_pairs(params, bodies):
    dev = DeviceWorld(params, bodies.copy())
    dev.step(1)
    p = dev.pairs()
    dev.close()
    return p


def _noalloc_pairs(params, bodies):
    lib = _ffi.load()
    cnt = C.c_uint64()
    cap = _ffi.NOALLOC_MAX_PAIRS
    pi = np.zeros(cap, np.uint32)
    pj = np.zeros(cap, np.uint32)
    rc = lib.ne_broadphase_pairs_noalloc(C.byref(params), C.byref(bodies.c), pi.ctypes.data_as(C.c_void_p),
                                         pj.ctypes.data_as(C.c_void_p), cap, C.byref(cnt))
    _ffi.check(rc, "ne_broadphase_pairs_noalloc")
    m = cnt.value
    return np.stack([pi[:m], pj[:m]], axis=1)


@pytest.mark.gpu
def test_noalloc_pairs_match_world_pairs_twice():
    # First call: a periodic sphere gas on the grid path (1,000 bodies).
    pa, ba = _still(*scenes.gas())
    # Second call: a reflective mixed-shape scene with a plane (grid + plane
    # pairs), smaller than the first, so stale pairs would show up as extras.
    pb, bb = _still(*scenes.mixed_shapes(n=300, half=9.0, periodic=False, with_plane=True, seed=21))
    for params, bodies in ((pa, ba), (pb, bb)):
        want = _world_pairs(params, bodies)
        got = _noalloc_pairs(params, bodies)
        assert got.shape == want.shape, f"{got.shape[0]} pairs, world step reports {want.shape[0]}"
        assert np.array_equal(got, want)


@pytest.mark.gpu
def test_noalloc_rejects_too_many_bodies():
    params, bodies = scenes.small_gas(n=_ffi.NOALLOC_MAX_BODIES + 1, half=60.0)
    lib = _ffi.load()
    cnt = C.c_uint64()
    rc = lib.ne_broadphase_pairs_noalloc(C.byref(params), C.byref(bodies.c), None, None, 0, C.byref(cnt))
    assert rc == _ffi.NE_ERR_CAPACITY
    assert b"NE_NOALLOC_MAX_BODIES" in lib.ne_last_error()
