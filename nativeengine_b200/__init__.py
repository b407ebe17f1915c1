"""nativeengine_b200 -- the B200 step() path of NativeEngine.

The product is ``libne_cuda.so`` (CUDA kernels for sm_100a behind the C-ABI in
include/ne_cuda.h) and the C++17 facade in ``host/``.  This Python package is
the loader and the test/benchmark plumbing: ``DeviceWorld`` drives one device
world through the C-ABI, ``bodies`` builds body arrays with the reference's
factory formulas, ``scenes`` builds the seeded benchmark worlds.
"""
from . import _ffi
from .bodies import (Body, BodyArrays, default_params, make_box, make_capsule, make_convex, make_cylinder,
                     make_kinematic, make_plane, make_sphere, make_static)
from .world import DeviceWorld

__all__ = [
    "_ffi", "Body", "BodyArrays", "DeviceWorld", "default_params", "make_box", "make_capsule", "make_convex",
    "make_cylinder", "make_kinematic", "make_plane", "make_sphere", "make_static",
]
