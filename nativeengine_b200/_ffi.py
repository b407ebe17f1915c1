"""ctypes mirror of include/ne_cuda.h and the loader for libne_cuda.so.

The library is built in-tree (``nativeengine_b200/_lib/libne_cuda.so``) by
``nativeengine_b200.build``.  There is no fallback: if the shared object is
missing, importing a device entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libne_cuda.so")

# status codes
NE_OK = 0
NE_ERR_ARG = 1
NE_ERR_CUDA = 2
NE_ERR_CAPACITY = 3
NE_ERR_UNSUPPORTED = 4
NE_ERR_TIMEOUT = 5
NE_ERR_NUMERIC = 6
NE_ERR_NO_DEVICE = 7
NUM_STAGES = 8
RECORD_PAIRS = 1
PRECISION_F64 = 0
PRECISION_F32 = 1
NOALLOC_MAX_BODIES = 2048
NOALLOC_MAX_PAIRS = 262144

# shapes (ne::Shape order)
SPHERE, CYLINDER, BOX, CAPSULE, CONVEX, PLANE, MESH, COMPOUND = range(8)
# combine modes (ne::World::Combine order)
AVERAGE, MIN, MAX, MULTIPLY, GEOMETRIC_MEAN = range(5)
# body flags
DYNAMIC, SLEEPING, KINEMATIC, SENSOR, CCD = 1, 2, 4, 8, 16

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)


class NeWorldParams(C.Structure):
    _fields_ = [
        ("half", C.c_double),
        ("periodic", C.c_int32),
        ("open_boundary", C.c_int32),
        ("dt", C.c_double),
        ("restitution", C.c_double),
        ("friction", C.c_double),
        ("contact_beta", C.c_double),
        ("gravity", C.c_double * 3),
        ("restitution_combine", C.c_int32),
        ("friction_combine", C.c_int32),
        ("warm_start", C.c_int32),
        ("force_brute_force", C.c_int32),
        ("capture_contacts", C.c_int32),
        ("sleep_enabled", C.c_int32),
        ("sleep_lin_vel", C.c_double),
        ("sleep_ang_vel", C.c_double),
        ("sleep_time", C.c_double),
        ("wake_vel", C.c_double),
        ("n_distance_joints", C.c_uint32),
        ("n_joints", C.c_uint32),
    ]


_i32cp = C.POINTER(C.c_int32)


class NeMeshData(C.Structure):
    _fields_ = [
        ("n_verts", C.c_uint32), ("verts", C.POINTER(C.c_double)),
        ("n_tris", C.c_uint32), ("tris", _i32cp), ("order", _i32cp),
        ("n_nodes", C.c_uint32), ("node_lo", C.POINTER(C.c_double)), ("node_hi", C.POINTER(C.c_double)),
        ("node_left", _i32cp), ("node_right", _i32cp), ("node_start", _i32cp), ("node_count", _i32cp),
    ]


class NeBodyArrays(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("x", _dp), ("q", _dp), ("v", _dp), ("w", _dp), ("force", _dp), ("torque", _dp),
        ("inv_mass", _dp), ("inv_inertia", _dp),
        ("shape", _i32p), ("radius", _dp), ("half_height", _dp), ("half_extents", _dp),
        ("vert_offset", _u32p), ("vert_count", _u32p), ("verts", _dp), ("n_verts", C.c_uint32),
        ("friction", _dp), ("restitution", _dp), ("linear_damping", _dp), ("angular_damping", _dp),
        ("gravity_scale", _dp),
        ("layer", _u32p), ("mask", _u32p), ("flags", _u32p),
        ("nocollide_offset", _u32p), ("nocollide_count", _u32p), ("nocollide", _u32p),
        ("n_nocollide", C.c_uint32),
        ("child_offset", _u32p), ("child_count", _u32p), ("n_children", C.c_uint32),
        ("child_shape", _i32p), ("child_pos", _dp), ("child_rot", _dp), ("child_radius", _dp),
        ("child_half_height", _dp), ("child_half_extents", _dp),
        ("mesh_index", _u32p), ("n_meshes", C.c_uint32), ("meshes", C.POINTER(NeMeshData)),
    ]


class NeContactArrays(C.Structure):
    _fields_ = [
        ("i", _u32p), ("j", _u32p), ("slot", _u32p),
        ("point", _dp), ("normal", _dp), ("depth", _dp), ("n_imp", _dp), ("t_imp", _dp),
    ]


class NeSolverShape(C.Structure):
    _fields_ = [("threads", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("team_max", C.c_uint32)]


_cdp = C.POINTER(C.c_double)


class NeStateGrad(C.Structure):
    _fields_ = [("x", _cdp), ("v", _cdp)]


class NeParamGrad(C.Structure):
    _fields_ = [("x", _cdp), ("q", _cdp), ("v", _cdp), ("w", _cdp), ("mass", _cdp), ("inv_mass", _cdp),
                ("inv_inertia", _cdp), ("friction", _cdp), ("restitution", _cdp)]


class NeStepStats(C.Structure):
    _fields_ = [
        ("pairs", C.c_uint64), ("survivors", C.c_uint64), ("contacts", C.c_uint64),
        ("islands", C.c_uint64), ("max_island", C.c_uint64), ("epa_cap_hits", C.c_uint64),
        ("steps", C.c_uint64), ("retries", C.c_uint64), ("candidates", C.c_uint64),
        ("graph_steps", C.c_uint64), ("graph_captures", C.c_uint64),
    ]


# Every extern "C" symbol the header declares (checked by the CPU test suite).
EXPORTS = {
    "ne_world_params_default": (None, [C.POINTER(NeWorldParams)]),
    "ne_world_create": (C.c_int, [C.POINTER(NeWorldParams), C.POINTER(C.c_void_p)]),
    "ne_world_destroy": (C.c_int, [C.c_void_p]),
    "ne_world_set_params": (C.c_int, [C.c_void_p, C.POINTER(NeWorldParams)]),
    "ne_world_upload": (C.c_int, [C.c_void_p, C.POINTER(NeBodyArrays)]),
    "ne_world_upload_batch": (C.c_int, [C.c_void_p, C.POINTER(NeWorldParams), C.c_uint32, C.c_void_p,
                                        C.POINTER(NeBodyArrays)]),
    "ne_world_upload_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ne_world_download": (C.c_int, [C.c_void_p, C.POINTER(NeBodyArrays)]),
    "ne_world_step": (C.c_int, [C.c_void_p, C.c_uint32]),
    "ne_world_reset_warm_cache": (C.c_int, [C.c_void_p]),
    "ne_world_stats": (C.c_int, [C.c_void_p, C.POINTER(NeStepStats)]),
    "ne_world_pairs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "ne_world_contacts": (C.c_int, [C.c_void_p, C.POINTER(NeContactArrays), C.c_uint64, C.POINTER(C.c_uint64)]),
    "ne_world_islands": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "ne_world_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "ne_world_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "ne_world_set_graph": (C.c_int, [C.c_void_p, C.c_int]),
    "ne_world_set_record": (C.c_int, [C.c_void_p, C.c_uint32]),
    "ne_world_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "ne_world_set_solver_shape": (C.c_int, [C.c_void_p, C.POINTER(NeSolverShape)]),
    "ne_world_get_solver_shape": (C.c_int, [C.c_void_p, C.POINTER(NeSolverShape)]),
    "ne_world_autotune": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(NeSolverShape)]),
    "ne_world_step_backward": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(NeStateGrad),
                                         C.POINTER(NeParamGrad)]),
    "ne_world_checkpoint": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "ne_world_restore": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ne_checkpoint_destroy": (C.c_int, [C.c_void_p]),
    "ne_world_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "ne_world_stage_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "ne_stage_name": (C.c_char_p, [C.c_int]),
    "ne_broadphase_pairs_noalloc": (C.c_int, [C.POINTER(NeWorldParams), C.POINTER(NeBodyArrays), C.c_void_p,
                                              C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "ne_status_string": (C.c_char_p, [C.c_int]),
    "ne_last_error": (C.c_char_p, []),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libne_cuda.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build the CUDA extension first "
            "(python -c 'import nativeengine_b200.build as b; b.build()')")
    lib = C.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class NeError(RuntimeError):
    def __init__(self, code: int, where: str):
        lib = load()
        msg = lib.ne_status_string(code).decode()
        detail = lib.ne_last_error().decode()
        super().__init__(f"{where}: {msg} ({code}): {detail}")
        self.code = code


def check(code: int, where: str) -> None:
    if code != NE_OK:
        raise NeError(code, where)
