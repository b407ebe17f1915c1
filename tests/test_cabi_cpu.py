"""The C-ABI library without a GPU: it loads, exports every function the
header declares, and its ctypes mirror has the C struct layouts."""
import os
import re
import subprocess
import tempfile

import pytest

from nativeengine_b200 import _ffi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ne_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ne_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    assert os.path.exists(_ffi.LIB_PATH), "libne_cuda.so not built"
    lib = _ffi.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ne_cuda.h but not exported"
        assert n in _ffi.EXPORTS, f"{n} missing from the ctypes mirror"


def test_status_strings():
    lib = _ffi.load()
    for code in range(8):
        assert lib.ne_status_string(code)
    assert lib.ne_stage_name(6) == b"solve"


def test_struct_layouts_match_c():
    src = r'''
#include <stddef.h>
#include <stdio.h>
#include "ne_cuda.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m))
int main(void) {
  printf("NeWorldParams %zu\nNeBodyArrays %zu\nNeContactArrays %zu\nNeStepStats %zu\nNeMeshData %zu\n",
         sizeof(NeWorldParams), sizeof(NeBodyArrays), sizeof(NeContactArrays), sizeof(NeStepStats),
         sizeof(NeMeshData));
  F(NeWorldParams, dt); F(NeWorldParams, gravity); F(NeWorldParams, sleep_lin_vel); F(NeWorldParams, n_joints);
  F(NeBodyArrays, x); F(NeBodyArrays, verts); F(NeBodyArrays, n_verts); F(NeBodyArrays, friction);
  F(NeBodyArrays, n_nocollide); F(NeBodyArrays, child_offset); F(NeBodyArrays, n_children);
  F(NeBodyArrays, child_half_extents); F(NeBodyArrays, mesh_index); F(NeBodyArrays, n_meshes);
  F(NeBodyArrays, meshes); F(NeMeshData, verts); F(NeMeshData, order); F(NeMeshData, n_nodes);
  F(NeMeshData, node_count);
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line.strip())
    import ctypes as C
    assert int(got["NeWorldParams"]) == C.sizeof(_ffi.NeWorldParams)
    assert int(got["NeBodyArrays"]) == C.sizeof(_ffi.NeBodyArrays)
    assert int(got["NeContactArrays"]) == C.sizeof(_ffi.NeContactArrays)
    assert int(got["NeStepStats"]) == C.sizeof(_ffi.NeStepStats)
    assert int(got["NeMeshData"]) == C.sizeof(_ffi.NeMeshData)
    for key, val in got.items():
        if "." in key:
            t, m = key.split(".")
            assert getattr(getattr(_ffi, t), m).offset == int(val), key
