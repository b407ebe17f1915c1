"""Build the CUDA library in-tree: nativeengine_b200/_lib/libne_cuda.so.

FP64 parity with the x86-64 reference needs ``--fmad=false`` (no fused
multiply-add contraction); division and square root stay IEEE-rounded
(nvcc's defaults -prec-div=true -prec-sqrt=true).  The batched FP32 form's
translation unit (ne_step_f32.cu) has no parity contract and is compiled with
contraction enabled.  Each source compiles to its own object (in parallel),
then nvcc links the shared library.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libne_cuda.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["ne_prims.cu", "ne_step.cu", "ne_step_f32.cu", "ne_adjoint.cu", "ne_capi.cu", "ne_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
# Per-source contraction setting: off everywhere except the FP32 form.
FMAD = {"ne_step_f32.cu": "--fmad=true"}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


HOST_SRC = os.path.join(HERE, "host", "src", "world.cpp")
HOST_SCENES = os.path.join(HERE, "host", "src", "scenes.cpp")
HOST_INC = os.path.join(HERE, "host", "include")
HOST_OUT = os.path.join(HERE, "_lib", "libne_host.so")


def build_host(force: bool = False, verbose: bool = False) -> str:
    """The C++17 facade (ne::World / ne::PhysicsWorld) over libne_cuda.so."""
    deps = [HOST_SRC, HOST_SCENES, OUT, os.path.join(HOST_INC, "ne", "world.hpp"),
            os.path.join(HOST_INC, "ne", "vmath.hpp"), os.path.join(CSRC, "ne_geom.cuh")]
    if force or _stale(HOST_OUT, deps):
        cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + HOST_INC,
               "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, HOST_SRC, HOST_SCENES,
               "-L" + os.path.dirname(OUT), "-lne_cuda",
               "-Wl,-rpath,$ORIGIN", "-o", HOST_OUT]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return HOST_OUT


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc()] + ARCH + FLAGS + [FMAD.get(src, "--fmad=false"), "-I" + os.path.join(ROOT, "include"),
                                     "-I" + CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "ne_cuda.h")]
    if force or _stale(OUT, deps):
        from concurrent.futures import ThreadPoolExecutor
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        os.makedirs(OBJDIR, exist_ok=True)
        with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
            objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
        cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_host(force=force, verbose=verbose)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
