"""Build the CUDA library in-tree: nativeengine_b200/_lib/libne_cuda.so.

FP64 parity with the x86-64 reference needs ``--fmad=false`` (no fused
multiply-add contraction); division and square root stay IEEE-rounded
(nvcc's defaults -prec-div=true -prec-sqrt=true).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libne_cuda.so")
SOURCES = ["ne_prims.cu", "ne_step.cu", "ne_capi.cu", "ne_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "--fmad=false", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


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


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "ne_cuda.h")]
    if force or _stale(OUT, deps):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        cmd = [nvcc()] + ARCH + FLAGS + ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-o", OUT]
        cmd += [os.path.join(CSRC, s) for s in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_host(force=force, verbose=verbose)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
