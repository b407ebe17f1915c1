"""The C++17 facade (ne::World / ne::PhysicsWorld) as reference client code
sees it: tests/cpp/facade_demo.cpp compiles against the facade headers and
links libne_host.so (CPU); on a GPU it runs and must reproduce the README
example's exact y and the stacking behaviour."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "nativeengine_b200", "_lib")


def build_demo(out_dir):
    exe = os.path.join(out_dir, "facade_demo")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "nativeengine_b200", "host", "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_demo.cpp"), "-L", LIB, "-lne_host", "-lne_cuda",
                    "-Wl,-rpath," + LIB, "-o", exe], check=True)
    return exe


def test_facade_compiles_and_links(tmp_path):
    assert os.path.exists(os.path.join(LIB, "libne_host.so")), "libne_host.so not built"
    assert os.path.exists(build_demo(str(tmp_path)))


@pytest.mark.gpu
def test_facade_demo_runs_on_device(tmp_path):
    exe = build_demo(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "readme y = 0.4890999999999725" in r.stdout


@pytest.mark.parametrize("rows,cols", [(3, 4), (8, 8), (13, 9)])
def test_facade_mesh_bvh_equals_the_reference_build(tmp_path, rows, cols):
    """ne::MeshData::build() of the facade makes the reference's BVH, node for
    node, so a mesh pair's contacts come in the reference's order."""
    import math
    import numpy as np
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference not built")
    exe = os.path.join(str(tmp_path), "mesh_bvh")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "nativeengine_b200", "host", "include"),
                    os.path.join(ROOT, "tests", "cpp", "mesh_bvh.cpp"), "-L", LIB, "-lne_host", "-lne_cuda",
                    "-Wl,-rpath," + LIB, "-o", exe], check=True)
    out = subprocess.run([exe, str(rows), str(cols)], capture_output=True, text=True, check=True).stdout.split("\n")
    order = [int(t) for t in out[0].split()[1:]]
    nodes = [line.split()[1:] for line in out[1:] if line.startswith("node")]
    verts = [(1.5 * c, 0.4 * math.sin(0.8 * c) * math.cos(0.6 * r), 1.5 * r) for r in range(rows) for c in range(cols)]
    tris = []
    for r in range(rows - 1):
        for c in range(cols - 1):
            a, b, d, e = r * cols + c, r * cols + c + 1, (r + 1) * cols + c, (r + 1) * cols + c + 1
            tris += [(a, d, b), (b, d, e)]
    ref = O.ref_mesh(verts, tris)
    assert order == ref.order.tolist()
    assert len(nodes) == len(ref.node_left)
    for k, nd in enumerate(nodes):
        assert [float(x) for x in nd[:3]] == ref.node_lo[k].tolist()
        assert [float(x) for x in nd[3:6]] == ref.node_hi[k].tolist()
        assert [int(x) for x in nd[6:]] == [ref.node_left[k], ref.node_right[k], ref.node_start[k], ref.node_count[k]]
