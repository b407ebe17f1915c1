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
