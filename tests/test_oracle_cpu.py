"""The oracle pinned to the reference's own tests and to the golden fixtures
(CPU only).  The reference is compiled unmodified from its sources by
oracle/Makefile; these tests skip where it has not been built."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_io

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (no reference sources here)")
SELFTEST = os.path.join(O.HERE, "_ref", "ne_selftest")


@needs_ref
@pytest.mark.skipif(not os.path.exists(SELFTEST), reason="reference selftest not built")
def test_reference_selftest_passes():
    r = subprocess.run([SELFTEST, "--selftest"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "Failed: 0" in r.stdout


@needs_ref
def test_readme_example_value():
    # README.md:61-72: a sphere dropped on a static ground box rests at y = 0.489.
    assert O.ref_readme_example() == 0.4890999999999725


@needs_ref
@pytest.mark.parametrize("name", golden_io.names())
def test_reference_reproduces_golden(name):
    params, bodies, expected = golden_io.load(name)
    ora = O.RefOracle(params, bodies)
    for s, e in enumerate(expected):
        ora.step(1)
        assert np.array_equal(ora.pairs(), e["pairs"]), f"{name} step {s}: pairs"
        c = ora.contacts()
        for k in ("i", "j", "point", "normal", "depth", "n_imp"):
            assert np.array_equal(c[k], e["c_" + k]), f"{name} step {s}: contact {k}"
        assert np.array_equal(ora.islands(), e["islands"])
        st = ora.state()
        for k in ("x", "q", "v", "w"):
            assert np.array_equal(st[k], e[k]), f"{name} step {s}: {k}"


@needs_ref
@pytest.mark.parametrize("kind,p,verts", [
    (0, [0.5], None), (0, [0.37], None), (1, [0.3, 0.8], None), (2, [0.25, 0.5, 0.75], None),
    (3, [0.25, 0.45], None), (4, [], [[0.1, 0.2, -0.3], [-0.4, 0.1, 0.2], [0.3, -0.2, 0.1], [0.0, 0.4, 0.05]]),
])
def test_factories_match_reference(kind, p, verts):
    """bodies.py's mass formulas give the reference factories' exact doubles."""
    from nativeengine_b200 import bodies as B
    if kind == 0:
        got = B.sphere_mass(p[0], 1.3)
    elif kind == 1:
        got = B.cylinder_mass(p[0], p[1], 1.3)
    elif kind == 2:
        got = B.box_mass(p, 1.3)
    elif kind == 3:
        got = B.capsule_mass(p[0], p[1], 1.3)
    else:
        got = B.convex_mass(verts, 1.3)
    want = O.ref_mass_props(kind, p, verts, 1.3)
    assert got[0] == want[0] and tuple(got[1]) == tuple(want[1])


needs_port = pytest.mark.skipif(not O.port_available(), reason="oracle/_build/libne_oracle.so not built")


@needs_port
@pytest.mark.parametrize("name", golden_io.names())
def test_port_reproduces_golden(name):
    """The C restatement (oracle/ne_oracle.c) gives the reference's bits."""
    params, bodies, expected = golden_io.load(name)
    port = O.PortOracle(params, bodies)
    for s, e in enumerate(expected):
        port.step(1)
        assert np.array_equal(port.pairs(), e["pairs"]), f"{name} step {s}: pairs"
        c = port.contacts()
        for k in ("i", "j", "slot", "point", "normal", "depth", "n_imp"):
            assert np.array_equal(c[k], e["c_" + k]), f"{name} step {s}: contact {k}"
        assert np.array_equal(port.islands(), e["islands"])
        st = port.state()
        for k in ("x", "q", "v", "w"):
            assert np.array_equal(st[k], e[k]), f"{name} step {s}: {k}"


@needs_ref
@needs_port
@pytest.mark.parametrize("make,steps", [
    (lambda: __import__("nativeengine_b200.scenes", fromlist=["x"]).box_pile(6, 6, 6), 60),
    (lambda: __import__("nativeengine_b200.scenes", fromlist=["x"]).gas(n=400, half=8.0), 60),
    (lambda: __import__("nativeengine_b200.scenes", fromlist=["x"]).mixed_shapes(n=150, seed=99), 40),
])
def test_port_matches_reference_trajectory(make, steps):
    params, bodies = make()
    ref = O.RefOracle(params, bodies.copy())
    port = O.PortOracle(params, bodies.copy())
    ref.step(steps)
    port.step(steps)
    a, b = ref.state(), port.state()
    for k in ("x", "q", "v", "w"):
        assert np.array_equal(a[k], b[k]), k
