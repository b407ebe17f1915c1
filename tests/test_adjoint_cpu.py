"""The per-world step program and its adjoint (csrc/ne_adjoint.cuh), built for
the host as test infrastructure (tests/cpp/adjoint_host.cpp):

* its forward is the reference's step bit for bit (against the oracle);
* its gradients of L = sum |x_T - t|^2 match central finite differences of the
  FP64 reference (the oracle) to 1e-4 relative, for initial velocities, masses,
  world friction and world restitution.

The device runs the same source (ne_adjoint.cu, tests/test_adjoint_gpu.py)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from nativeengine_b200 import _ffi, scenes
from nativeengine_b200.bodies import BodyArrays, make_box, make_plane, make_convex, default_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CAP = 4096


@pytest.fixture(scope="module")
def host_adj(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("adj") / "libadj_host.so")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I", cuda_inc,
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "nativeengine_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "adjoint_host.cpp"), "-o", out], check=True)
    lib = C.CDLL(out)
    dp = C.POINTER(C.c_double)
    lib.adjh_forward.argtypes = [C.POINTER(_ffi.NeWorldParams), C.POINTER(_ffi.NeBodyArrays), C.c_int, C.c_uint32,
                                 dp, dp, dp, dp]
    lib.adjh_grad.argtypes = [C.POINTER(_ffi.NeWorldParams), C.POINTER(_ffi.NeBodyArrays), C.c_int, C.c_uint32,
                              dp, dp, dp, dp, dp, dp, dp, dp, dp, dp]
    return lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def host_forward(lib, params, bodies, nsteps):
    n = bodies.n
    x, q, v, w = np.zeros((n, 3)), np.zeros((n, 4)), np.zeros((n, 3)), np.zeros((n, 3))
    rc = lib.adjh_forward(C.byref(params), C.byref(bodies.c), nsteps, CAP, _p(x), _p(q), _p(v), _p(w))
    assert rc == 0, rc
    return {"x": x, "q": q, "v": v, "w": w}


def host_grad(lib, params, bodies, nsteps, xbar):
    n = bodies.n
    out = {k: np.zeros(s) for k, s in (("x", (n, 3)), ("q", (n, 4)), ("v", (n, 3)), ("w", (n, 3)),
                                         ("invm", (n,)), ("invi", (n, 3)))}
    mu, e = C.c_double(), C.c_double()
    xb = np.ascontiguousarray(xbar, dtype=np.float64)
    rc = lib.adjh_grad(C.byref(params), C.byref(bodies.c), nsteps, CAP, _p(xb), None, _p(out["x"]), _p(out["q"]),
                       _p(out["v"]), _p(out["w"]), _p(out["invm"]), _p(out["invi"]), C.byref(mu), C.byref(e))
    assert rc == 0, rc
    out["mu"], out["e"] = mu.value, e.value
    inv_m = bodies.inv_mass
    dyn = inv_m > 0
    out["mass"] = np.where(dyn, -(out["invm"] * inv_m + (out["invi"] * bodies.inv_inertia).sum(1))
                           / np.where(dyn, 1.0 / np.where(dyn, inv_m, 1.0), 1.0), 0.0)
    return out


def _colliding():
    """Two boxes sliding into each other on a plane, one turned: box-box
    manifolds, plane contacts, friction and restitution."""
    bodies = [make_plane((0.0, 0.0, 0.0), (0.0, 1.0, 0.0))]
    a = make_box((-1.2, 0.5, 0.1), (1.0, 0.0, 0.0, 0.0), (0.5, 0.5, 0.5), 1.0)
    a.v = (3.0, 0.0, 0.2)
    c = 0.5 ** 0.5
    b = make_box((1.2, 0.55, -0.1), (np.cos(0.3), 0.0, np.sin(0.3), 0.0), (0.5, 0.55, 0.45), 1.0)
    b.v = (-2.5, 0.0, 0.0)
    bodies += [a, b]
    params = default_params(open_boundary=1, gravity=(0.0, -9.81, 0.0), dt=1.0 / 60.0, friction=0.45,
                            restitution=0.3)
    return params, BodyArrays(bodies)


FORWARD_CASES = {
    "sliding_3x3": (lambda: scenes.sliding_boxes(grid=3, seed=11), 40),
    "colliding": (_colliding, 40),
    "mixed_plane": (lambda: scenes.mixed_shapes(n=40, periodic=False, with_plane=True, gravity=(0, -9.81, 0),
                                                seed=23), 25),
    "gas_periodic": (lambda: scenes.small_gas(n=40, seed=3), 30),
}


@pytest.mark.parametrize("name", sorted(FORWARD_CASES))
def test_per_world_program_matches_the_reference(host_adj, oracle_cls, name):
    make, steps = FORWARD_CASES[name]
    params, bodies = make()
    got = host_forward(host_adj, params, bodies.copy(), steps)
    ref = oracle_cls(params, bodies.copy())
    ref.step(steps)
    want = ref.state()
    for k in ("x", "q", "v", "w"):
        assert np.array_equal(got[k], want[k]), f"{name}: {k} differs from the reference"


def _loss(x, targets, dyn):
    d = (x - targets)[dyn]
    return float((d * d).sum())


def _fd(oracle_cls, params, bodies, steps, targets, perturb, h):
    vals = []
    for s in (+1.0, -1.0):
        p2, b2 = perturb(params, bodies.copy(), s * h)
        o = oracle_cls(p2, b2)
        o.step(steps)
        vals.append(_loss(o.state()["x"], targets, bodies.inv_mass > 0))
    return (vals[0] - vals[1]) / (2.0 * h)


def _params_copy(p):
    q = _ffi.NeWorldParams()
    C.pointer(q)[0] = p
    return q


GRAD_CASES = {
    "sliding_2x2": (lambda: scenes.sliding_boxes(grid=2, seed=13, mu=0.45, e=0.3), 30),
    "colliding": (_colliding, 30),
}


@pytest.mark.parametrize("name", sorted(GRAD_CASES))
def test_adjoint_matches_reference_finite_differences(host_adj, oracle_cls, name):
    make, steps = GRAD_CASES[name]
    params, bodies = make()
    rng = np.random.default_rng(7)
    targets = rng.uniform(-5.0, 5.0, (bodies.n, 3))
    dyn = bodies.inv_mass > 0
    xT = host_forward(host_adj, params, bodies.copy(), steps)["x"]
    xbar = np.where(dyn[:, None], 2.0 * (xT - targets), 0.0)
    g = host_grad(host_adj, params, bodies.copy(), steps, xbar)

    checks = []
    for i in np.nonzero(dyn)[0]:
        for ax in (0, 2):
            def pert_v(p, b, d, i=i, ax=ax):
                b.v[i, ax] += d
                return p, b
            checks.append((f"v0[{i},{ax}]", g["v"][i, ax], pert_v, 1e-6 * max(1.0, abs(bodies.v[i, ax]))))

        def pert_m(p, b, d, i=i):
            m = 1.0 / b.inv_mass[i]
            m2 = m * (1.0 + d)
            b.inv_mass[i] = 1.0 / m2
            b.inv_inertia[i] *= m / m2
            return p, b
        m = 1.0 / bodies.inv_mass[i]
        checks.append((f"mass[{i}] (relative)", g["mass"][i] * m, pert_m, 1e-6))

    def pert_mu(p, b, d):
        p2 = _params_copy(p)
        p2.friction += d
        return p2, b

    def pert_e(p, b, d):
        p2 = _params_copy(p)
        p2.restitution += d
        return p2, b
    checks.append(("friction", g["mu"], pert_mu, 1e-6))
    checks.append(("restitution", g["e"], pert_e, 1e-6))

    bad = []
    for label, adj, pert, h in checks:
        fd = _fd(oracle_cls, params, bodies, steps, targets, pert, h)
        scale = max(abs(fd), abs(adj), 1e-3)
        rel = abs(adj - fd) / scale
        print(f"{name} {label}: adjoint {adj:+.9e} fd {fd:+.9e} rel {rel:.2e}")
        if rel > 1e-4:
            bad.append((label, adj, fd, rel))
    assert not bad, bad
