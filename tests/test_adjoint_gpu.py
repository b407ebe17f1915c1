"""stepBackward on the device (ne_world_step_backward): the same per-world
program and adjoint as the host build in test_adjoint_cpu.py, one thread per
world, with checkpoints.  Gradients of L = sum |x_T - t|^2 are checked against
the host build (identical source), across checkpoint intervals, and against
central finite differences of the FP64 reference on a batch of the adjoint
workload (boxes sliding on a plane, per-world friction and restitution)."""
import numpy as np
import pytest

from nativeengine_b200 import DeviceWorld, _ffi, scenes
from nativeengine_b200.shard import slice_bodies
from tests.test_adjoint_cpu import (GRAD_CASES, _colliding, _params_copy, host_adj, host_forward,  # noqa: F401
                                    host_grad)


def _dev_grad(params, bodies, steps, xbar, k=0):
    dev = DeviceWorld(params, bodies.copy(), record=False)
    g = dev.step_backward(steps, k, xbar=xbar)
    dev.close()
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GRAD_CASES))
def test_device_gradients_equal_the_host_build(host_adj, name):
    make, steps = GRAD_CASES[name]
    params, bodies = make()
    rng = np.random.default_rng(3)
    targets = rng.uniform(-5.0, 5.0, (bodies.n, 3))
    dyn = bodies.inv_mass > 0
    xT = host_forward(host_adj, params, bodies.copy(), steps)["x"]
    xbar = np.where(dyn[:, None], 2.0 * (xT - targets), 0.0)
    h = host_grad(host_adj, params, bodies.copy(), steps, xbar)
    d = _dev_grad(params, bodies, steps, xbar, k=7)
    for key, hk in (("x", "x"), ("q", "q"), ("v", "v"), ("w", "w"), ("inv_mass", "invm"), ("inv_inertia", "invi")):
        assert np.allclose(d[key], h[hk], rtol=1e-12, atol=1e-14), key
    assert abs(d["friction"][0] - h["mu"]) <= 1e-12 * max(1.0, abs(h["mu"]))
    assert abs(d["restitution"][0] - h["e"]) <= 1e-12 * max(1.0, abs(h["e"]))


@pytest.mark.gpu
def test_checkpoint_interval_does_not_change_gradients():
    params, bodies = _colliding()
    xbar = np.ones((bodies.n, 3))
    g = [_dev_grad(params, bodies, 24, xbar, k) for k in (0, 1, 5, 24)]
    for other in g[1:]:
        for key in ("x", "v", "w", "inv_mass", "friction", "restitution"):
            assert np.array_equal(g[0][key], other[key]), key


@pytest.mark.gpu
def test_step_backward_leaves_the_world_unchanged():
    params, bodies = scenes.sliding_boxes(grid=3, seed=2)
    dev = DeviceWorld(params, bodies.copy(), record=False)
    dev.step(5)
    before = dev.state()
    dev.step_backward(20, 5, xbar=np.ones((bodies.n, 3)))
    after = dev.state()
    for key in ("x", "q", "v", "w"):
        assert np.array_equal(before[key], after[key]), key
    dev.step(3)
    ref = DeviceWorld(params, bodies.copy(), record=False)
    ref.step(8)
    assert np.array_equal(dev.state()["x"], ref.state()["x"]), "warm cache or state disturbed"
    dev.close()
    ref.close()


@pytest.mark.gpu
def test_unsupported_world_is_refused():
    params, bodies = scenes.mixed_shapes(n=20, seed=5)   # capsules and cylinders
    dev = DeviceWorld(params, bodies.copy(), record=False)
    with pytest.raises(_ffi.NeError) as e:
        dev.step_backward(3, 0, xbar=np.ones((bodies.n, 3)))
    assert e.value.code == _ffi.NE_ERR_UNSUPPORTED
    dev.close()


def _world_loss(oracle_cls, params, bodies, steps, targets):
    o = oracle_cls(params, bodies)
    o.step(steps)
    x = o.state()["x"]
    dyn = bodies.inv_mass > 0
    d = (x - targets)[dyn]
    return float((d * d).sum())


@pytest.mark.gpu
def test_batch_gradients_match_reference_finite_differences(oracle_cls):
    steps, k = 40, 10
    params, bodies, begin, targets = scenes.adjoint_batch(nworlds=6, grid=4, seed=9)
    dev = DeviceWorld(params[0], None, record=False)
    dev.upload_batch(params, bodies.copy(), begin)
    with dev.checkpoint() as ck:
        dev.step(steps)
        xT = dev.state()["x"]
        dev.restore(ck)
    dyn = bodies.inv_mass > 0
    xbar = np.where(dyn[:, None], 2.0 * (xT - targets), 0.0)
    g = dev.step_backward(steps, k, xbar=xbar)
    dev.close()
    bad = []
    for wi in (0, 3, 5):
        part, _ = slice_bodies(bodies, begin, wi, wi + 1)
        tw = targets[begin[wi]:begin[wi + 1]]
        b0 = int(begin[wi])
        checks = []
        for li in (1, 6):
            for ax in (0, 2):
                def pv(p, b, dlt, li=li, ax=ax):
                    b.v[li, ax] += dlt
                    return p, b
                checks.append((f"w{wi} v0[{li},{ax}]", g["v"][b0 + li, ax], pv, 1e-6))

        def pm(p, b, dlt, li=5):
            m = 1.0 / b.inv_mass[li]
            m2 = m * (1.0 + dlt)
            b.inv_mass[li] = 1.0 / m2
            b.inv_inertia[li] *= m / m2
            return p, b
        checks.append((f"w{wi} mass[5] (relative)", g["mass"][b0 + 5] / part.inv_mass[5], pm, 1e-6))

        def pmu(p, b, dlt):
            q = _params_copy(p)
            q.friction += dlt
            return q, b

        def pe(p, b, dlt):
            q = _params_copy(p)
            q.restitution += dlt
            return q, b
        checks.append((f"w{wi} friction", g["friction"][wi], pmu, 1e-6))
        checks.append((f"w{wi} restitution", g["restitution"][wi], pe, 1e-6))
        for label, adj, pert, h in checks:
            vals = []
            for s in (1.0, -1.0):
                p2, b2 = pert(params[wi], part.copy(), s * h)
                vals.append(_world_loss(oracle_cls, p2, b2, steps, tw))
            fd = (vals[0] - vals[1]) / (2.0 * h)
            rel = abs(adj - fd) / max(abs(fd), abs(adj), 1e-3)
            print(f"{label}: adjoint {adj:+.9e} fd {fd:+.9e} rel {rel:.2e}")
            if rel > 1e-4:
                bad.append((label, adj, fd, rel))
    assert not bad, bad
