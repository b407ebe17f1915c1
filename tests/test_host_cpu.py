"""Host-side plumbing without a GPU: seeded scenes and body packing."""
import numpy as np

from nativeengine_b200 import _ffi, scenes
from nativeengine_b200.bodies import BodyArrays, make_box, make_plane, make_sphere, make_static


def test_scenes_are_deterministic():
    for make in (lambda: scenes.gas(n=200), lambda: scenes.box_pile(4, 4, 4), lambda: scenes.mixed_shapes(n=40)):
        (p1, b1), (p2, b2) = make(), make()
        for k in ("x", "q", "v", "w", "inv_mass", "inv_inertia", "verts"):
            assert np.array_equal(getattr(b1, k), getattr(b2, k))


def test_box_pile_config():
    params, b = scenes.box_pile()
    assert b.n == 4097
    assert b.shape[0] == _ffi.BOX and b.inv_mass[0] == 0.0
    assert np.all(b.half_extents[1:] >= 0.25) and np.all(b.half_extents[1:] <= 0.75)
    assert params.open_boundary == 1 and params.friction == 0.5 and params.restitution == 0.2
    assert tuple(params.gravity) == (0.0, -9.81, 0.0)
    assert abs(params.dt - 1.0 / 60.0) < 1e-18
    q = b.q[1:]
    assert np.allclose(np.einsum("ij,ij->i", q, q), 1.0)


def test_gas_config_no_overlap():
    params, b = scenes.gas()
    assert b.n == 1000 and params.periodic == 1 and params.half == 12.5
    L = 25.0
    d = b.x[:, None, :] - b.x[None, :, :]
    d -= L * np.floor(d / L + 0.5)
    r2 = np.einsum("ijk,ijk->ij", d, d) + np.eye(b.n) * 10
    assert r2.min() >= 1.0
    assert np.allclose(1.0 / b.inv_mass, 1.0)


def test_body_arrays_view():
    bodies = [make_static(make_box((0, -1, 0), (1, 0, 0, 0), (5, 1, 5), 1.0)), make_sphere((0, 1, 0), 0.5, 1.0),
              make_plane((0, 0, 0), (0, 2, 0))]
    ba = BodyArrays(bodies)
    c = ba.c
    assert c.n == 3 and c.shape[1] == _ffi.SPHERE and c.shape[2] == _ffi.PLANE
    assert c.half_extents[7] == 1.0      # plane normal normalised
    assert c.flags[0] & _ffi.DYNAMIC == 0 and c.flags[1] & _ffi.DYNAMIC
