"""Triangle meshes and compounds on the host side: the BVH builder's
invariants, the compound mass rule, packing into NeBodyArrays, and the
oracle's mesh and compound paths against the reference's own self-test
expectations (src/selftest.cpp:1300-1343)."""
import numpy as np
import pytest

from nativeengine_b200 import _ffi, scenes
from nativeengine_b200.bodies import (BodyArrays, MeshData, child_box, child_sphere, concat, make_compound,
                                      make_sphere, sphere_mass, take_range)


def _leaves(m: MeshData):
    out = []
    stack = [0] if len(m.node_left) else []
    while stack:
        k = stack.pop()
        if m.node_left[k] < 0:
            out.append(k)
        else:
            stack += [m.node_left[k], m.node_right[k]]
    return out


@pytest.mark.parametrize("rows,cols", [(2, 2), (5, 7), (12, 12)])
def test_mesh_bvh_covers_every_triangle_once(rows, cols):
    h = [0.3 * np.sin(0.5 * k) for k in range(rows * cols)]
    m = scenes.heightfield_mesh((0.0, 0.0, 0.0), 1.5, rows, cols, h)
    assert sorted(m.order.tolist()) == list(range(len(m.tris)))
    seen = []
    for k in _leaves(m):
        assert 0 < m.node_count[k] <= 4
        ids = m.order[m.node_start[k]:m.node_start[k] + m.node_count[k]]
        seen += ids.tolist()
        tv = m.verts[m.tris[ids]]
        assert np.all(tv.min(axis=(0, 1)) >= m.node_lo[k]) and np.all(tv.max(axis=(0, 1)) <= m.node_hi[k])
    assert sorted(seen) == list(range(len(m.tris)))


def test_compound_mass_is_the_parallel_axis_sum():
    r = 0.5
    c = make_compound((0, 0, 0), (1, 0, 0, 0), [child_sphere((-1, 0, 0), r), child_sphere((1, 0, 0), r)], 1.0)
    im, ii = sphere_mass(r, 1.0)
    m = 1.0 / im
    assert c.inv_mass == pytest.approx(1.0 / (2 * m), rel=1e-15)
    Ic = 1.0 / ii[0]
    assert c.inv_inertia[0] == pytest.approx(1.0 / (2 * Ic), rel=1e-15)
    assert c.inv_inertia[1] == pytest.approx(1.0 / (2 * (Ic + m)), rel=1e-15)


def test_children_and_meshes_survive_batching():
    p1, b1 = scenes.compound_pile(n=5)
    p2, b2 = scenes.mesh_floor()
    both, begin = concat([b1, b2])
    assert both.n_children == b1.n_children and len(both.meshes) == 1
    part = take_range(both, int(begin[1]), int(begin[2]))
    assert part.meshes[int(part.mesh_index[0])] is b2.meshes[0]
    part = take_range(both, 0, int(begin[1]))
    assert part.n_children == b1.n_children and np.array_equal(part.child_shape, b1.child_shape[:b1.n_children])
    s = both.c
    assert s.n_children == b1.n_children and s.n_meshes == 1


def test_reference_mesh_and_compound_self_test_settings(oracle_cls):
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference not built")
    params, bodies = scenes.mesh_floor()
    o = O.RefOracle(params, bodies.copy())
    o.step(1500)
    st = o.state()
    assert abs(st["x"][1, 1] - 0.5) < 0.05 and abs(st["x"][2, 1] - 0.5) < 0.08
    m = O.ref_mesh(bodies.meshes[0].verts, bodies.meshes[0].tris)
    assert sorted(m.order.tolist()) == [0, 1]
    with pytest.raises(NotImplementedError):
        O.PortOracle(params, bodies.copy())
