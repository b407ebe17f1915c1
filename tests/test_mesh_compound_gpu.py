"""Triangle meshes and compounds on the device against the reference compiled
in place (gatherContacts / meshContacts, src/world.cpp:53-121): pair lists,
contact lists (one per overlapping triangle, one per touching child), island
partitions and poses, bit for bit; and the same worlds in a batch, through the
CUDA graph, and in the FP32 form."""
import numpy as np
import pytest

from nativeengine_b200 import DeviceWorld, _ffi, scenes
from nativeengine_b200.bodies import BodyArrays, concat, make_box, make_mesh, make_sphere
from tests.parity import assert_same_contacts, assert_same_pairs, assert_same_state, max_state_err

SCENES = {
    "mesh_floor": (lambda: scenes.mesh_floor(), 700),
    "terrain_drop": (lambda: scenes.terrain_drop(), 150),
    "compound_pile": (lambda: scenes.compound_pile(), 150),
    "compound_on_mesh": (lambda: scenes.compound_pile(n=8, with_mesh=True), 150),
}


@pytest.fixture(scope="module")
def ref():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("the reference is not built (oracle/_ref)")
    return O


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
def test_single_steps_match_the_reference(ref, name):
    make, settle = SCENES[name]
    params, bodies = make()
    dev = DeviceWorld(params, bodies.copy())
    ora = ref.RefOracle(params, bodies.copy())
    dev.step(settle // 2)
    ora.step(settle // 2)
    seen = 0
    for s in range(4):
        dev.step(1)
        ora.step(1)
        what = f"{name} step {settle // 2 + s}"
        assert_same_pairs(dev, ora, what)
        assert_same_contacts(dev, ora, 0.0, what)
        assert_same_state(dev, ora, 0.0, what)
        assert np.array_equal(dev.islands(), ora.islands()), f"{what}: island partitions differ"
        seen += dev.stats()["contacts"]
    assert seen > 0, f"{name}: no contacts exercised"
    dev.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
def test_trajectories_match_the_reference(ref, name):
    make, steps = SCENES[name]
    params, bodies = make()
    dev = DeviceWorld(params, bodies.copy(), record=False)
    ora = ref.RefOracle(params, bodies.copy())
    dev.step(2 * steps)
    ora.step(2 * steps)
    assert max_state_err(dev, ora) == 0.0, name
    assert dev.stats()["graph_steps"] > 0
    dev.close()


@pytest.mark.gpu
def test_reference_built_bvh(ref):
    """The mesh's BVH as the reference's own MeshData::build() makes it: the
    contacts come in the reference's triangle order."""
    h = [0.5 * np.sin(0.7 * c) * np.cos(0.4 * r) for r in range(10) for c in range(10)]
    own = scenes.heightfield_mesh((-9.0, 0.0, -9.0), 2.0, 10, 10, h)
    mesh = ref.ref_mesh(own.verts, own.tris)
    rng = np.random.default_rng(3)
    bodies = [make_mesh((0.0, 0.0, 0.0), (1, 0, 0, 0), mesh)]
    for k in range(20):
        x = (float(rng.uniform(-6, 6)), float(1.5 + 0.9 * k), float(rng.uniform(-6, 6)))
        bodies.append(make_box(x, (1, 0, 0, 0), (0.9, 0.3, 0.7), 1.0) if k % 2 else make_sphere(x, 0.7, 1.0))
    params = scenes.default_params(half=1000.0, open_boundary=1, dt=1.0 / 120.0, gravity=(0.0, -9.81, 0.0),
                                   restitution=0.0, friction=0.4)
    ba = BodyArrays(bodies)
    dev = DeviceWorld(params, ba.copy())
    ora = ref.RefOracle(params, ba.copy())
    for s in range(200):
        dev.step(1)
        ora.step(1)
        if s % 40 == 39:
            assert_same_contacts(dev, ora, 0.0, f"step {s}")
            assert_same_state(dev, ora, 0.0, f"step {s}")
    assert dev.stats()["contacts"] > 0
    dev.close()


@pytest.mark.gpu
def test_batch_of_mesh_and_compound_worlds_matches_each_world_alone():
    made = [scenes.mesh_floor(), scenes.compound_pile(n=9), scenes.terrain_drop(n=16),
            scenes.compound_pile(n=6, seed=5, with_mesh=True)]
    params = [p for p, _ in made]
    both, begin = concat([b for _, b in made])
    dev = DeviceWorld(params[0], None, record=False)
    dev.upload_batch(params, both.copy(), begin)
    dev.step(120)
    got = dev.state()
    for k, (p, b) in enumerate(made):
        alone = DeviceWorld(p, b.copy(), record=False)
        alone.step(120)
        want = alone.state()
        for key in ("x", "q", "v", "w"):
            assert np.array_equal(got[key][begin[k]:begin[k + 1]], want[key]), (k, key)
        alone.close()
    dev.close()


@pytest.mark.gpu
def test_graph_and_eager_agree_with_meshes_and_compounds():
    out = []
    for graph in (True, False):
        params, bodies = scenes.terrain_drop()
        dev = DeviceWorld(params, bodies, record=False)
        dev.set_graph(graph)
        dev.step(90)
        out.append(dev.state())
        dev.close()
    for key in ("x", "q", "v", "w"):
        assert np.array_equal(out[0][key], out[1][key]), key


@pytest.mark.gpu
def test_fp32_form_steps_meshes_and_compounds_graph_and_eager_alike():
    """The FP32 form takes mesh and compound contacts from the FP64 passes;
    graph-replayed and kernel-by-kernel FP32 steps agree bit for bit."""
    out = []
    for graph in (True, False):
        params, bodies = scenes.compound_pile(n=10, with_mesh=True)
        dev = DeviceWorld(params, bodies, record=False, precision="f32")
        dev.set_graph(graph)
        dev.step(120)
        assert dev.stats()["contacts"] > 0
        out.append(dev.state())
        dev.close()
    for key in ("x", "q", "v", "w"):
        assert np.array_equal(out[0][key], out[1][key]), key
