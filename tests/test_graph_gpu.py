"""CUDA-graph stepping (ne_world_set_graph) against kernel-by-kernel stepping.

The captured step is the same kernel sequence with the same arguments, so the
two must agree bit for bit, also across the steps where a device buffer
overflows: the batch halts on the device, the host restores that step's
pre-step state, grows the buffer and re-captures.
"""
import numpy as np
import pytest

from nativeengine_b200 import DeviceWorld, scenes
from nativeengine_b200.bodies import BodyArrays, make_sphere

KEYS = ("x", "q", "v", "w")


def _pair(make, precision="f64", batch=False):
    out = []
    for graph in (True, False):
        made = make()
        if batch:
            params, bodies, begin = made[:3]
            dev = DeviceWorld(params[0], None, record=False, precision=precision)
            dev.upload_batch(params, bodies, begin)
        else:
            params, bodies = made
            dev = DeviceWorld(params, bodies, record=False, precision=precision)
        dev.set_graph(graph)
        out.append(dev)
    return out


def _same(a, b, label):
    sa, sb = a.state(), b.state()
    for k in KEYS:
        assert np.array_equal(sa[k], sb[k]), f"{label}: {k} differs between graph and eager stepping"


@pytest.mark.gpu
@pytest.mark.parametrize("name,precision", [("box_pile_216", "f64"), ("gas_periodic", "f64"),
                                            ("mixed_periodic", "f64"), ("batch_24", "f64"), ("batch_24", "f32")])
def test_graph_steps_match_eager_steps(name, precision):
    makes = {
        "box_pile_216": (lambda: scenes.box_pile(6, 6, 6, seed=4), False),
        "gas_periodic": (lambda: scenes.gas(n=400, half=6.0, seed=5), False),
        "mixed_periodic": (lambda: scenes.mixed_shapes(n=160, seed=17), False),
        "batch_24": (lambda: scenes.batch_mix(nworlds=24, lo=16, hi=300, seed=11), True),
    }
    make, batch = makes[name]
    g, e = _pair(make, precision, batch)
    for chunk in (1, 7, 64, 100):
        g.step(chunk)
        e.step(chunk)
        _same(g, e, f"{name}/{precision} after {chunk}")
    sg, se = g.stats(), e.stats()
    # A step that overflowed a buffer is taken once more outside the graph.
    assert 172 - sg["retries"] <= sg["graph_steps"] <= 172 and se["graph_steps"] == 0, (sg, se)
    assert sg["steps"] == se["steps"] == 172
    assert sg["contacts"] == se["contacts"] and sg["survivors"] == se["survivors"]
    assert g.launch_count() > 0
    g.close()
    e.close()


def _expanding_gas():
    """Open-boundary sphere gas flying apart: the cell coordinates widen, so
    the cell-key sort needs more bits as the run goes on."""
    params, bodies = scenes.gas(n=500, half=6.0, seed=21, sigma_v=4.0)
    params.periodic = 0
    params.open_boundary = 1
    return params, bodies


@pytest.mark.gpu
def test_graph_halts_and_regrows_key_bits(oracle_cls):
    g, e = _pair(_expanding_gas)
    for _ in range(6):
        g.step(50)
        e.step(50)
        _same(g, e, "expanding gas")
    assert g.stats()["retries"] > 0, "no step overflowed: the halt path was not exercised"
    assert g.stats()["graph_captures"] >= 2
    params, bodies = _expanding_gas()
    ref = oracle_cls(params, bodies.copy())
    ref.step(300)
    want, got = ref.state(), g.state()
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k
    g.close()
    e.close()


@pytest.mark.gpu
def test_graph_halts_and_regrows_pair_and_contact_buffers(oracle_cls):
    """Capacities are sized at the first upload; a tiny first world leaves
    them at their minimum, so the dense pile that replaces it overflows the
    survivor and contact buffers inside a replayed batch."""
    out = []
    for graph in (True, False):
        tiny = BodyArrays([make_sphere((0.0, 0.0, 0.0), 0.5, 1.0), make_sphere((3.0, 0.0, 0.0), 0.5, 1.0)])
        params, bodies = scenes.box_pile(8, 8, 8, seed=9)
        dev = DeviceWorld(params, tiny, record=False)
        dev.set_graph(graph)
        dev.upload(bodies)
        out.append(dev)
    g, e = out
    for _ in range(4):
        g.step(40)
        e.step(40)
        _same(g, e, "pile after growth")
    sg = g.stats()
    assert sg["retries"] > 0 and sg["graph_steps"] > 0, sg
    params, bodies = scenes.box_pile(8, 8, 8, seed=9)
    ref = oracle_cls(params, bodies.copy())
    ref.step(160)
    want, got = ref.state(), g.state()
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k
    g.close()
    e.close()
