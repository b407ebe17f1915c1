"""Device step vs oracle on the same seeded inputs (FP64, plain path).

Bar: pair lists, contact lists and island partitions bit-exact; contact
geometry, impulses and poses within 1e-12 relative (the device arithmetic is
order-faithful, so in practice they are bit-identical).
"""
import numpy as np
import pytest

from nativeengine_b200 import DeviceWorld, scenes
from tests.parity import assert_same_contacts, assert_same_pairs, assert_same_state, max_state_err

TOL = 1e-12

SCENES = {
    "small_gas_periodic": lambda: scenes.small_gas(),
    "small_gas_reflective": lambda: scenes.small_gas(periodic=False, seed=5),
    "gas_1000": lambda: scenes.gas(),
    "mixed_periodic": lambda: scenes.mixed_shapes(),
    "mixed_reflective_plane": lambda: scenes.mixed_shapes(periodic=False, with_plane=True, gravity=(0, -9.81, 0), seed=11),
    "box_stack": lambda: scenes.box_stack(),
    "box_pile_4x4x4": lambda: scenes.box_pile(4, 4, 4),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
def test_single_step_parity(name, oracle_cls):
    params, bodies = SCENES[name]()
    dev = DeviceWorld(params, bodies.copy())
    ora = oracle_cls(params, bodies.copy())
    for s in range(3):
        dev.step(1)
        ora.step(1)
        assert_same_pairs(dev, ora, f"{name} step {s}")
        assert_same_contacts(dev, ora, TOL, f"{name} step {s}")
        assert_same_state(dev, ora, TOL, f"{name} step {s}")
        assert np.array_equal(dev.islands(), ora.islands()), f"{name} step {s}: island partitions differ"


@pytest.mark.gpu
@pytest.mark.parametrize("name,steps", [("small_gas_periodic", 400), ("gas_1000", 120), ("mixed_periodic", 120),
                                        ("box_stack", 300), ("box_pile_4x4x4", 150)])
def test_trajectory_parity(name, steps, oracle_cls):
    params, bodies = SCENES[name]()
    dev = DeviceWorld(params, bodies.copy())
    ora = oracle_cls(params, bodies.copy())
    dev.step(steps)
    ora.step(steps)
    err = max_state_err(dev, ora)
    assert err <= TOL, f"{name}: {steps}-step trajectory rel err {err:.3e}"
