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


# Randomised scenes (size, box, boundary mode, planes), screened on the CPU so
# that the reference finishes them: on a few near-degenerate deep overlaps the
# reference's EPA face list grows without bound and its step does not return
# (see test_device_epa_stays_bounded), and parity cannot be checked there.
SWEEP_CASES = [
    (686, 7.802, "periodic", False, 976699), (172, 6.617, "reflective", True, 138781),
    (266, 5.181, "open", True, 241767), (563, 13.641, "periodic", False, 318534),
    (673, 8.41, "reflective", False, 254719), (451, 12.636, "open", True, 863757),
    (393, 10.599, "periodic", False, 674881), (94, 6.228, "reflective", True, 867087),
    (173, 12.704, "open", False, 60139), (167, 10.712, "periodic", False, 683689),
    (152, 4.601, "reflective", True, 178487), (685, 8.39, "open", False, 532595),
    (186, 6.513, "periodic", False, 3133), (482, 8.253, "reflective", True, 175990),
    (531, 13.22, "open", True, 153475), (575, 5.823, "periodic", False, 992259),
    (605, 4.869, "reflective", True, 878964), (361, 12.29, "open", True, 281052),
]


def _sweep_scene(n, half, mode, plane, seed):
    params, bodies = scenes.mixed_shapes(n=n, half=half, periodic=(mode == "periodic"), with_plane=plane, seed=seed,
                                         gravity=(0.0, -9.81, 0.0) if mode != "periodic" else (0, 0, 0))
    if mode == "open":
        params.open_boundary = 1
    return params, bodies


@pytest.mark.gpu
@pytest.mark.parametrize("k,n,half,mode,plane,seed", [(k,) + c for k, c in enumerate(SWEEP_CASES)])
def test_random_scene_parity(k, n, half, mode, plane, seed, oracle_cls):
    """The broadphase pair list, the contacts and the poses after two steps
    match the oracle on randomised scenes."""
    params, bodies = _sweep_scene(n, half, mode, plane, seed)
    dev = DeviceWorld(params, bodies.copy())
    ora = oracle_cls(params, bodies.copy())
    for s in range(2):
        dev.step(1)
        ora.step(1)
        what = f"case {k} ({mode}, n={n}, half={half:.2f}, plane={plane}) step {s}"
        assert_same_pairs(dev, ora, what)
        assert_same_contacts(dev, ora, TOL, what)
        assert_same_state(dev, ora, TOL, what)


@pytest.mark.gpu
def test_device_epa_stays_bounded():
    """A scene on which the reference's second step does not return: a sphere
    (body 135) deep inside a 12-point hull (body 374) drives its EPA into a face
    list that keeps multiplying.  The device EPA works in fixed budgets (68
    vertices, 192 faces, 64 iterations), so the step returns -- NE_OK, or
    NE_ERR_NUMERIC when a budget was hit -- with a finite state.  (No oracle:
    the reference cannot produce one.)"""
    from nativeengine_b200 import _ffi
    params, bodies = _sweep_scene(673, 8.410061220535114, "reflective", False, 254719)
    dev = DeviceWorld(params, bodies.copy())
    for _ in range(3):
        rc = dev.step(1)
        assert rc in (_ffi.NE_OK, _ffi.NE_ERR_NUMERIC)
    st = dev.state()
    assert all(np.isfinite(st[k]).all() for k in ("x", "q", "v", "w"))


def _long_lists(brute):
    """Piles whose partner lists reach every later body of the world: the
    ground box's list (577 bodies) and, under forced brute force, the first
    ~200 lists of 721 bodies -- more long lists than the device splits per
    step, so the rest take the one-warp walk."""
    if brute:
        params, bodies = scenes.box_pile(8, 9, 10, seed=6)
        params.force_brute_force = 1
        return params, bodies
    return scenes.box_pile(8, 8, 9, seed=7)


@pytest.mark.gpu
@pytest.mark.parametrize("brute", [False, True])
def test_long_partner_lists_match_the_oracle(brute, oracle_cls):
    params, bodies = _long_lists(brute)
    dev = DeviceWorld(params, bodies.copy())
    ora = oracle_cls(params, bodies.copy())
    for s in range(90):
        dev.step(1)
        ora.step(1)
        if s % 15 == 14:
            what = f"brute={brute} step {s}"
            assert_same_pairs(dev, ora, what)
            assert_same_contacts(dev, ora, 0.0, what)
            assert_same_state(dev, ora, 0.0, what)
    assert dev.stats()["contacts"] > 0
    dev.close()
