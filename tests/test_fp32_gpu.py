"""The batched FP32 form against the FP64 path, and the checkpoint API it is
measured with.

Error definition (one step from identical inputs): a device checkpoint holds
the state and the warm cache after a few settling steps; one FP64 step from
it and one FP32 step from it are compared per body:

    pose error  = |x32 - x64| / max(|x64|, 1)      (length unit ~ body size)
    orientation = |q32 - q64|                       (unit quaternions)

Bound: 1e-5 relative one-step pose error.
"""
import numpy as np
import pytest

from nativeengine_b200 import DeviceWorld, scenes
from nativeengine_b200.bodies import concat

POSE_TOL = 1e-5


def _batch_small():
    params, bodies, begin, _ = scenes.batch_mix(nworlds=24, lo=16, hi=300, seed=11)
    return params, bodies, begin


SCENES = {
    "box_pile_216": (lambda: scenes.box_pile(6, 6, 6, seed=4), 90),
    "gas_periodic": (lambda: scenes.gas(n=400, half=6.0, seed=5), 20),
    "mixed_periodic": (lambda: scenes.mixed_shapes(n=160, seed=17), 40),
    "mixed_plane": (lambda: scenes.mixed_shapes(n=120, periodic=False, with_plane=True,
                                                gravity=(0, -9.81, 0), seed=23), 60),
    "box_stack": (lambda: scenes.box_stack(levels=6), 120),
    "granular_2048": (lambda: scenes.granular_mix(n=2048, max_attempts=2000, seed=7), 10),
    "batch_24": (_batch_small, 60),
    "compound_pile": (lambda: scenes.compound_pile(), 120),
    "terrain_drop": (lambda: scenes.terrain_drop(), 120),
}


def _make(name):
    make, settle = SCENES[name]
    made = make()
    if len(made) == 3:
        params, bodies, begin = made
        dev = DeviceWorld(params[0], None, record=False)
        dev.upload_batch(params, bodies, begin)
    else:
        params, bodies = made
        dev = DeviceWorld(params, bodies, record=False)
    return dev, settle


def one_step_errors(dev):
    with dev.checkpoint() as ck:
        dev.set_precision("f64")
        dev.step(1)
        s64 = dev.state()
        c64 = dev.stats()["contacts"]
        dev.restore(ck)
        dev.set_precision("f32")
        dev.step(1)
        s32 = dev.state()
        c32 = dev.stats()["contacts"]
        dev.restore(ck)
        dev.set_precision("f64")
    ex = np.linalg.norm(s32["x"] - s64["x"], axis=1) / np.maximum(np.linalg.norm(s64["x"], axis=1), 1.0)
    eq = np.linalg.norm(s32["q"] - s64["q"], axis=1)
    ev = np.linalg.norm(s32["v"] - s64["v"], axis=1) / np.maximum(np.linalg.norm(s64["v"], axis=1), 1.0)
    return {"x": float(ex.max()), "q": float(eq.max()), "v": float(ev.max()), "contacts64": c64,
            "contacts32": c32, "changed": bool(np.any(s32["x"] != s64["x"]) or np.any(s32["v"] != s64["v"]))}


@pytest.mark.gpu
def test_checkpoint_restore_replays_bit_exactly():
    dev, _ = _make("box_pile_216")
    dev.step(40)
    with dev.checkpoint() as ck:
        dev.step(5)
        a = dev.state()
        dev.restore(ck)
        dev.step(5)
        b = dev.state()
    for key in ("x", "q", "v", "w"):
        assert np.array_equal(a[key], b[key]), key
    dev.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
def test_fp32_one_step_pose_error(name):
    dev, settle = _make(name)
    dev.step(settle)
    st = dev.stats()
    assert st["contacts"] > 0, "scene has no contacts to exercise the FP32 solve"
    err = one_step_errors(dev)
    print(f"{name}: contacts {err['contacts64']}/{err['contacts32']}  pose {err['x']:.3e}  "
          f"quat {err['q']:.3e}  vel {err['v']:.3e}")
    assert err["changed"], "the FP32 step reproduced FP64 bit for bit: the FP32 kernels did not run"
    assert err["x"] <= POSE_TOL, err
    assert err["q"] <= POSE_TOL, err
    dev.close()


@pytest.mark.gpu
def test_fp32_then_fp64_is_bit_exact_again(oracle_cls):
    """Switching back to FP64 restores the reference path exactly."""
    params, bodies = scenes.mixed_shapes(n=120, seed=29)
    dev = DeviceWorld(params, bodies.copy(), record=False, precision="f32")
    dev.step(3)
    st = dev.state()
    start = bodies.copy()
    for key in ("x", "q", "v", "w"):
        getattr(start, key)[:] = st[key]
    ref = oracle_cls(params, start)
    dev.set_precision("f64")
    dev.reset_warm_cache()
    dev.step(3)
    ref.step(3)
    a, b = dev.state(), ref.state()
    for key in ("x", "q", "v", "w"):
        assert np.array_equal(a[key], b[key]), key
    dev.close()


@pytest.mark.gpu
def test_autotune_keeps_state_and_results():
    dev_a, _ = _make("box_pile_216")
    dev_b, _ = _make("box_pile_216")
    dev_a.step(30)
    dev_b.step(30)
    shape = dev_b.autotune(steps=2)
    assert shape[0] % 32 == 0 and 64 <= shape[0] <= 512 and 1 <= shape[1] <= 4 and 1 <= shape[2] <= 64
    assert dev_b.solver_shape() == shape
    dev_a.step(4)
    dev_b.step(4)
    a, b = dev_a.state(), dev_b.state()
    for key in ("x", "q", "v", "w"):
        assert np.array_equal(a[key], b[key]), key
    dev_a.close()
    dev_b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_team_solver_matches_block_local(precision):
    """Big islands solved by teams of CTAs reproduce the one-CTA solver bit for bit."""
    dev_a, _ = _make("box_pile_216")
    dev_b, _ = _make("box_pile_216")
    for dev in (dev_a, dev_b):
        dev.set_precision(precision)
    dev_a.set_solver_shape(256, 1, 1)
    dev_b.set_solver_shape(128, 2, 8)
    dev_a.step(90)   # settle into one big island
    dev_b.step(90)
    for _ in range(3):
        dev_a.step(10)
        dev_b.step(10)
        a, b = dev_a.state(), dev_b.state()
        for key in ("x", "q", "v", "w"):
            assert np.array_equal(a[key], b[key]), key
    assert dev_b.stats()["max_island"] >= 48, "no big island exercised"
    dev_a.close()
    dev_b.close()


@pytest.mark.gpu
def test_fp32_pose_error_on_a_large_batch_after_fp32_steps():
    """Batch scale (256 worlds, piles up to ~2k boxes), state reached by FP32
    stepping: deep piles exercise near-touching GJK/EPA cases in FP32."""
    params, bodies, begin, _ = scenes.batch_mix(nworlds=256, seed=4)
    dev = DeviceWorld(params[0], None, record=False, precision="f32")
    dev.upload_batch(params, bodies, begin)
    dev.step(100)
    err = one_step_errors(dev)
    print(f"batch_256: contacts {err['contacts64']}/{err['contacts32']}  pose {err['x']:.3e}  "
          f"quat {err['q']:.3e}  vel {err['v']:.3e}")
    assert err["x"] <= POSE_TOL, err
    assert err["q"] <= POSE_TOL, err
    dev.close()
