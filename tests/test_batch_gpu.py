"""Batched worlds: every world of a batch evolves exactly as it does stepped
alone (device single-world path and the oracle), bit for bit."""
import numpy as np
import pytest

from nativeengine_b200 import DeviceWorld, scenes
from nativeengine_b200.bodies import concat

WORLDS = [
    lambda: scenes.small_gas(n=40, seed=3),                                   # brute force (n < 64)
    lambda: scenes.gas(n=300, half=8.0, seed=5),                              # periodic grid
    lambda: scenes.mixed_shapes(n=120, seed=17),                              # periodic, all shapes
    lambda: scenes.box_pile(4, 4, 4, seed=9),                                 # open, all-pairs grid
    lambda: scenes.mixed_shapes(n=90, periodic=False, with_plane=True, gravity=(0, -9.81, 0), seed=23),
    lambda: scenes.small_gas(n=70, periodic=False, seed=8),                   # reflective grid
]


def _split(state, begin, k):
    return {key: v[begin[k]:begin[k + 1]] for key, v in state.items()}


@pytest.mark.gpu
def test_batch_worlds_match_single_worlds(oracle_cls):
    made = [m() for m in WORLDS]
    params = [p for p, _ in made]
    bodies, begin = concat([b for _, b in made])
    dev = DeviceWorld(params[0], None)
    dev.upload_batch(params, bodies, begin)
    singles = [DeviceWorld(p, b.copy()) for p, b in made]
    oracles = [oracle_cls(p, b.copy()) for p, b in made]
    for step in range(4):
        dev.step(1)
        bs = dev.state()
        bp = dev.pairs()
        for k, (sw, ow) in enumerate(zip(singles, oracles)):
            sw.step(1)
            ow.step(1)
            ss, os_ = sw.state(), ow.state()
            part = _split(bs, begin, k)
            for key in ("x", "q", "v", "w"):
                assert np.array_equal(part[key], ss[key]), f"world {k} step {step}: {key} differs from single"
                assert np.array_equal(part[key], os_[key]), f"world {k} step {step}: {key} differs from oracle"
            sel = (bp[:, 0] >= begin[k]) & (bp[:, 0] < begin[k + 1])
            assert np.array_equal(bp[sel] - begin[k], sw.pairs()), f"world {k} step {step}: pairs"
            assert np.all(bp[sel][:, 1] < begin[k + 1]), "a pair crosses worlds"
