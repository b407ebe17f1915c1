"""Shared comparison helpers for the device-vs-oracle parity tests."""
import numpy as np


def assert_same_pairs(dev, ora, what=""):
    a, b = dev.pairs(), ora.pairs()
    assert a.shape == b.shape, f"{what}: pair count {a.shape[0]} != oracle {b.shape[0]}"
    assert np.array_equal(a, b), f"{what}: pair lists differ at {np.argwhere((a != b).any(1))[:5].ravel()}"


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size == 0:
        return 0.0
    scale = np.maximum(np.abs(b), 1.0)
    return float(np.max(np.abs(a - b) / scale))


def assert_same_contacts(dev, ora, tol=0.0, what=""):
    a, b = dev.contacts(), ora.contacts()
    assert a["i"].shape == b["i"].shape, f"{what}: contact count {a['i'].size} != oracle {b['i'].size}"
    assert np.array_equal(a["i"], b["i"]) and np.array_equal(a["j"], b["j"]), f"{what}: contact pairs differ"
    for k in ("point", "normal", "depth", "n_imp"):
        e = rel_err(a[k], b[k])
        assert e <= tol, f"{what}: contact {k} differs (rel err {e:.3e} > {tol})"


def assert_same_state(dev, ora, tol=0.0, what=""):
    a, b = dev.state(), ora.state()
    for k in ("x", "q", "v", "w"):
        e = rel_err(a[k], b[k])
        assert e <= tol, f"{what}: state {k} differs (rel err {e:.3e} > {tol})"


def max_state_err(dev, ora):
    a, b = dev.state(), ora.state()
    return max(rel_err(a[k], b[k]) for k in ("x", "q", "v", "w"))
