"""Load a golden fixture (tests/golden/*.npz) as (params, BodyArrays, expected)."""
import os

import numpy as np

from nativeengine_b200 import _ffi
from nativeengine_b200.bodies import BodyArrays

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN_DIR) if f.endswith(".npz"))


def load(name):
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    b = BodyArrays.__new__(BodyArrays)
    for k in z.files:
        if k.startswith("in_"):
            v = z[k]
            setattr(b, k[3:], int(v) if v.ndim == 0 else np.ascontiguousarray(v))
    b.n = int(b.x.shape[0])
    b._c = None
    p = _ffi.NeWorldParams()
    for fname, _ in p._fields_:
        v = z["param_" + fname]
        if fname == "gravity":
            for a in range(3):
                p.gravity[a] = float(v[a])
        else:
            setattr(p, fname, v.item())
    steps = sorted({int(k[1:k.index("_")]) for k in z.files if k.startswith("s") and "_" in k and k[1].isdigit()})
    expected = []
    for s in steps:
        e = {"pairs": z[f"s{s}_pairs"], "islands": z[f"s{s}_islands"]}
        for k in ("i", "j", "slot", "point", "normal", "depth", "n_imp"):
            e["c_" + k] = z[f"s{s}_c_{k}"]
        for k in ("x", "q", "v", "w"):
            e[k] = z[f"s{s}_{k}"]
        expected.append(e)
    return p, b, expected
