"""Regenerate the golden fixtures from the reference implementation.

Runs the NativeEngine reference, compiled unmodified from its own sources into
oracle/_ref/libneref.so (oracle/Makefile), on small seeded scenes and stores,
per step, the broadphase pair list, the contacts with their converged normal
impulses, the island labels and the body state.  The inputs are stored too, so
the fixtures do not depend on the scene generators staying bit-stable.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from nativeengine_b200 import scenes  # noqa: E402
from nativeengine_b200.bodies import params_dict  # noqa: E402
from oracle.oracle import RefOracle  # noqa: E402

STEPS = 3

SCENES = {
    "gas_periodic_50": lambda: scenes.small_gas(),
    "gas_reflective_50": lambda: scenes.small_gas(periodic=False, seed=5),
    "mixed_periodic_96": lambda: scenes.mixed_shapes(),
    "mixed_plane_reflective_96": lambda: scenes.mixed_shapes(periodic=False, with_plane=True,
                                                             gravity=(0, -9.81, 0), seed=11),
    "box_stack_6": lambda: scenes.box_stack(),
    "box_pile_64": lambda: scenes.box_pile(4, 4, 4),
}

ARRAYS = ("x", "q", "v", "w", "force", "torque", "inv_mass", "inv_inertia", "shape", "radius", "half_height",
          "half_extents", "vert_offset", "vert_count", "verts", "friction", "restitution", "linear_damping",
          "angular_damping", "gravity_scale", "layer", "mask", "flags", "nocollide_offset", "nocollide_count",
          "nocollide")


def main():
    for name, make in SCENES.items():
        params, bodies = make()
        out = {"in_" + k: getattr(bodies, k) for k in ARRAYS}
        out["in_n_verts"] = np.array(bodies.n_verts)
        out["in_n_nocollide"] = np.array(bodies.n_nocollide)
        for k, v in params_dict(params).items():
            out["param_" + k] = np.array(v)
        ora = RefOracle(params, bodies.copy())
        for s in range(STEPS):
            ora.step(1)
            out[f"s{s}_pairs"] = ora.pairs()
            c = ora.contacts()
            for k in ("i", "j", "slot", "point", "normal", "depth", "n_imp"):
                out[f"s{s}_c_{k}"] = c[k]
            out[f"s{s}_islands"] = ora.islands()
            st = ora.state()
            for k in ("x", "q", "v", "w"):
                out[f"s{s}_{k}"] = st[k]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, bodies.n, "bodies", len(out["s0_pairs"]), "pairs")


if __name__ == "__main__":
    main()
