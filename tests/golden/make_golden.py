"""Generates the golden fixtures in tests/golden/ from the reference engine
(oracle/_ref/librbps_ref.so, built from the reference's own sources by
oracle/Makefile).

    python tests/golden/make_golden.py

Each fixture is an .npz holding the scene arrays, the reference state after
1 and 10 steps, the SAP pairs and the ContactList of step 1.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from rbps_b200 import scenes  # noqa: E402
from oracle import ref  # noqa: E402

def settled(factory, dt, sub, steps):
    """The scene after `steps` reference steps, as a fresh scene: bodies start
    at the reference's poses and velocities (many resting contacts)."""
    spec = factory()
    w = ref.RefWorld(spec, dt, sub)
    w.step(steps)
    st = w.state()
    b = spec.bodies.copy()
    b["position"] = st["position"]
    b["orientation"] = st["orientation"]
    b["linear_velocity"] = st["linear_velocity"]
    b["angular_velocity"] = st["angular_velocity"]
    return scenes.WorldSpec(b, spec.forces, spec.colliders, spec.joints, spec.hulls)


CASES = {
    # name: (world factory, timestep, substeps)
    "boxsphere64_seed1": (lambda: scenes.small_world(seed=1, n=64), 1.0 / 60.0, 10),
    "capsules32_seed2": (lambda: scenes.capsule_world(seed=2, n=32), 1.0 / 60.0, 10),
    "chain13_seed3": (lambda: scenes.chain_world(seed=3, n_bodies=12), 1.0 / 120.0, 4),
    "boxsphere64_settled": (lambda: settled(lambda: scenes.small_world(seed=1, n=64), 1.0 / 60.0, 10, 150),
                            1.0 / 60.0, 10),
    "capsules32_settled": (lambda: settled(lambda: scenes.capsule_world(seed=2, n=32), 1.0 / 60.0, 10, 120),
                           1.0 / 60.0, 10),
    "chain13_settled": (lambda: settled(lambda: scenes.chain_world(seed=3, n_bodies=12), 1.0 / 120.0, 4, 300),
                        1.0 / 120.0, 4),
}


def record(name, factory, dt, sub):
    spec = factory()
    w = ref.RefWorld(spec, dt, sub)
    out = {"bodies": spec.bodies, "forces": spec.forces, "colliders": spec.colliders, "joints": spec.joints,
           "timestep": dt, "substeps": sub}
    w.step(1)
    s1 = w.state()
    out.update({f"s1_{k}": v for k, v in s1.items()})
    out["s1_pairs"] = w.pairs()
    c = w.contacts()
    out["s1_contacts"] = c
    w.step(9)
    s10 = w.state()
    out.update({f"s10_{k}": v for k, v in s10.items()})
    out["s10_pairs"] = w.pairs()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "bodies", len(spec.bodies), "pairs@1", len(out["s1_pairs"]), "contacts@1", len(c),
          "pairs@10", len(out["s10_pairs"]))


if __name__ == "__main__":
    for name, (f, dt, sub) in CASES.items():
        record(name, f, dt, sub)
