"""Shared helpers of the parity tests."""
import glob
import os

import numpy as np

from rbps_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    spec = scenes.WorldSpec(d["bodies"], d["forces"], d["colliders"], d["joints"], [])
    sc = scenes.Scene(name, float(d["timestep"]), int(d["substeps"]), 10, [spec])
    return sc, d


def rel_err(a, b, floor=1.0):
    """max |a-b| / max(|b|, floor) over all entries (NaN-safe: NaN -> inf)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size == 0:
        return 0.0
    e = np.abs(a - b) / np.maximum(np.abs(b), floor)
    e[~np.isfinite(e)] = np.inf
    return float(e.max())


def quat_err(a, b):
    """Relative error of quaternions with the sign ambiguity removed."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.sign(np.sum(a * b, axis=1, keepdims=True))
    s[s == 0] = 1
    return rel_err(a * s, b)


def state_err(st, ref_st):
    return {"position": rel_err(st["position"], ref_st["position"]),
            "orientation": quat_err(st["orientation"], ref_st["orientation"]),
            "linear_velocity": rel_err(st["linear_velocity"], ref_st["linear_velocity"]),
            "angular_velocity": rel_err(st["angular_velocity"], ref_st["angular_velocity"])}


def bit_equal(st, ref_st):
    return all(np.array_equal(np.asarray(st[k]), np.asarray(ref_st[k])) for k in ("position", "orientation"))
