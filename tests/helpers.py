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


def _qrot(q, v):
    w, u = q[:, :1], q[:, 1:]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def joint_gaps(spec, st):
    """(attachment gap in m, swing angle between the bodies' `axis` in
    degrees) of every joint of a world spec in state st."""
    J, q, x = spec.joints, st["orientation"], st["position"]
    b1, b2 = J["body_1"], J["body_2"]
    p1 = x[b1] + _qrot(q[b1], J["r_1"])
    p2 = x[b2] + _qrot(q[b2], J["r_2"])
    a1 = _qrot(q[b1], J["axis"])
    a2 = _qrot(q[b2], J["axis"])
    ang = np.degrees(np.arccos(np.clip((a1 * a2).sum(1), -1.0, 1.0)))
    return np.linalg.norm(p1 - p2, axis=1), ang
