"""Error and drift measures of batched world states (host side, numpy).

These are the per-config error reports of the batched FP32 path against the
FP64 engine (which equals the reference bit for bit): one-step state error,
contact and joint residuals, and energy and momentum drift over N steps.
Trajectories are chaotic, so nothing here compares long horizons point by
point.

States are dicts of per-body arrays as ``Batch.state`` returns them
(position (n, 3), orientation (n, 4) wxyz, linear_velocity (n, 3),
angular_velocity (n, 3)).
"""
import numpy as np

from . import abi

GRAVITY = 9.81


def state_error(a, r):
    """Relative one-step error of state a against reference state r, per
    body: max over the body's position coordinates of |a - r| / max(|r|, 1)
    and over its orientation components (sign-aligned quaternions).
    Returns (n,) float64; non-finite entries give inf."""
    ep = np.abs(a["position"] - r["position"]) / np.maximum(np.abs(r["position"]), 1.0)
    sign = np.where((a["orientation"] * r["orientation"]).sum(1, keepdims=True) < 0, -1.0, 1.0)
    eq = np.abs(a["orientation"] * sign - r["orientation"])
    e = np.maximum(ep.max(1), eq.max(1))
    e[~np.isfinite(e)] = np.inf
    return e


def _qrot(q, v):
    w, u = q[:, :1], q[:, 1:]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def joint_gaps(spec, st):
    """Attachment gap |p1 - p2| in m of every joint of a world (the
    positional error every joint type constrains to zero, Joint.cpp:107-111)."""
    J = spec.joints
    if len(J) == 0:
        return np.zeros(0)
    q, x = st["orientation"], st["position"]
    b1, b2 = J["body_1"].astype(np.int64), J["body_2"].astype(np.int64)
    p1 = x[b1] + _qrot(q[b1], J["r_1"])
    p2 = x[b2] + _qrot(q[b2], J["r_2"])
    return np.linalg.norm(p1 - p2, axis=1)


def world_energy(spec, st, g=GRAVITY):
    """Kinetic + potential energy of a world's dynamic bodies (potential
    measured from the lowest static body, the ground plane's body)."""
    b = spec.bodies
    dyn = b["type"] == abi.BODY_DYNAMIC
    if not dyn.any():
        return 0.0
    x, v, om, q = st["position"], st["linear_velocity"], st["angular_velocity"], st["orientation"]
    m = b["mass"]
    inert = b["inertia"][:, :3]
    # body-frame angular velocity: conj(q) * omega * q
    qc = q.copy()
    qc[:, 1:] *= -1.0
    ob = _qrot(qc, om)
    stat = ~dyn
    y0 = float(x[stat][:, 1].min()) if stat.any() else 0.0
    ke = 0.5 * m * (v * v).sum(1) + 0.5 * (inert * ob * ob).sum(1)
    pe = m * g * (x[:, 1] - y0)
    return float((ke + pe)[dyn].sum())


def world_momentum(spec, st):
    """Total linear momentum of a world's dynamic bodies (3,)."""
    dyn = spec.bodies["type"] == abi.BODY_DYNAMIC
    return (spec.bodies["mass"][dyn, None] * st["linear_velocity"][dyn]).sum(0)


def chain_links(spec):
    """Indices of the bodies that carry a joint."""
    J = spec.joints
    if len(J) == 0:
        return np.zeros(0, np.int64)
    return np.unique(np.concatenate([J["body_1"], J["body_2"]]).astype(np.int64))


def jointed_component(spec, contacts):
    """Bodies connected to any jointed body through joints or through the
    given contacts (rbps_contact records), static bodies excluded from the
    connections: the bodies whose one-step motion the joints can reach."""
    n = len(spec.bodies)
    parent = np.arange(n)

    def find(i):
        while parent[i] != i:
            parent[i] = parent[parent[i]]
            i = parent[i]
        return i

    dyn = spec.bodies["type"] == abi.BODY_DYNAMIC
    edges = [(int(a), int(b)) for a, b in zip(spec.joints["body_1"], spec.joints["body_2"])]
    edges += [(int(a), int(b)) for a, b in zip(contacts["body_a"], contacts["body_b"])]
    for a, b in edges:
        if a < n and b < n and dyn[a] and dyn[b]:
            ra, rb = find(a), find(b)
            if ra != rb:
                parent[ra] = rb
    links = chain_links(spec)
    roots = {find(int(i)) for i in links}
    return np.array([i for i in range(n) if find(i) in roots], np.int64)


def summary(e):
    """Distribution of per-world errors (NaN entries are skipped)."""
    e = np.asarray(e, np.float64)
    g = e[~np.isnan(e)]
    if len(g) == 0:
        return {"worlds": 0}
    return {"worlds": int(len(g)), "median": float(np.median(g)), "p90": float(np.percentile(g, 90)),
            "p99": float(np.percentile(g, 99)), "max": float(g.max()),
            "within_1e-5": int((g <= 1e-5).sum()), "fraction_within_1e-5": float((g <= 1e-5).mean())}


def perturb_ulp(st, seed=0):
    """The state rounded to float32 with every position and orientation
    coordinate then moved by one float32 ulp up or down (seeded random
    signs): the smallest change a float state can carry, to measure how
    strongly one step amplifies it."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = dict(st)
    for k in ("position", "orientation"):
        f = np.asarray(st[k], np.float32)
        to = np.where(rng.random(f.shape) < 0.5, np.float32(np.inf), np.float32(-np.inf))
        out[k] = np.nextafter(f, to.astype(np.float32)).astype(np.float64)
    return out
