"""The oracle's ball joint (RBPS_JOINT_SPHERICAL), checked without a GPU.

The reference has no ball joint, so the oracle restates one on the
reference's rows (oracle/ref_harness.cpp, SphJoint) and no reference test
pins it.  These tests pin its behaviour instead: a pendulum keeps its
attachment, the swing cone pulls a link that starts outside it back to the
cone and leaves one inside it alone, and hanging chains stay together.
"""
import numpy as np
import pytest

from rbps_b200 import scenes
from helpers import joint_gaps


def _run(ref, sc, steps):
    w = ref.RefWorld(sc.worlds[0], sc.timestep, sc.substeps)
    out = []
    for _ in range(steps):
        w.step(1)
        out.append(joint_gaps(sc.worlds[0], w.state()))
    return out


def test_pendulum_keeps_attachment(ref):
    sc = scenes.config2(seed=2, n_chains=1, n_links=1, max_angle_deg=20.0)
    for gap, ang in _run(ref, sc, 120):
        assert gap.max() < 1e-3
        assert ang.max() < 60.0


@pytest.mark.parametrize("limited", [1, 0])
def test_cone_acts_only_outside(ref, limited):
    """A link started 80 degrees off its anchor's axis: with the cone it is
    inside the cone after one step (the correction also sets it swinging
    back, as XPBD derives velocities from the corrected poses); without it,
    it stays near 80 degrees."""
    sc = scenes.config2(seed=2, n_chains=1, n_links=1, max_angle_deg=0.0)
    spec = sc.worlds[0]
    a = np.radians(80.0)
    q = np.array([np.cos(a / 2), np.sin(a / 2), 0.0, 0.0])  # about x
    pivot = np.zeros(3)
    reach = spec.joints["r_2"][0][1]
    w, u = q[0], q[1:]
    up = np.array([0.0, reach, 0.0])
    t = 2.0 * np.cross(u, up)
    spec.bodies["orientation"][1] = q
    spec.bodies["position"][1] = pivot - (up + w * t + np.cross(u, t))
    spec.joints["limited"] = limited
    (gap, ang), = _run(ref, sc, 1)
    # the cone row, solved after the attachment row, turns the link about
    # its centre and opens the attachment until the next substep
    assert gap.max() < (0.02 if limited else 1e-3), gap
    if limited:
        assert ang[0] < 61.0, ang
    else:
        assert ang[0] > 75.0, ang


def test_hanging_chains_stay_together(ref):
    sc = scenes.config2(seed=3, n_chains=4, n_links=12)
    for k, (gap, ang) in enumerate(_run(ref, sc, 60)):
        assert np.isfinite(gap).all(), k
        assert gap.max() < 0.02, (k, gap.max())
        assert np.percentile(ang, 95) < 62.0, (k, np.percentile(ang, 95))
