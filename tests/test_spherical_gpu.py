"""Ball joints with a swing cone (RBPS_JOINT_SPHERICAL) on the device
against the oracle's own restatement (oracle/ref_harness.cpp, SphJoint: the
reference has no ball joint, so this parity is unpinned by any reference
test; the restatement reuses the reference's rows, impulse routines and
compute_angle_limit_correction).

* FP64 reference order, hanging capsule chains (scenes.config2 at small
  sizes): the state after every step bit-identical to the oracle's, with
  the initial bends inside the cone (U[-30, 30] degrees) and beyond it
  (U[-75, 75] degrees, so the cone row acts from the first substep).
* FP32, the same chains: in reference order one step within 1e-3 of the
  FP64 oracle (a hanging chain's stiff rows amplify float rounding: about
  1e-4 measured); colored (joints and contacts relaxed colour by colour,
  so the order and the result differ from the oracle's) finite with the
  joints held over 21 steps: attachment gaps below 0.15 m, the 99th
  percentile of the swing angles below 75 degrees (0.078 m and 66.6
  degrees measured; reference order gives 0.060 m and 61.3 degrees).
"""
import numpy as np
import pytest

from rbps_b200 import abi, scenes
from helpers import bit_equal, joint_gaps, state_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("max_angle", [30.0, 75.0])
def test_fp64_chains_match_oracle(rbps, ref, max_angle):
    sc = scenes.config2(seed=5, n_chains=4, n_links=8, max_angle_deg=max_angle)
    spec = sc.worlds[0]
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)
    w = ref.RefWorld(spec, sc.timestep, sc.substeps)
    cone_hit = False
    for step in range(1, 31):
        b.step(1)
        w.step(1)
        st, rs = b.state(0), w.state()
        assert np.isfinite(rs["position"]).all(), f"oracle went non-finite at step {step}"
        assert bit_equal(st, rs), f"step {step}: {state_err(st, rs)}"
        gap, ang = joint_gaps(spec, rs)
        cone_hit = cone_hit or bool((ang > 59.0).any())
    assert gap.max() < 0.02, gap.max()
    if max_angle > 60.0:
        assert cone_hit


def test_fp32_chains(rbps, ref):
    sc = scenes.config2(seed=6, n_chains=16, n_links=16)
    spec = sc.worlds[0]
    w = ref.RefWorld(spec, sc.timestep, sc.substeps)
    w.step(1)
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_REFERENCE_ORDER)
    b.step(1)
    err = state_err(b.state(0), w.state())
    assert max(err["position"], err["orientation"]) <= 1e-3, err
    c = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    c.step(21)
    st = c.state(0)
    for k in st:
        assert np.isfinite(st[k]).all(), k
    gap, ang = joint_gaps(spec, st)
    assert gap.max() < 0.15, gap.max()
    assert np.percentile(ang, 99) < 75.0, np.percentile(ang, 99)
    assert c.stats()["max_colors"] >= 2
