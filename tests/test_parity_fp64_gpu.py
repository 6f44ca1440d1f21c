"""FP64 reference-order GPU engine against the reference engine.

The FP64 instantiation keeps the reference's operation order and runs
without FMA contraction, so on the same inputs it must reproduce the
reference: the SAP pair list bit for bit (order included), the ContactList
and the body state to 1e-12 relative (bit-exact in practice), and the
one-step state within the 1e-5 relative gate in every case.
"""
import numpy as np
import pytest

from rbps_b200 import abi, scenes
from helpers import golden_names, load_golden, state_err, bit_equal

pytestmark = pytest.mark.gpu

ONE_STEP_TOL = 1e-5     # gate: one-step state error vs the FP64 reference
EXACT_TOL = 1e-12       # FP64 restatement: round-off only


def _batch(rbps, sc):
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)
    b.set_dump(True)
    return b


@pytest.mark.parametrize("name", ["chain13_seed3", "boxsphere64_settled"])
def test_sap_state_matches_reference(rbps, ref, name):
    """Persistent SAP state (fat AABBs, endpoint order and values) bit-equal
    to the reference BroadPhaseState after commit and after each step."""
    sc, _ = load_golden(name)
    b = _batch(rbps, sc)
    w = ref.RefWorld(sc.worlds[0], sc.timestep, sc.substeps)
    for step in range(4):
        fat, ids, vals = b.sap_state(0)
        rfat, rids, rvals = w.sap_state()
        np.testing.assert_array_equal(fat, rfat, err_msg=f"fat, step {step}")
        np.testing.assert_array_equal(vals, rvals, err_msg=f"values, step {step}")
        if step:  # before the first sort the GPU keeps insertion order too
            np.testing.assert_array_equal(ids, rids, err_msg=f"endpoint order, step {step}")
        b.step(1)
        w.step(1)


@pytest.mark.parametrize("name", golden_names())
def test_golden_step1(rbps, name):
    sc, g = load_golden(name)
    b = _batch(rbps, sc)
    b.step(1)
    st = b.state(0)
    ref1 = {k: g["s1_" + k] for k in ("position", "orientation", "linear_velocity", "angular_velocity")}
    err = state_err(st, ref1)
    assert max(err.values()) <= EXACT_TOL, err
    # SAP pairs: identical list, identical order
    np.testing.assert_array_equal(b.pairs(0), g["s1_pairs"])
    # ContactList of the last substep
    c, rc = b.contacts(0), g["s1_contacts"]
    assert len(c) == len(rc)
    for f in ("body_a", "body_b", "collider_a", "collider_b", "collision"):
        np.testing.assert_array_equal(c[f], rc[f], err_msg=f)
    for f in ("normal", "r_a_local", "r_b_local", "point_on_a", "point_on_b", "penetration_depth",
              "normal_lambda", "tangent_lambda", "relative_velocity", "restitution", "static_friction",
              "dynamic_friction"):
        np.testing.assert_allclose(c[f], rc[f], rtol=EXACT_TOL, atol=EXACT_TOL, err_msg=f)


@pytest.mark.parametrize("name", golden_names())
def test_golden_step10(rbps, name):
    sc, g = load_golden(name)
    b = _batch(rbps, sc)
    b.step(10)
    st = b.state(0)
    ref10 = {k: g["s10_" + k] for k in ("position", "orientation", "linear_velocity", "angular_velocity")}
    err = state_err(st, ref10)
    assert max(err["position"], err["orientation"]) <= ONE_STEP_TOL, err
    np.testing.assert_array_equal(b.pairs(0), g["s10_pairs"])


def test_config0_live_oracle(rbps, ref):
    """Config 0 as specified (512 boxes + spheres over a plane, FP64, dt
    1/60, 10 substeps, 600 steps): the pair list identical to the live
    reference's every step for all 600 steps, the state after step 1 within
    the gate and the state bit-identical at every 50th step."""
    sc = scenes.config0(seed=0, steps=600)
    w_ref = ref.RefWorld(sc.worlds[0], sc.timestep, sc.substeps)
    b = _batch(rbps, sc)
    for step in range(1, 601):
        w_ref.step(1)
        b.step(1)
        np.testing.assert_array_equal(b.pairs(0), w_ref.pairs(), err_msg=f"step {step}")
        if step == 1:
            err = state_err(b.state(0), w_ref.state())
            assert max(err.values()) <= ONE_STEP_TOL, err
        if step % 50 == 0:
            st, rs = b.state(0), w_ref.state()
            assert bit_equal(st, rs), f"step {step}: {state_err(st, rs)}"


def test_hull_world_live_oracle(rbps, ref):
    """Convex hulls, boxes and spheres falling onto a plane (FP64, reference
    order): hull-vs-anything pairs go through the device GJK / EPA /
    manifold pass.  Pair lists identical every step for 40 steps; state after
    step 1 within the gate; hull contacts do occur."""
    spec = scenes.hull_world(seed=4, n=24)
    sc = scenes.Scene("hulls", 1.0 / 60.0, 10, 40, [spec])
    w_ref = ref.RefWorld(spec, sc.timestep, sc.substeps)
    b = _batch(rbps, sc)
    hull_colliders = set(np.nonzero(spec.colliders["shape"] == abi.SHAPE_CONVEX_HULL)[0].tolist())
    saw_hull_pair = False
    for step in range(1, 41):
        w_ref.step(1)
        b.step(1)
        np.testing.assert_array_equal(b.pairs(0), w_ref.pairs(), err_msg=f"step {step}")
        if step == 1:
            err = state_err(b.state(0), w_ref.state())
            assert max(err.values()) <= ONE_STEP_TOL, err
        c = w_ref.contacts()
        saw_hull_pair = saw_hull_pair or any(
            0 not in (int(x), int(y)) and (int(x) in hull_colliders or int(y) in hull_colliders)
            for x, y in zip(c["collider_a"], c["collider_b"]))
    assert saw_hull_pair, "the scene must produce hull contacts that are not hull-vs-plane"
    st, rs = b.state(0), w_ref.state()
    assert bit_equal(st, rs) or max(state_err(st, rs).values()) <= 1e-6


def test_round_world_live_oracle(rbps, ref):
    """Ellipsoids, cylinders, cones, boxes and spheres falling onto a plane
    (FP64, reference order): their plane routines (PlaneCollision.hpp:40-61,
    416-536) and GJK / EPA pairs on the device.  Pair lists identical every
    step for 40 steps, state after step 1 within the exact gate, and contacts
    between round shapes occur."""
    spec = scenes.round_world(seed=8, n=24)
    sc = scenes.Scene("round", 1.0 / 60.0, 10, 40, [spec])
    w_ref = ref.RefWorld(spec, sc.timestep, sc.substeps)
    b = _batch(rbps, sc)
    rounds = set(np.nonzero(np.isin(spec.colliders["shape"], (abi.SHAPE_ELLIPSOID, abi.SHAPE_CYLINDER,
                                                               abi.SHAPE_CONE)))[0].tolist())
    saw_round_pair = False
    for step in range(1, 41):
        w_ref.step(1)
        b.step(1)
        np.testing.assert_array_equal(b.pairs(0), w_ref.pairs(), err_msg=f"step {step}")
        if step == 1:
            err = state_err(b.state(0), w_ref.state())
            assert max(err.values()) <= EXACT_TOL, err
        c = w_ref.contacts()
        saw_round_pair = saw_round_pair or any(
            0 not in (int(x), int(y)) and (int(x) in rounds or int(y) in rounds)
            for x, y in zip(c["collider_a"], c["collider_b"]))
    assert saw_round_pair, "the scene must produce contacts between round shapes"
    st, rs = b.state(0), w_ref.state()
    assert bit_equal(st, rs) or max(state_err(st, rs).values()) <= 1e-6
