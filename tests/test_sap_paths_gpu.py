"""The one-CTA SAP paths of the frame against the live reference (FP64,
reference order), on worlds built to reach each branch:

- the single-pass sweep with its hits staged in shared memory, and its
  fallback (a pile dense enough that the hits exceed the staging lists);
- the endpoint sort as a merge of the moved endpoints, and its fallback to
  the full radix sort (every object fast enough to leave its fat box every
  step, so more endpoints move than the merge takes).

Each must leave the reference's pair list, order included, every step.
"""
import numpy as np
import pytest

from rbps_b200 import abi, scenes
from helpers import bit_equal, state_err

pytestmark = pytest.mark.gpu

MERGE_MAX = 512  # moved endpoints the merge takes


def stage_cap(n_objects):
    """Staging-list entries of the sweep: what the frame's 9,280-word
    staging area leaves after two words per endpoint, halved."""
    return (9280 - 4 * n_objects) // 2


def _world(seed, n, lo, hi, speed=0.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    bodies, forces, colliders = scenes.box_sphere_world(rng, n, lo=lo, hi=hi)
    spec = scenes._finish(bodies, forces, colliders, [])
    if speed:
        dyn = spec.bodies["type"] == abi.BODY_DYNAMIC
        spec.bodies["linear_velocity"][dyn] = rng.uniform(-speed, speed, (int(dyn.sum()), 3))
    return spec


def _run(rbps, ref, spec, steps):
    sc = scenes.Scene("sap_paths", 1.0 / 60.0, 4, steps, [spec])
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER, max_pairs_per_world=65536)
    b.set_dump(True)
    w = ref.RefWorld(spec, sc.timestep, sc.substeps)
    counts = []
    for step in range(1, steps + 1):
        b.step(1)
        w.step(1)
        rp = w.pairs()
        np.testing.assert_array_equal(b.pairs(0), rp, err_msg=f"step {step}")
        counts.append(len(rp))
    st, rs = b.state(0), w.state()
    assert bit_equal(st, rs) or max(state_err(st, rs).values()) <= 1e-9
    return counts


def test_dense_pile_exceeds_the_staging_lists(rbps, ref):
    """700 bodies packed into 6 x 5 x 6 m: 6,000 to 17,000 pairs a step,
    more than the staging lists hold, so the sweep falls back to the global
    emit and sort."""
    counts = _run(rbps, ref, _world(11, 700, (-3.0, 0.5, -3.0), (3.0, 5.5, 3.0)), 6)
    assert max(counts) > stage_cap(700), counts


def test_moderate_pile_stays_staged(rbps, ref):
    """300 bodies in an 8 x 5 x 8 m box: 1,100 to 2,300 pairs a step, which
    fit the staging lists."""
    counts = _run(rbps, ref, _world(12, 300, (-4.0, 0.5, -4.0), (4.0, 5.5, 4.0)), 6)
    assert 0 < max(counts) <= stage_cap(300), counts


def test_fast_bodies_exceed_the_merge(rbps, ref):
    """300 bodies at up to 20 m/s: every fat box is left every step, 600+
    endpoints move, and the sort falls back from the merge to the radix
    sort."""
    spec = _world(13, 300, (-20.0, 1.0, -20.0), (20.0, 30.0, 20.0), speed=20.0)
    assert 2 * 300 > MERGE_MAX
    _run(rbps, ref, spec, 6)


def test_slow_bodies_merge(rbps, ref):
    """The same bodies at rest high above the plane: a few endpoints move a
    step, and the merge places them."""
    _run(rbps, ref, _world(13, 300, (-20.0, 1.0, -20.0), (20.0, 30.0, 20.0)), 6)
