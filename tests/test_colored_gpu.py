"""Colored (graph-coloured Gauss-Seidel) FP32 path.

Colour validity is checked exactly: no two candidates of one colour share a
dynamic body.  Physics is checked against the FP64 reference one step ahead
(tolerance 1e-2 relative: Gauss-Seidel order differs, FP32 arithmetic) and
for plausibility over many steps (finite, resting on the ground).
"""
import numpy as np
import pytest

from rbps_b200 import abi, scenes
from helpers import bit_equal, load_golden, state_err

pytestmark = pytest.mark.gpu


def colour_valid(colors, ba, bb, dynamic):
    seen = {}
    for c, a, b in zip(colors, ba, bb):
        if c >= 64:      # 64 = serial overflow colour, 65 = no contact rows this substep
            continue
        for x in (a, b):
            if dynamic[x]:
                key = (int(c), int(x))
                if key in seen:
                    return False
                seen[key] = True
    return True


@pytest.mark.parametrize("precision", [abi.PRECISION_FP32, abi.PRECISION_FP64])
def test_colouring_is_valid(rbps, precision):
    sc, _ = load_golden("boxsphere64_settled")
    b = rbps.Batch.from_scene(sc, precision, abi.SOLVE_COLORED)
    b.set_dump(True)
    b.step(3)
    col, ba, bb = b.colors(0)
    dyn = sc.worlds[0].bodies["type"] == abi.BODY_DYNAMIC
    assert len(col) > 0
    assert colour_valid(col, ba, bb, dyn)
    assert b.stats()["max_colors"] >= 2
    # only candidates with contact rows are coloured; the rest are idle
    assert set(np.unique(col).tolist()) <= set(range(66))
    n_active = int((col < 65).sum())
    assert 0 < n_active < len(col)
    assert n_active <= len(b.contacts(0))  # every active candidate has >= 1 row


def test_colored_fp32_one_step_close(rbps):
    sc, g = load_golden("boxsphere64_settled")
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    b.step(1)
    ref1 = {k: g["s1_" + k] for k in ("position", "orientation", "linear_velocity", "angular_velocity")}
    err = state_err(b.state(0), ref1)
    assert err["position"] < 1e-2 and err["orientation"] < 1e-2, err


def test_colored_batch_settles(rbps):
    sc = scenes.config3(seed=5, n_worlds=16, steps=240)
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    b.step(240)
    st = b.state_all(("position",))
    assert np.isfinite(st["position"]).all()
    # everything has fallen onto the ground plane (y >= -0.1) and stays low
    assert st["position"][:, 1].min() > -0.2


def test_batches_of_different_sizes_coexist(rbps):
    """Colored batches share the substep kernel's shared-memory limit on a
    device: a batch created after one with larger worlds must not lower it
    (the larger batch's steps would then fail to launch)."""
    big = rbps.Batch.from_scene(scenes.config3(seed=2, n_worlds=8, lo_bodies=300, hi_bodies=512),
                                abi.PRECISION_FP32, abi.SOLVE_COLORED)
    small = rbps.Batch.from_scene(scenes.config3(seed=3, n_worlds=8, lo_bodies=8, hi_bodies=16),
                                  abi.PRECISION_FP32, abi.SOLVE_COLORED)
    big.step(2)
    small.step(2)
    big.step(2)
    for b in (big, small):
        assert np.isfinite(b.state_all()["position"]).all()


def test_large_world_colouring(rbps):
    """Worlds above 4,096 bodies colour by claims on (body, colour) slots,
    many contacts of one body per round.  Tangled chains (scenes.config2,
    196 chains of 32 capsules: 6,468 bodies, up to 25 contacts per body by
    step 28): the colouring is valid, nothing is left to the serial bucket,
    the colour count lies between the largest body degree (a lower bound)
    and twice it, and two batches stepped from the same scene agree bit for
    bit (the colouring is deterministic, and so is relaxing the trailing
    small colours on one CTA)."""
    sc = scenes.config2(seed=0, n_chains=196, n_links=32)
    dyn = sc.worlds[0].bodies["type"] == abi.BODY_DYNAMIC
    runs = []
    for _ in range(2):
        b = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED, max_pairs_per_world=1 << 20)
        b.set_dump(True)
        b.step(28)
        col, ba, bb = b.colors(0)
        st = b.stats()
        runs.append((b.state(0), col))
    assert colour_valid(col, ba, bb, dyn)
    act = col < 64
    a, c = ba[act], bb[act]
    deg = np.bincount(np.concatenate([a[dyn[a]], c[dyn[c]]]))
    assert deg.max() >= 12, deg.max()  # tangled enough to need many colours
    assert st["serial_overflow"] == 0, st
    ncol = int(col[act].max()) + 1
    assert deg.max() <= ncol <= 2 * deg.max(), (ncol, deg.max())
    assert bit_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
