"""The launch-shape autotuner (rbps_batch_autotune): it times its candidate
configurations on the batch's own worlds from one device snapshot, keeps the
fastest and rewinds.  The state after the call equals the state before it,
and because a configuration only changes launch shapes, stepping on gives
the same bits as an untuned twin batch."""
import numpy as np
import pytest

from rbps_b200 import abi, scenes

pytestmark = pytest.mark.gpu

FIELDS = ("position", "orientation", "linear_velocity", "angular_velocity")


def test_autotune_keeps_state_and_results(rbps):
    sc = scenes.config3(seed=9, n_worlds=96, lo_bodies=8, hi_bodies=300)
    tuned = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    plain = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    for b in (tuned, plain):
        b.step(10)
    before = tuned.state_all(FIELDS)
    r = tuned.autotune(trial_steps=2)
    assert r["trials"] >= 2 and r["frame_block"] in (128, 256) and r["narrow_grid"] >= 1
    assert r["narrow_per_warp"] in (32, 64, 128, 256) and r["color_chunk"] in (64, 128, 256)
    assert r["ms_per_step"] <= r["ms_per_step_default"]
    after = tuned.state_all(FIELDS)
    for k in FIELDS:
        np.testing.assert_array_equal(after[k], before[k], err_msg=k)
    for b in (tuned, plain):
        b.step(6)
    a, p = tuned.state_all(FIELDS), plain.state_all(FIELDS)
    for k in FIELDS:
        np.testing.assert_array_equal(a[k], p[k], err_msg=k)


@pytest.mark.parametrize("cfg", [dict(narrow_per_warp=256, color_chunk=32, team_bodies=64, frame_block=128),
                                 dict(narrow_per_warp=64, color_chunk=128, team_bodies=192, narrow_grid=37),
                                 dict(team_bodies=400, pair_bodies=16),
                                 dict(team_bodies=128, pair_bodies=128)])
def test_launch_shape_does_not_change_results(rbps, cfg):
    """Every knob of the autotuner, set by hand away from its default: the
    same bits as a batch at the defaults."""
    sc = scenes.config3(seed=4, n_worlds=80, lo_bodies=8, hi_bodies=300)
    a = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    p = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    a.set_launch(**cfg)
    for b in (a, p):
        b.step(12)
    x, y = a.state_all(FIELDS), p.state_all(FIELDS)
    for k in FIELDS:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)


def test_set_launch_rejects_bad_shapes(rbps):
    sc = scenes.config3(seed=4, n_worlds=4, lo_bodies=8, hi_bodies=40)
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    for bad in (dict(frame_block=96), dict(narrow_per_warp=48), dict(color_chunk=512)):
        with pytest.raises(rbps.RbpsError) as ei:
            b.set_launch(**bad)
        assert ei.value.code == abi.ERR_INVALID
