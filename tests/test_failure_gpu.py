"""Failure detection on small worlds, with every failure made on the host.

- Pair capacity: a batch whose max_pairs_per_world is far below the pairs
  its worlds produce returns RBPS_ERR_CAPACITY from the next synchronising
  call, without hanging, and stays usable: the error is cleared once
  reported, state reads work, the next step reports it again, and a
  snapshot taken before the overflow restores bit for bit.  The reference
  asserts inside its broadphase instead (BroadPhase.cpp:201,215).
- Non-finite state: a NaN position injected through rbps_batch_set_state
  makes the next step's synchronising call return RBPS_ERR_STATE naming the
  world; the other worlds of the batch step exactly as in a twin batch
  without the NaN; replacing the bad world's state clears the failure; with
  the check off the NaN propagates silently, as in the reference.
"""
import numpy as np
import pytest

from rbps_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _dense_scene(n_worlds=3, n=48, seed=5):
    """Bodies packed into a 2 x 2 x 2 m box: hundreds of SAP pairs each."""
    worlds = []
    for w in range(n_worlds):
        rng = np.random.Generator(np.random.PCG64(seed + w))
        bodies, forces, colliders = scenes.box_sphere_world(rng, n, lo=(-1.0, 1.0, -1.0), hi=(1.0, 3.0, 1.0))
        worlds.append(scenes._finish(bodies, forces, colliders, []))
    return scenes.Scene("dense", 1.0 / 60.0, 4, 10, worlds)


MODES = [(abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER), (abi.PRECISION_FP32, abi.SOLVE_COLORED)]


@pytest.mark.parametrize("prec,solve", MODES)
def test_pair_capacity_overflow_reported_and_recoverable(rbps, prec, solve):
    sc = _dense_scene()
    full = rbps.Batch.from_scene(sc, prec, solve)
    full.set_dump(True)
    full.step(1)
    assert min(len(full.pairs(w)) for w in range(len(sc.worlds))) > 16
    b = rbps.Batch.from_scene(sc, prec, solve, max_pairs_per_world=8)
    snap = b.snapshot()
    st0 = b.state_all(("position", "orientation"))
    b.step(1)
    with pytest.raises(rbps.RbpsError) as ei:
        b.synchronize()
    assert ei.value.code == abi.ERR_CAPACITY
    assert "capacity" in str(ei.value)
    st = b.state(0)  # usable: the error was cleared when it was reported
    assert np.isfinite(st["position"]).all()
    b.step(1)
    with pytest.raises(rbps.RbpsError) as ei:
        b.synchronize()
    assert ei.value.code == abi.ERR_CAPACITY
    b.restore(snap)
    b.synchronize()
    st1 = b.state_all(("position", "orientation"))
    for k in st0:
        np.testing.assert_array_equal(st1[k], st0[k])
    b.close()
    full.close()


@pytest.mark.parametrize("prec,solve", MODES)
def test_nan_state_reported_world_isolated(rbps, prec, solve):
    sc = scenes.Scene("three", 1.0 / 120.0, 4, 10, [scenes.chain_world(seed=s, n_bodies=24) for s in (1, 2, 3)])
    a = rbps.Batch.from_scene(sc, prec, solve)
    twin = rbps.Batch.from_scene(sc, prec, solve)
    a.step(3)
    twin.step(3)
    st = a.state(1)
    st["position"][5, 1] = np.nan
    a.set_state(1, st)
    a.step(1)
    twin.step(1)
    with pytest.raises(rbps.RbpsError) as ei:
        a.synchronize()
    assert ei.value.code == abi.ERR_STATE
    assert "world 1" in str(ei.value)
    # the other worlds are untouched by world 1's NaN
    for w in (0, 2):
        sa, st_ = a.state(w), twin.state(w)
        for k in ("position", "orientation", "linear_velocity", "angular_velocity"):
            np.testing.assert_array_equal(sa[k], st_[k])
    # replacing the bad world's state clears the failure
    a.set_state(1, twin.state(1))
    a.step(2)
    twin.step(2)
    a.synchronize()
    for w in (0, 2):
        np.testing.assert_array_equal(a.state(w)["position"], twin.state(w)["position"])
    # world 1 steps on from the replaced state (its SAP bounds were rebuilt
    # from the NaN pose, so only finiteness is asserted there)
    assert np.isfinite(a.state(1)["position"]).all()
    a.close()
    twin.close()


def test_nan_state_unchecked_propagates(rbps):
    sc = scenes.Scene("one", 1.0 / 120.0, 4, 10, [scenes.small_world(seed=4, n=16)])
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)
    b.set_state_check(False)
    st = b.state(0)
    st["orientation"][3, 0] = np.nan
    b.set_state(0, st)
    b.step(2)
    b.synchronize()  # no error: the reference's behaviour
    assert not np.isfinite(b.state(0)["orientation"]).all()
    b.set_state_check(True)
    b.step(1)
    with pytest.raises(rbps.RbpsError) as ei:
        b.synchronize()
    assert ei.value.code == abi.ERR_STATE
    b.close()
