"""Multi-GPU sharding on one GPU: the worlds of one set split into two parts
by balanced body count (rbps_b200.shard, as bench.py splits them across
ranks) and stepped as two batches give every world exactly the state it
has in the batch of the whole set.  Worlds share nothing, so a rank's
result cannot depend on which other worlds it holds."""
import numpy as np
import pytest

from rbps_b200 import abi, scenes, shard

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,solve", [(abi.PRECISION_FP32, abi.SOLVE_COLORED),
                                        (abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)])
def test_two_parts_equal_the_whole(rbps, prec, solve):
    full = scenes.config3(seed=2, n_worlds=40)
    assert max(w.n_bodies for w in full.worlds) >= 128  # both team kinds of the colored kernel
    whole = rbps.Batch.from_scene(full, prec, solve)
    whole.set_state_check(False)
    whole.step(20)
    want = [whole.state(w) for w in range(len(full.worlds))]
    whole.close()
    for part in range(2):
        sub, idx = shard.shard_scene(full, 2, part)
        b = rbps.Batch.from_scene(sub, prec, solve)
        b.set_state_check(False)
        b.step(20)
        for k, w in enumerate(idx):
            got = b.state(k)
            for f in ("position", "orientation", "linear_velocity", "angular_velocity"):
                np.testing.assert_array_equal(got[f], want[w][f], err_msg=f"part {part} world {w} {f}")
        b.close()
