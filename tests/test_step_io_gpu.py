"""Host I/O entry points: rbps_batch_step_io (returns with the poses on the
host) and rbps_batch_step_io_async (copies on a second stream, overlapping
the neighbouring steps; final after rbps_batch_synchronize) give the same
bits as rbps_batch_step followed by a state read, step after step, with the
forces changed every step."""
import numpy as np
import pytest

from rbps_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _scene():
    return scenes.config3(seed=7, n_worlds=64, lo_bodies=8, hi_bodies=64)


@pytest.mark.parametrize("mode", ["sync", "async"])
def test_step_io_matches_step(rbps, mode):
    sc = _scene()
    ref = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    io = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    n, _ = io.total_bodies()
    f0 = np.ascontiguousarray(np.concatenate([w.forces for w in sc.worlds]))
    outs = []
    for k in range(6):
        f = np.ascontiguousarray(f0 * (1.0 + 0.1 * k))
        pos, rot = np.zeros((n, 3)), np.zeros((n, 4))
        outs.append((f, pos, rot))
        call = io.step_io if mode == "sync" else io.step_io_async
        call(f.ctypes.data, pos.ctypes.data, rot.ctypes.data)
    io.synchronize()
    for k, (f, pos, rot) in enumerate(outs):
        ref.set_forces_all(f)
        ref.step(1)
        st = ref.state_all()
        np.testing.assert_array_equal(pos, st["position"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rot, st["orientation"], err_msg=f"step {k}")
