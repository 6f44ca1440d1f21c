"""The C++ drop-in rbps_gpu::World (include/rbps_gpu_world.hpp) against the
reference's own rbps::World, through the compiled test program
tests/cpp/test_world_gpu.cpp: every scenario of the reference's
tests/rbps/API/test_world.cpp, plus every collidable shape and the three
joint types, built by the same calls in both worlds and required to agree
bit for bit after every step (FP64, reference order).

The program is built with the oracle (`make -C oracle world_test`, which
needs the reference's headers); where it has not been built the test is
skipped.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_world_gpu")


def test_cpp_world_matches_reference_world():
    if not os.path.exists(BIN):
        pytest.skip("C++ world test not built (make -C oracle world_test)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out
    passed = [ln for ln in out.splitlines() if ln.startswith("PASS ")]
    assert len(passed) == 16, out
