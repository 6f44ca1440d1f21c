"""Device scan and stable radix sort (the primitives every step phase uses)
against numpy, on one CTA and on a cooperative grid, for ragged sizes."""
import numpy as np
import pytest

import rbps_b200

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 2, 31, 32, 33, 127, 128, 129, 1000, 4097, 70000]
TEAMS = [(False, 32), (False, 128), (False, 256), (True, 128), (True, 256)]


@pytest.mark.parametrize("grid,block", TEAMS)
@pytest.mark.parametrize("n", SIZES)
def test_scan(rbps, grid, block, n):
    rng = np.random.default_rng(n)
    v = rng.integers(0, 50, n).astype(np.uint32)
    out, tot = rbps_b200.selftest_scan(v, grid, block)
    exp = np.concatenate([[0], np.cumsum(v, dtype=np.uint64)[:-1]]).astype(np.uint32) if n else v
    np.testing.assert_array_equal(out, exp)
    assert tot == int(v.sum())


@pytest.mark.parametrize("grid,block", TEAMS)
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("bits", [7, 11, 32])
def test_stable_sort(rbps, grid, block, n, bits):
    rng = np.random.default_rng(1000 + n)
    keys = rng.integers(0, 2 ** min(bits, 31), n).astype(np.uint32)
    if bits < 32:
        keys &= np.uint32((1 << bits) - 1)
    else:
        keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 4] = keys[0] if n else 0  # many ties
    ko, vo = rbps_b200.selftest_sort(keys, bits, grid, block)
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(vo, order)
    np.testing.assert_array_equal(ko, keys[order])
