"""The allocation-free SAP query (rbps_sap_pairs_static) against the
allocating GPU broadphase (rbps_bp_*), called through the C ABI.

rbps_sap_pairs_static is for callers that cannot allocate device memory while
running; it works out of a static device array shared by all calls.  The test
makes two calls in a row on different inputs (the second must not see the
first's leftovers) and requires the pair lists, emission order included, to
equal what the allocating broadphase returns for the same fat AABBs.  Integer
output: exact equality.  This file is collected last so a failure here never
hides the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(seed, n, spread):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 3))
    h = rng.uniform(0.2, 1.5, (n, 1))
    return np.concatenate([c - h, c + h], 1), rng.permutation(10 * n)[:n].astype(np.uint32)


def _allocating(rbps, tight, ids):
    bp = rbps.BroadPhase()
    handles = [bp.insert(int(u), t) for u, t in zip(ids, tight)]
    bp.update()
    fat = np.stack([bp.fat_aabb(h) for h in handles])
    return bp.pairs(), fat


def _static(rbps, fat, ids, pair_cap):
    import torch
    dev = torch.device("cuda", 0)
    d_fat = torch.from_numpy(np.ascontiguousarray(fat)).to(dev)
    d_ids = torch.from_numpy(ids.view(np.int32)).to(dev)
    d_pairs = torch.zeros(2 * pair_cap, dtype=torch.int32, device=dev)
    d_n = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = rbps.lib().rbps_sap_pairs_static(d_fat.data_ptr(), d_ids.data_ptr(), len(ids), d_pairs.data_ptr(),
                                          pair_cap, d_n.data_ptr(), C.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    n = int(d_n.cpu().numpy().view(np.uint32)[0])
    return d_pairs.cpu().numpy().view(np.uint32).reshape(-1, 2)[:min(n, pair_cap)], n


def test_static_matches_allocating_two_calls(rbps):
    first = _scene(7, 3000, 30.0)
    second = _scene(8, 1200, 12.0)  # fewer objects, denser: leftovers of call 1 must not leak
    for tight, ids in (first, second):
        want, fat = _allocating(rbps, tight, ids)
        got, n = _static(rbps, fat, ids, pair_cap=65536)
        assert n == len(want) and n > 0
        np.testing.assert_array_equal(got, want)


def test_static_rejects_oversize(rbps):
    rc = rbps.lib().rbps_sap_pairs_static(None, None, 8193, None, 0, C.c_void_p(1), None)
    assert rc == rbps.abi.ERR_INVALID
