"""The allocation-free SAP query (rbps_sap_pairs_static) against the
allocating GPU broadphase (rbps_bp_*) and the reference's own broadphase,
called through the C ABI.

rbps_sap_pairs_static is for callers that cannot allocate device memory while
running; it works out of a static device array shared by all calls.  The
tests make calls in a row on different inputs (a later call must not see an
earlier one's leftovers) and require the pair lists, emission order
included, to equal what the allocating broadphase and the reference return
for the same fat AABBs.  Integer output: exact equality.  They also cover
the edge returns: zero objects, a pair buffer smaller than the pair count,
more pairs than the array holds (0xFFFFFFFF, pairs left unwritten), and
that a call allocates no device memory.  This file is collected last so a
failure here never hides the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OVERFLOW = 0xFFFFFFFF


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


class _Static:
    """Device buffers for one query, made before any call so that the calls
    themselves run with no allocation by anyone."""

    def __init__(self, fat, ids, pair_cap, fill=0):
        import torch
        dev = torch.device("cuda", 0)
        n = len(ids)
        self.n_objects = n
        self.pair_cap = pair_cap
        fat = np.ascontiguousarray(fat, np.float64).reshape(n, 6) if n else np.zeros((1, 6))
        ids = np.ascontiguousarray(ids, np.uint32) if n else np.zeros(1, np.uint32)
        self.fat = torch.from_numpy(fat).to(dev)
        self.ids = torch.from_numpy(ids.view(np.int32)).to(dev)
        self.pairs = torch.full((max(2 * pair_cap, 2),), fill, dtype=torch.int32, device=dev)
        self.n = torch.zeros(1, dtype=torch.int32, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def call(self, rbps):
        rc = rbps.lib().rbps_sap_pairs_static(self.fat.data_ptr(), self.ids.data_ptr(), self.n_objects,
                                              self.pairs.data_ptr(), self.pair_cap, self.n.data_ptr(),
                                              C.c_void_p(self.stream.cuda_stream))
        assert rc == 0
        self.stream.synchronize()
        return int(self.n.cpu().numpy().view(np.uint32)[0])

    def pair_list(self, n):
        return self.pairs.cpu().numpy().view(np.uint32).reshape(-1, 2)[:min(n, self.pair_cap)]


def _static(rbps, fat, ids, pair_cap):
    q = _Static(fat, ids, pair_cap)
    n = q.call(rbps)
    return q.pair_list(n), n


def test_static_matches_allocating_two_calls(rbps):
    first = _scene(7, 3000, 30.0)
    second = _scene(8, 1200, 12.0)  # fewer objects, denser: leftovers of call 1 must not leak
    for tight, ids in (first, second):
        want, fat = _allocating(rbps, tight, ids)
        got, n = _static(rbps, fat, ids, pair_cap=65536)
        assert n == len(want) and n > 0
        np.testing.assert_array_equal(got, want)


def test_static_matches_reference_broadphase(rbps, ref):
    """The reference's own SAP (BroadPhase.cpp, compiled unmodified) fills
    its fat AABBs from the tight ones; the static query on those fat AABBs
    must emit the reference's pair list, order included."""
    for seed, n, spread in ((11, 2500, 25.0), (12, 700, 6.0)):
        tight, ids = _scene(seed, n, spread)
        bp = ref.RefBroadPhase()
        handles = [bp.insert(int(u), t) for u, t in zip(ids, tight)]
        bp.update()
        want = bp.pairs()
        fat = np.stack([bp.fat_aabb(h) for h in handles])
        got, cnt = _static(rbps, fat, ids, pair_cap=65536)
        assert cnt == len(want) and cnt > 0
        np.testing.assert_array_equal(got, want)


def test_static_zero_objects(rbps):
    q = _Static(np.zeros((0, 6)), np.zeros(0, np.uint32), 16, fill=-7)
    q.n.fill_(123)
    assert q.call(rbps) == 0
    assert (q.pairs.cpu().numpy() == -7).all()


def test_static_pair_cap_smaller_than_pairs(rbps):
    """With room for fewer pairs than found, the count is the full count and
    the buffer holds the first pair_cap pairs of the emission order."""
    tight, ids = _scene(9, 3000, 30.0)
    want, fat = _allocating(rbps, tight, ids)
    assert len(want) > 100
    q = _Static(fat, ids, 100)
    n = q.call(rbps)
    assert n == len(want)
    np.testing.assert_array_equal(q.pair_list(n), want[:100])


def test_static_overflow_sentinel(rbps):
    """400 boxes over one another give 79,800 pairs, more than the static
    array's 65,536: the count is 0xFFFFFFFF and the pairs are left
    unwritten; the next call on ordinary input is correct again."""
    n = 400
    tight = np.tile(np.array([[-1.0, -1.0, -1.0, 1.0, 1.0, 1.0]]), (n, 1))
    ids = np.arange(n, dtype=np.uint32)
    bp = rbps.BroadPhase()
    handles = [bp.insert(int(u), t) for u, t in zip(ids, tight)]
    bp.update()
    fat = np.stack([bp.fat_aabb(h) for h in handles])
    q = _Static(fat, ids, 1024, fill=-7)
    assert q.call(rbps) == OVERFLOW
    assert (q.pairs.cpu().numpy() == -7).all()
    tight2, ids2 = _scene(10, 800, 10.0)
    want, fat2 = _allocating(rbps, tight2, ids2)
    got, cnt = _static(rbps, fat2, ids2, pair_cap=65536)
    assert cnt == len(want)
    np.testing.assert_array_equal(got, want)


def test_static_allocates_nothing(rbps):
    """After a first call (which looks up the array's address), further
    calls leave the device's free memory unchanged."""
    import torch
    tight, ids = _scene(13, 2000, 20.0)
    want, fat = _allocating(rbps, tight, ids)
    q = _Static(fat, ids, 65536)
    assert q.call(rbps) == len(want)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        n = q.call(rbps)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert n == len(want)
    np.testing.assert_array_equal(q.pair_list(n), want)


def test_static_rejects_oversize(rbps):
    rc = rbps.lib().rbps_sap_pairs_static(None, None, 8193, None, 0, C.c_void_p(1), None)
    assert rc == rbps.abi.ERR_INVALID
