"""The algebra behind the frame's one-CTA SAP fast paths, on the CPU.

- Endpoint sort as a merge: when the endpoints that did not move (R) are
  still in key order, merging them with the moved ones (M, ranked by key,
  then previous position) gives the stable sort of the whole array -- the
  order the reference's insertion sort leaves (BroadPhase.cpp:80-94).
- Sweep without a pair sort: grouping the hits (i, j) by the later opening
  position j and ranking each group by i gives the order of a stable sort
  of the pairs emitted per i by j (BroadPhase.cpp:104-152).

These restate the index arithmetic of merge_moved_endpoints and
sweep_staged in numpy and compare them with the plain definitions on random
arrays rich in ties; the device code is compared with the reference itself
by tests/test_sap_paths_gpu.py.
"""
import numpy as np
import pytest


def merge_moved(keys, moved):
    """Final position of each previous position, by the merge."""
    n = len(keys)
    m_idx = np.nonzero(moved)[0]
    r_idx = np.nonzero(~moved)[0]
    rk, mk = keys[r_idx], keys[m_idx]
    if np.any(rk[1:] < rk[:-1]):
        return None  # R out of order: the device falls back to the radix sort
    # rank of each moved endpoint among the moved ones by (key, position)
    rank = np.array([np.sum((mk < mk[u]) | ((mk == mk[u]) & (np.arange(len(mk)) < u))) for u in range(len(mk))],
                    dtype=np.int64)
    final = np.empty(n, np.int64)
    smk = np.empty(len(mk), keys.dtype)
    smp = np.empty(len(mk), np.int64)
    smk[rank] = mk
    smp[rank] = m_idx
    for u, p in enumerate(m_idx):  # + R entries before (key, p)
        final[p] = rank[u] + np.sum((rk < mk[u]) | ((rk == mk[u]) & (r_idx < p)))
    for r, p in enumerate(r_idx):  # + M entries before (key, p)
        final[p] = r + np.sum((smk < rk[r]) | ((smk == rk[r]) & (smp < p)))
    return final


@pytest.mark.parametrize("seed", range(40))
def test_merge_equals_stable_sort(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 200))
    keys = np.sort(rng.integers(0, 40, n))           # last frame's sorted keys (ties)
    moved = rng.random(n) < rng.choice([0.0, 0.05, 0.3, 1.0])
    keys = keys.copy()
    keys[moved] = rng.integers(0, 40, int(moved.sum()))  # the update rewrites the moved keys
    final = merge_moved(keys, moved)
    assert final is not None  # R keeps its order: its keys were sorted and unchanged
    order = np.argsort(keys, kind="stable")          # previous order breaks ties
    expect = np.empty(n, np.int64)
    expect[order] = np.arange(n)
    np.testing.assert_array_equal(final, expect)


def test_merge_refuses_unsorted_rest():
    keys = np.array([3, 1, 2, 5])
    assert merge_moved(keys, np.zeros(4, bool)) is None


def grouped_pairs(hits):
    """Hits (i, j) in any order -> the device's final order: groups by j
    (scan of the per-j counts), each ranked by i."""
    hits = list(hits)
    js = np.array([j for _, j in hits], np.int64)
    nep = int(js.max()) + 1 if len(hits) else 0
    hist = np.bincount(js, minlength=nep)
    first = np.concatenate([[0], np.cumsum(hist)[:-1]]) if nep else np.zeros(0, np.int64)
    out = [None] * len(hits)
    for i, j in hits:
        r = sum(1 for i2, j2 in hits if j2 == j and i2 < i)
        out[first[j] + r] = (i, j)
    return out


@pytest.mark.parametrize("seed", range(40))
def test_grouping_equals_sorted_emission(seed):
    rng = np.random.default_rng(100 + seed)
    nep = int(rng.integers(4, 120))
    # emission by opening endpoint i, each i's partners j > i ascending
    emitted = []
    for i in range(nep):
        js = np.nonzero(rng.random(nep - i - 1) < 0.15)[0] + i + 1
        emitted += [(i, int(j)) for j in js]
    if not emitted:
        return
    expect = [emitted[k] for k in np.argsort([j for _, j in emitted], kind="stable")]
    shuffled = [emitted[k] for k in rng.permutation(len(emitted))]  # the atomic slots' arbitrary order
    assert grouped_pairs(shuffled) == expect
