"""GPU SAP broadphase (rbps_bp_*) against the reference rbc broadphase.

Cases follow the reference's own tests (tests/rbc/test_broad_phase.cpp:34-348:
empty / single / overlapping / separated / lifecycle / swept moves) plus
randomised stress with moves, removals and slot reuse; the pair list must
match bit for bit, emission order included.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def box(c, half):
    c = np.asarray(c, np.float64)
    return np.concatenate([c - half, c + half])


# (single CTA, threads): the cooperative grid, and the one-CTA team that the
# batched engine runs each world's broadphase on
TEAMS = [(False, 256), (True, 128), (True, 256), (True, 32)]


@pytest.fixture(params=TEAMS, ids=lambda t: f"{'cta' if t[0] else 'grid'}{t[1]}")
def team(request):
    return request.param


def both(rbps, ref, team=(False, 256)):
    return rbps.BroadPhase(single_cta=team[0], block=team[1]), ref.RefBroadPhase()


def check(g, r):
    g.update()
    r.update()
    np.testing.assert_array_equal(g.pairs(), r.pairs())
    return len(r.pairs())


def test_reference_cases(rbps, ref, team):
    g, r = both(rbps, ref, team)
    assert check(g, r) == 0                                  # empty_scene_no_pairs
    for bp in (g, r):
        bp.insert(0, box((0, 0, 0), 1.0))
    assert check(g, r) == 0                                  # single_object_no_pairs
    for bp in (g, r):
        bp.insert(1, box((1, 0, 0), 1.0))
    assert check(g, r) == 1                                  # two_overlapping_objects_one_pair
    for bp in (g, r):
        bp.insert(2, box((20, 0, 0), 1.0))
    assert check(g, r) == 1                                  # three_objects_only_adjacent_pair
    for bp in (g, r):
        bp.insert(3, box((0.5, 0, 0), 2.0))
    assert check(g, r) == 3
    for bp in (g, r):
        bp.remove(1)                                         # remove_eliminates_pair
    check(g, r)
    for bp in (g, r):
        h = bp.insert(7, box((0.2, 0.1, 0), 0.5))            # slot reuse after remove
    check(g, r)
    for bp in (g, r):
        bp.move(0, box((30, 0, 0), 1.0))                     # move out of range
    check(g, r)
    for bp in (g, r):
        bp.move_swept(0, box((0, 0, 0), 1.0), (3.0, -2.0, 0.5), 1.0 / 60.0)
    check(g, r)
    for h in (0, 2, 3):
        np.testing.assert_array_equal(g.fat_aabb(h), r.fat_aabb(h))


def test_touching_and_signed_zero(rbps, ref, team):
    """Inclusive overlap on touching faces and -0.0 / +0.0 key ties."""
    g, r = both(rbps, ref, team)
    aabbs = [(-0.1, -1, -1, 0.9, 1, 1), (-0.1, -1, -1, 1.1, 1, 1), (1.1, -1, -1, 3.0, 1, 1),
             (-0.2, 0.5, 0.5, -0.1, 2, 2), (-2.0, -1, -1, -0.1, 1, 1)]
    for i, a in enumerate(aabbs):
        for bp in (g, r):
            bp.insert(i, a)
    check(g, r)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_stress(rbps, ref, seed, team):
    rng = np.random.default_rng(seed)
    g, r = both(rbps, ref, team)
    n = 3000
    centers = rng.uniform(-40, 40, (n, 3))
    halves = rng.uniform(0.2, 1.5, n)
    handles = []
    for i in range(n):
        a = box(centers[i], halves[i])
        hg, hr = g.insert(i, a), r.insert(i, a)
        assert hg == hr
        handles.append(hg)
    check(g, r)
    alive = set(handles)
    next_id = n
    for it in range(6):
        for h in rng.choice(sorted(alive), size=len(alive) // 3, replace=False):
            d = rng.normal(0, 0.3 if it % 2 else 2.0, 3)
            centers[h] += d
            a = box(centers[h], halves[h])
            if rng.random() < 0.5:
                v = rng.normal(0, 3, 3)
                g.move_swept(h, a, v, 1 / 60)
                r.move_swept(h, a, v, 1 / 60)
            else:
                g.move(h, a)
                r.move(h, a)
        if it == 2:
            for h in rng.choice(sorted(alive), size=200, replace=False):
                g.remove(h)
                r.remove(h)
                alive.discard(h)
            for k in range(100):
                a = box(rng.uniform(-40, 40, 3), 1.0)
                hg, hr = g.insert(next_id, a), r.insert(next_id, a)
                assert hg == hr
                alive.add(hg)
                centers[hg] = (a[:3] + a[3:]) / 2
                halves[hg] = 1.0
                next_id += 1
        check(g, r)
