"""The oracle, pinned without a GPU.

* oracle/_ref (the reference compiled from its own sources) reproduces every
  committed golden fixture bit for bit: states after 1 and 10 steps, SAP
  pairs, the ContactList of step 1;
* oracle/sap.py (the pure-Python restatement of the SAP broadphase) matches
  the compiled reference on the reference's own broadphase test cases
  (tests/rbc/test_broad_phase.cpp) and on random insert / move / swept-move
  / remove sequences: identical pair lists (emission order included) and
  identical fat AABBs.
"""
import numpy as np
import pytest

from helpers import golden_names, load_golden
from oracle import sap

STATE_KEYS = ("position", "orientation", "linear_velocity", "angular_velocity")


@pytest.mark.parametrize("name", golden_names())
def test_oracle_reproduces_golden(ref, name):
    sc, g = load_golden(name)
    w = ref.RefWorld(sc.worlds[0], sc.timestep, sc.substeps)
    w.step(1)
    s1 = w.state()
    for k in STATE_KEYS:
        np.testing.assert_array_equal(s1[k], g["s1_" + k], err_msg=k)
    np.testing.assert_array_equal(w.pairs(), g["s1_pairs"])
    c = w.contacts()
    assert len(c) == len(g["s1_contacts"])
    for f in ("body_a", "body_b", "normal", "point_on_a", "point_on_b", "penetration_depth", "normal_lambda",
              "tangent_lambda"):
        np.testing.assert_array_equal(c[f], g["s1_contacts"][f], err_msg=f)
    w.step(9)
    s10 = w.state()
    for k in STATE_KEYS:
        np.testing.assert_array_equal(s10[k], g["s10_" + k], err_msg=k)
    np.testing.assert_array_equal(w.pairs(), g["s10_pairs"])


def make_aabb(cx, cy, cz, half):
    """make_aabb of test_broad_phase.cpp:16-20 (float arguments)."""
    f = np.float32
    c = [float(f(cx)), float(f(cy)), float(f(cz))]
    h = float(f(half))
    return [c[0] - h, c[1] - h, c[2] - h, c[0] + h, c[1] + h, c[2] + h]


class Both:
    """The restatement and the compiled reference driven in lockstep."""

    def __init__(self, ref):
        self.p = sap.SapBroadPhase()
        self.r = ref.RefBroadPhase()

    def insert(self, uid, a):
        hp, hr = self.p.insert(uid, a), self.r.insert(uid, np.asarray(a, np.float64))
        assert hp == hr
        return hp

    def remove(self, h):
        self.p.remove(h)
        self.r.remove(h)

    def move(self, h, a):
        self.p.move(h, a)
        self.r.move(h, np.asarray(a, np.float64))

    def move_swept(self, h, a, v, dt):
        self.p.move_swept(h, a, v, dt)
        self.r.move_swept(h, np.asarray(a, np.float64), np.asarray(v, np.float64), dt)

    def update(self):
        pp = self.p.update()
        self.r.update()
        rp = [tuple(int(x) for x in row) for row in self.r.pairs()]
        assert pp == rp
        return pp

    def fat_equal(self, h):
        np.testing.assert_array_equal(np.array(self.p.fat_aabb(h)), self.r.fat_aabb(h))


def has_pair(pairs, a, b):
    return (min(a, b), max(a, b)) in pairs


# tests/rbc/test_broad_phase.cpp, one function per reference test
def test_empty_scene_no_pairs(ref):                                       # :34
    assert Both(ref).update() == []


def test_single_object_no_pairs(ref):                                     # :42
    b = Both(ref)
    b.insert(0, make_aabb(0, 0, 0, 1.0))
    assert b.update() == []


def test_two_overlapping_objects_one_pair(ref):                          # :55
    b = Both(ref)
    b.insert(0, make_aabb(0, 0, 0, 1.0))
    b.insert(1, make_aabb(1, 0, 0, 1.0))
    p = b.update()
    assert len(p) == 1 and has_pair(p, 0, 1)


def test_two_separated_objects_no_pair(ref):                             # :69
    b = Both(ref)
    b.insert(0, make_aabb(-5, 0, 0, 1.0))
    b.insert(1, make_aabb(5, 0, 0, 1.0))
    assert b.update() == []


def test_three_objects_only_adjacent_pair(ref):                          # :82
    b = Both(ref)
    b.insert(0, make_aabb(0, 0, 0, 1.0))
    b.insert(1, make_aabb(1, 0, 0, 1.0))
    b.insert(2, make_aabb(20, 0, 0, 1.0))
    p = b.update()
    assert len(p) == 1 and has_pair(p, 0, 1)


def test_all_three_overlapping(ref):                                     # :97
    b = Both(ref)
    b.insert(0, make_aabb(0.0, 0, 0, 2.0))
    b.insert(1, make_aabb(1.0, 0, 0, 2.0))
    b.insert(2, make_aabb(0.5, 0, 0, 2.0))
    p = b.update()
    assert len(p) == 3 and has_pair(p, 0, 1) and has_pair(p, 0, 2) and has_pair(p, 1, 2)


def test_remove_eliminates_pair(ref):                                    # :117
    b = Both(ref)
    b.insert(0, make_aabb(0, 0, 0, 1.0))
    h1 = b.insert(1, make_aabb(1, 0, 0, 1.0))
    assert len(b.update()) == 1
    b.remove(h1)
    assert b.update() == []


def test_handle_slot_reused_after_remove(ref):                           # :133
    b = Both(ref)
    h0 = b.insert(42, make_aabb(0, 0, 0, 1.0))
    b.remove(h0)
    h1 = b.insert(99, make_aabb(0, 0, 0, 1.0))
    assert h1 == h0
    assert b.update() == []


def test_move_into_overlap_creates_pair(ref):                            # :150
    b = Both(ref)
    h0 = b.insert(0, make_aabb(-10, 0, 0, 1.0))
    b.insert(1, make_aabb(10, 0, 0, 1.0))
    assert b.update() == []
    b.move(h0, make_aabb(9.5, 0, 0, 1.0))
    assert has_pair(b.update(), 0, 1)


def test_move_out_of_overlap_removes_pair(ref):                          # :168
    b = Both(ref)
    b.insert(0, make_aabb(0, 0, 0, 1.0))
    h1 = b.insert(1, make_aabb(1, 0, 0, 1.0))
    assert len(b.update()) == 1
    b.move(h1, make_aabb(10, 0, 0, 1.0))
    assert b.update() == []


def test_small_move_keeps_fat_aabb(ref):                                  # :185
    b = Both(ref)
    h = b.insert(0, make_aabb(0, 0, 0, 1.0))
    b.update()
    b.move(h, make_aabb(0.01, 0, 0, 1.0))
    assert not b.p.dirty
    b.fat_equal(h)


def test_large_move_refits_fat_aabb(ref):                                 # :202
    b = Both(ref)
    h = b.insert(0, make_aabb(0, 0, 0, 1.0))
    b.update()
    b.move(h, make_aabb(5.0, 0, 0, 1.0))
    assert b.p.dirty
    b.fat_equal(h)


def test_swept_move_detects_fast_approaching_object(ref):                # :252
    b = Both(ref)
    b.insert(0, make_aabb(5, 0, 0, 1.0))
    hb = b.insert(1, make_aabb(-1, 0, 0, 1.0))
    assert b.update() == []
    b.move_swept(hb, make_aabb(-1, 0, 0, 1.0), (50, 0, 0), 0.1)
    assert has_pair(b.update(), 0, 1)


def test_swept_move_slow_object_no_false_pair(ref):                      # :278
    b = Both(ref)
    b.insert(0, make_aabb(5, 0, 0, 1.0))
    hb = b.insert(1, make_aabb(-1, 0, 0, 1.0))
    b.update()
    b.move_swept(hb, make_aabb(-1, 0, 0, 1.0), (1, 0, 0), 0.016)
    assert b.update() == []


def test_swept_move_velocity_away_no_pair(ref):                          # :301
    b = Both(ref)
    b.insert(0, make_aabb(5, 0, 0, 1.0))
    hb = b.insert(1, make_aabb(-1, 0, 0, 1.0))
    b.update()
    b.move_swept(hb, make_aabb(-1, 0, 0, 1.0), (-50, 0, 0), 0.1)
    assert b.update() == []


def test_swept_zero_velocity_matches_standard_move(ref):                 # :326
    s, m = Both(ref), Both(ref)
    tight = make_aabb(0, 0, 0, 1.0)
    hs, hm = s.insert(0, tight), m.insert(0, tight)
    s.move_swept(hs, tight, (0, 0, 0), 0.016)
    m.move(hm, tight)
    assert s.p.fat_aabb(hs) == m.p.fat_aabb(hm)
    s.fat_equal(hs)
    m.fat_equal(hm)


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_random_sequences(ref, seed):
    """Inserts, removals with slot reuse, plain and swept moves, with float
    key ties (coarse grid positions) and touching boxes."""
    rng = np.random.default_rng(seed)
    b = Both(ref)
    n = 120
    grid = seed % 2 == 0  # coarse positions produce equal endpoint keys
    centers = (np.round(rng.uniform(-6, 6, (n, 3)) * 2) / 2) if grid else rng.uniform(-6, 6, (n, 3))
    halves = np.where(rng.random(n) < 0.5, 0.5, rng.uniform(0.1, 1.0, n))
    live = {}
    uid = 0
    for i in range(n):
        a = list(centers[i] - halves[i]) + list(centers[i] + halves[i])
        live[b.insert(uid, a)] = i
        uid += 1
    b.update()
    for it in range(8):
        for h in rng.choice(sorted(live), size=len(live) // 3, replace=False):
            i = live[h]
            centers[i] += rng.normal(0, 0.05 if it % 2 else 0.6, 3)
            a = list(centers[i] - halves[i]) + list(centers[i] + halves[i])
            if rng.random() < 0.5:
                b.move_swept(h, a, rng.normal(0, 3, 3), 1.0 / 60.0)
            else:
                b.move(h, a)
        for h in rng.choice(sorted(live), size=5, replace=False):
            b.remove(h)
            del live[h]
        for _ in range(4):
            i = int(rng.integers(n))
            a = list(centers[i] - halves[i]) + list(centers[i] + halves[i])
            live[b.insert(uid, a)] = i
            uid += 1
        b.update()
        for h in live:
            b.fat_equal(h)


def _hull_cases():
    import narrow_cases as NC
    import rbps_b200
    rng = np.random.default_rng(11)
    cases = [("tet", NC.TET_VERTS, NC.TET_FACES), ("cube", NC.CUBE_VERTS, NC.CUBE_FACES)]
    for k, n in enumerate((8, 16, 24, 32)):
        d = rng.normal(size=(n, 3))
        pts = d / np.linalg.norm(d, axis=1, keepdims=True) * rng.uniform(0.2, 1.0, 3)
        cases.append((f"ellipsoid{n}", pts, rbps_b200.quickhull(pts)))
    # a box as a point cloud: quickhull splits each face into triangles that must merge back
    corners = np.array([[x, y, z] for x in (-0.3, 0.3) for y in (-0.5, 0.5) for z in (-0.2, 0.2)])
    cases.append(("box_cloud", corners, rbps_b200.quickhull(corners)))
    # a hexagonal prism: faces of 6 vertices
    ang = np.arange(6) * np.pi / 3
    ring = np.stack([np.cos(ang), np.zeros(6), np.sin(ang)], 1)
    prism = np.vstack([ring + [0, -0.4, 0], ring + [0, 0.4, 0]])
    cases.append(("hex_prism", prism, rbps_b200.quickhull(prism)))
    return cases


def test_hull_tables_match_reference(ref):
    """The library's polygon / adjacency tables (the restatement of
    convex_hull_data_create, ConvexHull.hpp:149-420) equal the reference's."""
    import rbps_b200
    from rbps_b200 import abi, scenes
    cases = _hull_cases()
    b = np.zeros(1, abi.BODY_DT)
    b[0] = abi.body_default()
    spec = scenes.WorldSpec(b, np.zeros((1, 3)), np.zeros(0, abi.COLLIDER_DT), np.zeros(0, abi.JOINT_DT),
                            [(v, t) for _, v, t in cases])
    rw = ref.RefWorld(spec, 1 / 60, 1)
    for hid, (name, verts, tris) in enumerate(cases):
        mine = rbps_b200.hull_tables(verts, tris)
        theirs = rw.hull_tables(hid)
        nv = len(verts)
        assert len(theirs["poly_offsets"]) > 1, name
        for key in ("poly_offsets", "poly_indices", "p2p_offsets", "p2p_indices", "v2p_indices", "v2n_indices"):
            np.testing.assert_array_equal(mine[key], theirs[key], err_msg=f"{name}.{key}")
        for key in ("v2p_offsets", "v2n_offsets"):
            np.testing.assert_array_equal(mine[key][:nv + 1], theirs[key][:nv + 1], err_msg=f"{name}.{key}")
        np.testing.assert_array_equal(mine["poly_normals"], theirs["poly_normals"], err_msg=f"{name}.normals")
