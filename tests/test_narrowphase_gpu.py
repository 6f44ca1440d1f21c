"""Narrowphase parity: the device rbc::dispatch (rbps_batch_collide) against
the oracle (the reference's own rbc::dispatch, Dispatcher.hpp:208-213).

* the reference's analytic test cases (tests/rbc/analytic/*.cpp), FP64:
  manifold bit-identical to the oracle, and the reference test's own
  assertion holds;
* collide(A, B) against collide(B, A) for the reference's symmetry tests;
* seeded pose sweeps of every analytic shape pairing, FP64 bit-identical;
  FP32 within a stated tolerance where both engines agree on the contact
  feature.
"""
import zlib

import numpy as np
import pytest

from rbps_b200 import abi, scenes

import narrow_cases as NC

pytestmark = pytest.mark.gpu


def _world_with_hulls():
    """An empty world holding the fixture hulls (ids as narrow_cases.HULL_IDS)."""
    b = np.zeros(1, abi.BODY_DT)
    b[0] = abi.body_default()
    b[0]["type"] = abi.BODY_STATIC
    c = np.zeros(1, abi.COLLIDER_DT)
    c[0] = abi.collider_default()
    c[0]["shape"] = abi.SHAPE_PLANE
    c[0]["params"] = (0, 1, 0, 0)
    c[0]["is_static"] = 1
    return scenes.WorldSpec(b, np.zeros((1, 3)), c, np.zeros(0, abi.JOINT_DT), NC.hull_list())


@pytest.fixture(scope="module")
def engines(rbps, ref):
    spec = _world_with_hulls()
    out = {}
    for prec in (abi.PRECISION_FP64, abi.PRECISION_FP32):
        bt = rbps.Batch(1, 1.0 / 60.0, 1, precision=prec)
        bt.add_world(0, spec)
        bt.commit()
        out[prec] = bt
    rw = ref.RefWorld(spec, 1.0 / 60.0, 1)
    yield out, rw
    for bt in out.values():
        bt.close()


def _run(engines, prec, sa, ta, sb, tb):
    batches, rw = engines
    return batches[prec].collide(sa, ta, sb, tb), rw.collide(sa, ta, sb, tb)


def _same(g, r):
    """Bit-identical manifolds (status, count, normal, points, depths)."""
    if int(g["status"]) != int(r["status"]) or int(g["n_points"]) != int(r["n_points"]):
        return False
    if int(g["status"]) != abi.COLLIDE_HIT:
        return True
    k = int(g["n_points"])
    return (np.array_equal(g["normal"], r["normal"]) and np.array_equal(g["position"][:k], r["position"][:k])
            and np.array_equal(g["depth"][:k], r["depth"][:k]))


def _check_expectation(m, exp, ta):
    hit = int(m["status"]) == abi.COLLIDE_HIT
    assert hit == exp["hit"]
    if not hit:
        return
    k = int(m["n_points"])
    if "depth" in exp:
        v, tol = exp["depth"]
        assert abs(m["depth"][0] - v) <= tol
    if exp.get("depth_positive"):
        assert m["depth"][0] > 0
        assert all(m["depth"][i] > 0 for i in range(k))
    if "n_points" in exp:
        assert k == exp["n_points"]
    if "all_depths" in exp:
        v, tol = exp["all_depths"]
        assert all(abs(m["depth"][i] - v) <= tol for i in range(k))
    if "normal" in exp:
        ax, v, tol = exp["normal"][:3]
        got = m["normal"][ax] if len(exp["normal"]) > 3 else abs(m["normal"][ax])
        assert abs(got - v) <= tol
    if "max_depth_from_verts" in exp:
        name, tol = exp["max_depth_from_verts"]
        verts = NC.HULLS[name][0]
        q = ta[3:]
        wy = np.array([NC.rotate(q, v)[1] + ta[1] for v in verts])
        assert abs(max(m["depth"][:k]) - max(0.0, -wy.min())) <= tol
    assert abs(np.linalg.norm(m["normal"]) - 1.0) < 1e-9


@pytest.mark.parametrize("case", NC.REF_CASES, ids=[c[0] for c in NC.REF_CASES])
def test_reference_analytic_case(engines, case):
    name, where, a, ta, b, tb, exp = case
    sa, sb = NC.descs([a]), NC.descs([b])
    g, r = _run(engines, abi.PRECISION_FP64, sa, np.array([ta]), sb, np.array([tb]))
    assert _same(g[0], r[0]), f"{name} ({where}): device {g[0]} vs oracle {r[0]}"
    _check_expectation(g[0], exp, np.array(ta))


@pytest.mark.parametrize("case", NC.SYMMETRY_CASES, ids=[c[0] for c in NC.SYMMETRY_CASES])
def test_reference_symmetry_case(engines, case):
    name, where, a, ta, b, tb = case
    sa, sb = NC.descs([a, b]), NC.descs([b, a])
    tfa, tfb = np.array([ta, tb]), np.array([tb, ta])
    g, r = _run(engines, abi.PRECISION_FP64, sa, tfa, sb, tfb)
    for i in range(2):
        assert _same(g[i], r[i]), f"{name} ({where}) order {i}"
    assert abs(g[0]["depth"][0] - g[1]["depth"][0]) <= 1e-3
    assert np.allclose(g[0]["normal"], -g[1]["normal"], atol=1e-3)


PAIRINGS = [(a, b) for i, a in enumerate(NC.ANALYTIC_KINDS) for b in NC.ANALYTIC_KINDS[i:]]
PAIRINGS += [(b, a) for (a, b) in PAIRINGS if a != b]
PAIRINGS += [(a, "plane") for a in NC.ANALYTIC_KINDS] + [("hull", "plane")]
# GJK / EPA / manifold pairs (no analytic routine): hull against everything
PAIRINGS += [("hull", k) for k in NC.ANALYTIC_KINDS] + [(k, "hull") for k in NC.ANALYTIC_KINDS] + [("hull", "hull")]


# ellipsoid / cylinder / cone: their plane routines, and GJK / EPA (one EPA
# point, ContactManifoldGenerator.cpp:405-412) against every convex shape
ROUND_PAIRINGS = [(k, "plane") for k in NC.ROUND_KINDS]
ROUND_PAIRINGS += [(k, m) for k in NC.ROUND_KINDS for m in NC.ANALYTIC_KINDS + NC.ROUND_KINDS + ("hull",)]
ROUND_PAIRINGS += [(m, k) for k in NC.ROUND_KINDS for m in NC.ANALYTIC_KINDS + ("hull",)]


@pytest.mark.parametrize("pairing", PAIRINGS + ROUND_PAIRINGS,
                         ids=[f"{a}-{b}" for a, b in PAIRINGS + ROUND_PAIRINGS])
def test_random_poses_fp64_bit_exact(engines, pairing):
    ka, kb = pairing
    sa, ta, sb, tb = NC.random_pairs(zlib.crc32(f"{ka}-{kb}".encode()), ka, kb, 2000)
    g, r = _run(engines, abi.PRECISION_FP64, sa, ta, sb, tb)
    hits = int((r["status"] == abi.COLLIDE_HIT).sum())
    assert hits > 100, "sweep should produce contacts"
    bad = [i for i in range(len(g)) if not _same(g[i], r[i])]
    assert not bad, f"{len(bad)} of {len(g)} differ; first {bad[0]}: device {g[bad[0]]} oracle {r[bad[0]]}"
    if pairing == ("hull", "hull"):
        # clipped polygon manifolds (ContactManifoldGenerator.cpp:176-379) occur
        assert int((g["n_points"] >= 2).sum()) > 50


@pytest.mark.parametrize("pairing", PAIRINGS, ids=[f"{a}-{b}" for a, b in PAIRINGS])
def test_random_poses_fp32(engines, pairing):
    """FP32 device arithmetic against the FP64 oracle.  Where both report a
    contact with the same point count and normals within 2e-3:
      * the deepest depth agrees to 2e-4 m (GJK pairs: within the 3 % below);
      * the point sets agree to 2e-4 m + 1.5 m x |normal difference| (a
        point sits up to a shape size, <= 0.6 m, along the normal from a
        centre, and near-coincident centres amplify the FP32 error of the
        normal), except that at most 3 % of the pairs may keep a different
        subset of clip points (the 4-point reduction breaks near-ties
        differently in FP32);
    hit/miss may differ only for grazing contacts (depth < 1e-3 m)."""
    ka, kb = pairing
    sa, ta, sb, tb = NC.random_pairs(zlib.crc32(f"{ka}-{kb}".encode()), ka, kb, 2000)
    g, r = _run(engines, abi.PRECISION_FP32, sa, ta, sb, tb)
    # GJK / EPA / clipping run in double in both precisions, but the FP32
    # library compiles them with FMA contraction: a degenerate polytope or
    # clip can then take another path, which the 3 % allowance covers
    gjk_pair = "hull" in pairing and "plane" not in pairing
    same_feature = 0
    other_subset = 0
    for i in range(len(g)):
        gh, rh = int(g[i]["status"]) == 1, int(r[i]["status"]) == 1
        if gh != rh:
            d = (g[i] if gh else r[i])["depth"][0]
            assert d < 1e-3, f"pair {i}: hit/miss differ at depth {d}"
            continue
        if not gh or g[i]["n_points"] != r[i]["n_points"]:
            continue
        dn = np.abs(g[i]["normal"] - r[i]["normal"]).max()
        if dn > 2e-3:
            continue  # a different SAT axis / feature was chosen (near-tie)
        k = int(g[i]["n_points"])
        if k == 0:
            continue  # a hit without points (both engines agree)
        same_feature += 1
        deep_ok = abs(g[i]["depth"][:k].max() - r[i]["depth"][:k].max()) < 2e-4
        if not gjk_pair:
            assert deep_ok, f"pair {i}"
        # point order can differ inside a face clip: compare as sets
        gp = np.sort(g[i]["position"][:k], axis=0)
        rp = np.sort(r[i]["position"][:k], axis=0)
        if not deep_ok or np.abs(gp - rp).max() >= 2e-4 + 1.5 * dn:
            other_subset += 1
    assert same_feature > 0.8 * int((r["status"] == 1).sum())
    assert other_subset <= 0.03 * same_feature, f"{other_subset} of {same_feature} pairs keep other clip points"


def test_hull_pairs_run_gjk(engines):
    """Hull against a non-plane shape runs GJK / EPA / the manifold on the
    device (no RBPS_COLLIDE_UNSUPPORTED) and gives the oracle's bits."""
    sa = NC.descs([NC.hull("cube"), NC.sphere(0.5), NC.hull("ellA"), NC.hull("cube")])
    sb = NC.descs([NC.box(0.5, 0.5, 0.5), NC.hull("tet"), NC.capsule(0.4, 0.2), NC.hull("cube")])
    ta = np.array([NC.tf(0, 0, 0), NC.tf(0, 0, 0), NC.tf(0, 0, 0), NC.tf(0, 0, 0)])
    tb = np.array([NC.tf(1.2, 0, 0), NC.tf(0.5, 0.5, 0), NC.tf(0.3, 0.3, 0.1),
                   NC.tf(0.2, 1.8, 0.1, NC.axis_quat((0, 0, 1), 0.3))])
    g, r = _run(engines, abi.PRECISION_FP64, sa, ta, sb, tb)
    assert abi.COLLIDE_UNSUPPORTED not in list(g["status"])
    assert int((g["status"] == abi.COLLIDE_HIT).sum()) >= 3
    for i in range(len(g)):
        assert _same(g[i], r[i]), f"pair {i}: device {g[i]} oracle {r[i]}"


@pytest.mark.parametrize("pairing", ROUND_PAIRINGS, ids=[f"{a}-{b}" for a, b in ROUND_PAIRINGS])
def test_round_shapes_fp32(engines, pairing):
    """Ellipsoid / cylinder / cone in the FP32 library against the FP64
    oracle: hit/miss may differ only for grazing contacts (depth < 1e-3 m);
    where both hit, the deepest depths agree to 1e-3 m and the normals to
    1e-2 for at least 97 % of the pairs (EPA / GJK run in double, but the
    plane routines and the transforms are float)."""
    ka, kb = pairing
    sa, ta, sb, tb = NC.random_pairs(zlib.crc32(f"{ka}-{kb}".encode()), ka, kb, 2000)
    g, r = _run(engines, abi.PRECISION_FP32, sa, ta, sb, tb)
    both = close = 0
    for i in range(len(g)):
        gh, rh = int(g[i]["status"]) == 1, int(r[i]["status"]) == 1
        if gh != rh:
            d = (g[i] if gh else r[i])["depth"][0]
            assert d < 1e-3, f"pair {i}: hit/miss differ at depth {d}"
            continue
        if not gh or int(g[i]["n_points"]) == 0 or int(r[i]["n_points"]) == 0:
            continue
        both += 1
        kg, kr = int(g[i]["n_points"]), int(r[i]["n_points"])
        dd = abs(g[i]["depth"][:kg].max() - r[i]["depth"][:kr].max())
        dn = np.abs(g[i]["normal"] - r[i]["normal"]).max()
        close += int(dd < 1e-3 and dn < 1e-2)
    assert both > 100
    assert close >= 0.97 * both, f"{close} of {both}"
