"""Triangle-mesh colliders (RBPS_SHAPE_MESH) against the reference
(MeshCollision.hpp, TriangleUtils.hpp, RBC_PLANE_SPEC(Mesh)), FP64
bit-exact:

* rbps_batch_collide of seeded sphere / capsule / box / plane / mesh poses
  against a closed mesh (a quickhull of points on an ellipsoid) and an open
  grid mesh, both argument orders, and shapes without a mesh routine
  (ellipsoid, heightmap) finding no contact, as in the reference;
* a world of spheres, boxes and capsules falling onto a static bumpy mesh:
  SAP pairs identical every step for 40 steps, state after step 1 exact.
"""
import zlib

import numpy as np
import pytest

import rbps_b200
from rbps_b200 import abi, scenes
from helpers import state_err, bit_equal
import narrow_cases as NC

pytestmark = pytest.mark.gpu


def _closed_mesh():
    rng = np.random.default_rng(17)
    d = rng.standard_normal((40, 3))
    pts = d / np.linalg.norm(d, axis=1, keepdims=True) * np.array([0.8, 0.5, 0.6])
    return pts, rbps_b200.quickhull(pts)


@pytest.fixture(scope="module")
def meshes(rbps, ref):
    spec = scenes.mesh_world(seed=3, n=0)
    spec.meshes = [_closed_mesh(), spec.meshes[0]]
    b = rbps.Batch(1, 1.0 / 60.0, 1, precision=abi.PRECISION_FP64)
    b.add_world(0, spec)
    b.commit()
    rw = ref.RefWorld(spec, 1.0 / 60.0, 1)
    yield b, rw
    b.close()


def _same(g, r):
    if int(g["status"]) != int(r["status"]) or int(g["n_points"]) != int(r["n_points"]):
        return False
    if int(g["status"]) != abi.COLLIDE_HIT:
        return True
    k = int(g["n_points"])
    return (np.array_equal(g["normal"], r["normal"]) and np.array_equal(g["position"][:k], r["position"][:k])
            and np.array_equal(g["depth"][:k], r["depth"][:k]))


def _mesh(mesh_id):
    return (abi.SHAPE_MESH, (0, 0, 0, 0), mesh_id)


@pytest.mark.parametrize("mesh_id", [0, 1], ids=["closed", "grid"])
@pytest.mark.parametrize("kind", ["sphere", "capsule", "box", "plane", "mesh", "ellipsoid"])
def test_shape_vs_mesh(meshes, kind, mesh_id):
    b, rw = meshes
    rng = np.random.default_rng(zlib.crc32(f"{kind}{mesh_id}".encode()))
    n = 600 if kind == "mesh" else 1500
    if kind == "plane":
        shapes = [NC.plane(*(lambda v: (*(v / np.linalg.norm(v)), 0.0))(rng.normal(size=3))) for _ in range(n)]
    elif kind == "mesh":
        shapes = [_mesh(0) for _ in range(n)]
    else:
        shapes = [NC.random_shape(rng, kind) for _ in range(n)]
    sa = NC.descs(shapes)
    sb = NC.descs([_mesh(mesh_id)] * n)
    q = NC.random_quats(rng, n)
    spread = (1.2, 1.0, 1.2) if mesh_id == 0 else (5.0, 1.0, 5.0)
    x = rng.uniform(-np.array(spread), np.array(spread), (n, 3))
    ta = np.concatenate([x, q], 1)
    qb = NC.random_quats(rng, n) if mesh_id == 0 else np.tile([1.0, 0, 0, 0], (n, 1))
    tb = np.concatenate([rng.uniform(-0.2, 0.2, (n, 3)), qb], 1)
    for A, TA, B, TB in ((sa, ta, sb, tb), (sb, tb, sa, ta)):
        g, r = b.collide(A, TA, B, TB), rw.collide(A, TA, B, TB)
        bad = [i for i in range(n) if not _same(g[i], r[i])]
        assert not bad, f"{len(bad)} differ; first {bad[0]}: device {g[bad[0]]} oracle {r[bad[0]]}"
        hits = int((r["status"] == abi.COLLIDE_HIT).sum())
        if kind == "ellipsoid":
            assert hits == 0
        elif kind != "mesh":
            assert hits > 50, hits


def test_mesh_world_live_oracle(rbps, ref):
    spec = scenes.mesh_world(seed=5, n=24)
    sc = scenes.Scene("mesh", 1.0 / 60.0, 10, 40, [spec])
    w = ref.RefWorld(spec, sc.timestep, sc.substeps)
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)
    b.set_dump(True)
    saw_mesh = False
    for step in range(1, 41):
        w.step(1)
        b.step(1)
        np.testing.assert_array_equal(b.pairs(0), w.pairs(), err_msg=f"step {step}")
        if step == 1:
            err = state_err(b.state(0), w.state())
            assert max(err.values()) <= 1e-12, err
        c = w.contacts()
        saw_mesh = saw_mesh or bool((c["collider_a"] == 0).any() or (c["collider_b"] == 0).any())
    assert saw_mesh
    st, rs = b.state(0), w.state()
    assert bit_equal(st, rs) or max(state_err(st, rs).values()) <= 1e-6


def test_fp32_mesh_world_runs(rbps, ref):
    """The FP32 colored engine on the bumpy-mesh world: finite, and one step
    within 1e-4 of the FP64 oracle (the step before any body lands)."""
    spec = scenes.mesh_world(seed=5, n=24)
    sc = scenes.Scene("mesh", 1.0 / 60.0, 10, 60, [spec])
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
