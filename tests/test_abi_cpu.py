"""The C-ABI boundary, checked without a GPU.

* librbps_b200.so loads and exports every function include/rbps_gpu.h
  declares, and the Python binding binds exactly those;
* the numpy mirrors of the descriptor structs have the C layout (a probe
  compiled from the header with the host C compiler prints sizeof/offsetof);
* the descriptor defaults equal the reference's parameter defaults
  (BodyParams{}, ColliderParams{}, *JointParams{}, World{},
  BroadPhaseConfig{}), read from the oracle;
* argument errors come back as RBPS_ERR_INVALID with a message, before any
  device work;
* the host convex-hull builder (rbps_quickhull) returns closed, outward,
  counter-clockwise hulls.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import rbps_b200
from rbps_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rbps_gpu.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"RBPS_API\s+[\w\s\*]+?\b(rbps_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(rbps_b200.LIB_PATH):
        from rbps_b200 import build
        build.build()
    return rbps_b200.lib()


def test_header_declares_the_boundary():
    names = header_functions()
    for required in ("rbps_batch_create", "rbps_world_add_body", "rbps_world_add_collider", "rbps_world_add_joint",
                     "rbps_batch_commit", "rbps_batch_step", "rbps_batch_get_state", "rbps_batch_set_state",
                     "rbps_batch_get_pairs", "rbps_batch_get_contacts", "rbps_batch_get_stats",
                     "rbps_batch_destroy", "rbps_last_error", "rbps_batch_collide", "rbps_bp_update"):
        assert required in names
    assert len(names) >= 45


def test_library_exports_every_header_symbol(lib):
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_header(lib):
    bound = {n for n in header_functions() if getattr(lib, n).argtypes is not None}
    # the *_default helpers and single-item adds are bound lazily; everything
    # the Python classes call must carry a signature
    unbound = set(header_functions()) - bound - {"rbps_body_desc_default", "rbps_collider_desc_default",
                                                 "rbps_joint_desc_default", "rbps_world_set_body_force"}
    assert not unbound, f"no ctypes signature for {sorted(unbound)}"


def test_version_string(lib):
    assert lib.rbps_version().decode().startswith("rbps_b200")


LAYOUT_PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "rbps_gpu.h"
#define F(S, f) printf("%s %s %zu\n", #S, #f, offsetof(S, f));
#define Z(S) printf("%s sizeof %zu\n", #S, sizeof(S));
int main(void) {
  Z(rbps_body_desc) F(rbps_body_desc, type) F(rbps_body_desc, mass) F(rbps_body_desc, inertia)
  F(rbps_body_desc, position) F(rbps_body_desc, orientation) F(rbps_body_desc, linear_velocity)
  F(rbps_body_desc, angular_velocity)
  Z(rbps_collider_desc) F(rbps_collider_desc, shape) F(rbps_collider_desc, params) F(rbps_collider_desc, hull)
  F(rbps_collider_desc, body_id) F(rbps_collider_desc, is_static) F(rbps_collider_desc, local_pos)
  F(rbps_collider_desc, local_rot) F(rbps_collider_desc, restitution) F(rbps_collider_desc, static_friction)
  F(rbps_collider_desc, dynamic_friction)
  Z(rbps_joint_desc) F(rbps_joint_desc, type) F(rbps_joint_desc, body_1) F(rbps_joint_desc, body_2)
  F(rbps_joint_desc, axis) F(rbps_joint_desc, limit_axis) F(rbps_joint_desc, r_1) F(rbps_joint_desc, r_2)
  F(rbps_joint_desc, actuation) F(rbps_joint_desc, compliance) F(rbps_joint_desc, damping)
  F(rbps_joint_desc, limited) F(rbps_joint_desc, lower_limit) F(rbps_joint_desc, upper_limit)
  F(rbps_joint_desc, target_position) F(rbps_joint_desc, target_speed)
  Z(rbps_contact) F(rbps_contact, body_a) F(rbps_contact, body_b) F(rbps_contact, collider_a)
  F(rbps_contact, collider_b) F(rbps_contact, normal) F(rbps_contact, r_a_local) F(rbps_contact, r_b_local)
  F(rbps_contact, point_on_a) F(rbps_contact, point_on_b) F(rbps_contact, penetration_depth)
  F(rbps_contact, normal_lambda) F(rbps_contact, tangent_lambda) F(rbps_contact, relative_velocity)
  F(rbps_contact, restitution) F(rbps_contact, static_friction) F(rbps_contact, dynamic_friction)
  F(rbps_contact, collision) F(rbps_contact, pad_)
  Z(rbps_manifold) F(rbps_manifold, status) F(rbps_manifold, n_points) F(rbps_manifold, normal)
  F(rbps_manifold, position) F(rbps_manifold, depth)
  return 0;
}
"""


def test_struct_layout_matches_numpy_mirrors(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(LAYOUT_PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    seen = set()
    for line in filter(None, out):
        struct, field, value = line.split()
        dt = abi.DTYPES[struct]
        if field == "sizeof":
            assert dt.itemsize == int(value) == abi.STRUCT_SIZES[struct], struct
        else:
            assert dt.fields[field][1] == int(value), f"{struct}.{field}"
            seen.add((struct, field))
    for struct, dt in abi.DTYPES.items():
        assert {(struct, f) for f in dt.names} <= seen, f"probe misses a field of {struct}"


def _c_default(lib, fn, dtype, *extra):
    rec = np.zeros(1, dtype)
    getattr(lib, fn).argtypes = [C.c_void_p] + [C.c_int32] * len(extra)
    getattr(lib, fn).restype = None
    getattr(lib, fn)(C.c_void_p(rec.ctypes.data), *extra)
    return rec[0]


def _assert_records_equal(a, b):
    for name in a.dtype.names:
        np.testing.assert_array_equal(a[name], b[name], err_msg=name)


def test_defaults_match_reference_params(lib, ref):
    body, coll, rev, pri, fix, world = ref.default_descs()
    _assert_records_equal(_c_default(lib, "rbps_body_desc_default", abi.BODY_DT), body)
    _assert_records_equal(_c_default(lib, "rbps_collider_desc_default", abi.COLLIDER_DT), coll)
    _assert_records_equal(_c_default(lib, "rbps_joint_desc_default", abi.JOINT_DT, abi.JOINT_REVOLUTE), rev)
    _assert_records_equal(_c_default(lib, "rbps_joint_desc_default", abi.JOINT_DT, abi.JOINT_PRISMATIC), pri)
    _assert_records_equal(_c_default(lib, "rbps_joint_desc_default", abi.JOINT_DT, abi.JOINT_FIXED), fix)
    # the Python mirrors agree too
    _assert_records_equal(abi.body_default(), body)
    _assert_records_equal(abi.collider_default(), coll)
    _assert_records_equal(abi.joint_default(abi.JOINT_REVOLUTE), rev)
    _assert_records_equal(abi.joint_default(abi.JOINT_FIXED), fix)
    d = rbps_b200.BatchDesc()
    lib.rbps_batch_desc_default(C.byref(d))
    assert (d.timestep, d.substeps, d.fat_margin, d.reinsert_threshold) == tuple(world)


def _last_error(lib):
    buf = C.create_string_buffer(512)
    lib.rbps_last_error(buf, 512)
    return buf.value.decode()


def test_invalid_arguments_rejected_before_device_work(lib):
    d = rbps_b200.BatchDesc()
    lib.rbps_batch_desc_default(C.byref(d))
    h = C.c_void_p()
    for field, bad in (("n_worlds", 0), ("substeps", 0), ("timestep", -1.0), ("precision", 7),
                       ("solve_mode", 3), ("block_threads", 100)):
        e = rbps_b200.BatchDesc()
        C.memmove(C.byref(e), C.byref(d), C.sizeof(d))
        setattr(e, field, bad)
        assert lib.rbps_batch_create(C.byref(e), C.byref(h)) == abi.ERR_INVALID, field
        assert "rbps_batch_create" in _last_error(lib)
    assert lib.rbps_batch_create(None, C.byref(h)) == abi.ERR_INVALID
    assert lib.rbps_batch_step(None, 1) == abi.ERR_INVALID
    assert lib.rbps_batch_commit(None) == abi.ERR_INVALID
    assert lib.rbps_batch_destroy(None) in (abi.OK, abi.ERR_INVALID)
    assert lib.rbps_sap_pairs_static(None, None, 9000, None, 0, None, None) == abi.ERR_INVALID


def test_no_device_is_a_cuda_error(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    d = rbps_b200.BatchDesc()
    lib.rbps_batch_desc_default(C.byref(d))
    h = C.c_void_p()
    assert lib.rbps_batch_create(C.byref(d), C.byref(h)) == abi.ERR_CUDA
    assert "no CUDA device" in _last_error(lib)


def _hull_ok(points, tris):
    pts = np.asarray(points, np.float64)
    v = sorted(set(tris.ravel().tolist()))
    # closed 2-manifold: every directed edge appears once and its reverse once
    edges = {}
    for a, b, c in tris:
        for e in ((a, b), (b, c), (c, a)):
            assert e not in edges
            edges[e] = True
    assert all((b, a) in edges for (a, b) in edges)
    assert len(v) - len(edges) // 2 + len(tris) == 2  # Euler characteristic
    centroid = pts[v].mean(axis=0)
    scale = np.abs(pts).max()
    for a, b, c in tris:
        n = np.cross(pts[b] - pts[a], pts[c] - pts[a])
        assert np.dot(n, pts[a] - centroid) > 0  # counter-clockwise seen from outside
        nn = n / np.linalg.norm(n)
        assert ((pts - pts[a]) @ nn <= 1e-9 * scale + 1e-12).all()  # every point inside or on the face plane


@pytest.mark.parametrize("seed", range(6))
def test_quickhull_random_clouds(lib, seed):
    rng = np.random.default_rng(seed)
    n = [4, 8, 16, 32, 64, 200][seed]
    if seed % 2:
        d = rng.normal(size=(n, 3))
        pts = d / np.linalg.norm(d, axis=1, keepdims=True) * rng.uniform(0.2, 1.0, 3)  # on an ellipsoid
    else:
        pts = rng.uniform(-1, 1, (n, 3))
    tris = rbps_b200.quickhull(pts)
    assert len(tris) >= 4
    _hull_ok(pts, tris)


def test_quickhull_cube_with_interior_points(lib):
    corners = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float64)
    inner = np.random.default_rng(3).uniform(-0.9, 0.9, (50, 3))
    tris = rbps_b200.quickhull(np.vstack([corners, inner]))
    assert set(tris.ravel().tolist()) == set(range(8))
    _hull_ok(np.vstack([corners, inner]), tris)


def test_quickhull_rejects_degenerate(lib):
    flat = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0.5, 0.5, 0]], np.float64)
    with pytest.raises(rbps_b200.RbpsError):
        rbps_b200.quickhull(flat)
