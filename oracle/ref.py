"""ctypes binding of the oracle: the unmodified reference engine built from
its own sources into oracle/_ref/librbps_ref.so (see oracle/Makefile).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product never imports it.
"""
import ctypes as C
import os

import numpy as np

from rbps_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "librbps_ref.so")
_lib = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_U = C.POINTER(C.c_uint32)


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
        L = C.CDLL(LIB_PATH)
        L.ref_world_create.restype = _P
        L.ref_world_create.argtypes = [C.c_double, C.c_int, C.c_double, C.c_double]
        L.ref_world_destroy.argtypes = [_P]
        L.ref_hull_create.restype = C.c_uint32
        L.ref_hull_create.argtypes = [_P, _D, C.c_uint32, _U, C.c_uint32]
        L.ref_mesh_create.restype = C.c_uint32
        L.ref_mesh_create.argtypes = [_P, _D, C.c_uint32, _U, C.c_uint32]
        L.ref_heightmap_create.restype = C.c_uint32
        L.ref_heightmap_create.argtypes = [_P, C.POINTER(C.c_float), C.c_uint32, C.c_uint32, _D, _D]
        L.ref_add_body.restype = C.c_uint32
        L.ref_add_body.argtypes = [_P, _P]
        L.ref_set_body_force.argtypes = [_P, C.c_uint32, _D, _D]
        L.ref_add_collider.restype = C.c_uint32
        L.ref_add_collider.argtypes = [_P, _P]
        L.ref_add_joint.restype = C.c_uint32
        L.ref_add_joint.argtypes = [_P, _P]
        L.ref_collide.restype = C.c_int
        L.ref_collide.argtypes = [_P, C.c_uint32, _P, _D, _P, _D, _P]
        L.ref_default_descs.argtypes = [_P, _P, _P, _P, _P, _D]
        L.ref_hull_tables.restype = C.c_int
        L.ref_hull_tables.argtypes = [_P, C.c_uint32, C.c_uint32, _U, _U, _U, _D, _U, _U, _U, _U, _U, _U]
        L.ref_step.argtypes = [_P, C.c_int]
        L.ref_body_count.restype = C.c_uint32
        L.ref_body_count.argtypes = [_P]
        L.ref_get_state.argtypes = [_P, _D, _D, _D, _D]
        L.ref_set_state.argtypes = [_P, _D, _D, _D, _D]
        L.ref_get_pairs.restype = C.c_uint32
        L.ref_get_pairs.argtypes = [_P, _U, C.c_uint32]
        L.ref_get_contacts.restype = C.c_uint32
        L.ref_get_contacts.argtypes = [_P, _P, C.c_uint32]
        L.ref_get_sap_state.restype = C.c_uint32
        L.ref_get_sap_state.argtypes = [_P, _D, _U, C.POINTER(C.c_float)]
        L.ref_collision_groups.restype = C.c_uint32
        L.ref_collision_groups.argtypes = [_P, _U, C.c_uint32]
        L.ref_step_worlds.restype = C.c_double
        L.ref_step_worlds.argtypes = [C.POINTER(_P), C.c_uint32, C.c_int, C.c_int]
        L.ref_bp_create.restype = _P
        L.ref_bp_create.argtypes = [C.c_double, C.c_double]
        L.ref_bp_destroy.argtypes = [_P]
        L.ref_bp_insert.restype = C.c_uint32
        L.ref_bp_insert.argtypes = [_P, C.c_uint32, _D]
        L.ref_bp_remove.argtypes = [_P, C.c_uint32]
        L.ref_bp_move.argtypes = [_P, C.c_uint32, _D]
        L.ref_bp_move_swept.argtypes = [_P, C.c_uint32, _D, _D, C.c_double]
        L.ref_bp_update.argtypes = [_P]
        L.ref_bp_get_pairs.restype = C.c_uint32
        L.ref_bp_get_pairs.argtypes = [_P, _U, C.c_uint32]
        L.ref_bp_get_fat_aabb.argtypes = [_P, C.c_uint32, _D]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_D)


class RefWorld:
    """One reference rbps::World built from a scenes.WorldSpec."""

    def __init__(self, spec, timestep, substeps, fat_margin=0.1, reinsert_threshold=0.05):
        L = lib()
        self.h = L.ref_world_create(timestep, substeps, fat_margin, reinsert_threshold)
        for verts, tris in spec.hulls:
            v = np.ascontiguousarray(verts, np.float64)
            t = np.ascontiguousarray(tris, np.uint32)
            L.ref_hull_create(self.h, _dp(v), len(v), t.ctypes.data_as(_U), len(t))
        for verts, faces in getattr(spec, "meshes", []):
            v = np.ascontiguousarray(verts, np.float64)
            f = np.ascontiguousarray(faces, np.uint32)
            L.ref_mesh_create(self.h, _dp(v), len(v), f.ctypes.data_as(_U), len(f))
        for heights, scale, origin in getattr(spec, "heightmaps", []):
            hh = np.ascontiguousarray(heights, np.float32)
            sc = np.ascontiguousarray(scale, np.float64)
            og = np.ascontiguousarray(origin, np.float64)
            L.ref_heightmap_create(self.h, hh.ctypes.data_as(C.POINTER(C.c_float)), hh.shape[0], hh.shape[1],
                                   _dp(sc), _dp(og))
        bodies = np.ascontiguousarray(spec.bodies)
        for i in range(len(bodies)):
            L.ref_add_body(self.h, C.c_void_p(bodies.ctypes.data + i * bodies.itemsize))
        forces = np.ascontiguousarray(spec.forces, np.float64)
        for i in range(len(bodies)):
            L.ref_set_body_force(self.h, i, _dp(forces[i]), None)
        cols = np.ascontiguousarray(spec.colliders)
        for i in range(len(cols)):
            L.ref_add_collider(self.h, C.c_void_p(cols.ctypes.data + i * cols.itemsize))
        joints = np.ascontiguousarray(spec.joints)
        for i in range(len(joints)):
            L.ref_add_joint(self.h, C.c_void_p(joints.ctypes.data + i * joints.itemsize))
        self.n = L.ref_body_count(self.h)

    def close(self):
        if self.h:
            lib().ref_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        lib().ref_step(self.h, n)

    def state(self):
        n = self.n
        pos, quat = np.zeros((n, 3)), np.zeros((n, 4))
        vel, omega = np.zeros((n, 3)), np.zeros((n, 3))
        lib().ref_get_state(self.h, _dp(pos), _dp(quat), _dp(vel), _dp(omega))
        return {"position": pos, "orientation": quat, "linear_velocity": vel, "angular_velocity": omega}

    def set_state(self, st):
        a = {k: np.ascontiguousarray(v, np.float64) for k, v in st.items()}
        lib().ref_set_state(self.h, _dp(a["position"]), _dp(a["orientation"]),
                            _dp(a["linear_velocity"]), _dp(a["angular_velocity"]))

    def pairs(self):
        L = lib()
        n = L.ref_get_pairs(self.h, None, 0)
        out = np.zeros((max(n, 1), 2), np.uint32)
        L.ref_get_pairs(self.h, out.ctypes.data_as(_U), n)
        return out[:n]

    def contacts(self):
        L = lib()
        n = L.ref_get_contacts(self.h, None, 0)
        out = np.zeros(max(n, 1), abi.CONTACT_DT)
        L.ref_get_contacts(self.h, C.c_void_p(out.ctypes.data), n)
        return out[:n]

    def sap_state(self):
        L = lib()
        n = L.ref_get_sap_state(self.h, None, None, None)
        fat = np.zeros((max(n, 1), 6))
        ids = np.zeros(max(2 * n, 1), np.uint32)
        vals = np.zeros(max(2 * n, 1), np.float32)
        L.ref_get_sap_state(self.h, _dp(fat), ids.ctypes.data_as(_U), vals.ctypes.data_as(C.POINTER(C.c_float)))
        return fat[:n], ids[:2 * n], vals[:2 * n]

    def collide(self, a, tf_a, b, tf_b):
        """rbc::dispatch on n shape pairs (collider descriptors; hull ids name
        this world's hulls); tf_*: (n, 7) position + quaternion wxyz."""
        a = np.ascontiguousarray(a, abi.COLLIDER_DT)
        b = np.ascontiguousarray(b, abi.COLLIDER_DT)
        ta = np.ascontiguousarray(tf_a, np.float64).reshape(-1, 7)
        tb = np.ascontiguousarray(tf_b, np.float64).reshape(-1, 7)
        n = len(a)
        out = np.zeros(max(n, 1), abi.MANIFOLD_DT)
        rc = lib().ref_collide(self.h, n, C.c_void_p(a.ctypes.data), _dp(ta), C.c_void_p(b.ctypes.data), _dp(tb),
                               C.c_void_p(out.ctypes.data))
        if rc != 0:
            raise ValueError("ref_collide: unknown shape or hull")
        return out[:n]

    def hull_tables(self, hull, cap=4096):
        """The reference's polygon / adjacency tables of this world's hull."""
        return _tables(lambda *a: lib().ref_hull_tables(self.h, hull, cap, *a), cap)

    def collision_groups(self):
        c = self.contacts()
        colors = np.zeros(max(len(c), 1), np.uint32)
        ng = lib().ref_collision_groups(self.h, colors.ctypes.data_as(_U), len(c))
        return colors[:len(c)], ng


TABLE_NAMES = ("poly_offsets", "poly_indices", "poly_normals", "v2p_offsets", "v2p_indices", "v2n_offsets",
               "v2n_indices", "p2p_offsets", "p2p_indices")


def _tables(fn, cap):
    """Calls a table dump with cap-sized buffers; vertex offset tables come
    back at full length (callers slice vert_count + 1)."""
    counts = np.zeros(5, np.uint32)
    arrs = [np.zeros(cap, np.uint32), np.zeros(cap, np.uint32), np.zeros(3 * cap, np.float64)] + \
        [np.zeros(cap, np.uint32) for _ in range(6)]
    ptrs = [a.ctypes.data_as(_D) if a.dtype == np.float64 else a.ctypes.data_as(_U) for a in arrs]
    rc = fn(counts.ctypes.data_as(_U), *ptrs)
    if rc != 0:
        raise ValueError(f"hull tables: status {rc}")
    npoly, nidx, nv2p, nv2n, np2p = (int(x) for x in counts)
    return {"poly_offsets": arrs[0][:npoly + 1], "poly_indices": arrs[1][:nidx],
            "poly_normals": arrs[2][:3 * npoly].reshape(-1, 3), "v2p_offsets": arrs[3],
            "v2p_indices": arrs[4][:nv2p], "v2n_offsets": arrs[5], "v2n_indices": arrs[6][:nv2n],
            "p2p_offsets": arrs[7][:npoly + 1], "p2p_indices": arrs[8][:np2p]}


def default_descs():
    """The reference's parameter defaults as descriptor records:
    (body, collider, revolute, prismatic, fixed, world_cfg)."""
    body = np.zeros(1, abi.BODY_DT)
    coll = np.zeros(1, abi.COLLIDER_DT)
    joints = np.zeros(3, abi.JOINT_DT)
    cfg = np.zeros(4)
    jp = joints.ctypes.data
    lib().ref_default_descs(C.c_void_p(body.ctypes.data), C.c_void_p(coll.ctypes.data), C.c_void_p(jp),
                            C.c_void_p(jp + joints.itemsize), C.c_void_p(jp + 2 * joints.itemsize), _dp(cfg))
    return body[0], coll[0], joints[0], joints[1], joints[2], cfg


def step_worlds(worlds, steps, threads):
    """Steps every RefWorld `steps` times on `threads` host threads; returns
    wall seconds."""
    arr = (_P * len(worlds))(*[w.h for w in worlds])
    return lib().ref_step_worlds(arr, len(worlds), steps, threads)


class RefBroadPhase:
    """The reference rbc SAP broadphase (BroadPhase.cpp), unmodified."""

    def __init__(self, fat_margin=0.1, reinsert_threshold=0.05):
        self.h = lib().ref_bp_create(fat_margin, reinsert_threshold)

    def __del__(self):
        try:
            lib().ref_bp_destroy(self.h)
        except Exception:
            pass

    def insert(self, user_id, aabb):
        return lib().ref_bp_insert(self.h, user_id, _dp(np.asarray(aabb, np.float64)))

    def remove(self, handle):
        lib().ref_bp_remove(self.h, handle)

    def move(self, handle, aabb):
        lib().ref_bp_move(self.h, handle, _dp(np.asarray(aabb, np.float64)))

    def move_swept(self, handle, aabb, vel, dt):
        lib().ref_bp_move_swept(self.h, handle, _dp(np.asarray(aabb, np.float64)),
                                _dp(np.asarray(vel, np.float64)), dt)

    def update(self):
        lib().ref_bp_update(self.h)

    def pairs(self):
        L = lib()
        n = L.ref_bp_get_pairs(self.h, None, 0)
        out = np.zeros((max(n, 1), 2), np.uint32)
        L.ref_bp_get_pairs(self.h, out.ctypes.data_as(_U), n)
        return out[:n]

    def fat_aabb(self, handle):
        out = np.zeros(6)
        lib().ref_bp_get_fat_aabb(self.h, handle, _dp(out))
        return out
