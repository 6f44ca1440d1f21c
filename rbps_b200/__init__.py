"""rbps_b200 - B200 (sm_100a) implementation of the RBPS per-step hot path.

Python binding of the C ABI in include/rbps_gpu.h (librbps_b200.so, built
in-tree by ``python -m rbps_b200.build``).  The classes mirror the
reference's setup surface:

* :class:`World` - one ``rbps::World`` (World.hpp:87-213): ``create_body``,
  ``create_collider``, ``create_revolute_joint`` ... then ``step()``.
* :class:`Batch` - many independent worlds stepped together.
* :class:`BroadPhase` - the rbc SAP broadphase API (BroadPhase.hpp:151-260)
  with the sort and sweep on the GPU.

There is no CPU fallback: every call goes through the CUDA library, and a
missing library or device raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

__all__ = ["lib", "Batch", "World", "BroadPhase", "RbpsError", "abi", "quickhull", "hull_tables"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RBPS_B200_LIB") or os.path.join(_HERE, "librbps_b200.so")
_lib = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_U = C.POINTER(C.c_uint32)


class RbpsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rbps error {code}: {msg}")
        self.code = code


class BatchDesc(C.Structure):
    _fields_ = [("n_worlds", C.c_uint32), ("timestep", C.c_double), ("substeps", C.c_int32),
                ("precision", C.c_int32), ("solve_mode", C.c_int32), ("fat_margin", C.c_double),
                ("reinsert_threshold", C.c_double), ("use_velocity_expansion", C.c_int32),
                ("device", C.c_int32), ("stream", C.c_void_p), ("max_pairs_per_world", C.c_uint32),
                ("block_threads", C.c_uint32)]


class StateView(C.Structure):
    _fields_ = [("position", _D), ("orientation", _D), ("linear_velocity", _D), ("angular_velocity", _D)]


class TuneResult(C.Structure):
    _fields_ = [("frame_block", C.c_int32), ("narrow_grid", C.c_int32), ("ms_per_step", C.c_double),
                ("ms_per_step_default", C.c_double), ("trials", C.c_uint32), ("team_bodies", C.c_uint32),
                ("narrow_per_warp", C.c_uint32), ("color_chunk", C.c_uint32), ("pair_bodies", C.c_uint32),
                ("pad_", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("pairs", C.c_uint64), ("candidates", C.c_uint64),
                ("contacts", C.c_uint64), ("max_colors", C.c_uint32), ("serial_overflow", C.c_uint32),
                ("device_error", C.c_int32), ("graph", C.c_uint32), ("kernel_launches", C.c_uint64),
                ("gjk_pairs", C.c_uint64)]


def lib():
    """Loads librbps_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m rbps_b200.build`")
        L = C.CDLL(LIB_PATH)
        i = C.c_int
        sig = {
            "rbps_batch_desc_default": (None, [C.POINTER(BatchDesc)]),
            "rbps_batch_create": (i, [C.POINTER(BatchDesc), C.POINTER(_P)]),
            "rbps_batch_destroy": (i, [_P]),
            "rbps_hull_create": (i, [_P, _D, C.c_uint32, _U, C.c_uint32, _U]),
            "rbps_heightmap_create": (i, [_P, C.POINTER(C.c_float), C.c_uint32, C.c_uint32, _D, _D, _U]),
            "rbps_mesh_create": (i, [_P, _D, C.c_uint32, _U, C.c_uint32, _U]),
            "rbps_quickhull": (i, [_D, C.c_uint32, _U, C.c_uint32, _U]),
            "rbps_hull_tables": (i, [_D, C.c_uint32, _U, C.c_uint32, C.c_uint32, _U, _U, _U, _D, _U, _U, _U, _U, _U,
                                     _U]),
            "rbps_world_add_body": (i, [_P, C.c_uint32, _P, _U]),
            "rbps_world_add_bodies": (i, [_P, C.c_uint32, C.c_uint32, _P, _U]),
            "rbps_world_set_body_force": (i, [_P, C.c_uint32, C.c_uint32, _D, _D]),
            "rbps_world_set_body_forces": (i, [_P, C.c_uint32, C.c_uint32, C.c_uint32, _D]),
            "rbps_batch_step_io": (i, [_P, C.c_void_p, C.c_void_p, C.c_void_p]),
            "rbps_batch_step_io_async": (i, [_P, C.c_void_p, C.c_void_p, C.c_void_p]),
            "rbps_batch_snapshot": (i, [_P, C.POINTER(C.c_uint32)]),
            "rbps_batch_snapshot_update": (i, [_P, C.c_uint32]),
            "rbps_batch_restore": (i, [_P, C.c_uint32]),
            "rbps_batch_autotune": (i, [_P, C.c_int32, C.POINTER(TuneResult)]),
            "rbps_batch_set_launch": (i, [_P, C.POINTER(TuneResult)]),
            "rbps_world_add_collider": (i, [_P, C.c_uint32, _P, _U]),
            "rbps_world_add_colliders": (i, [_P, C.c_uint32, C.c_uint32, _P, _U]),
            "rbps_world_add_joint": (i, [_P, C.c_uint32, _P, _U]),
            "rbps_batch_commit": (i, [_P]),
            "rbps_batch_step": (i, [_P, C.c_int32]),
            "rbps_batch_synchronize": (i, [_P]),
            "rbps_batch_set_state_check": (i, [_P, C.c_int32]),
            "rbps_batch_get_state": (i, [_P, C.c_uint32, C.POINTER(StateView)]),
            "rbps_batch_set_state": (i, [_P, C.c_uint32, C.POINTER(StateView)]),
            "rbps_batch_get_state_all": (i, [_P, C.POINTER(StateView)]),
            "rbps_batch_set_forces_all": (i, [_P, _D]),
            "rbps_batch_body_count": (i, [_P, C.c_uint32, _U]),
            "rbps_batch_total_bodies": (i, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "rbps_batch_set_dump": (i, [_P, C.c_int32]),
            "rbps_batch_get_pairs": (i, [_P, C.c_uint32, _U, C.c_uint32, _U]),
            "rbps_batch_get_contacts": (i, [_P, C.c_uint32, _P, C.c_uint32, _U]),
            "rbps_batch_get_colors": (i, [_P, C.c_uint32, _U, _U, _U, C.c_uint32, _U]),
            "rbps_batch_get_stats": (i, [_P, C.POINTER(Stats)]),
            "rbps_batch_get_sap_state": (i, [_P, C.c_uint32, _D, _U, C.POINTER(C.c_float), _U]),
            "rbps_debug_broadphase": (i, [_P, C.c_uint32, _U]),
            "rbps_batch_collide": (i, [_P, C.c_uint32, _P, _D, _P, _D, _P]),
            "rbps_batch_set_profile": (i, [_P, C.c_int32]),
            "rbps_batch_get_profile": (i, [_P, C.POINTER(C.c_uint64), C.c_uint32]),
            "rbps_bp_create": (i, [C.c_double, C.c_double, C.POINTER(_P)]),
            "rbps_bp_destroy": (i, [_P]),
            "rbps_bp_insert": (i, [_P, C.c_uint32, _D, _U]),
            "rbps_bp_remove": (i, [_P, C.c_uint32]),
            "rbps_bp_move": (i, [_P, C.c_uint32, _D]),
            "rbps_bp_move_swept": (i, [_P, C.c_uint32, _D, _D, C.c_double]),
            "rbps_bp_update": (i, [_P]),
            "rbps_bp_get_pairs": (i, [_P, _U, C.c_uint32, _U]),
            "rbps_bp_get_fat_aabb": (i, [_P, C.c_uint32, _D]),
            "rbps_bp_configure": (i, [_P, C.c_int32, C.c_int32]),
            "rbps_sap_pairs_static": (i, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                          C.c_void_p]),
            "rbps_selftest_sort": (i, [_U, C.c_uint32, C.c_int32, C.c_int32, C.c_int32, _U, _U]),
            "rbps_selftest_scan": (i, [_U, C.c_uint32, C.c_int32, C.c_int32, _U, _U]),
            "rbps_last_error": (i, [C.c_char_p, C.c_size_t]),
            "rbps_version": (C.c_char_p, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        buf = C.create_string_buffer(1024)
        lib().rbps_last_error(buf, 1024)
        raise RbpsError(rc, buf.value.decode())
    return rc


def _dp(a):
    return a.ctypes.data_as(_D)


def quickhull(points):
    """CCW outward triangles (m, 3) of the convex hull of `points` (n, 3)."""
    pts = np.ascontiguousarray(points, np.float64)
    cap = 4 * len(pts) + 16
    tris = np.zeros((cap, 3), np.uint32)
    n = C.c_uint32(0)
    _check(lib().rbps_quickhull(_dp(pts), len(pts), tris.ctypes.data_as(_U), cap, C.byref(n)))
    return tris[:n.value].copy()


def hull_tables(verts, tris, cap=4096):
    """The merged-polygon and adjacency tables the library builds for a hull
    (dict of numpy arrays; vertex offset tables at full cap length)."""
    v = np.ascontiguousarray(verts, np.float64)
    t = np.ascontiguousarray(tris, np.uint32)
    counts = np.zeros(5, np.uint32)
    arrs = [np.zeros(cap, np.uint32), np.zeros(cap, np.uint32), np.zeros(3 * cap, np.float64)] + \
        [np.zeros(cap, np.uint32) for _ in range(6)]
    ptrs = [a.ctypes.data_as(_D) if a.dtype == np.float64 else a.ctypes.data_as(_U) for a in arrs]
    _check(lib().rbps_hull_tables(_dp(v), len(v), t.ctypes.data_as(_U), len(t), cap, counts.ctypes.data_as(_U),
                                  *ptrs))
    npoly, nidx, nv2p, nv2n, np2p = (int(x) for x in counts)
    return {"poly_offsets": arrs[0][:npoly + 1], "poly_indices": arrs[1][:nidx],
            "poly_normals": arrs[2][:3 * npoly].reshape(-1, 3), "v2p_offsets": arrs[3],
            "v2p_indices": arrs[4][:nv2p], "v2n_offsets": arrs[5], "v2n_indices": arrs[6][:nv2n],
            "p2p_offsets": arrs[7][:npoly + 1], "p2p_indices": arrs[8][:np2p]}


class Batch:
    """Independent worlds stepped together (one rbps_batch)."""

    def __init__(self, n_worlds, timestep, substeps, precision=abi.PRECISION_FP64,
                 solve_mode=abi.SOLVE_REFERENCE_ORDER, fat_margin=0.1, reinsert_threshold=0.05,
                 device=0, max_pairs_per_world=0, block_threads=0, stream=None):
        L = lib()
        d = BatchDesc()
        L.rbps_batch_desc_default(C.byref(d))
        d.n_worlds = n_worlds
        d.timestep = timestep
        d.substeps = substeps
        d.precision = precision
        d.solve_mode = solve_mode
        d.fat_margin = fat_margin
        d.reinsert_threshold = reinsert_threshold
        d.device = device
        d.max_pairs_per_world = max_pairs_per_world
        d.block_threads = block_threads
        d.stream = stream
        h = _P()
        _check(L.rbps_batch_create(C.byref(d), C.byref(h)))
        self.h = h
        self.n_worlds = n_worlds
        self.precision = precision
        self.committed = False
        self._counts = [0] * n_worlds

    @classmethod
    def from_scene(cls, scene, precision=abi.PRECISION_FP64, solve_mode=abi.SOLVE_REFERENCE_ORDER, **kw):
        b = cls(len(scene.worlds), scene.timestep, scene.substeps, precision, solve_mode, **kw)
        for w, spec in enumerate(scene.worlds):
            b.add_world(w, spec)
        b.commit()
        return b

    def add_world(self, w, spec):
        L = lib()
        hull_base = []
        for verts, tris in spec.hulls:
            v = np.ascontiguousarray(verts, np.float64)
            t = np.ascontiguousarray(tris, np.uint32)
            hid = C.c_uint32(0)
            _check(L.rbps_hull_create(self.h, _dp(v), len(v), t.ctypes.data_as(_U), len(t), C.byref(hid)))
            hull_base.append(hid.value)
        bodies = np.ascontiguousarray(spec.bodies)
        first = C.c_uint32(0)
        _check(L.rbps_world_add_bodies(self.h, w, len(bodies), C.c_void_p(bodies.ctypes.data), C.byref(first)))
        forces = np.ascontiguousarray(spec.forces, np.float64)
        if len(bodies):
            _check(L.rbps_world_set_body_forces(self.h, w, first.value, len(bodies), _dp(forces)))
        hm_base = []
        for heights, scale, origin in getattr(spec, "heightmaps", []):
            hh = np.ascontiguousarray(heights, np.float32)
            sc = np.ascontiguousarray(scale, np.float64)
            og = np.ascontiguousarray(origin, np.float64)
            hid = C.c_uint32(0)
            _check(L.rbps_heightmap_create(self.h, hh.ctypes.data_as(C.POINTER(C.c_float)), hh.shape[0], hh.shape[1],
                                           _dp(sc), _dp(og), C.byref(hid)))
            hm_base.append(hid.value)
        mesh_base = []
        for verts, faces in getattr(spec, "meshes", []):
            v = np.ascontiguousarray(verts, np.float64)
            f = np.ascontiguousarray(faces, np.uint32)
            mid = C.c_uint32(0)
            _check(L.rbps_mesh_create(self.h, _dp(v), len(v), f.ctypes.data_as(_U), len(f), C.byref(mid)))
            mesh_base.append(mid.value)
        cols = np.ascontiguousarray(spec.colliders).copy()
        if mesh_base:
            m = cols["shape"] == abi.SHAPE_MESH
            cols["hull"][m] = np.asarray(mesh_base, np.uint32)[cols["hull"][m]]
        if hull_base:
            m = cols["shape"] == abi.SHAPE_CONVEX_HULL
            cols["hull"][m] = np.asarray(hull_base, np.uint32)[cols["hull"][m]]
        if hm_base:
            m = cols["shape"] == abi.SHAPE_HEIGHTMAP
            cols["hull"][m] = np.asarray(hm_base, np.uint32)[cols["hull"][m]]
        if len(cols):
            _check(L.rbps_world_add_colliders(self.h, w, len(cols), C.c_void_p(cols.ctypes.data), None))
        joints = np.ascontiguousarray(spec.joints)
        for i in range(len(joints)):
            _check(L.rbps_world_add_joint(self.h, w, C.c_void_p(joints.ctypes.data + i * joints.itemsize), None))
        self._counts[w] = len(bodies)

    def add_hull(self, verts, tris):
        """Registers a convex hull (before commit); returns its hull id."""
        v = np.ascontiguousarray(verts, np.float64)
        t = np.ascontiguousarray(tris, np.uint32)
        hid = C.c_uint32(0)
        _check(lib().rbps_hull_create(self.h, _dp(v), len(v), t.ctypes.data_as(_U), len(t), C.byref(hid)))
        return hid.value

    def commit(self):
        _check(lib().rbps_batch_commit(self.h))
        self.committed = True

    PROFILE_PHASES = ("broadphase", "candidates", "narrowphase", "colouring", "integrate", "contact_pos",
                      "joint_pos", "vel_update", "vel_solve", "stats")

    def set_profile(self, on=True):
        """Per-world phase timers (SM cycles); enabling zeroes them."""
        _check(lib().rbps_batch_set_profile(self.h, 1 if on else 0))

    def profile(self):
        """(n_worlds, 16) uint64: phase cycles (PROFILE_PHASES order), then
        slot 12 = CTA, 13 / 14 = start / end globaltimer ns of the last step.
        For worlds on one CTA, slots 10, 11 and 15 split the broadphase: the
        endpoint sort, the sweep and the pair order (cycles)."""
        out = np.zeros((self.n_worlds, 16), np.uint64)
        _check(lib().rbps_batch_get_profile(self.h, out.ctypes.data_as(C.POINTER(C.c_uint64)), self.n_worlds))
        return out

    def collide(self, a, tf_a, b, tf_b):
        """Device narrowphase (rbc::dispatch) of n shape pairs: collider
        descriptors a, b (abi.COLLIDER_DT) and transforms (n, 7) = position +
        quaternion wxyz.  Returns abi.MANIFOLD_DT records."""
        a = np.ascontiguousarray(a, abi.COLLIDER_DT)
        b = np.ascontiguousarray(b, abi.COLLIDER_DT)
        ta = np.ascontiguousarray(tf_a, np.float64).reshape(-1, 7)
        tb = np.ascontiguousarray(tf_b, np.float64).reshape(-1, 7)
        n = len(a)
        if not (len(b) == n and len(ta) == n and len(tb) == n):
            raise ValueError("collide: a, b, tf_a and tf_b must have the same length")
        out = np.zeros(max(n, 1), abi.MANIFOLD_DT)
        _check(lib().rbps_batch_collide(self.h, n, C.c_void_p(a.ctypes.data), _dp(ta), C.c_void_p(b.ctypes.data),
                                        _dp(tb), C.c_void_p(out.ctypes.data)))
        return out[:n]

    def step(self, n=1):
        _check(lib().rbps_batch_step(self.h, n))

    def synchronize(self):
        _check(lib().rbps_batch_synchronize(self.h))

    def set_state_check(self, on=True):
        """Failure detection (on by default): a non-finite body state makes
        the next synchronising call raise RbpsError(ERR_STATE).  Off
        reproduces the reference, which lets a NaN propagate."""
        _check(lib().rbps_batch_set_state_check(self.h, 1 if on else 0))

    def step_io(self, force_ptr, pos_ptr, rot_ptr):
        """One step with host I/O through raw host pointers (ints or None)."""
        _check(lib().rbps_batch_step_io(self.h, force_ptr, pos_ptr, rot_ptr))

    def autotune(self, trial_steps=3):
        """Times the launch-shape candidates on this batch's own worlds from
        one snapshot, keeps the fastest, rewinds; returns the choice."""
        r = TuneResult()
        _check(lib().rbps_batch_autotune(self.h, trial_steps, C.byref(r)))
        return {k: getattr(r, k) for k, _ in TuneResult._fields_ if k != "pad_"}

    def set_launch(self, **cfg):
        """Applies launch-shape fields (frame_block, narrow_grid, team_bodies,
        pair_bodies, narrow_per_warp, color_chunk) as rbps_batch_set_launch;
        others keep their values.  Results do not depend on them."""
        r = TuneResult()
        for k, v in cfg.items():
            setattr(r, k, v)
        _check(lib().rbps_batch_set_launch(self.h, C.byref(r)))

    def snapshot(self):
        """Device-side snapshot of the whole batch state; returns its slot."""
        slot = C.c_uint32(0)
        _check(lib().rbps_batch_snapshot(self.h, C.byref(slot)))
        return slot.value

    def snapshot_update(self, slot):
        _check(lib().rbps_batch_snapshot_update(self.h, slot))

    def restore(self, slot):
        """Rewinds every world to snapshot `slot`."""
        _check(lib().rbps_batch_restore(self.h, slot))

    def step_io_async(self, force_ptr, pos_ptr, rot_ptr):
        """step_io without the wait: the copies overlap neighbouring steps;
        the host buffers are final after synchronize()."""
        _check(lib().rbps_batch_step_io_async(self.h, force_ptr, pos_ptr, rot_ptr))

    def set_dump(self, on=True):
        _check(lib().rbps_batch_set_dump(self.h, 1 if on else 0))

    def n_bodies(self, w):
        n = C.c_uint32(0)
        _check(lib().rbps_batch_body_count(self.h, w, C.byref(n)))
        return n.value

    def total_bodies(self):
        n, nd = C.c_uint64(0), C.c_uint64(0)
        _check(lib().rbps_batch_total_bodies(self.h, C.byref(n), C.byref(nd)))
        return n.value, nd.value

    def state(self, w):
        n = self.n_bodies(w)
        pos, quat = np.zeros((n, 3)), np.zeros((n, 4))
        vel, omega = np.zeros((n, 3)), np.zeros((n, 3))
        v = StateView(_dp(pos), _dp(quat), _dp(vel), _dp(omega))
        _check(lib().rbps_batch_get_state(self.h, w, C.byref(v)))
        return {"position": pos, "orientation": quat, "linear_velocity": vel, "angular_velocity": omega}

    def state_all(self, fields=("position", "orientation")):
        n, _ = self.total_bodies()
        out = {"position": np.zeros((n, 3)), "orientation": np.zeros((n, 4)),
               "linear_velocity": np.zeros((n, 3)), "angular_velocity": np.zeros((n, 3))}
        ptr = {k: (_dp(out[k]) if k in fields else None) for k in out}
        v = StateView(ptr["position"], ptr["orientation"], ptr["linear_velocity"], ptr["angular_velocity"])
        _check(lib().rbps_batch_get_state_all(self.h, C.byref(v)))
        return {k: out[k] for k in fields}

    def set_state(self, w, st):
        a = {k: np.ascontiguousarray(st[k], np.float64) if k in st else None
             for k in ("position", "orientation", "linear_velocity", "angular_velocity")}
        v = StateView(*[(_dp(a[k]) if a[k] is not None else None)
                        for k in ("position", "orientation", "linear_velocity", "angular_velocity")])
        _check(lib().rbps_batch_set_state(self.h, w, C.byref(v)))

    def set_forces_all(self, force):
        f = np.ascontiguousarray(force, np.float64)
        _check(lib().rbps_batch_set_forces_all(self.h, _dp(f)))

    def pairs(self, w):
        L = lib()
        n = C.c_uint32(0)
        _check(L.rbps_batch_get_pairs(self.h, w, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 2), np.uint32)
        _check(L.rbps_batch_get_pairs(self.h, w, out.ctypes.data_as(_U), n.value, C.byref(n)))
        return out[:n.value]

    def contacts(self, w):
        L = lib()
        n = C.c_uint32(0)
        _check(L.rbps_batch_get_contacts(self.h, w, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), abi.CONTACT_DT)
        _check(L.rbps_batch_get_contacts(self.h, w, C.c_void_p(out.ctypes.data), n.value, C.byref(n)))
        return out[:n.value]

    def colors(self, w):
        L = lib()
        n = C.c_uint32(0)
        _check(L.rbps_batch_get_colors(self.h, w, None, None, None, 0, C.byref(n)))
        col = np.zeros(max(n.value, 1), np.uint32)
        ba = np.zeros_like(col)
        bb = np.zeros_like(col)
        _check(L.rbps_batch_get_colors(self.h, w, col.ctypes.data_as(_U), ba.ctypes.data_as(_U),
                                       bb.ctypes.data_as(_U), n.value, C.byref(n)))
        return col[:n.value], ba[:n.value], bb[:n.value]

    def sap_state(self, w):
        """(fat AABBs (n, 6), endpoint ids in list order, endpoint values)."""
        L = lib()
        n = C.c_uint32(0)
        _check(L.rbps_batch_get_sap_state(self.h, w, None, None, None, C.byref(n)))
        fat = np.zeros((max(n.value, 1), 6))
        ids = np.zeros(max(2 * n.value, 1), np.uint32)
        vals = np.zeros(max(2 * n.value, 1), np.float32)
        _check(L.rbps_batch_get_sap_state(self.h, w, _dp(fat), ids.ctypes.data_as(_U),
                                          vals.ctypes.data_as(C.POINTER(C.c_float)), C.byref(n)))
        return fat[:n.value], ids[:2 * n.value], vals[:2 * n.value]

    def stats(self):
        s = Stats()
        _check(lib().rbps_batch_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_ if k != "pad_"}

    def close(self):
        if getattr(self, "h", None):
            lib().rbps_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class World:
    """rbps::World on the GPU (World.hpp:87-213): create bodies, colliders and
    joints, then ``step()``.  State is read with :meth:`state`."""

    def __init__(self, timestep=1.0 / 60.0, substeps=20, precision=abi.PRECISION_FP64,
                 solve_mode=abi.SOLVE_REFERENCE_ORDER, **kw):
        self.timestep = timestep
        self.substeps = substeps
        self._batch = Batch(1, timestep, substeps, precision, solve_mode, **kw)
        self._forces = {}

    def create_body(self, type=abi.BODY_DYNAMIC, mass=1.0, inertia_tensor=(1.0, 1.0, 1.0, 0.0, 0.0, 0.0),
                    position=(0.0, 0.0, 0.0), orientation=(1.0, 0.0, 0.0, 0.0),
                    linear_velocity=(0.0, 0.0, 0.0), angular_velocity=(0.0, 0.0, 0.0)):
        """BodyParams (BodyAPI.hpp:22-31) -> body ID."""
        d = abi.body_default()
        d["type"], d["mass"], d["inertia"] = type, mass, inertia_tensor
        d["position"], d["orientation"] = position, orientation
        d["linear_velocity"], d["angular_velocity"] = linear_velocity, angular_velocity
        arr = np.array([d], abi.BODY_DT)
        bid = C.c_uint32(0)
        _check(lib().rbps_world_add_body(self._batch.h, 0, C.c_void_p(arr.ctypes.data), C.byref(bid)))
        return bid.value

    def set_force(self, body, force, torque=None):
        f = np.asarray(force, np.float64)
        t = np.asarray(torque, np.float64) if torque is not None else None
        _check(lib().rbps_world_set_body_force(self._batch.h, 0, body, _dp(f), _dp(t) if t is not None else None))

    def create_collider(self, shape=abi.SHAPE_SPHERE, params=(0.5,), body_id=0, is_static=False,
                        local_pos=(0.0, 0.0, 0.0), local_rot=(1.0, 0.0, 0.0, 0.0), restitution=0.5,
                        static_friction=0.5, dynamic_friction=0.5, hull=0):
        """ColliderParams (ColliderAPI.hpp:17-27) -> collider ID."""
        d = abi.collider_default()
        d["shape"] = shape
        d["params"] = list(params) + [0.0] * (4 - len(params))
        d["hull"], d["body_id"], d["is_static"] = hull, body_id, int(is_static)
        d["local_pos"], d["local_rot"] = local_pos, local_rot
        d["restitution"], d["static_friction"], d["dynamic_friction"] = restitution, static_friction, dynamic_friction
        arr = np.array([d], abi.COLLIDER_DT)
        cid = C.c_uint32(0)
        _check(lib().rbps_world_add_collider(self._batch.h, 0, C.c_void_p(arr.ctypes.data), C.byref(cid)))
        return cid.value

    def _joint(self, jtype, **kw):
        d = abi.joint_default(jtype)
        for k, v in kw.items():
            d[k] = v
        arr = np.array([d], abi.JOINT_DT)
        jid = C.c_uint32(0)
        _check(lib().rbps_world_add_joint(self._batch.h, 0, C.c_void_p(arr.ctypes.data), C.byref(jid)))
        return jid.value

    def create_revolute_joint(self, body_1, body_2, aligned_axis=(1.0, 0.0, 0.0), limit_axis=(0.0, 1.0, 0.0),
                              r_1=(0.0, 0.0, 0.0), r_2=(0.0, 0.0, 0.0), actuation=abi.ACTUATION_FREE,
                              compliance=0.0, damping=0.0, limited=False, lower_limit=0.0, upper_limit=0.0):
        """RevoluteJointParams (JointAPI.hpp:43-57)."""
        return self._joint(abi.JOINT_REVOLUTE, body_1=body_1, body_2=body_2, axis=aligned_axis,
                           limit_axis=limit_axis, r_1=r_1, r_2=r_2, actuation=actuation, compliance=compliance,
                           damping=damping, limited=int(limited), lower_limit=lower_limit, upper_limit=upper_limit)

    def create_prismatic_joint(self, body_1, body_2, moving_axis=(1.0, 0.0, 0.0), r_1=(0.0, 0.0, 0.0),
                               r_2=(0.0, 0.0, 0.0), actuation=abi.ACTUATION_FREE, compliance=0.0, damping=0.0,
                               limited=False, lower_limit=0.0, upper_limit=0.0):
        """PrismaticJointParams (JointAPI.hpp:24-36)."""
        return self._joint(abi.JOINT_PRISMATIC, body_1=body_1, body_2=body_2, axis=moving_axis, r_1=r_1, r_2=r_2,
                           actuation=actuation, compliance=compliance, damping=damping, limited=int(limited),
                           lower_limit=lower_limit, upper_limit=upper_limit)

    def create_fixed_joint(self, body_1, body_2, r_1=(0.0, 0.0, 0.0), r_2=(0.0, 0.0, 0.0)):
        """FixedJointParams (JointAPI.hpp:59-65)."""
        return self._joint(abi.JOINT_FIXED, body_1=body_1, body_2=body_2, r_1=r_1, r_2=r_2)

    def step(self, n=1):
        """World::step (World.hpp:192-212); commits the world on first use."""
        if not self._batch.committed:
            self._batch.commit()
        self._batch.step(n)

    def state(self):
        if not self._batch.committed:
            self._batch.commit()
        return self._batch.state(0)

    @property
    def batch(self):
        return self._batch


def selftest_sort(keys, bits=32, grid=False, block=128):
    """Device stable radix sort of `keys` by the low `bits` bits; returns
    (sorted keys, original positions)."""
    k = np.ascontiguousarray(keys, np.uint32)
    ko, vo = np.zeros_like(k), np.zeros_like(k)
    _check(lib().rbps_selftest_sort(k.ctypes.data_as(_U), len(k), bits, int(grid), block,
                                    ko.ctypes.data_as(_U), vo.ctypes.data_as(_U)))
    return ko, vo


def selftest_scan(values, grid=False, block=128):
    """Device exclusive scan; returns (scan, total)."""
    v = np.ascontiguousarray(values, np.uint32)
    out = np.zeros_like(v)
    tot = C.c_uint32(0)
    _check(lib().rbps_selftest_scan(v.ctypes.data_as(_U), len(v), int(grid), block, out.ctypes.data_as(_U),
                                    C.byref(tot)))
    return out, tot.value


class BroadPhase:
    """GPU SAP broadphase with the rbc API (BroadPhase.hpp:151-260)."""

    def __init__(self, fat_margin=0.1, reinsert_threshold=0.05, single_cta=False, block=256):
        h = _P()
        _check(lib().rbps_bp_create(fat_margin, reinsert_threshold, C.byref(h)))
        self.h = h
        if single_cta or block != 256:
            _check(lib().rbps_bp_configure(h, int(single_cta), block))

    def __del__(self):
        try:
            lib().rbps_bp_destroy(self.h)
        except Exception:
            pass

    def insert(self, user_id, aabb):
        hd = C.c_uint32(0)
        _check(lib().rbps_bp_insert(self.h, user_id, _dp(np.asarray(aabb, np.float64)), C.byref(hd)))
        return hd.value

    def remove(self, handle):
        _check(lib().rbps_bp_remove(self.h, handle))

    def move(self, handle, aabb):
        _check(lib().rbps_bp_move(self.h, handle, _dp(np.asarray(aabb, np.float64))))

    def move_swept(self, handle, aabb, vel, dt):
        _check(lib().rbps_bp_move_swept(self.h, handle, _dp(np.asarray(aabb, np.float64)),
                                        _dp(np.asarray(vel, np.float64)), dt))

    def update(self):
        _check(lib().rbps_bp_update(self.h))

    def pairs(self):
        L = lib()
        n = C.c_uint32(0)
        _check(L.rbps_bp_get_pairs(self.h, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 2), np.uint32)
        _check(L.rbps_bp_get_pairs(self.h, out.ctypes.data_as(_U), n.value, C.byref(n)))
        return out[:n.value]

    def fat_aabb(self, handle):
        out = np.zeros(6)
        _check(lib().rbps_bp_get_fat_aabb(self.h, handle, _dp(out)))
        return out
