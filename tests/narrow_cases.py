"""Shape-pair cases of the narrowphase parity tests.

REF_CASES restates the inputs and expected results of the reference's own
analytic collision tests (tests/rbc/analytic/*.cpp, file:line per case) as
data: shapes, poses, and what the reference test asserts about the
manifold (hit or miss, depth, dominant normal component, point count).
random_pairs() draws seeded poses near contact for every shape pairing the
device handles analytically.
"""
import math

import numpy as np

from rbps_b200 import abi

# tests/rbc/analytic: convex-hull fixtures (test_convex_hull_plane.cpp:9-67)
TET_VERTS = np.array([[1, 1, 1], [-1, -1, 1], [-1, 1, -1], [1, -1, -1]], np.float64)
TET_FACES = np.array([[0, 1, 2], [0, 3, 1], [0, 2, 3], [1, 3, 2]], np.uint32)
CUBE_VERTS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                       [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float64)
CUBE_FACES = np.array([[0, 1, 2], [0, 2, 3], [4, 6, 5], [4, 7, 6], [0, 5, 1], [0, 4, 5],
                       [2, 6, 3], [3, 6, 7], [0, 3, 7], [0, 7, 4], [1, 5, 6], [1, 6, 2]], np.uint32)

def _ellipsoid_hull(seed, n, axes):
    """n points uniform on an ellipsoid surface and their hull triangles
    (from a fixed point set, so the fixture does not depend on a build)."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    return d / np.linalg.norm(d, axis=1, keepdims=True) * np.asarray(axes)


ELLIPSOID_A = _ellipsoid_hull(21, 16, (0.5, 0.3, 0.4))
ELLIPSOID_B = _ellipsoid_hull(22, 24, (0.35, 0.5, 0.3))
HULLS = {"tet": (TET_VERTS, TET_FACES), "cube": (CUBE_VERTS, CUBE_FACES),
         "ellA": (ELLIPSOID_A, None), "ellB": (ELLIPSOID_B, None)}
HULL_IDS = {"tet": 0, "cube": 1, "ellA": 2, "ellB": 3}


def hull_list():
    """[(verts, tris)] in HULL_IDS order; ellipsoid triangles from quickhull."""
    import rbps_b200
    out = []
    for name in sorted(HULL_IDS, key=HULL_IDS.get):
        v, t = HULLS[name]
        out.append((v, t if t is not None else rbps_b200.quickhull(v)))
    return out


def sphere(r):
    return (abi.SHAPE_SPHERE, (r, 0, 0, 0), 0)


def box(hx, hy, hz):
    return (abi.SHAPE_BOX, (hx, hy, hz, 0), 0)


def capsule(half_height, radius):
    return (abi.SHAPE_CAPSULE, (half_height, radius, 0, 0), 0)


def ellipsoid(a, b, c):
    return (abi.SHAPE_ELLIPSOID, (a, b, c, 0), 0)


def cylinder(half_height, radius):
    return (abi.SHAPE_CYLINDER, (half_height, radius, 0, 0), 0)


def cone(half_height, radius):
    return (abi.SHAPE_CONE, (half_height, radius, 0, 0), 0)


def plane(nx, ny, nz, d):
    return (abi.SHAPE_PLANE, (nx, ny, nz, d), 0)


def hull(name):
    return (abi.SHAPE_CONVEX_HULL, (0, 0, 0, 0), HULL_IDS[name])


def axis_quat(axis, angle):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    s = math.sin(angle * 0.5)
    return (math.cos(angle * 0.5), a[0] * s, a[1] * s, a[2] * s)


def tf(x, y, z, q=(1.0, 0.0, 0.0, 0.0)):
    return (x, y, z) + tuple(q)


QUARTER_PI = math.pi / 4
HALF_PI = math.pi / 2
S2 = math.sqrt(2.0)
INV_S2 = 1.0 / math.sqrt(2.0)

# Four of these files are not built by the reference (CMakeLists.txt:215-260
# registers sphere_sphere, box_box, sphere_box, sphere_capsule and the
# convex-hull tests only): test_plane_sphere.cpp, test_plane_box.cpp,
# test_plane_capsule.cpp and test_capsule_capsule.cpp.  Three of their
# assertions disagree with the reference code as it stands, and the cases
# below state what the code does (the oracle runs that code):
#   * X-vs-Plane normals point from A into the plane, i.e. minus the plane
#     normal (PlaneCollision.hpp, "n = -world_n"); the stale tests expect +n;
#   * a box corner exactly on the plane is a contact: corners within the
#     1e-4f slop are kept (PlaneCollision.hpp:310);
#   * parallel capsules project s and t from the first endpoints separately
#     (CapsuleCapsule.hpp:52-55), so collinear capsules touching end to end
#     report no contact.
# (name, reference file:line, shape A, tf A, shape B, tf B, expectation)
# expectation: {"hit": bool, "depth": (value, tol), "normal": (axis, |value|, tol) or (axis, value, tol, "signed"),
#               "n_points": k}
REF_CASES = [
    ("sphere_sphere_separated", "test_sphere_sphere.cpp:4", sphere(1), tf(0, 0, 0), sphere(1), tf(3, 0, 0),
     {"hit": False}),
    ("sphere_sphere_touching", "test_sphere_sphere.cpp:14", sphere(1), tf(0, 0, 0), sphere(1), tf(2, 0, 0),
     {"hit": False}),
    ("sphere_sphere_overlapping_depth", "test_sphere_sphere.cpp:25", sphere(1), tf(0, 0, 0), sphere(1),
     tf(1.5, 0, 0), {"hit": True, "depth": (0.5, 0.01), "normal": (0, 1.0, 0.01)}),
    ("sphere_sphere_diagonal_overlap", "test_sphere_sphere.cpp:41", sphere(1), tf(0, 0, 0), sphere(1),
     tf(1, 1, 0), {"hit": True}),
    ("sphere_sphere_coincident_centres", "test_sphere_sphere.cpp:53", sphere(1), tf(0, 0, 0), sphere(1),
     tf(0, 0, 0), {"hit": True, "depth": (2.0, 0.01)}),
    ("sphere_box_separated", "test_sphere_box.cpp:4", sphere(1), tf(0, 0, 0), box(1, 1, 1), tf(4, 0, 0),
     {"hit": False}),
    ("sphere_box_face_overlap_x", "test_sphere_box.cpp:14", sphere(1), tf(0, 0, 0), box(1, 1, 1),
     tf(1.8, 0, 0), {"hit": True, "normal": (0, 1.0, 0.05)}),
    ("sphere_box_face_overlap_y", "test_sphere_box.cpp:28", sphere(1), tf(0, 0, 0), box(1, 1, 1),
     tf(0, 1.7, 0), {"hit": True, "depth": (0.3, 0.05), "normal": (1, 1.0, 0.05)}),
    ("sphere_box_corner_region_no_hit", "test_sphere_box.cpp:43", sphere(1), tf(2, 2, 2), box(1, 1, 1),
     tf(0, 0, 0), {"hit": False}),
    ("sphere_box_corner_region_hit", "test_sphere_box.cpp:56", sphere(1), tf(1.5, 1.5, 1.5), box(1, 1, 1),
     tf(0, 0, 0), {"hit": True, "depth": (1.0 - 0.866, 0.01)}),
    ("sphere_box_centre_inside_box", "test_sphere_box.cpp:70", sphere(0.3), tf(0.1, 0.1, 0.1), box(2, 2, 2),
     tf(0, 0, 0), {"hit": True, "depth_positive": True}),
    ("sphere_capsule_separated", "test_sphere_capsule.cpp:6", sphere(1), tf(0, 4, 0), capsule(1, 0.5),
     tf(0, 0, 0), {"hit": False}),
    ("sphere_capsule_overlap_shaft", "test_sphere_capsule.cpp:18", sphere(1), tf(1.2, 0, 0), capsule(1, 0.5),
     tf(0, 0, 0), {"hit": True, "depth": (0.3, 0.02), "normal": (0, 1.0, 0.05)}),
    ("sphere_capsule_overlap_endpoint", "test_sphere_capsule.cpp:35", sphere(1), tf(0, 2, 0), capsule(1, 0.5),
     tf(0, 0, 0), {"hit": True, "depth": (0.5, 0.02)}),
    ("sphere_capsule_no_hit_endpoint", "test_sphere_capsule.cpp:52", sphere(1), tf(0, 3, 0), capsule(1, 0.5),
     tf(0, 0, 0), {"hit": False}),
    ("capsule_capsule_separated_parallel", "test_capsule_capsule.cpp:7", capsule(1, 0.5), tf(0, 0, 0),
     capsule(1, 0.5), tf(3, 0, 0), {"hit": False}),
    ("capsule_capsule_overlap_parallel", "test_capsule_capsule.cpp:17", capsule(1, 0.5), tf(0, 0, 0),
     capsule(1, 0.5), tf(0.8, 0, 0), {"hit": True, "depth": (0.2, 0.02), "normal": (0, 1.0, 0.05)}),
    ("capsule_capsule_overlap_perpendicular", "test_capsule_capsule.cpp:34", capsule(1, 0.5), tf(0, 0, 0),
     capsule(1, 0.5), tf(0, 0, 0, axis_quat((0, 0, 1), HALF_PI)), {"hit": True, "depth": (1.0, 0.05)}),
    ("capsule_capsule_overlap_crossing_offset", "test_capsule_capsule.cpp:52", capsule(1, 0.5), tf(0, 0, 0),
     capsule(1, 0.5), tf(0, 0, 0.6, axis_quat((0, 0, 1), HALF_PI)), {"hit": True, "depth": (0.4, 0.02)}),
    ("capsule_capsule_endpoint_to_endpoint", "test_capsule_capsule.cpp:68", capsule(1, 0.5), tf(0, 0, 0),
     capsule(1, 0.5), tf(0, 2.4, 0), {"hit": False}),  # collinear quirk (stale test expects a hit)
    ("capsule_capsule_separated_endpoint_gap", "test_capsule_capsule.cpp:84", capsule(1, 0.5), tf(0, 0, 0),
     capsule(1, 0.5), tf(0, 3.5, 0), {"hit": False}),
    ("box_box_separated_x", "test_box_box.cpp:8", box(1, 1, 1), tf(0, 0, 0), box(1, 1, 1), tf(2.5, 0, 0),
     {"hit": False}),
    ("box_box_face_overlap_x", "test_box_box.cpp:18", box(1, 1, 1), tf(0, 0, 0), box(1, 1, 1), tf(1.6, 0, 0),
     {"hit": True, "depth": (0.4, 0.01), "normal": (0, 1.0, 0.01)}),
    ("box_box_face_overlap_z", "test_box_box.cpp:33", box(1, 1, 1), tf(0, 0, 0), box(1, 1, 1), tf(0, 0, 1.8),
     {"hit": True, "depth": (0.2, 0.01), "normal": (2, 1.0, 0.01)}),
    ("box_box_minimum_axis_chosen", "test_box_box.cpp:48", box(1, 1, 1), tf(0, 0, 0), box(1, 1, 1),
     tf(0.5, 0.5, 1.8), {"hit": True, "depth": (0.2, 0.01), "normal": (2, 1.0, 0.01)}),
    ("box_box_deep_penetration", "test_box_box.cpp:64", box(3, 3, 3), tf(0, 0, 0), box(1, 1, 1),
     tf(0.2, 0, 0), {"hit": True, "depth_positive": True}),
    ("sphere_plane_above_no_hit", "test_plane_sphere.cpp:13", sphere(1), tf(0, 2, 0), plane(0, 1, 0, 0),
     tf(0, 0, 0), {"hit": False}),
    ("sphere_plane_just_touching_no_hit", "test_plane_sphere.cpp:24", sphere(1), tf(0, 1, 0), plane(0, 1, 0, 0),
     tf(0, 0, 0), {"hit": False}),
    ("sphere_plane_penetrating", "test_plane_sphere.cpp:34", sphere(1), tf(0, 0.7, 0), plane(0, 1, 0, 0),
     tf(0, 0, 0), {"hit": True, "depth": (0.3, 0.001), "normal": (1, -1.0, 0.001, "signed")}),
    ("sphere_plane_centre_on_plane", "test_plane_sphere.cpp:48", sphere(1), tf(0, 0, 0), plane(0, 1, 0, 0),
     tf(0, 0, 0), {"hit": True, "depth": (1.0, 0.001), "normal": (1, -1.0, 0.001, "signed")}),
    ("sphere_plane_deep_below", "test_plane_sphere.cpp:60", sphere(1), tf(0, -5, 0), plane(0, 1, 0, 0),
     tf(0, 0, 0), {"hit": True, "depth": (6.0, 0.001), "normal": (1, -1.0, 0.001, "signed")}),
    ("sphere_plane_diagonal_plane", "test_plane_sphere.cpp:72", sphere(1), tf(1, 1, 0),
     plane(INV_S2, INV_S2, 0, 0), tf(0, 0, 0), {"hit": False}),
    ("box_plane_above_no_hit", "test_plane_box.cpp:8", box(1, 1, 1), tf(0, 2, 0), plane(0, 1, 0, 0), tf(0, 0, 0),
     {"hit": False}),
    ("box_plane_face_penetrating", "test_plane_box.cpp:18", box(1, 1, 1), tf(0, 0.7, 0), plane(0, 1, 0, 0),
     tf(0, 0, 0), {"hit": True, "depth": (0.3, 0.001), "normal": (1, -1.0, 0.001, "signed")}),
    ("box_plane_corner_touching_no_hit", "test_plane_box.cpp:32", box(1, 1, 1),
     tf(0, S2, 0, axis_quat((0, 0, 1), QUARTER_PI)), plane(0, 1, 0, 0), tf(0, 0, 0),
     {"hit": True, "depth": (0.0, 1e-9)}),  # corner on the plane: kept by the 1e-4f slop
    ("box_plane_rotated_penetrating", "test_plane_box.cpp:44", box(1, 1, 1),
     tf(0, 1.2, 0, axis_quat((0, 0, 1), QUARTER_PI)), plane(0, 1, 0, 0), tf(0, 0, 0),
     {"hit": True, "depth": (S2 - 1.2, 0.01), "normal": (1, -1.0, 0.001, "signed")}),
    ("box_plane_fully_below", "test_plane_box.cpp:58", box(1, 1, 1), tf(0, -3, 0), plane(0, 1, 0, 0),
     tf(0, 0, 0), {"hit": True, "depth": (4.0, 0.001)}),
    ("capsule_plane_above_no_hit", "test_plane_capsule.cpp:7", capsule(1, 0.5), tf(0, 2, 0), plane(0, 1, 0, 0),
     tf(0, 0, 0), {"hit": False}),
    ("capsule_plane_upright_penetrating", "test_plane_capsule.cpp:18", capsule(1, 0.5), tf(0, 1, 0),
     plane(0, 1, 0, 0), tf(0, 0, 0), {"hit": True, "depth": (0.5, 0.001), "normal": (1, -1.0, 0.001, "signed")}),
    ("capsule_plane_horizontal_penetrating", "test_plane_capsule.cpp:32", capsule(1, 0.5),
     tf(0, 0.3, 0, axis_quat((0, 0, 1), HALF_PI)), plane(0, 1, 0, 0), tf(0, 0, 0),
     {"hit": True, "depth": (0.2, 0.01), "normal": (1, -1.0, 0.001, "signed")}),
    ("capsule_plane_tilted_45_penetrating", "test_plane_capsule.cpp:46", capsule(1, 0.5),
     tf(0, 1, 0, axis_quat((0, 0, 1), QUARTER_PI)), plane(0, 1, 0, 0), tf(0, 0, 0),
     {"hit": True, "depth": (math.sin(QUARTER_PI) + 0.5 - 1.0, 0.01), "normal": (1, -1.0, 0.001, "signed")}),
    ("convex_hull_plane_separated", "test_convex_hull_plane.cpp:104", hull("tet"), tf(0, 5, 0),
     plane(0, 1, 0, 0), tf(0, 0, 0), {"hit": False}),
    ("convex_hull_plane_penetrating", "test_convex_hull_plane.cpp:117", hull("tet"), tf(0, 0.7, 0),
     plane(0, 1, 0, 0), tf(0, 0, 0),
     {"hit": True, "n_points": 2, "depth_positive": True, "normal": (1, -1.0, 0.01, "signed")}),
    ("convex_hull_plane_reduction_4pts", "test_convex_hull_plane.cpp:143", hull("cube"), tf(0, 0.5, 0),
     plane(0, 1, 0, 0), tf(0, 0, 0),
     {"hit": True, "n_points": 4, "all_depths": (0.5, 0.01), "normal": (1, -1.0, 0.01, "signed")}),
    ("convex_hull_plane_deepest_always_kept", "test_convex_hull_plane.cpp:169", hull("cube"),
     tf(0, 0.5, 0, axis_quat((0, 0, 1), math.radians(30.0))), plane(0, 1, 0, 0), tf(0, 0, 0),
     {"hit": True, "max_depth_from_verts": ("cube", 0.01)}),
]

# Symmetry checks of the reference tests: collide(A, B) and collide(B, A)
# give the same depth and opposite normals.
SYMMETRY_CASES = [
    ("box_sphere_symmetry", "test_sphere_box.cpp:82", sphere(1), tf(0, 0, 0), box(1, 1, 1), tf(0, 1.7, 0)),
    ("sphere_capsule_symmetry", "test_sphere_capsule.cpp:62", sphere(1), tf(1.2, 0, 0), capsule(1, 0.5),
     tf(0, 0, 0)),
    ("sphere_plane_symmetry_plane_sphere", "test_plane_sphere.cpp:84", sphere(1), tf(0, 0.7, 0),
     plane(0, 1, 0, 0), tf(0, 0, 0)),
]


def descs(shapes):
    """Collider descriptor array from (kind, params, hull) tuples."""
    out = np.zeros(len(shapes), abi.COLLIDER_DT)
    for i, (kind, params, hid) in enumerate(shapes):
        out[i]["shape"] = kind
        out[i]["params"] = params
        out[i]["hull"] = hid
        out[i]["local_rot"] = (1, 0, 0, 0)
    return out


def rotate(q, v):
    w, x, y, z = q
    u = np.array([x, y, z])
    v = np.asarray(v, np.float64)
    return v + 2.0 * np.cross(u, np.cross(u, v) + w * v)


def random_quats(rng, n):
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


ANALYTIC_KINDS = ("sphere", "box", "capsule")
# convex shapes without analytic pair routines (GJK / EPA, one EPA point),
# with their own plane routines (PlaneCollision.hpp:40-61, 416-536)
ROUND_KINDS = ("ellipsoid", "cylinder", "cone")
HULL_NAMES = ("tet", "cube", "ellA", "ellB")
# hull scale: the fixture tet / cube span [-1, 1]; the ellipsoids ~0.5


def random_shape(rng, kind):
    if kind == "sphere":
        return sphere(rng.uniform(0.2, 0.6))
    if kind == "box":
        return box(*rng.uniform(0.2, 0.6, 3))
    if kind == "capsule":
        return capsule(rng.uniform(0.1, 0.5), rng.uniform(0.1, 0.3))
    if kind == "ellipsoid":
        return ellipsoid(*rng.uniform(0.2, 0.6, 3))
    if kind == "cylinder":
        return cylinder(rng.uniform(0.1, 0.5), rng.uniform(0.15, 0.5))
    if kind == "cone":
        return cone(rng.uniform(0.15, 0.5), rng.uniform(0.15, 0.5))
    raise ValueError(kind)


def random_pairs(seed, kind_a, kind_b, n, spread=1.2):
    """n shape pairs of the given kinds at random orientations, B placed
    around A within `spread` so that about half of them overlap.  Planes
    are the ground plane y = 0 (B) with A around it."""
    rng = np.random.default_rng(seed)
    sa, sb, ta, tb = [], [], [], []
    qa = random_quats(rng, n)
    qb = random_quats(rng, n)
    for i in range(n):
        a = random_shape(rng, kind_a) if kind_a != "hull" else hull(HULL_NAMES[i % 4])
        if kind_b == "plane":
            b = plane(0, 1, 0, 0)
            pa = (rng.uniform(-2, 2), rng.uniform(-0.6, 1.2), rng.uniform(-2, 2))
            pb = (0.0, 0.0, 0.0)
            qbi = (1.0, 0.0, 0.0, 0.0)
        else:
            b = random_shape(rng, kind_b) if kind_b != "hull" else hull(HULL_NAMES[(i // 4) % 4])
            pa = tuple(rng.uniform(-3, 3, 3))
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            pb = tuple(np.asarray(pa) + d * rng.uniform(0.0, spread))
            qbi = tuple(qb[i])
        sa.append(a)
        sb.append(b)
        ta.append(pa + tuple(qa[i]))
        tb.append(pb + qbi)
    return descs(sa), np.array(ta), descs(sb), np.array(tb)
