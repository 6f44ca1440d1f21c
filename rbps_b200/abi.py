"""numpy mirrors of the C ABI descriptor structs in include/rbps_gpu.h.

The dtypes use C alignment (``align=True``) so an array of them can be
passed to the ``rbps_world_add_*`` bulk entry points (and to the oracle
harness) as a plain pointer.
"""
import numpy as np

# status codes
OK = 0
ERR_INVALID = -1
ERR_CAPACITY = -2
ERR_CUDA = -3
ERR_NOT_CONVERGED = -4
ERR_STATE = -5
ERR_INTERNAL = -6

COLLIDE_MISS = 0
COLLIDE_HIT = 1
COLLIDE_UNSUPPORTED = 2

PRECISION_FP64 = 0
PRECISION_FP32 = 1
PRECISION_FP32_POS64 = 2

SOLVE_REFERENCE_ORDER = 0
SOLVE_COLORED = 1

BODY_STATIC = 0
BODY_DYNAMIC = 1

# rbc::Shape variant indices (rbc/shapes/ShapeTypes.hpp:67-69)
SHAPE_SPHERE = 0
SHAPE_BOX = 1
SHAPE_ELLIPSOID = 2
SHAPE_CAPSULE = 3
SHAPE_CYLINDER = 4
SHAPE_CONE = 5
SHAPE_PLANE = 6
SHAPE_HEIGHTMAP = 7
SHAPE_MESH = 8
SHAPE_CONVEX_HULL = 9

JOINT_PRISMATIC = 0
JOINT_REVOLUTE = 1
JOINT_FIXED = 2
JOINT_SPHERICAL = 3    # ball joint with a swing cone; no reference counterpart

ACTUATION_FREE = 0
ACTUATION_POSITION = 1
ACTUATION_SPEED = 2

BODY_DT = np.dtype([
    ("type", np.int32),
    ("mass", np.float64),
    ("inertia", np.float64, 6),
    ("position", np.float64, 3),
    ("orientation", np.float64, 4),
    ("linear_velocity", np.float64, 3),
    ("angular_velocity", np.float64, 3),
], align=True)

COLLIDER_DT = np.dtype([
    ("shape", np.int32),
    ("params", np.float64, 4),
    ("hull", np.uint32),
    ("body_id", np.uint32),
    ("is_static", np.int32),
    ("local_pos", np.float64, 3),
    ("local_rot", np.float64, 4),
    ("restitution", np.float64),
    ("static_friction", np.float64),
    ("dynamic_friction", np.float64),
], align=True)

JOINT_DT = np.dtype([
    ("type", np.int32),
    ("body_1", np.uint32),
    ("body_2", np.uint32),
    ("axis", np.float64, 3),
    ("limit_axis", np.float64, 3),
    ("r_1", np.float64, 3),
    ("r_2", np.float64, 3),
    ("actuation", np.int32),
    ("compliance", np.float64),
    ("damping", np.float64),
    ("limited", np.int32),
    ("lower_limit", np.float64),
    ("upper_limit", np.float64),
    ("target_position", np.float64),
    ("target_speed", np.float64),
], align=True)

CONTACT_DT = np.dtype([
    ("body_a", np.uint32), ("body_b", np.uint32),
    ("collider_a", np.uint32), ("collider_b", np.uint32),
    ("normal", np.float64, 3),
    ("r_a_local", np.float64, 3),
    ("r_b_local", np.float64, 3),
    ("point_on_a", np.float64, 3),
    ("point_on_b", np.float64, 3),
    ("penetration_depth", np.float64),
    ("normal_lambda", np.float64),
    ("tangent_lambda", np.float64),
    ("relative_velocity", np.float64),
    ("restitution", np.float64),
    ("static_friction", np.float64),
    ("dynamic_friction", np.float64),
    ("collision", np.int32),
    ("pad_", np.int32),
], align=True)

MANIFOLD_DT = np.dtype([
    ("status", np.int32),
    ("n_points", np.int32),
    ("normal", np.float64, 3),
    ("position", np.float64, (4, 3)),
    ("depth", np.float64, 4),
], align=True)

# byte sizes of the C structs (the CPU tests compile the header to check them)
STRUCT_SIZES = {"rbps_body_desc": 168, "rbps_collider_desc": 136, "rbps_joint_desc": 176, "rbps_contact": 200,
                "rbps_manifold": 160}
DTYPES = {"rbps_body_desc": BODY_DT, "rbps_collider_desc": COLLIDER_DT, "rbps_joint_desc": JOINT_DT,
          "rbps_contact": CONTACT_DT, "rbps_manifold": MANIFOLD_DT}


def body_default():
    """rbps::BodyParams{} (BodyAPI.hpp:22-31)."""
    b = np.zeros(1, BODY_DT)[0]
    b["type"] = BODY_DYNAMIC
    b["mass"] = 1.0
    b["inertia"] = (1.0, 1.0, 1.0, 0.0, 0.0, 0.0)
    b["orientation"] = (1.0, 0.0, 0.0, 0.0)
    return b


def collider_default():
    """rbps::ColliderParams{} (ColliderAPI.hpp:17-27); shape = Sphere{0.5}."""
    c = np.zeros(1, COLLIDER_DT)[0]
    c["shape"] = SHAPE_SPHERE
    c["params"] = (0.5, 0.0, 0.0, 0.0)
    c["local_rot"] = (1.0, 0.0, 0.0, 0.0)
    c["restitution"] = 0.5
    c["static_friction"] = 0.5
    c["dynamic_friction"] = 0.5
    return c


def joint_default(jtype=JOINT_REVOLUTE):
    """Revolute/Prismatic/FixedJointParams{} (JointAPI.hpp:24-57); a
    spherical joint defaults like a prismatic one (swing axis +x, no cone)."""
    j = np.zeros(1, JOINT_DT)[0]
    j["type"] = jtype
    if jtype != JOINT_FIXED:
        j["axis"] = (1.0, 0.0, 0.0)
    if jtype == JOINT_REVOLUTE:
        j["limit_axis"] = (0.0, 1.0, 0.0)
    return j
