"""Seeded synthetic scenes for the RBPS hot-path workloads.

Every scene is plain data (numpy arrays of the C ABI descriptor structs), so
the identical scene can be built in the GPU engine and in the reference
engine.  One ``numpy.random.Generator(PCG64(seed))`` per scene draws, per
body and in this order: shape type, size, orientation (normalised 4-D
Gaussian), position, velocity.

Mass properties use density 1000 kg/m^3 and the reference's unit-density
formulas (Sphere.hpp:54-80, Box.hpp:72-86, Capsule.hpp:83-118); gravity is
set explicitly through the body force, ``(0, -g*m, 0)``.
"""
from dataclasses import dataclass, field
from typing import List, Optional, Tuple
import math

import numpy as np

from . import abi

DENSITY = 1000.0
PI = 3.14159265358979323846


@dataclass
class WorldSpec:
    bodies: np.ndarray                 # abi.BODY_DT
    forces: np.ndarray                 # (n, 3) float64
    colliders: np.ndarray              # abi.COLLIDER_DT
    joints: np.ndarray                 # abi.JOINT_DT
    hulls: List[Tuple[np.ndarray, np.ndarray]] = field(default_factory=list)
    # (heights (rows, cols) float32, scale (3,), origin (3,)); a heightmap
    # collider's `hull` field indexes this list
    heightmaps: List[Tuple[np.ndarray, np.ndarray, np.ndarray]] = field(default_factory=list)
    # (vertices (n, 3), faces (m, 3)); a mesh collider's `hull` indexes this
    meshes: List[Tuple[np.ndarray, np.ndarray]] = field(default_factory=list)

    @property
    def n_bodies(self):
        return len(self.bodies)

    @property
    def n_dynamic(self):
        return int(np.count_nonzero(self.bodies["type"] == abi.BODY_DYNAMIC))


@dataclass
class Scene:
    name: str
    timestep: float
    substeps: int
    steps: int
    worlds: List[WorldSpec]
    description: str = ""

    @property
    def n_bodies(self):
        return sum(w.n_bodies for w in self.worlds)

    @property
    def n_dynamic(self):
        return sum(w.n_dynamic for w in self.worlds)


# ------------------------------------------------------------ mass properties
def sphere_mass(r):
    vol = (4.0 / 3.0) * PI * r * r * r
    i = (2.0 / 5.0) * vol * r * r
    return vol * DENSITY, np.array([i, i, i, 0.0, 0.0, 0.0]) * DENSITY


def box_mass(h):
    x2, y2, z2 = 4.0 * h[0] * h[0], 4.0 * h[1] * h[1], 4.0 * h[2] * h[2]
    vol = 8.0 * h[0] * h[1] * h[2]
    return vol * DENSITY, np.array([(1.0 / 12.0) * vol * (y2 + z2),
                                    (1.0 / 12.0) * vol * (x2 + z2),
                                    (1.0 / 12.0) * vol * (x2 + y2), 0.0, 0.0, 0.0]) * DENSITY


def capsule_mass(hh, r):
    r2, h2 = r * r, hh * hh
    vol = PI * r * r * (2.0 * hh + (4.0 / 3.0) * r)
    m_cyl = PI * r2 * 2.0 * hh
    m_hemi = vol - m_cyl
    iyy = (m_cyl * r2 / 2.0) + (m_hemi * 2.0 * r2 / 5.0)
    d = hh + 3.0 * r / 8.0
    ixx = m_cyl * (r2 / 4.0 + h2 / 3.0) + m_hemi * (2.0 * r2 / 5.0 + d * d)
    return vol * DENSITY, np.array([ixx, iyy, ixx, 0.0, 0.0, 0.0]) * DENSITY


def ellipsoid_mass(a):
    """Ellipsoid.hpp compute_volume / compute_inertia_tensor (x density)."""
    vol = (4.0 / 3.0) * PI * a[0] * a[1] * a[2]
    ax2, ay2, az2 = a[0] * a[0], a[1] * a[1], a[2] * a[2]
    inertia = np.array([(2.0 / 5.0) * vol * (ay2 + az2), (2.0 / 5.0) * vol * (ax2 + az2),
                        (2.0 / 5.0) * vol * (ax2 + ay2), 0.0, 0.0, 0.0])
    return vol * DENSITY, inertia * DENSITY


def cylinder_mass(hh, r):
    """Cylinder.hpp compute_volume / compute_inertia_tensor (x density)."""
    vol = PI * r * r * (2.0 * hh)
    r2, h2 = r * r, (2.0 * hh) * (2.0 * hh)
    iyy = 0.5 * vol * r2
    ixx = (1.0 / 12.0) * vol * (3.0 * r2 + h2)
    return vol * DENSITY, np.array([ixx, iyy, ixx, 0.0, 0.0, 0.0]) * DENSITY


def cone_mass(hh, r):
    """Cone.hpp compute_volume / compute_inertia_tensor (x density)."""
    vol = (1.0 / 3.0) * PI * r * r * (2.0 * hh)
    r2, h = r * r, 2.0 * hh
    iyy = (3.0 / 10.0) * vol * r2
    ixx_apex = (3.0 / 5.0) * vol * (r2 / 4.0 + h * h)
    d = 3.0 * h / 8.0 - hh
    return vol * DENSITY, np.array([ixx_apex - vol * d * d, iyy, ixx_apex - vol * d * d, 0.0, 0.0, 0.0]) * DENSITY


def hull_mass(verts, tris):
    """Volume and inertia about the origin of a closed CCW triangle mesh
    (signed tetrahedra from the origin), scaled by the density."""
    a, b, c = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    det = np.einsum("ij,ij->i", a, np.cross(b, c))
    vol = det.sum() / 6.0
    # second moments of each tetra (origin, a, b, c)
    def s(u, v):
        return (a[:, u] * a[:, v] + b[:, u] * b[:, v] + c[:, u] * c[:, v]
                + (a[:, u] + b[:, u] + c[:, u]) * (a[:, v] + b[:, v] + c[:, v])) / 120.0 * det
    sxx, syy, szz = s(0, 0).sum(), s(1, 1).sum(), s(2, 2).sum()
    sxy, sxz, syz = s(0, 1).sum(), s(0, 2).sum(), s(1, 2).sum()
    inertia = np.array([syy + szz, sxx + szz, sxx + syy, -sxy, -sxz, -syz])
    return vol * DENSITY, inertia * DENSITY


# ------------------------------------------------------------------ helpers
def random_quats(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def _ground(bodies, colliders, forces, friction, restitution, offset=(0.0, 0.0, 0.0)):
    """Static ground body (id 0) with Plane{(0,1,0), 0} (Plane.hpp:32-58)."""
    b = abi.body_default()
    b["type"] = abi.BODY_STATIC
    b["mass"] = 0.0
    b["position"] = offset
    bodies.append(b)
    forces.append((0.0, 0.0, 0.0))
    c = abi.collider_default()
    c["shape"] = abi.SHAPE_PLANE
    c["params"] = (0.0, 1.0, 0.0, 0.0)
    c["body_id"] = 0
    c["is_static"] = 1
    c["restitution"] = restitution
    c["static_friction"] = friction
    c["dynamic_friction"] = friction
    colliders.append(c)


def _dyn_body(pos, quat, mass, inertia, vel=(0.0, 0.0, 0.0), g=9.81):
    b = abi.body_default()
    b["type"] = abi.BODY_DYNAMIC
    b["mass"] = mass
    b["inertia"] = inertia
    b["position"] = pos
    b["orientation"] = quat
    b["linear_velocity"] = vel
    return b, (0.0, -g * mass, 0.0)


def _collider(shape, params, body, friction, restitution, hull=0):
    c = abi.collider_default()
    c["shape"] = shape
    p = list(params) + [0.0] * (4 - len(params))
    c["params"] = p
    c["hull"] = hull
    c["body_id"] = body
    c["restitution"] = restitution
    c["static_friction"] = friction
    c["dynamic_friction"] = friction
    return c


def _finish(bodies, forces, colliders, joints, hulls=None):
    return WorldSpec(
        bodies=np.array(bodies, dtype=abi.BODY_DT),
        forces=np.array(forces, dtype=np.float64).reshape(-1, 3),
        colliders=np.array(colliders, dtype=abi.COLLIDER_DT),
        joints=np.array(joints, dtype=abi.JOINT_DT) if joints else np.zeros(0, abi.JOINT_DT),
        hulls=hulls or [])


def box_sphere_world(rng, n, friction=0.5, restitution=0.0,
                     lo=(-5.0, 1.0, -5.0), hi=(5.0, 21.0, 5.0), g=9.81,
                     ground=True, size=(0.2, 0.5)):
    """A ground plane plus n bodies, each a box (half-extents U[size]^3) or a
    sphere (radius U[size]) with probability 1/2, uniform random orientation,
    position uniform in [lo, hi], at rest.  Returns lists of descriptor
    records (bodies, forces, colliders) that callers may extend."""
    bodies, forces, colliders = [], [], []
    if ground:
        _ground(bodies, colliders, forces, friction, restitution)
    is_box = rng.random(n) < 0.5
    box_h = rng.uniform(size[0], size[1], (n, 3))
    sph_r = rng.uniform(size[0], size[1], n)
    quats = random_quats(rng, n)
    pos = rng.uniform(lo, hi, (n, 3))
    # vectorised mass properties (same formulas as box_mass / sphere_mass)
    hx, hy, hz = box_h[:, 0], box_h[:, 1], box_h[:, 2]
    bvol = 8.0 * hx * hy * hz
    x2, y2, z2 = 4.0 * hx * hx, 4.0 * hy * hy, 4.0 * hz * hz
    binert = np.stack([(1.0 / 12.0) * bvol * (y2 + z2), (1.0 / 12.0) * bvol * (x2 + z2),
                       (1.0 / 12.0) * bvol * (x2 + y2)], 1)
    svol = (4.0 / 3.0) * PI * sph_r * sph_r * sph_r
    sinert = (2.0 / 5.0) * svol * sph_r * sph_r
    b = np.zeros(n, abi.BODY_DT)
    b["type"] = abi.BODY_DYNAMIC
    b["mass"] = np.where(is_box, bvol, svol) * DENSITY
    inert = np.zeros((n, 6))
    inert[:, :3] = np.where(is_box[:, None], binert, sinert[:, None]) * DENSITY
    b["inertia"] = inert
    b["position"] = pos
    b["orientation"] = quats
    c = np.zeros(n, abi.COLLIDER_DT)
    c["shape"] = np.where(is_box, abi.SHAPE_BOX, abi.SHAPE_SPHERE)
    params = np.zeros((n, 4))
    params[:, :3] = np.where(is_box[:, None], box_h, np.stack([sph_r, np.zeros(n), np.zeros(n)], 1))
    c["params"] = params
    c["body_id"] = np.arange(len(bodies), len(bodies) + n)
    c["local_rot"] = (1.0, 0.0, 0.0, 0.0)
    c["restitution"] = restitution
    c["static_friction"] = friction
    c["dynamic_friction"] = friction
    f = np.zeros((n, 3))
    f[:, 1] = -g * b["mass"]
    bodies.extend(list(b))
    forces.extend(list(map(tuple, f)))
    colliders.extend(list(c))
    return bodies, forces, colliders


def capsule_chain(bodies, forces, colliders, joints, origin, n_links=13, radius=0.1,
                  half_height=0.2, friction=0.5, restitution=0.0, g=9.81,
                  limit=None, compliance=0.0, damping=0.0, gap=0.02):
    """n_links capsules laid along +X from `origin`, each link's local Y axis
    mapped to world X, joined by revolute joints about world Z
    (RevoluteJointParams, JointAPI.hpp:43-57) at anchors `gap` beyond the
    capsule tips.  The defaults are the settings under which the reference
    engine stays finite: with tips touching (gap=0), or with joint damping /
    angle limits among falling bodies, the reference's joint rows and
    contacts fight and its chains blow up to NaN within a few hundred steps."""
    q = (math.cos(-PI / 4.0), 0.0, 0.0, math.sin(-PI / 4.0))  # local +Y -> world +X
    reach = half_height + radius + gap
    m, inertia = capsule_mass(half_height, radius)
    first = len(bodies)
    for k in range(n_links):
        pos = (origin[0] + k * 2.0 * reach, origin[1], origin[2])
        b, f = _dyn_body(pos, q, m, inertia, g=g)
        bid = len(bodies)
        bodies.append(b)
        forces.append(f)
        colliders.append(_collider(abi.SHAPE_CAPSULE, [half_height, radius], bid, friction, restitution))
    for k in range(n_links - 1):
        j = abi.joint_default(abi.JOINT_REVOLUTE)
        j["body_1"] = first + k
        j["body_2"] = first + k + 1
        j["axis"] = (0.0, 0.0, 1.0)
        j["limit_axis"] = (0.0, 1.0, 0.0)
        j["r_1"] = (0.0, reach, 0.0)
        j["r_2"] = (0.0, -reach, 0.0)
        j["compliance"] = compliance
        j["damping"] = damping
        j["limited"] = 1 if limit is not None else 0
        j["lower_limit"] = -(limit or 0.0)
        j["upper_limit"] = (limit or 0.0)
        joints.append(j)


# ------------------------------------------------------------------ configs
def config0(seed=0, n_bodies=512, steps=600):
    """Plain single world, FP64: 256 boxes + 256 spheres (equal split of the
    types, shuffled), sizes U[0.2,0.5], random orientation, positions in
    [-5,5]x[1,21]x[-5,5] over a static ground plane, at rest, g=-9.81,
    dt=1/60, 10 substeps, friction 0.5, restitution 0."""
    rng = np.random.Generator(np.random.PCG64(seed))
    bodies, forces, colliders = [], [], []
    _ground(bodies, colliders, forces, 0.5, 0.0)
    types = np.array([1] * (n_bodies // 2) + [0] * (n_bodies - n_bodies // 2))
    rng.shuffle(types)
    box_h = rng.uniform(0.2, 0.5, (n_bodies, 3))
    sph_r = rng.uniform(0.2, 0.5, n_bodies)
    quats = random_quats(rng, n_bodies)
    pos = rng.uniform((-5.0, 1.0, -5.0), (5.0, 21.0, 5.0), (n_bodies, 3))
    for i in range(n_bodies):
        bid = len(bodies)
        if types[i]:
            m, inertia = box_mass(box_h[i])
            c = _collider(abi.SHAPE_BOX, box_h[i], bid, 0.5, 0.0)
        else:
            m, inertia = sphere_mass(sph_r[i])
            c = _collider(abi.SHAPE_SPHERE, [sph_r[i]], bid, 0.5, 0.0)
        b, f = _dyn_body(pos[i], quats[i], m, inertia)
        bodies.append(b)
        forces.append(f)
        colliders.append(c)
    w = _finish(bodies, forces, colliders, [])
    return Scene("config0_plain_fp64", 1.0 / 60.0, 10, steps, [w],
                 f"{n_bodies} boxes+spheres over a ground plane, seed {seed}")


def config1(seed=0, n_bodies=65536, steps=1, n_hull_shapes=None, extent=200.0):
    """Collision stress, one world: n_bodies split equally (shuffled) among
    spheres (r U[0.2,0.5]), boxes (half-extents U[0.2,0.5]^3), capsules
    (half-height U[0.1,0.5], r U[0.1,0.3]) and convex hulls (quickhull of
    16-32 points on an ellipsoid with semi-axes U[0.2,1]); random
    orientation, positions U[0, extent]^3, velocities N(0, 2 m/s) per axis;
    no ground plane, g=-9.81, dt=1/60, 10 substeps.

    Every hull body gets its own hull shape unless n_hull_shapes caps the
    number of distinct shapes (then body k uses shape k mod n_hull_shapes).
    Points are Gaussian directions scaled by the semi-axes."""
    import rbps_b200
    rng = np.random.Generator(np.random.PCG64(seed))
    q = n_bodies // 4
    types = np.array([0] * (n_bodies - 3 * q) + [1] * q + [2] * q + [3] * q)
    rng.shuffle(types)
    n_hull = int(np.count_nonzero(types == 3))
    n_shapes = n_hull if n_hull_shapes is None else max(1, min(n_hull, n_hull_shapes))
    hulls = []
    for _ in range(n_shapes):
        m = int(rng.integers(16, 33))
        d = rng.standard_normal((m, 3))
        pts = d / np.linalg.norm(d, axis=1, keepdims=True) * rng.uniform(0.2, 1.0, 3)
        hulls.append((pts, rbps_b200.quickhull(pts)))
    hull_props = [hull_mass(v, t) for v, t in hulls]
    sph_r = rng.uniform(0.2, 0.5, n_bodies)
    box_h = rng.uniform(0.2, 0.5, (n_bodies, 3))
    cap_hh = rng.uniform(0.1, 0.5, n_bodies)
    cap_r = rng.uniform(0.1, 0.3, n_bodies)
    quats = random_quats(rng, n_bodies)
    pos = rng.uniform(0.0, extent, (n_bodies, 3))
    vel = rng.normal(0.0, 2.0, (n_bodies, 3))
    bodies, forces, colliders = [], [], []
    k_hull = 0
    for i in range(n_bodies):
        t = types[i]
        if t == 0:
            m, inertia = sphere_mass(sph_r[i])
            c = _collider(abi.SHAPE_SPHERE, [sph_r[i]], i, 0.5, 0.0)
        elif t == 1:
            m, inertia = box_mass(box_h[i])
            c = _collider(abi.SHAPE_BOX, box_h[i], i, 0.5, 0.0)
        elif t == 2:
            m, inertia = capsule_mass(cap_hh[i], cap_r[i])
            c = _collider(abi.SHAPE_CAPSULE, [cap_hh[i], cap_r[i]], i, 0.5, 0.0)
        else:
            h = k_hull % n_shapes
            k_hull += 1
            m, inertia = hull_props[h]
            c = _collider(abi.SHAPE_CONVEX_HULL, [], i, 0.5, 0.0, hull=h)
        b, f = _dyn_body(pos[i], quats[i], m, inertia, vel=vel[i])
        bodies.append(b)
        forces.append(f)
        colliders.append(c)
    w = _finish(bodies, forces, colliders, [], hulls)
    return Scene("config1_collision_stress", 1.0 / 60.0, 10, steps, [w],
                 f"{n_bodies} spheres/boxes/capsules/hulls in {extent:g}^3 m, seed {seed}")


def config2(seed=0, n_chains=1024, n_links=32, steps=300, radius=0.05, half_height=0.15, mass=1.0,
            spacing=1.0, cone_deg=60.0, compliance=1e-6, max_angle_deg=30.0, gap=0.04, friction=0.5):
    """Joint-heavy single world: n_chains chains of n_links capsules (radius
    0.05 m, segment 2 * half_height = 0.3 m, 1 kg each) hanging from static
    anchors on a square grid `spacing` m apart, joined by ball joints with a
    60 degree swing cone about the links' axes and compliance 1e-6; every
    joint starts bent by an angle U[-30, 30] degrees about a random
    horizontal axis of its parent; no ground, g=-9.81, dt=1/60, 8 substeps.

    A link's local +Y is its capsule axis (identity = hanging straight
    down, pivot above the centre); pivots sit `gap`/2 beyond the capsule
    tips, so neighbouring links clear each other anywhere inside the cone."""
    rng = np.random.Generator(np.random.PCG64(seed))
    side = int(math.ceil(math.sqrt(n_chains)))
    reach = half_height + radius + 0.5 * gap
    m0, inertia0 = capsule_mass(half_height, radius)
    inertia = inertia0 * (mass / m0)
    cone = cone_deg * PI / 180.0
    amax = max_angle_deg * PI / 180.0
    bodies, forces, colliders, joints = [], [], [], []

    def qmul(a, b):
        return (a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
                a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
                a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
                a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0])

    def qrot(q, v):
        w, x, y, z = q
        u = np.array([x, y, z])
        v = np.asarray(v, np.float64)
        t = 2.0 * np.cross(u, v)
        return v + w * t + np.cross(u, t)

    for c in range(n_chains):
        anchor = np.array([(c % side) * spacing, 0.0, (c // side) * spacing])
        a = abi.body_default()
        a["type"] = abi.BODY_STATIC
        a["mass"] = 0.0
        a["position"] = anchor
        parent = len(bodies)
        bodies.append(a)
        forces.append((0.0, 0.0, 0.0))
        q_par = (1.0, 0.0, 0.0, 0.0)
        pivot = anchor
        for k in range(n_links):
            phi = rng.uniform(0.0, 2.0 * PI)
            ang = rng.uniform(-amax, amax)
            s = math.sin(0.5 * ang)
            q = qmul(q_par, (math.cos(0.5 * ang), math.cos(phi) * s, 0.0, math.sin(phi) * s))
            n = math.sqrt(sum(x * x for x in q))
            q = tuple(x / n for x in q)
            pos = pivot - qrot(q, (0.0, reach, 0.0))
            b, f = _dyn_body(tuple(pos), q, mass, inertia)
            bid = len(bodies)
            bodies.append(b)
            forces.append(f)
            colliders.append(_collider(abi.SHAPE_CAPSULE, [half_height, radius], bid, friction, 0.0))
            j = abi.joint_default(abi.JOINT_SPHERICAL)
            j["body_1"] = parent
            j["body_2"] = bid
            j["axis"] = (0.0, 1.0, 0.0)
            j["r_1"] = (0.0, 0.0, 0.0) if k == 0 else (0.0, -reach, 0.0)
            j["r_2"] = (0.0, reach, 0.0)
            j["compliance"] = compliance
            j["limited"] = 1
            j["upper_limit"] = cone
            joints.append(j)
            parent, q_par = bid, q
            pivot = pos - qrot(q, (0.0, reach, 0.0))
    w = _finish(bodies, forces, colliders, joints)
    return Scene("config2_joint_heavy", 1.0 / 60.0, 8, steps, [w],
                 f"{n_chains} chains x {n_links} capsules, ball joints with a {cone_deg:g} deg cone, seed {seed}")


def config3(seed=0, n_worlds=4096, steps=1000, lo_bodies=8, hi_bodies=512, chain=True):
    """Batched uneven worlds: per world n ~ log-uniform[8,512] boxes/spheres
    (as config0) + one 13-link revolute capsule chain + ground plane,
    dt=1/120, 4 substeps.  chain=False leaves the chains out and keeps every
    other draw (the same boxes and spheres)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = np.floor(np.exp(rng.uniform(math.log(lo_bodies), math.log(hi_bodies + 1), n_worlds))).astype(int)
    counts = np.clip(counts, lo_bodies, hi_bodies)
    worlds = []
    for w in range(n_worlds):
        bodies, forces, colliders = box_sphere_world(rng, int(counts[w]))
        joints = []
        origin = (rng.uniform(-4.5, -3.5), rng.uniform(1.0, 21.0), rng.uniform(-5.0, 5.0))
        if chain:
            capsule_chain(bodies, forces, colliders, joints, origin)
        worlds.append(_finish(bodies, forces, colliders, joints))
    return Scene("config3_batched_fp32", 1.0 / 120.0, 4, steps, worlds,
                 f"{n_worlds} worlds, bodies log-uniform[{lo_bodies},{hi_bodies}] + 13-link chain, seed {seed}")


def config4(seed=0, n_worlds=256, steps=2000, height=64, offset=1.0e4, mass_ratio=1.0e-3):
    """Precision stress: per world a tower of `height` boxes (half-extent
    0.5), densities alternating 1:1000 (`mass_ratio`; 1.0 gives a uniform
    tower), offset `offset` m from the origin plus a uniform horizontal
    jitter, ground plane at the offset, friction 0.8, 20 substeps."""
    rng = np.random.Generator(np.random.PCG64(seed))
    worlds = []
    for w in range(n_worlds):
        ox = offset + rng.uniform(-50.0, 50.0)
        oz = offset + rng.uniform(-50.0, 50.0)
        bodies, forces, colliders = [], [], []
        _ground(bodies, colliders, forces, 0.8, 0.0, offset=(ox, 0.0, oz))
        h = np.array([0.5, 0.5, 0.5])
        for k in range(height):
            m, inertia = box_mass(h)
            scale = 1.0 if k % 2 == 0 else mass_ratio
            b, f = _dyn_body((ox, 0.5 + k * 1.0, oz), (1.0, 0.0, 0.0, 0.0), m * scale, inertia * scale)
            bid = len(bodies)
            bodies.append(b)
            forces.append(f)
            colliders.append(_collider(abi.SHAPE_BOX, h, bid, 0.8, 0.0))
        worlds.append(_finish(bodies, forces, colliders, []))
    return Scene("config4_precision", 1.0 / 60.0, 20, steps, worlds,
                 f"{n_worlds} towers of {height} boxes at {offset} m, seed {seed}")


def small_world(seed=0, n=64, **kw):
    """A config0-style world with n bodies (for fast parity tests)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    bodies, forces, colliders = box_sphere_world(rng, n, **kw)
    return _finish(bodies, forces, colliders, [])


def chain_world(seed=0, n_bodies=16, n_links=13, **kw):
    rng = np.random.Generator(np.random.PCG64(seed))
    bodies, forces, colliders = box_sphere_world(rng, n_bodies)
    joints = []
    origin = (rng.uniform(-4.5, -3.5), rng.uniform(1.0, 21.0), rng.uniform(-5.0, 5.0))
    capsule_chain(bodies, forces, colliders, joints, origin, n_links=n_links, **kw)
    return _finish(bodies, forces, colliders, joints)


def capsule_world(seed=0, n=48, friction=0.5, restitution=0.0):
    """Ground plane + a mix of capsules, boxes and spheres (exercises the
    capsule pair routines)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    bodies, forces, colliders = [], [], []
    _ground(bodies, colliders, forces, friction, restitution)
    kind = rng.integers(0, 3, n)
    quats = random_quats(rng, n)
    pos = rng.uniform((-3.0, 1.0, -3.0), (3.0, 9.0, 3.0), (n, 3))
    for i in range(n):
        bid = len(bodies)
        if kind[i] == 0:
            hh, r = rng.uniform(0.1, 0.5), rng.uniform(0.1, 0.3)
            m, inertia = capsule_mass(hh, r)
            c = _collider(abi.SHAPE_CAPSULE, [hh, r], bid, friction, restitution)
        elif kind[i] == 1:
            h = rng.uniform(0.2, 0.5, 3)
            m, inertia = box_mass(h)
            c = _collider(abi.SHAPE_BOX, h, bid, friction, restitution)
        else:
            r = rng.uniform(0.2, 0.5)
            m, inertia = sphere_mass(r)
            c = _collider(abi.SHAPE_SPHERE, [r], bid, friction, restitution)
        b, f = _dyn_body(pos[i], quats[i], m, inertia)
        bodies.append(b)
        forces.append(f)
        colliders.append(c)
    return _finish(bodies, forces, colliders, [])


def round_world(seed=0, n=24, friction=0.5, restitution=0.0):
    """Ground plane + ellipsoids, cylinders, cones, boxes and spheres
    dropped close to the ground: the ellipsoid / cylinder / cone plane
    routines and their GJK / EPA pairs."""
    rng = np.random.Generator(np.random.PCG64(seed))
    bodies, forces, colliders = [], [], []
    _ground(bodies, colliders, forces, friction, restitution)
    kind = rng.integers(0, 5, n)
    quats = random_quats(rng, n)
    pos = rng.uniform((-2.0, 0.6, -2.0), (2.0, 3.0, 2.0), (n, 3))
    for i in range(n):
        bid = len(bodies)
        if kind[i] == 0:
            a = rng.uniform(0.2, 0.45, 3)
            m, inertia = ellipsoid_mass(a)
            c = _collider(abi.SHAPE_ELLIPSOID, a, bid, friction, restitution)
        elif kind[i] == 1:
            hh, r = rng.uniform(0.15, 0.4), rng.uniform(0.15, 0.4)
            m, inertia = cylinder_mass(hh, r)
            c = _collider(abi.SHAPE_CYLINDER, [hh, r], bid, friction, restitution)
        elif kind[i] == 2:
            hh, r = rng.uniform(0.15, 0.4), rng.uniform(0.15, 0.4)
            m, inertia = cone_mass(hh, r)
            c = _collider(abi.SHAPE_CONE, [hh, r], bid, friction, restitution)
        elif kind[i] == 3:
            h = rng.uniform(0.2, 0.4, 3)
            m, inertia = box_mass(h)
            c = _collider(abi.SHAPE_BOX, h, bid, friction, restitution)
        else:
            r = rng.uniform(0.2, 0.4)
            m, inertia = sphere_mass(r)
            c = _collider(abi.SHAPE_SPHERE, [r], bid, friction, restitution)
        b, f = _dyn_body(pos[i], quats[i], m, inertia)
        bodies.append(b)
        forces.append(f)
        colliders.append(c)
    return _finish(bodies, forces, colliders, [])


def terrain_heights(rng, rows=33, cols=33, amp=0.6):
    """Smooth random terrain: a sum of a few random bumps (float32)."""
    r, c = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    h = np.zeros((rows, cols))
    for _ in range(6):
        cr, cc = rng.uniform(0, rows), rng.uniform(0, cols)
        w = rng.uniform(3.0, 8.0)
        h += rng.uniform(-1.0, 1.0) * np.exp(-((r - cr) ** 2 + (c - cc) ** 2) / (2.0 * w * w))
    return (amp * h).astype(np.float32)


def terrain_world(seed=0, n=32, rows=33, cols=33, cell=0.5, friction=0.5, restitution=0.0):
    """A static heightmap terrain (rows x cols samples, `cell` m apart,
    centred on the origin) with spheres, boxes and capsules dropped onto it
    (HeightmapCollision.hpp's sphere / capsule / box routines)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    heights = terrain_heights(rng, rows, cols)
    origin = np.array([-0.5 * (cols - 1) * cell, 0.0, -0.5 * (rows - 1) * cell])
    scale = np.array([cell, 1.0, cell])
    bodies, forces, colliders = [], [], []
    g = abi.body_default()
    g["type"] = abi.BODY_STATIC
    g["mass"] = 0.0
    bodies.append(g)
    forces.append((0.0, 0.0, 0.0))
    c = abi.collider_default()
    c["shape"] = abi.SHAPE_HEIGHTMAP
    c["hull"] = 0
    c["body_id"] = 0
    c["is_static"] = 1
    c["restitution"] = restitution
    c["static_friction"] = friction
    c["dynamic_friction"] = friction
    colliders.append(c)
    kind = rng.integers(0, 3, n)
    quats = random_quats(rng, n)
    half = 0.4 * (cols - 1) * cell
    pos = rng.uniform((-half, 1.2, -half), (half, 3.5, half), (n, 3))
    for i in range(n):
        bid = len(bodies)
        if kind[i] == 0:
            r = rng.uniform(0.2, 0.4)
            m, inertia = sphere_mass(r)
            cl = _collider(abi.SHAPE_SPHERE, [r], bid, friction, restitution)
        elif kind[i] == 1:
            h = rng.uniform(0.2, 0.4, 3)
            m, inertia = box_mass(h)
            cl = _collider(abi.SHAPE_BOX, h, bid, friction, restitution)
        else:
            hh, r = rng.uniform(0.1, 0.4), rng.uniform(0.1, 0.25)
            m, inertia = capsule_mass(hh, r)
            cl = _collider(abi.SHAPE_CAPSULE, [hh, r], bid, friction, restitution)
        b, f = _dyn_body(pos[i], quats[i], m, inertia)
        bodies.append(b)
        forces.append(f)
        colliders.append(cl)
    w = _finish(bodies, forces, colliders, [])
    w.heightmaps = [(heights, scale, origin)]
    return w


def grid_mesh(heights, cell, origin):
    """An open triangle mesh over a height grid (2 triangles per cell, CCW
    seen from +Y): vertices (rows * cols, 3) and faces (m, 3)."""
    rows, cols = heights.shape
    r, c = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    verts = np.stack([origin[0] + c * cell, heights.astype(np.float64), origin[2] + r * cell], -1).reshape(-1, 3)
    faces = []
    for i in range(rows - 1):
        for j in range(cols - 1):
            v00, v01, v10, v11 = i * cols + j, i * cols + j + 1, (i + 1) * cols + j, (i + 1) * cols + j + 1
            faces.append((v00, v10, v01))
            faces.append((v10, v11, v01))
    return verts, np.array(faces, np.uint32)


def mesh_world(seed=0, n=24, rows=17, cols=17, cell=0.75, friction=0.5, restitution=0.0):
    """A static bumpy ground mesh (an open grid mesh) with spheres, boxes
    and capsules dropped onto it (MeshCollision.hpp's routines)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    heights = terrain_heights(rng, rows, cols, amp=0.5)
    origin = np.array([-0.5 * (cols - 1) * cell, 0.0, -0.5 * (rows - 1) * cell])
    verts, faces = grid_mesh(heights, cell, origin)
    bodies, forces, colliders = [], [], []
    g = abi.body_default()
    g["type"] = abi.BODY_STATIC
    g["mass"] = 0.0
    bodies.append(g)
    forces.append((0.0, 0.0, 0.0))
    c = abi.collider_default()
    c["shape"] = abi.SHAPE_MESH
    c["hull"] = 0
    c["body_id"] = 0
    c["is_static"] = 1
    c["restitution"] = restitution
    c["static_friction"] = friction
    c["dynamic_friction"] = friction
    colliders.append(c)
    kind = rng.integers(0, 3, n)
    quats = random_quats(rng, n)
    half = 0.4 * (cols - 1) * cell
    pos = rng.uniform((-half, 1.2, -half), (half, 3.5, half), (n, 3))
    for i in range(n):
        bid = len(bodies)
        if kind[i] == 0:
            r = rng.uniform(0.2, 0.4)
            m, inertia = sphere_mass(r)
            cl = _collider(abi.SHAPE_SPHERE, [r], bid, friction, restitution)
        elif kind[i] == 1:
            h = rng.uniform(0.2, 0.4, 3)
            m, inertia = box_mass(h)
            cl = _collider(abi.SHAPE_BOX, h, bid, friction, restitution)
        else:
            hh, r = rng.uniform(0.1, 0.4), rng.uniform(0.1, 0.25)
            m, inertia = capsule_mass(hh, r)
            cl = _collider(abi.SHAPE_CAPSULE, [hh, r], bid, friction, restitution)
        b, f = _dyn_body(pos[i], quats[i], m, inertia)
        bodies.append(b)
        forces.append(f)
        colliders.append(cl)
    w = _finish(bodies, forces, colliders, [])
    w.meshes = [(verts, faces)]
    return w


def hull_world(seed=0, n=24, n_shapes=4, friction=0.5, restitution=0.0):
    """Ground plane + convex hulls, boxes and spheres dropped close to the
    ground (exercises GJK / EPA and the hull manifolds).  Hull shapes are the
    quickhull of 16-32 points on ellipsoids with semi-axes U[0.2, 0.6]; hull
    mass and inertia from the closed mesh about the vertex origin."""
    import rbps_b200
    rng = np.random.Generator(np.random.PCG64(seed))
    hulls = []
    for k in range(n_shapes):
        m = int(rng.integers(16, 33))
        d = rng.standard_normal((m, 3))
        pts = d / np.linalg.norm(d, axis=1, keepdims=True) * rng.uniform(0.2, 0.6, 3)
        hulls.append((pts, rbps_b200.quickhull(pts)))
    bodies, forces, colliders = [], [], []
    _ground(bodies, colliders, forces, friction, restitution)
    kind = rng.integers(0, 4, n)
    quats = random_quats(rng, n)
    pos = rng.uniform((-2.0, 0.6, -2.0), (2.0, 3.0, 2.0), (n, 3))
    for i in range(n):
        bid = len(bodies)
        if kind[i] <= 1:
            h = int(rng.integers(0, n_shapes))
            m, inertia = hull_mass(hulls[h][0], hulls[h][1])
            c = _collider(abi.SHAPE_CONVEX_HULL, [], bid, friction, restitution, hull=h)
        elif kind[i] == 2:
            h = rng.uniform(0.2, 0.4, 3)
            m, inertia = box_mass(h)
            c = _collider(abi.SHAPE_BOX, h, bid, friction, restitution)
        else:
            r = rng.uniform(0.2, 0.4)
            m, inertia = sphere_mass(r)
            c = _collider(abi.SHAPE_SPHERE, [r], bid, friction, restitution)
        b, f = _dyn_body(pos[i], quats[i], m, inertia)
        bodies.append(b)
        forces.append(f)
        colliders.append(c)
    return _finish(bodies, forces, colliders, [], hulls)


def with_state(scene, states, worlds=None):
    """The same worlds restarted from given states: a new Scene whose bodies
    start at `states[k]` (dicts with position, orientation, linear_velocity,
    angular_velocity per body, as Batch.state returns) for world
    `worlds[k]` (default: the first len(states) worlds).  Colliders, joints,
    forces and hulls are shared; joint and contact multipliers start from
    zero, as at any commit."""
    idx = list(range(len(states))) if worlds is None else list(worlds)
    out = []
    for k, st in zip(idx, states):
        w = scene.worlds[k]
        b = w.bodies.copy()
        for f in ("position", "orientation", "linear_velocity", "angular_velocity"):
            b[f] = np.asarray(st[f], np.float64)
        out.append(WorldSpec(b, w.forces, w.colliders, w.joints, w.hulls,
                             getattr(w, "heightmaps", []), getattr(w, "meshes", [])))
    return Scene(scene.name, scene.timestep, scene.substeps, scene.steps, out, scene.description)


def config3_separated(seed=0, n_worlds=256, steps=1000, lo_bodies=8, hi_bodies=512):
    """config3's worlds (same shape, size and count distributions, the same
    13-link chain per world) with no two bodies' bounding spheres
    overlapping at the start and every body clear of the ground: each body's
    position is redrawn until its bounding sphere (box: |half-extents|,
    sphere: radius, chain link: half-height + radius) is clear of every body
    placed before it.  At rest; the first step is free fall plus the chain
    joints."""
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = np.floor(np.exp(rng.uniform(math.log(lo_bodies), math.log(hi_bodies + 1), n_worlds))).astype(int)
    counts = np.clip(counts, lo_bodies, hi_bodies)
    worlds = []
    for w in range(n_worlds):
        bodies, forces, colliders = box_sphere_world(rng, int(counts[w]))
        joints = []
        origin = (rng.uniform(-4.5, -3.5), rng.uniform(2.0, 21.0), rng.uniform(-5.0, 5.0))
        capsule_chain(bodies, forces, colliders, joints, origin)
        B = np.array(bodies, dtype=abi.BODY_DT)
        Cl = np.array(colliders, dtype=abi.COLLIDER_DT)
        rad = np.zeros(len(B))
        for c in Cl:
            p = c["params"]
            if c["shape"] == abi.SHAPE_BOX:
                rad[c["body_id"]] = float(np.linalg.norm(p[:3]))
            elif c["shape"] == abi.SHAPE_SPHERE:
                rad[c["body_id"]] = float(p[0])
            elif c["shape"] == abi.SHAPE_CAPSULE:
                rad[c["body_id"]] = float(p[0] + p[1])
        dyn = np.nonzero(B["type"] == abi.BODY_DYNAMIC)[0]
        chain = dyn[-13:]
        P = np.zeros((len(B), 3))
        R = np.zeros(len(B))
        P[:13], R[:13] = B["position"][chain], rad[chain]
        n_placed = 13
        for i in dyn[:-13]:
            for _ in range(10000):
                p = B["position"][i]
                gap = np.linalg.norm(P[:n_placed] - p, axis=1) - R[:n_placed]
                if p[1] - rad[i] > 0.05 and (gap > rad[i]).all():
                    break
                B["position"][i] = rng.uniform((-5.0, 1.0, -5.0), (5.0, 21.0, 5.0))
            P[n_placed], R[n_placed] = B["position"][i], rad[i]
            n_placed += 1
        worlds.append(_finish(list(B), forces, list(Cl), joints))
    return Scene("config3_separated", 1.0 / 120.0, 4, steps, worlds,
                 f"{n_worlds} config-3 worlds without initial overlap, seed {seed}")
