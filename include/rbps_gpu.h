/*
 * rbps_gpu.h - C ABI of the B200 (sm_100a) implementation of the RBPS
 * per-step hot path: SAP broadphase, narrowphase + contact manifolds and the
 * XPBD substep (integrate, contact/joint position solve, velocity update,
 * restitution/friction velocity solve, joint damping).
 *
 * Every entry point returns an int status (RBPS_OK == 0, negative on error);
 * rbps_last_error() gives the message of the last failing call on the
 * calling thread.  No torch or CUDA types appear in the signatures: the
 * stream is passed as an opaque pointer (a cudaStream_t or NULL).
 *
 * The surface mirrors the reference facade rbps::World
 * (include/rbps/API/World.hpp:87-213) and its parameter structs
 * (BodyAPI.hpp:22-31, ColliderAPI.hpp:17-27, JointAPI.hpp:24-57), generalised
 * to a batch of independent worlds that step together on one GPU.  IDs follow
 * the reference's "ID == slot == index" rule for collections without
 * removals (storage/Soa.hpp:465,577): the n-th body / collider / joint added
 * to a world gets ID n.
 *
 * Ownership: the caller owns every host buffer; the library owns all device
 * memory.  One host thread drives a batch at a time (the reference World is
 * likewise not thread-safe).
 */
#ifndef RBPS_GPU_H
#define RBPS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RBPS_API __attribute__((visibility("default")))
#else
#define RBPS_API
#endif

/* ---------------------------------------------------------------- status */
enum {
    RBPS_OK = 0,
    RBPS_ERR_INVALID = -1,       /* bad argument / call order              */
    RBPS_ERR_CAPACITY = -2,      /* a device buffer (pairs, contacts, ...) overflowed */
    RBPS_ERR_CUDA = -3,          /* CUDA runtime failure                   */
    RBPS_ERR_NOT_CONVERGED = -4, /* an iterative kernel hit its iteration cap */
    RBPS_ERR_STATE = -5,         /* non-finite body state detected          */
    RBPS_ERR_INTERNAL = -6       /* a device consistency check failed       */
};

/* ------------------------------------------------------------------ enums */
/* Arithmetic of the device state and solver. */
enum {
    RBPS_PRECISION_FP64 = 0,       /* everything double, reference operation order */
    RBPS_PRECISION_FP32 = 1,       /* everything float                              */
    RBPS_PRECISION_FP32_POS64 = 2  /* float solver; body positions float relative   */
                                   /* to a per-world double origin (far-from-origin) */
};

/* Order in which contact and joint rows are relaxed inside a substep. */
enum {
    RBPS_SOLVE_REFERENCE_ORDER = 0, /* sequential Gauss-Seidel in ContactList order (Contact.cpp:295-309) */
    RBPS_SOLVE_COLORED = 1          /* graph-coloured Gauss-Seidel, one thread per pair per colour       */
};

/* rbps::BodyType (Body.hpp: enum BodyType { STATIC, DYNAMIC }). */
enum { RBPS_BODY_STATIC = 0, RBPS_BODY_DYNAMIC = 1 };

/* Shape kinds; the values are the rbc::Shape variant indices
 * (rbc/shapes/ShapeTypes.hpp:67-69). */
enum {
    RBPS_SHAPE_SPHERE = 0,
    RBPS_SHAPE_BOX = 1,
    RBPS_SHAPE_ELLIPSOID = 2,   /* params = semi-axes a, b, c (Ellipsoid.hpp)        */
    RBPS_SHAPE_CAPSULE = 3,
    RBPS_SHAPE_CYLINDER = 4,    /* params = half_height, base_radius; axis local +Y  */
    RBPS_SHAPE_CONE = 5,        /* params = half_height, base_radius; apex at +Y     */
    RBPS_SHAPE_PLANE = 6,
    RBPS_SHAPE_HEIGHTMAP = 7,   /* collider `hull` = heightmap id (rbps_heightmap_create) */
    RBPS_SHAPE_MESH = 8,        /* collider `hull` = mesh id (rbps_mesh_create)           */
    RBPS_SHAPE_CONVEX_HULL = 9
};

/* rbps::JointType / JointActuationType (constraints/Joint.hpp).
 * RBPS_JOINT_SPHERICAL has no counterpart in the reference, whose joint
 * types stop at FIXED (a ball joint is only planned there): a ball joint in
 * the reference's row framework (Constraint.cpp:5-46) with two rows,
 *   [0] POSITIONAL  attachment p1 - p2, as the revolute's row 1
 *                   (Joint.cpp:107-111); carries the joint's compliance
 *   [1] ROTATIONAL  swing cone: when the angle between the two bodies'
 *                   `axis` exceeds upper_limit, the correction of
 *                   compute_angle_limit_correction (Joint.cpp:73-90) about
 *                   normalize(a1 x a2) with limits [-upper_limit, upper_limit]
 * `limited` switches the cone on; lower_limit, limit_axis, actuation and
 * damping are ignored.  Unlike the reference's joint rows, whose lambda is
 * never reset, both rows restart lambda at 0 every substep (standard XPBD),
 * so the compliance acts as a fixed-stiffness spring.  Both rows take the direction value / |value|
 * whenever |value| > 1e-9 (set_value's normalize() would leave a zero
 * direction for |value| in (1e-9, 3.2e-5)). */
enum { RBPS_JOINT_PRISMATIC = 0, RBPS_JOINT_REVOLUTE = 1, RBPS_JOINT_FIXED = 2, RBPS_JOINT_SPHERICAL = 3 };
enum { RBPS_ACTUATION_FREE = 0, RBPS_ACTUATION_POSITION = 1, RBPS_ACTUATION_SPEED = 2 };

/* ---------------------------------------------------------- descriptors */
typedef struct rbps_batch_desc {
    uint32_t n_worlds;          /* independent worlds in the batch                 */
    double timestep;            /* World::timestep (World.hpp:97)                  */
    int32_t substeps;           /* World::substeps (World.hpp:98)                  */
    int32_t precision;          /* RBPS_PRECISION_*                                */
    int32_t solve_mode;         /* RBPS_SOLVE_*                                    */
    double fat_margin;          /* BroadPhaseConfig::fat_margin (BroadPhase.hpp:116)        */
    double reinsert_threshold;  /* BroadPhaseConfig::reinsert_threshold (BroadPhase.hpp:124) */
    int32_t use_velocity_expansion; /* CollisionPipelineConfig (CollisionPipeline.hpp:146-154) */
    int32_t device;             /* CUDA device ordinal                             */
    void *stream;               /* cudaStream_t, NULL = the library's own stream   */
    uint32_t max_pairs_per_world;   /* broadphase pair capacity per world, 0 = automatic */
    uint32_t block_threads;     /* threads per world-CTA, 0 = automatic (autotuned)  */
} rbps_batch_desc;

/* Mirrors rbps::BodyParams (BodyAPI.hpp:22-31).  inertia = {xx,yy,zz,xy,xz,yz}
 * (m3d::smat3 field order), orientation = {w,x,y,z}.  As in create_body
 * (BodyAPI.hpp:61) the body's force defaults to (0, -9.8f*mass, 0). */
typedef struct rbps_body_desc {
    int32_t type;
    double mass;
    double inertia[6];
    double position[3];
    double orientation[4];
    double linear_velocity[3];
    double angular_velocity[3];
} rbps_body_desc;

/* Mirrors rbps::ColliderParams (ColliderAPI.hpp:17-27).
 *   sphere : params = {radius}
 *   box    : params = {hx, hy, hz}
 *   capsule: params = {half_height, radius}   (segment along local Y)
 *   plane  : params = {nx, ny, nz, d}         (normal . x = d)
 *   hull   : hull = id returned by rbps_hull_create */
typedef struct rbps_collider_desc {
    int32_t shape;
    double params[4];
    uint32_t hull;
    uint32_t body_id;
    int32_t is_static;
    double local_pos[3];
    double local_rot[4];
    double restitution;
    double static_friction;
    double dynamic_friction;
} rbps_collider_desc;

/* Mirrors Prismatic/Revolute/FixedJointParams (JointAPI.hpp:24-57).
 * axis = moving_axis (prismatic), aligned_axis (revolute) or the swing
 * axis in both bodies' frames (spherical). */
typedef struct rbps_joint_desc {
    int32_t type;
    uint32_t body_1;
    uint32_t body_2;
    double axis[3];
    double limit_axis[3];
    double r_1[3];
    double r_2[3];
    int32_t actuation;
    double compliance;
    double damping;
    int32_t limited;
    double lower_limit;
    double upper_limit;
    double target_position;
    double target_speed;
} rbps_joint_desc;

/* Host views of body state (length n bodies each; NULL fields are skipped). */
typedef struct rbps_state_view {
    double *position;          /* 3n */
    double *orientation;       /* 4n, w,x,y,z */
    double *linear_velocity;   /* 3n */
    double *angular_velocity;  /* 3n */
} rbps_state_view;

/* One row of the reference ContactList (CollisionPipeline.hpp:46-82) as
 * produced by the last narrowphase pass of the last step. */
typedef struct rbps_contact {
    uint32_t body_a, body_b, collider_a, collider_b;
    double normal[3];
    double r_a_local[3];
    double r_b_local[3];
    double point_on_a[3];
    double point_on_b[3];
    double penetration_depth;
    double normal_lambda;
    double tangent_lambda;
    double relative_velocity;
    double restitution, static_friction, dynamic_friction;
    int32_t collision;
    int32_t pad_;
} rbps_contact;

typedef struct rbps_stats {
    uint64_t steps;            /* steps run since commit                        */
    uint64_t pairs;            /* SAP pairs of the last step, all worlds         */
    uint64_t candidates;       /* narrowphase candidates (pairs + plane tests)   */
    uint64_t contacts;         /* contact points of the last substep             */
    uint32_t max_colors;       /* largest colour count of any world, last step   */
    uint32_t serial_overflow;  /* pairs that needed the serial fallback colour   */
    int32_t device_error;      /* last device error word (RBPS_ERR_* or 0)       */
    uint32_t graph;            /* 1 when steps replay a captured CUDA graph      */
    uint64_t kernel_launches;  /* kernels launched by the last rbps_batch_step  */
    uint64_t gjk_pairs;        /* pairs run through GJK / EPA in the last step  */
} rbps_stats;

/* Result of one shape-pair test (rbc::ContactManifold, Contact.hpp:37-51). */
enum {
    RBPS_COLLIDE_MISS = 0,        /* no overlap                                  */
    RBPS_COLLIDE_HIT = 1,         /* overlap; n_points >= 1 points are valid     */
    RBPS_COLLIDE_UNSUPPORTED = 2  /* reserved: every supported shape pair has a device routine */
};

typedef struct rbps_manifold {
    int32_t status;           /* RBPS_COLLIDE_*                                 */
    int32_t n_points;         /* 0..4                                           */
    double normal[3];         /* unit, from shape A toward shape B              */
    double position[4][3];    /* world-space contact points                     */
    double depth[4];          /* penetration depth of each point (> 0 overlap)  */
} rbps_manifold;

typedef struct rbps_batch rbps_batch;

/* ---------------------------------------------------------------- batch */
RBPS_API void rbps_batch_desc_default(rbps_batch_desc *desc);
RBPS_API void rbps_body_desc_default(rbps_body_desc *desc);      /* BodyParams{} */
RBPS_API void rbps_collider_desc_default(rbps_collider_desc *desc); /* ColliderParams{} */
RBPS_API void rbps_joint_desc_default(rbps_joint_desc *desc, int32_t type);

/* Replaces World::World(timestep, substeps) (World.hpp:103) for n worlds. */
RBPS_API int rbps_batch_create(const rbps_batch_desc *desc, rbps_batch **out);
RBPS_API int rbps_batch_destroy(rbps_batch *batch);

/* Convex hull from CCW triangles, like convex_hull_data_create
 * (ConvexHull.hpp:126-420); the data is copied.  verts = 3*n_verts doubles. */
RBPS_API int rbps_hull_create(rbps_batch *batch, const double *verts, uint32_t n_verts,
                              const uint32_t *tris, uint32_t n_tris, uint32_t *hull_id);
/* Replaces heightmap_data_create (Heightmap.hpp): rows x cols float height
 * samples (row-major; sample (r, c) sits at origin + (c * scale.x,
 * h * scale.y, r * scale.z) in world space), copied at call time.  Colliders
 * with shape RBPS_SHAPE_HEIGHTMAP name the returned id in their `hull` field;
 * spheres, capsules and boxes collide with it (HeightmapCollision.hpp), other
 * shapes do not, as in the reference.  Before rbps_batch_commit. */
RBPS_API int rbps_heightmap_create(rbps_batch *batch, const float *heights, uint32_t rows, uint32_t cols,
                                   const double *scale, const double *origin, uint32_t *heightmap_id);
/* Replaces mesh_data_create (Mesh.hpp): a triangle mesh of n_verts local
 * vertices (3 doubles each) and n_faces triangles (3 indices each), copied
 * at call time, face normals and local AABB precomputed as the reference
 * does.  Colliders with shape RBPS_SHAPE_MESH name the returned id in their
 * `hull` field; spheres, capsules, boxes, planes and meshes collide with it
 * (MeshCollision.hpp, PlaneCollision.hpp), other shapes do not, as in the
 * reference.  Before rbps_batch_commit. */
RBPS_API int rbps_mesh_create(rbps_batch *batch, const double *verts, uint32_t n_verts, const uint32_t *indices,
                              uint32_t n_faces, uint32_t *mesh_id);
/* Quickhull helper (the reference ships no hull builder, ConvexHull.hpp:29-33):
 * CCW outward triangles of the convex hull of n points.  Writes at most
 * tri_cap triangles; *n_tris receives the count. */
/* The merged-polygon and adjacency tables the library builds for a hull
 * (those of convex_hull_data_create, ConvexHull.hpp:149-420), host only:
 * counts = {polygons, polygon indices, vertex->polygon entries,
 * vertex->neighbour entries, polygon->polygon entries}; each output array
 * (any may be NULL) needs at most `cap` entries (poly_normals: 3 per polygon;
 * the *_offsets arrays: polygons + 1 or vertices + 1).  Returns
 * RBPS_ERR_CAPACITY with counts filled when cap is too small. */
RBPS_API int rbps_hull_tables(const double *verts, uint32_t n_verts, const uint32_t *tris, uint32_t n_tris,
                              uint32_t cap, uint32_t *counts, uint32_t *poly_offsets, uint32_t *poly_indices,
                              double *poly_normals, uint32_t *v2p_offsets, uint32_t *v2p_indices,
                              uint32_t *v2n_offsets, uint32_t *v2n_indices, uint32_t *p2p_offsets,
                              uint32_t *p2p_indices);
RBPS_API int rbps_quickhull(const double *points, uint32_t n_points,
                            uint32_t *tris, uint32_t tri_cap, uint32_t *n_tris);

/* Replaces World::create_body (World.hpp:113 -> BodyAPI.hpp:53-80). */
RBPS_API int rbps_world_add_body(rbps_batch *batch, uint32_t world,
                                 const rbps_body_desc *desc, uint32_t *id_out);
/* Bulk form: n bodies, ids first_id .. first_id+n-1. */
RBPS_API int rbps_world_add_bodies(rbps_batch *batch, uint32_t world, uint32_t n,
                                   const rbps_body_desc *descs, uint32_t *first_id);
/* Bulk form of rbps_world_set_body_force for bodies first .. first+n-1
 * (3 doubles each). */
RBPS_API int rbps_world_set_body_forces(rbps_batch *batch, uint32_t world, uint32_t first, uint32_t n,
                                        const double *force);
/* Writes bodies.force / bodies.torque (Body.hpp BODY_FIELDS) of one body. */
RBPS_API int rbps_world_set_body_force(rbps_batch *batch, uint32_t world, uint32_t body,
                                       const double force[3], const double torque[3]);
/* Replaces World::create_collider (World.hpp:124-132 -> ColliderAPI.hpp:61-91). */
RBPS_API int rbps_world_add_collider(rbps_batch *batch, uint32_t world,
                                     const rbps_collider_desc *desc, uint32_t *id_out);
RBPS_API int rbps_world_add_colliders(rbps_batch *batch, uint32_t world, uint32_t n,
                                      const rbps_collider_desc *descs, uint32_t *first_id);
/* Replaces World::create_{prismatic,revolute,fixed}_joint (World.hpp:141-156). */
RBPS_API int rbps_world_add_joint(rbps_batch *batch, uint32_t world,
                                  const rbps_joint_desc *desc, uint32_t *id_out);

/* Uploads every world, builds offsets, the initial SAP state (the
 * broad_phase_insert of each collider, BroadPhase.cpp:169-197), plane
 * candidate lists and joint colouring.  No adds are allowed afterwards. */
RBPS_API int rbps_batch_commit(rbps_batch *batch);

/* Replaces World::step (World.hpp:192-212), n_steps times, on every world.
 * Asynchronous on the batch stream; device errors surface at the next
 * rbps_batch_synchronize / get_* call. */
RBPS_API int rbps_batch_step(rbps_batch *batch, int32_t n_steps);
/* Waits for every step and copy enqueued on the batch (both its streams). */
RBPS_API int rbps_batch_synchronize(rbps_batch *batch);
/* Failure detection, on by default: at the end of every step each world's
 * bodies are checked for a non-finite position, orientation or velocity,
 * and the next rbps_batch_synchronize / get_* call returns RBPS_ERR_STATE
 * naming the first such world (the error is then cleared; the world keeps
 * its state until rbps_batch_set_state or rbps_batch_restore replaces it).
 * The reference has no such check (a NaN just propagates through
 * World::step), so enable = 0 restores its behaviour exactly. */
RBPS_API int rbps_batch_set_state_check(rbps_batch *batch, int32_t enable);
/* One World::step of every world with host I/O, for callers that feed
 * forces and read poses every frame: copies force_in (3 doubles per body,
 * all worlds in world order; NULL keeps the current forces) host -> device,
 * steps, and copies positions (3 doubles per body) and orientations (4
 * doubles, w,x,y,z) device -> host (either may be NULL).  Returns when the
 * outputs are written.  Host buffers should be page-locked for full copy
 * bandwidth. */
RBPS_API int rbps_batch_step_io(rbps_batch *batch, const double *force_in, double *position_out,
                                double *orientation_out);
/* rbps_batch_step_io without the wait, for a caller that steps frame after
 * frame: enqueues the force copy, the step and the pose copies and returns.
 * The copies run on a second stream and overlap the neighbouring steps'
 * compute (two staging slots on the device alternate between calls).  The
 * call's host buffers must stay untouched until rbps_batch_synchronize
 * returns (force_in may be reused after the next call returns).  The same
 * World::step as rbps_batch_step_io (World.hpp:192-212); no reference
 * counterpart for the pipelining. */
RBPS_API int rbps_batch_step_io_async(rbps_batch *batch, const double *force_in, double *position_out,
                                      double *orientation_out);

/* Device-side snapshot of every world's simulation state -- bodies (poses,
 * previous poses, velocities, forces), the persistent SAP state (fat AABBs,
 * endpoint order and keys) and the joints' state (drive targets, rows and
 * their multipliers) -- for callers that fork rollouts from one state and
 * rewind (sample-based MPC, determinism replays).  The reference has no
 * snapshot API; its design note (docs/design/world-snapshot-restore/
 * world-snapshot-restore.md) asks for a pool of pre-allocated slots and a
 * bit-exact restore, which this provides on the device.  Each call takes a
 * new slot (device memory owned by the batch, freed with it), copies
 * asynchronously on the batch stream and returns its id in *slot_out. */
RBPS_API int rbps_batch_snapshot(rbps_batch *batch, uint32_t *slot_out);
/* Copies snapshot `slot` back over the batch state (asynchronous on the
 * batch stream); stepping on from it repeats the original run bit for bit. */
RBPS_API int rbps_batch_restore(rbps_batch *batch, uint32_t slot);
/* Overwrites snapshot `slot` with the current state. */
RBPS_API int rbps_batch_snapshot_update(rbps_batch *batch, uint32_t slot);

/* Launch configuration chosen by rbps_batch_autotune. */
typedef struct rbps_tune_result {
    int32_t frame_block;          /* threads per CTA of the frame (SAP) kernel */
    int32_t narrow_grid;          /* CTAs of the narrowphase kernels           */
    double ms_per_step;           /* trial time of the chosen configuration    */
    double ms_per_step_default;   /* trial time of the configuration before    */
    uint32_t trials;              /* configurations timed                      */
    uint32_t team_bodies;         /* worlds this large step on a whole CTA     */
    uint32_t narrow_per_warp;     /* narrowphase candidates a warp takes per pass */
    uint32_t color_chunk;         /* active candidates coloured per staged batch  */
    uint32_t pair_bodies;         /* worlds this large (below team_bodies) step on half a CTA */
    uint32_t pad_;
} rbps_tune_result;

/* Project autotuner (no reference counterpart; the batched design picks its
 * launch shapes by measurement): times `trial_steps` steps of the batch's
 * own worlds under each candidate configuration -- frame kernel at 128 or
 * 256 threads, narrowphase grid at 1/2, 1 or 2 times its occupancy bound,
 * then the body counts from which a world steps on a whole CTA or on half
 * a CTA instead of a warp, then the narrowphase candidates a warp takes per pass
 * (32 to 256) and the colouring's batch of staged candidates (64 to 256) --
 * from the same device snapshot, keeps the fastest and rewinds the batch to
 * the snapshot, so the state is as before the call.  The configuration
 * changes launch shapes only: results stay bit for bit the same.  Blocks
 * the host until done. */
RBPS_API int rbps_batch_autotune(rbps_batch *batch, int32_t trial_steps, rbps_tune_result *result);
/* Applies a launch configuration without timing anything (no reference
 * counterpart): e.g. one rbps_batch_autotune chose for a batch of the same
 * worlds earlier.  Fields frame_block (128 or 256), narrow_grid, team_bodies,
 * pair_bodies, narrow_per_warp (a multiple of 32) and color_chunk (32 to 256)
 * are used;
 * 0 keeps the current value; the timing fields are ignored.  Results do not
 * depend on the configuration. */
RBPS_API int rbps_batch_set_launch(rbps_batch *batch, const rbps_tune_result *config);

/* Per-world body state, host doubles (converted from the device precision). */
RBPS_API int rbps_batch_get_state(rbps_batch *batch, uint32_t world, const rbps_state_view *view);
RBPS_API int rbps_batch_set_state(rbps_batch *batch, uint32_t world, const rbps_state_view *view);
/* All worlds at once: bodies in world order (world 0 bodies, world 1 bodies, ...). */
RBPS_API int rbps_batch_get_state_all(rbps_batch *batch, const rbps_state_view *view);
/* Per-body force (3 doubles each) for all worlds, copied host -> device. */
RBPS_API int rbps_batch_set_forces_all(rbps_batch *batch, const double *force);
RBPS_API int rbps_batch_body_count(rbps_batch *batch, uint32_t world, uint32_t *n_bodies);
RBPS_API int rbps_batch_total_bodies(rbps_batch *batch, uint64_t *n_bodies, uint64_t *n_dynamic);

/* Parity dumps (enable before stepping; they cost extra device copies). */
RBPS_API int rbps_batch_set_dump(rbps_batch *batch, int32_t enable);
/* BroadPhaseState::pairs of the last step (BroadPhase.hpp:141), as
 * (id_a, id_b) uint32 pairs in emission order. */
RBPS_API int rbps_batch_get_pairs(rbps_batch *batch, uint32_t world, uint32_t *pairs,
                                  uint32_t cap, uint32_t *n_out);
/* ContactList of the last substep of the last step, in list order. */
RBPS_API int rbps_batch_get_contacts(rbps_batch *batch, uint32_t world, rbps_contact *out,
                                     uint32_t cap, uint32_t *n_out);
/* Colour of every narrowphase candidate of the last step (colored mode);
 * candidates in list order (SAP pairs, then plane tests); bodies of each. */
RBPS_API int rbps_batch_get_colors(rbps_batch *batch, uint32_t world, uint32_t *colors,
                                   uint32_t *body_a, uint32_t *body_b, uint32_t cap,
                                   uint32_t *n_out);
RBPS_API int rbps_batch_get_stats(rbps_batch *batch, rbps_stats *stats);
/* Persistent SAP state of one world, as the reference BroadPhaseState holds
 * it (BroadPhase.hpp:88-143): fat AABB of each SAP object (6 doubles; object
 * order = collider order, planes skipped) and the endpoint list in its
 * current order as (object*2 + is_max) with the float values.  Any pointer
 * may be NULL; *n_objects receives the object count. */
RBPS_API int rbps_batch_get_sap_state(rbps_batch *batch, uint32_t world, double *fat, uint32_t *ep_ids,
                                      float *ep_values, uint32_t *n_objects);

/* Narrowphase on the device for n independent shape pairs: the GPU
 * counterpart of rbc::dispatch(a, tf_a, b, tf_b, manifold)
 * (rbc/Dispatcher.hpp:208-213), in the batch's precision.  Shapes are
 * collider descriptors (only shape, params and hull are read; hull ids name
 * hulls created on this batch, which must be committed when any is used).
 * tf_a / tf_b: 7 doubles per pair (position xyz, orientation wxyz).  Host
 * buffers; synchronous. */
RBPS_API int rbps_batch_collide(rbps_batch *batch, uint32_t n, const rbps_collider_desc *a, const double *tf_a,
                                const rbps_collider_desc *b, const double *tf_b, rbps_manifold *out);
/* Diagnostics: per-world phase timers.  With profiling enabled every step
 * adds, per world, the SM cycles of each phase (read by the team leader
 * after the phase's closing barrier) to RBPS_PROFILE_SLOTS uint64 slots:
 *   0 broadphase, 1 candidate build, 2 narrowphase, 3 colouring,
 *   4 integrate, 5 contact position solve (reference order: with joints),
 *   6 joint position solve, 7 velocity update, 8 velocity solve, 9 stats;
 *   12 = CTA that stepped the world, 13 / 14 = globaltimer ns at the start
 *   and end of the world's last step.
 * Enabling (re)zeroes the counters; it costs a few clock reads per phase. */
#define RBPS_PROFILE_SLOTS 16
RBPS_API int rbps_batch_set_profile(rbps_batch *batch, int32_t enable);
/* Copies RBPS_PROFILE_SLOTS values per world for the first cap_worlds worlds. */
RBPS_API int rbps_batch_get_profile(rbps_batch *batch, uint64_t *out, uint32_t cap_worlds);
/* Diagnostics: the broadphase + candidate build of one world (the first
 * phase of a step) on its own, at the current poses; counts[0] = SAP pairs,
 * counts[1] = narrowphase candidates.  It updates the SAP state as a step
 * would (a repeat at unchanged poses changes nothing). */
RBPS_API int rbps_debug_broadphase(rbps_batch *batch, uint32_t world, uint32_t *counts);

/* ------------------------------------------------- standalone broadphase
 * GPU drop-in for the rbc SAP API (rbc/BroadPhase.hpp:151-260): objects are
 * inserted / moved on the host exactly as in the reference, and
 * rbps_bp_update runs the sort and sweep on the device.  Pairs come back in
 * the reference emission order. */
typedef struct rbps_bp rbps_bp;
RBPS_API int rbps_bp_create(double fat_margin, double reinsert_threshold, rbps_bp **out);
RBPS_API int rbps_bp_destroy(rbps_bp *bp);
/* aabb = {min.x,min.y,min.z,max.x,max.y,max.z} */
RBPS_API int rbps_bp_insert(rbps_bp *bp, uint32_t user_id, const double aabb[6], uint32_t *handle);
RBPS_API int rbps_bp_remove(rbps_bp *bp, uint32_t handle);
RBPS_API int rbps_bp_move(rbps_bp *bp, uint32_t handle, const double aabb[6]);
RBPS_API int rbps_bp_move_swept(rbps_bp *bp, uint32_t handle, const double aabb[6],
                                const double linear_velocity[3], double dt);
RBPS_API int rbps_bp_update(rbps_bp *bp);
RBPS_API int rbps_bp_get_pairs(rbps_bp *bp, uint32_t *pairs, uint32_t cap, uint32_t *n_out);
RBPS_API int rbps_bp_get_fat_aabb(rbps_bp *bp, uint32_t handle, double aabb[6]);
/* Runs the sort + sweep on one CTA of block_threads threads instead of a
 * cooperative grid (cheaper for small object counts). */
RBPS_API int rbps_bp_configure(rbps_bp *bp, int32_t single_cta, int32_t block_threads);

/* ------------------------------------------------- allocation-free query
 * No counterpart in the reference: it serves callers that cannot allocate
 * device memory once running (real-time loops, where cudaMalloc can block and
 * synchronise the device; hosts that own a fixed device-memory budget).  The
 * SAP sort + sweep of n_objects fat AABBs as a freshly filled broadphase holds
 * them (endpoints in object order), with no allocation: working memory is a
 * file-scope device array of about 2.3 MB per GPU, held until exit.
 *   fat_aabbs : device, 6 doubles per object {min.xyz, max.xyz}
 *   user_ids  : device, 1 per object
 *   pairs     : device, 2 * pair_cap; (id_a, id_b), id_a < id_b, in the
 *               reference emission order; the first min(pair count,
 *               pair_cap) pairs are written
 *   n_pairs   : device, receives the pair count (may exceed pair_cap), or
 *               0xFFFFFFFF when more than 65,536 pairs were found, or
 *               0xFFFFFFFE when an internal consistency check of the sort
 *               failed; with either value `pairs` is left unwritten
 * At most 8,192 objects (larger counts return RBPS_ERR_INVALID); zero
 * objects give zero pairs.  Runs asynchronously on `stream`.  The first call
 * on a device looks up the array's device address; make that first call
 * before any stream capture, and do not call it again on a device after a
 * cudaDeviceReset of that device (the array may move).  Calls share the
 * array: calls that overlap on the GPU race, so order them on one stream. */
RBPS_API int rbps_sap_pairs_static(const double *fat_aabbs, const uint32_t *user_ids, uint32_t n_objects,
                                   uint32_t *pairs, uint32_t pair_cap, uint32_t *n_pairs, void *stream);

/* ------------------------------------------------------------ self tests
 * Self-checking runs of the device primitives every step phase is built on:
 * a stable radix sort of keys (values = original positions) by their low
 * `bits` bits, and an exclusive scan, on one CTA (grid = 0) or a cooperative
 * grid (grid = 1) of block_threads threads per CTA. */
RBPS_API int rbps_selftest_sort(const uint32_t *keys, uint32_t n, int32_t bits, int32_t grid,
                                int32_t block_threads, uint32_t *keys_out, uint32_t *vals_out);
RBPS_API int rbps_selftest_scan(const uint32_t *in, uint32_t n, int32_t grid, int32_t block_threads,
                                uint32_t *out, uint32_t *total);

/* ------------------------------------------------------------- errors */
RBPS_API int rbps_last_error(char *buf, size_t size);
RBPS_API const char *rbps_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RBPS_GPU_H */
