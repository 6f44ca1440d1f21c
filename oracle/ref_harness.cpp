// ref_harness.cpp - TEST INFRASTRUCTURE ONLY (the oracle).
//
// A thin extern "C" shim around the UNMODIFIED reference engine
// (rbps::World, include/rbps/API/World.hpp:87-213, and the rbc SAP
// broadphase, include/rbc/BroadPhase.hpp:151-260), compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/librbps_ref.so.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// it; the product library never links or calls it.
//
// It takes the same descriptor structs as the product C ABI (rbps_gpu.h) so a
// parity test builds the identical scene in both engines.  One addition is
// the oracle's own: the ball joint with a swing cone (RBPS_JOINT_SPHERICAL),
// which the reference does not have, restated on the reference's own rows
// and limit routine (SphJoint below).  Its parity is unpinned by any
// reference test.

#include "rbps/API/World.hpp"
#include "rbc/BroadPhase.hpp"
#include "rbc/Dispatcher.hpp"
#include "rbps_gpu.h"

#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

namespace
{
    struct HullStore
    {
        std::vector<m3d::vec3> verts;
        std::vector<uint32_t> tris;
        rbc::ConvexHullData *data = nullptr;
        ~HullStore() { rbc::convex_hull_data_destroy(data); }
    };

    // A ball joint with a swing cone (RBPS_JOINT_SPHERICAL).  The reference
    // has no such joint type; this is the oracle's own restatement in the
    // reference's row framework: its two rows live in the world's
    // ConstraintCollection (created in joint order, so solve_constraints
    // relaxes them in the same order as the other joints' rows), and their
    // errors are set every substep by sph_joint_errors below.
    struct SphJoint
    {
        uint32_t b1, b2;
        m3d::vec3 r1, r2, axis;
        bool limited;
        double cone;
        uint32_t row_attach, row_cone; // constraint ids
    };

    struct HeightmapStore
    {
        std::vector<float> heights;
        rbc::HeightmapData *data = nullptr;
        ~HeightmapStore() { rbc::heightmap_data_destroy(data); }
    };

    struct MeshStore
    {
        std::vector<m3d::vec3> verts;
        std::vector<uint32_t> idx;
        rbc::MeshData *data = nullptr;
        ~MeshStore() { rbc::mesh_data_destroy(data); }
    };

    struct RefWorld
    {
        rbps::World w;
        std::vector<std::unique_ptr<MeshStore>> meshes;
        std::vector<std::unique_ptr<HullStore>> hulls;
        std::vector<std::unique_ptr<HeightmapStore>> heightmaps;
        std::vector<SphJoint> sph;
        RefWorld(double dt, int substeps) : w(dt, substeps) {}
    };

    // set_value (Constraint.cpp:5-12) for the ball joint's rows, with the
    // direction value / |value| whenever |value| > EPSILON: normalize()
    // would return the zero vector for |value| in (1e-9, 3.2e-5), and a
    // rotational row with compliance 0 then divides by zero.
    void sph_set_value(rbps::ConstraintCollection &cc, uint32_t i, const m3d::vec3 &value)
    {
        const double mag = m3d::magnitude(value);
        cc.magnitude[i] = mag;
        cc.direction[i] = mag > m3d::EPSILON ? value * (1.0 / mag) : m3d::vec3{1.0, 0.0, 0.0};
    }

    // Ball-joint row error, evaluated on the current poses right before the
    // row is solved: the attachment as the revolute joint's
    // (Joint.cpp:107-111), the swing cone through the reference's own
    // compute_angle_limit_correction (Joint.cpp:73-90) with the swing angle
    // phi = atan2(|a1 x a2|, a1 . a2) about n = normalize(a1 x a2) and limits
    // [-cone, cone].  Both rows restart lambda every substep (standard XPBD,
    // Mueller et al. 2020, Alg. 2), so the compliant attachment row is a
    // spring of fixed stiffness.
    void sph_row_error(RefWorld *rw, const SphJoint &j, bool cone, uint32_t i)
    {
        rbps::BodyCollection &bc = rw->w.bodies;
        rbps::ConstraintCollection &cc = rw->w.constraints;
        cc.lambda[i] = 0.0;
        if (!cone)
        {
            const m3d::vec3 r1_wc = m3d::rotate(bc.orientation[j.b1], j.r1);
            const m3d::vec3 r2_wc = m3d::rotate(bc.orientation[j.b2], j.r2);
            const m3d::vec3 p1 = bc.position[j.b1] + r1_wc;
            const m3d::vec3 p2 = bc.position[j.b2] + r2_wc;
            sph_set_value(cc, i, p1 - p2);
            return;
        }
        m3d::vec3 err{0.0, 0.0, 0.0};
        if (j.limited)
        {
            const m3d::vec3 a1 = m3d::rotate(bc.orientation[j.b1], j.axis);
            const m3d::vec3 a2 = m3d::rotate(bc.orientation[j.b2], j.axis);
            const m3d::vec3 c = m3d::cross(a1, a2);
            double phi = m3d::atan2(m3d::magnitude(c), m3d::dot(a1, a2));
            err = rbps::compute_angle_limit_correction(phi, m3d::normalize(c), a1, a2, -j.cone, j.cone);
        }
        sph_set_value(cc, i, -err);
    }

    // solve_constraints (Constraint.cpp:90-106): every row in pool order,
    // with a ball joint's row evaluated right before it is solved.  The
    // other joints' rows keep the errors compute_joint_errors set before
    // the loop, as in the reference; on a hanging chain those stale errors
    // over-correct and the chain diverges within a few steps, which is why
    // the ball joint evaluates its rows in place.
    void solve_rows_with_sph(RefWorld *rw, double inv_h)
    {
        rbps::BodyCollection &bc = rw->w.bodies;
        rbps::ConstraintCollection &cc = rw->w.constraints;
        std::vector<int64_t> tag(cc.count(), -1);
        for (size_t k = 0; k < rw->sph.size(); ++k)
        {
            tag[cc.index_of(rw->sph[k].row_attach)] = (int64_t)(2 * k);
            tag[cc.index_of(rw->sph[k].row_cone)] = (int64_t)(2 * k + 1);
        }
        for (uint32_t i = 0; i < cc.count(); ++i)
        {
            if (tag[i] >= 0)
                sph_row_error(rw, rw->sph[tag[i] / 2], (tag[i] & 1) != 0, i);
            switch (cc.type[i])
            {
            case rbps::ConstraintType::POSITIONAL: rbps::compute_positional_constraint_impulse(bc, cc, i, inv_h); break;
            case rbps::ConstraintType::ROTATIONAL: rbps::compute_rotational_constraint_impulse(bc, cc, i, inv_h); break;
            default: break;
            }
        }
    }

    // World::step (World.hpp:192-212) with solve_constraints replaced by
    // solve_rows_with_sph.
    void step_with_sph(RefWorld *rw)
    {
        rbps::World &w = rw->w;
        const double h = w.timestep / w.substeps;
        const double inv_h = 1.0 / h;
        rbps::update_broad_phase_aabbs(w.colliders, w.broad_phase_state, w.bodies, w.timestep, true);
        rbc::broad_phase_update(w.broad_phase_state);
        w.contacts.reserve(w.broad_phase_state.pairs.size() * 4);
        for (int i = 0; i < w.substeps; ++i)
        {
            w.contacts.clear();
            rbps::run_narrow_phase(w.broad_phase_state, w.colliders, w.bodies, w.contacts);
            rbps::update_position_and_orientation(w.bodies, h);
            rbps::solve_contacts_position_level(w.contacts, w.bodies, inv_h);
            rbps::compute_joint_errors(w.joints, w.bodies, w.constraints, h);
            solve_rows_with_sph(rw, inv_h);
            rbps::update_velocities(w.bodies, inv_h);
            rbps::solve_contacts_velocity_level(w.contacts, w.bodies, h);
            rbps::apply_joint_damping(w.joints, w.bodies, h);
        }
    }

    m3d::vec3 v3(const double *p) { return m3d::vec3(p[0], p[1], p[2]); }
    m3d::quat q4(const double *p) { return m3d::quat(p[0], p[1], p[2], p[3]); }
    void put3(double *o, const m3d::vec3 &v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }
    void put4(double *o, const m3d::quat &q) { o[0] = q.w; o[1] = q.x; o[2] = q.y; o[3] = q.z; }
    void aabb_in(const double *a, rbc::AABB &out)
    {
        out.min = m3d::vec3(a[0], a[1], a[2]);
        out.max = m3d::vec3(a[3], a[4], a[5]);
    }
    // rbc::Shape of a collider descriptor (hull ids index the world's hulls).
    bool make_shape(RefWorld *rw, const rbps_collider_desc *d, rbc::Shape &out)
    {
        switch (d->shape)
        {
        case RBPS_SHAPE_SPHERE: out = rbc::Sphere(d->params[0]); return true;
        case RBPS_SHAPE_BOX: out = rbc::Box(v3(d->params)); return true;
        case RBPS_SHAPE_CAPSULE: out = rbc::Capsule(d->params[0], d->params[1]); return true;
        case RBPS_SHAPE_ELLIPSOID: out = rbc::Ellipsoid(v3(d->params)); return true;
        case RBPS_SHAPE_CYLINDER: out = rbc::Cylinder(d->params[0], d->params[1]); return true;
        case RBPS_SHAPE_CONE: out = rbc::Cone(d->params[0], d->params[1]); return true;
        case RBPS_SHAPE_PLANE: out = rbc::Plane(v3(d->params), d->params[3]); return true;
        case RBPS_SHAPE_MESH:
            if (d->hull >= rw->meshes.size())
                return false;
            out = rbc::Mesh(rw->meshes[d->hull]->data);
            return true;
        case RBPS_SHAPE_HEIGHTMAP:
            if (d->hull >= rw->heightmaps.size())
                return false;
            out = rbc::Heightmap(rw->heightmaps[d->hull]->data);
            return true;
        case RBPS_SHAPE_CONVEX_HULL:
            if (d->hull >= rw->hulls.size())
                return false;
            out = rbc::ConvexHull(rw->hulls[d->hull]->data);
            return true;
        default: return false;
        }
    }
} // namespace

extern "C"
{
    void *ref_world_create(double timestep, int substeps, double fat_margin, double reinsert_threshold)
    {
        auto *rw = new RefWorld(timestep, substeps);
        rbc::BroadPhaseConfig cfg;
        cfg.fat_margin = fat_margin;
        cfg.reinsert_threshold = reinsert_threshold;
        rbc::broad_phase_init(rw->w.broad_phase_state, cfg);
        return rw;
    }

    void ref_world_destroy(void *h) { delete static_cast<RefWorld *>(h); }

    uint32_t ref_hull_create(void *h, const double *verts, uint32_t n_verts,
                             const uint32_t *tris, uint32_t n_tris)
    {
        auto *rw = static_cast<RefWorld *>(h);
        auto hs = std::make_unique<HullStore>();
        hs->verts.resize(n_verts);
        for (uint32_t i = 0; i < n_verts; ++i)
            hs->verts[i] = v3(verts + 3 * i);
        hs->tris.assign(tris, tris + 3 * n_tris);
        hs->data = rbc::convex_hull_data_create(hs->verts.data(), n_verts,
                                                hs->tris.data(), n_tris);
        rw->hulls.push_back(std::move(hs));
        return static_cast<uint32_t>(rw->hulls.size() - 1);
    }

    uint32_t ref_heightmap_create(void *h, const float *heights, uint32_t rows, uint32_t cols, const double *scale,
                                  const double *origin)
    {
        auto *rw = static_cast<RefWorld *>(h);
        auto hs = std::make_unique<HeightmapStore>();
        hs->heights.assign(heights, heights + (size_t)rows * cols);
        hs->data = rbc::heightmap_data_create(hs->heights.data(), rows, cols, v3(scale), v3(origin));
        rw->heightmaps.push_back(std::move(hs));
        return static_cast<uint32_t>(rw->heightmaps.size() - 1);
    }

    uint32_t ref_mesh_create(void *h, const double *verts, uint32_t n_verts, const uint32_t *idx, uint32_t n_faces)
    {
        auto *rw = static_cast<RefWorld *>(h);
        auto ms = std::make_unique<MeshStore>();
        ms->verts.resize(n_verts);
        for (uint32_t i = 0; i < n_verts; ++i)
            ms->verts[i] = v3(verts + 3 * i);
        ms->idx.assign(idx, idx + 3 * (size_t)n_faces);
        ms->data = rbc::mesh_data_create(ms->verts.data(), n_verts, ms->idx.data(), n_faces);
        rw->meshes.push_back(std::move(ms));
        return static_cast<uint32_t>(rw->meshes.size() - 1);
    }

    uint32_t ref_add_body(void *h, const rbps_body_desc *d)
    {
        auto *rw = static_cast<RefWorld *>(h);
        rbps::BodyParams p;
        p.type = d->type == RBPS_BODY_STATIC ? rbps::STATIC : rbps::DYNAMIC;
        p.mass = d->mass;
        p.inertia_tensor = m3d::smat3(d->inertia[0], d->inertia[1], d->inertia[2],
                                      d->inertia[3], d->inertia[4], d->inertia[5]);
        p.position = v3(d->position);
        p.orientation = q4(d->orientation);
        p.linear_velocity = v3(d->linear_velocity);
        p.angular_velocity = v3(d->angular_velocity);
        return rw->w.create_body(p);
    }

    void ref_set_body_force(void *h, uint32_t body, const double *force, const double *torque)
    {
        auto *rw = static_cast<RefWorld *>(h);
        const uint32_t i = rw->w.bodies.index_of(body);
        if (force)
            rw->w.bodies.force[i] = v3(force);
        if (torque)
            rw->w.bodies.torque[i] = v3(torque);
    }

    uint32_t ref_add_collider(void *h, const rbps_collider_desc *d)
    {
        auto *rw = static_cast<RefWorld *>(h);
        rbps::ColliderParams p;
        if (!make_shape(rw, d, p.shape))
            return UINT32_MAX;
        p.body_id = d->body_id;
        p.is_static = d->is_static != 0;
        p.local_pos = v3(d->local_pos);
        p.local_rot = q4(d->local_rot);
        p.restitution = d->restitution;
        p.static_friction = d->static_friction;
        p.dynamic_friction = d->dynamic_friction;
        return rw->w.create_collider(p);
    }

    uint32_t ref_add_joint(void *h, const rbps_joint_desc *d)
    {
        auto *rw = static_cast<RefWorld *>(h);
        uint32_t id = UINT32_MAX;
        const auto act = static_cast<rbps::JointActuationType>(d->actuation);
        if (d->type == RBPS_JOINT_REVOLUTE)
        {
            rbps::RevoluteJointParams p;
            p.body_1 = d->body_1; p.body_2 = d->body_2;
            p.aligned_axis = v3(d->axis); p.limit_axis = v3(d->limit_axis);
            p.r_1 = v3(d->r_1); p.r_2 = v3(d->r_2);
            p.actuation_type = act; p.compliance = d->compliance; p.damping = d->damping;
            p.limited = d->limited != 0; p.lower_limit = d->lower_limit; p.upper_limit = d->upper_limit;
            id = rw->w.create_revolute_joint(p);
        }
        else if (d->type == RBPS_JOINT_PRISMATIC)
        {
            rbps::PrismaticJointParams p;
            p.body_1 = d->body_1; p.body_2 = d->body_2;
            p.moving_axis = v3(d->axis);
            p.r_1 = v3(d->r_1); p.r_2 = v3(d->r_2);
            p.actuation_type = act; p.compliance = d->compliance; p.damping = d->damping;
            p.limited = d->limited != 0; p.lower_limit = d->lower_limit; p.upper_limit = d->upper_limit;
            id = rw->w.create_prismatic_joint(p);
        }
        else if (d->type == RBPS_JOINT_FIXED)
        {
            rbps::FixedJointParams p;
            p.body_1 = d->body_1; p.body_2 = d->body_2;
            p.r_1 = v3(d->r_1); p.r_2 = v3(d->r_2);
            id = rw->w.create_fixed_joint(p);
        }
        else if (d->type == RBPS_JOINT_SPHERICAL)
        {
            SphJoint j;
            j.b1 = d->body_1; j.b2 = d->body_2;
            j.r1 = v3(d->r_1); j.r2 = v3(d->r_2); j.axis = v3(d->axis);
            j.limited = d->limited != 0;
            j.cone = d->upper_limit;
            auto &cc = rw->w.constraints;
            j.row_attach = rbps::create_constraint(cc, {.body_1 = d->body_1, .body_2 = d->body_2,
                                                        .type = rbps::ConstraintType::POSITIONAL,
                                                        .r_1 = j.r1, .r_2 = j.r2, .compliance = d->compliance});
            j.row_cone = rbps::create_constraint(cc, {.body_1 = d->body_1, .body_2 = d->body_2,
                                                      .type = rbps::ConstraintType::ROTATIONAL,
                                                      .r_1 = j.r1, .r_2 = j.r2, .compliance = 0.0});
            rw->sph.push_back(j);
            return 0x80000000u | (uint32_t)(rw->sph.size() - 1);
        }
        if (id != UINT32_MAX)
        {
            const uint32_t j = rw->w.joints.index_of(id);
            rw->w.joints.target_position[j] = d->target_position;
            rw->w.joints.target_speed[j] = d->target_speed;
        }
        return id;
    }

    // rbc::dispatch (Dispatcher.hpp:208-213) on n shape pairs.  tf_* hold 7
    // doubles per pair (position xyz, orientation wxyz).  out receives one
    // rbps_manifold per pair (hit flag, points, normal A->B, depths).
    // Returns -1 when a descriptor names an unknown shape or hull.
    int ref_collide(void *h, uint32_t n, const rbps_collider_desc *a, const double *tf_a,
                    const rbps_collider_desc *b, const double *tf_b, rbps_manifold *out)
    {
        auto *rw = static_cast<RefWorld *>(h);
        for (uint32_t i = 0; i < n; ++i)
        {
            rbc::Shape sa, sb;
            if (!make_shape(rw, a + i, sa) || !make_shape(rw, b + i, sb))
                return -1;
            const m3d::tf ta(v3(tf_a + 7 * i), q4(tf_a + 7 * i + 3));
            const m3d::tf tb(v3(tf_b + 7 * i), q4(tf_b + 7 * i + 3));
            rbc::ContactManifold m;
            const bool hit = rbc::dispatch(sa, ta, sb, tb, m);
            rbps_manifold &o = out[i];
            std::memset(&o, 0, sizeof(o));
            o.status = hit ? RBPS_COLLIDE_HIT : RBPS_COLLIDE_MISS;
            o.n_points = hit ? m.num_points : 0;
            if (hit)
            {
                put3(o.normal, m.normal);
                for (int k = 0; k < m.num_points && k < 4; ++k)
                {
                    put3(o.position[k], m.points[k].position);
                    o.depth[k] = m.points[k].penetration_depth;
                }
            }
        }
        return 0;
    }

    // The reference's parameter defaults (BodyParams{}, ColliderParams{},
    // Revolute/Prismatic/FixedJointParams{}, World{}, BroadPhaseConfig{})
    // written into the C ABI descriptors; world_cfg = {timestep, substeps,
    // fat_margin, reinsert_threshold}.
    void ref_default_descs(rbps_body_desc *body, rbps_collider_desc *coll, rbps_joint_desc *revolute,
                           rbps_joint_desc *prismatic, rbps_joint_desc *fixed, double *world_cfg)
    {
        const rbps::BodyParams bp{};
        std::memset(body, 0, sizeof(*body));
        body->type = bp.type == rbps::STATIC ? RBPS_BODY_STATIC : RBPS_BODY_DYNAMIC;
        body->mass = bp.mass;
        const m3d::smat3 &I = bp.inertia_tensor;
        const double iv[6] = {I.xx, I.yy, I.zz, I.xy, I.xz, I.yz};
        std::memcpy(body->inertia, iv, sizeof(iv));
        put3(body->position, bp.position);
        put4(body->orientation, bp.orientation);
        put3(body->linear_velocity, bp.linear_velocity);
        put3(body->angular_velocity, bp.angular_velocity);

        const rbps::ColliderParams cp{};
        std::memset(coll, 0, sizeof(*coll));
        coll->shape = static_cast<int32_t>(cp.shape.v.index());
        coll->params[0] = std::get<rbc::Sphere>(cp.shape.v).radius;
        coll->body_id = cp.body_id;
        coll->is_static = cp.is_static ? 1 : 0;
        put3(coll->local_pos, cp.local_pos);
        put4(coll->local_rot, cp.local_rot);
        coll->restitution = cp.restitution;
        coll->static_friction = cp.static_friction;
        coll->dynamic_friction = cp.dynamic_friction;

        const rbps::RevoluteJointParams rp{};
        std::memset(revolute, 0, sizeof(*revolute));
        revolute->type = RBPS_JOINT_REVOLUTE;
        revolute->body_1 = (uint32_t)rp.body_1; revolute->body_2 = (uint32_t)rp.body_2;
        put3(revolute->axis, rp.aligned_axis); put3(revolute->limit_axis, rp.limit_axis);
        put3(revolute->r_1, rp.r_1); put3(revolute->r_2, rp.r_2);
        revolute->actuation = static_cast<int32_t>(rp.actuation_type);
        revolute->compliance = rp.compliance; revolute->damping = rp.damping;
        revolute->limited = rp.limited ? 1 : 0;
        revolute->lower_limit = rp.lower_limit; revolute->upper_limit = rp.upper_limit;

        const rbps::PrismaticJointParams pp{};
        std::memset(prismatic, 0, sizeof(*prismatic));
        prismatic->type = RBPS_JOINT_PRISMATIC;
        prismatic->body_1 = (uint32_t)pp.body_1; prismatic->body_2 = (uint32_t)pp.body_2;
        put3(prismatic->axis, pp.moving_axis);
        put3(prismatic->r_1, pp.r_1); put3(prismatic->r_2, pp.r_2);
        prismatic->actuation = static_cast<int32_t>(pp.actuation_type);
        prismatic->compliance = pp.compliance; prismatic->damping = pp.damping;
        prismatic->limited = pp.limited ? 1 : 0;
        prismatic->lower_limit = pp.lower_limit; prismatic->upper_limit = pp.upper_limit;

        const rbps::FixedJointParams fp{};
        std::memset(fixed, 0, sizeof(*fixed));
        fixed->type = RBPS_JOINT_FIXED;
        fixed->body_1 = (uint32_t)fp.body_1; fixed->body_2 = (uint32_t)fp.body_2;
        put3(fixed->r_1, fp.r_1); put3(fixed->r_2, fp.r_2);

        const rbps::World w{};
        const rbc::BroadPhaseConfig bc{};
        world_cfg[0] = w.timestep;
        world_cfg[1] = w.substeps;
        world_cfg[2] = bc.fat_margin;
        world_cfg[3] = bc.reinsert_threshold;
    }

    // The reference's polygon / adjacency tables of hull `hull` of world h
    // (ConvexHullData, ConvexHull.hpp:60-98), in the layout of
    // rbps_hull_tables; returns -1 for an unknown hull, -2 when cap is small.
    int ref_hull_tables(void *h, uint32_t hull, uint32_t cap, uint32_t *counts, uint32_t *poly_offsets,
                        uint32_t *poly_indices, double *poly_normals, uint32_t *v2p_offsets, uint32_t *v2p_indices,
                        uint32_t *v2n_offsets, uint32_t *v2n_indices, uint32_t *p2p_offsets, uint32_t *p2p_indices)
    {
        auto *rw = static_cast<RefWorld *>(h);
        if (hull >= rw->hulls.size())
            return -1;
        const rbc::ConvexHullData *d = rw->hulls[hull]->data;
        const uint32_t np = d->poly_count, nv = d->vert_count;
        counts[0] = np;
        counts[1] = np ? d->poly_offsets[np] : 0;
        counts[2] = np ? d->vertex_to_polys_offsets[nv] : 0;
        counts[3] = np ? d->vertex_to_neighbors_offsets[nv] : 0;
        counts[4] = np ? d->poly_to_polys_offsets[np] : 0;
        uint32_t need = np + 1;
        for (int k = 1; k < 5; ++k)
            need = counts[k] > need ? counts[k] : need;
        if (np && nv + 1 > need)
            need = nv + 1;
        if (need > cap)
            return -2;
        if (!np)
        {
            poly_offsets[0] = 0;
            return 0;
        }
        std::memcpy(poly_offsets, d->poly_offsets, 4 * (np + 1));
        std::memcpy(poly_indices, d->poly_indices, 4 * counts[1]);
        for (uint32_t p = 0; p < np; ++p)
            put3(poly_normals + 3 * p, d->poly_normals[p]);
        std::memcpy(v2p_offsets, d->vertex_to_polys_offsets, 4 * (nv + 1));
        std::memcpy(v2p_indices, d->vertex_to_polys_indices, 4 * counts[2]);
        std::memcpy(v2n_offsets, d->vertex_to_neighbors_offsets, 4 * (nv + 1));
        std::memcpy(v2n_indices, d->vertex_to_neighbors_indices, 4 * counts[3]);
        std::memcpy(p2p_offsets, d->poly_to_polys_offsets, 4 * (np + 1));
        std::memcpy(p2p_indices, d->poly_to_polys_indices, 4 * counts[4]);
        return 0;
    }

    void ref_step(void *h, int n)
    {
        auto *rw = static_cast<RefWorld *>(h);
        for (int i = 0; i < n; ++i)
        {
            if (rw->sph.empty())
                rw->w.step();
            else
                step_with_sph(rw);
        }
    }

    uint32_t ref_body_count(void *h) { return static_cast<RefWorld *>(h)->w.bodies.count(); }

    void ref_get_state(void *h, double *pos, double *quat, double *vel, double *omega)
    {
        auto &b = static_cast<RefWorld *>(h)->w.bodies;
        for (uint32_t i = 0; i < b.count(); ++i)
        {
            if (pos) put3(pos + 3 * i, b.position[i]);
            if (quat) put4(quat + 4 * i, b.orientation[i]);
            if (vel) put3(vel + 3 * i, b.linear_velocity[i]);
            if (omega) put3(omega + 3 * i, b.angular_velocity[i]);
        }
    }

    void ref_set_state(void *h, const double *pos, const double *quat, const double *vel, const double *omega)
    {
        auto &b = static_cast<RefWorld *>(h)->w.bodies;
        for (uint32_t i = 0; i < b.count(); ++i)
        {
            if (pos) b.position[i] = v3(pos + 3 * i);
            if (quat) b.orientation[i] = q4(quat + 4 * i);
            if (vel) b.linear_velocity[i] = v3(vel + 3 * i);
            if (omega) b.angular_velocity[i] = v3(omega + 3 * i);
        }
    }

    uint32_t ref_get_pairs(void *h, uint32_t *out, uint32_t cap)
    {
        const auto &pairs = static_cast<RefWorld *>(h)->w.broad_phase_state.pairs;
        const uint32_t n = static_cast<uint32_t>(pairs.size());
        for (uint32_t i = 0; i < n && i < cap; ++i)
        {
            out[2 * i] = pairs[i].id_a;
            out[2 * i + 1] = pairs[i].id_b;
        }
        return n;
    }

    uint32_t ref_get_contacts(void *h, rbps_contact *out, uint32_t cap)
    {
        const auto &c = static_cast<RefWorld *>(h)->w.contacts;
        const uint32_t n = c.n_contacts;
        for (uint32_t i = 0; i < n && i < cap; ++i)
        {
            rbps_contact &o = out[i];
            std::memset(&o, 0, sizeof(o));
            o.body_a = c.body_a[i]; o.body_b = c.body_b[i];
            o.collider_a = c.collider_a[i]; o.collider_b = c.collider_b[i];
            put3(o.normal, c.normal[i]);
            put3(o.r_a_local, c.r_a_local[i]);
            put3(o.r_b_local, c.r_b_local[i]);
            put3(o.point_on_a, c.point_on_a[i]);
            put3(o.point_on_b, c.point_on_b[i]);
            o.penetration_depth = c.penetration_depth[i];
            o.normal_lambda = c.normal_lambda[i];
            o.tangent_lambda = c.tangent_lambda[i];
            o.relative_velocity = c.relative_velocity[i];
            o.restitution = c.restitution[i];
            o.static_friction = c.static_friction[i];
            o.dynamic_friction = c.dynamic_friction[i];
            o.collision = c.collision[i] ? 1 : 0;
        }
        return n;
    }

    // BroadPhaseState of the world: fat AABB per object slot and the endpoint
    // list as (slot*2 + is_max) with values; returns the object count.
    uint32_t ref_get_sap_state(void *h, double *fat, uint32_t *ep_ids, float *ep_values)
    {
        const auto &bp = static_cast<RefWorld *>(h)->w.broad_phase_state;
        for (size_t o = 0; o < bp.objects.size(); ++o)
            if (fat)
            {
                put3(fat + 6 * o, bp.objects[o].fat_aabb.min);
                put3(fat + 6 * o + 3, bp.objects[o].fat_aabb.max);
            }
        for (size_t i = 0; i < bp.endpoints.size(); ++i)
        {
            if (ep_ids)
                ep_ids[i] = 2u * bp.endpoints[i].slot + bp.endpoints[i].is_max;
            if (ep_values)
                ep_values[i] = bp.endpoints[i].value;
        }
        return static_cast<uint32_t>(bp.objects.size());
    }

    // Colouring of the current ContactList by the reference's own
    // get_collision_groups (CollisionPipeline.cpp:223-293): writes the colour
    // of each contact and returns the number of groups.
    uint32_t ref_collision_groups(void *h, uint32_t *color_of_contact, uint32_t cap)
    {
        auto *rw = static_cast<RefWorld *>(h);
        auto groups = rbps::get_collision_groups(rw->w.contacts, rw->w.bodies);
        for (uint32_t g = 0; g < groups.size(); ++g)
            for (uint32_t c : groups[g])
                if (c < cap)
                    color_of_contact[c] = g;
        return static_cast<uint32_t>(groups.size());
    }

    // CPU baseline: steps n independent worlds `steps` times on `threads`
    // host threads (one World per thread at a time; worlds share no state)
    // and returns the wall-clock seconds.
    double ref_step_worlds(void **worlds, uint32_t n, int steps, int threads)
    {
        if (threads < 1)
            threads = 1;
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t)
            pool.emplace_back([=]() {
                for (uint32_t i = t; i < n; i += threads)
                    ref_step(worlds[i], steps);
            });
        for (auto &th : pool)
            th.join();
        const auto t1 = std::chrono::steady_clock::now();
        return std::chrono::duration<double>(t1 - t0).count();
    }

    // ---- the rbc SAP broadphase, unmodified (BroadPhase.cpp:160-245) ----
    void *ref_bp_create(double fat_margin, double reinsert_threshold)
    {
        auto *bp = new rbc::BroadPhaseState();
        rbc::BroadPhaseConfig cfg;
        cfg.fat_margin = fat_margin;
        cfg.reinsert_threshold = reinsert_threshold;
        rbc::broad_phase_init(*bp, cfg);
        return bp;
    }
    void ref_bp_destroy(void *h) { delete static_cast<rbc::BroadPhaseState *>(h); }
    uint32_t ref_bp_insert(void *h, uint32_t user_id, const double *aabb)
    {
        rbc::AABB a;
        aabb_in(aabb, a);
        return rbc::broad_phase_insert(*static_cast<rbc::BroadPhaseState *>(h), user_id, a);
    }
    void ref_bp_remove(void *h, uint32_t handle)
    {
        rbc::broad_phase_remove(*static_cast<rbc::BroadPhaseState *>(h), handle);
    }
    void ref_bp_move(void *h, uint32_t handle, const double *aabb)
    {
        rbc::AABB a;
        aabb_in(aabb, a);
        rbc::broad_phase_move(*static_cast<rbc::BroadPhaseState *>(h), handle, a);
    }
    void ref_bp_move_swept(void *h, uint32_t handle, const double *aabb, const double *vel, double dt)
    {
        rbc::AABB a;
        aabb_in(aabb, a);
        rbc::broad_phase_move_swept(*static_cast<rbc::BroadPhaseState *>(h), handle, a, v3(vel), dt);
    }
    void ref_bp_update(void *h) { rbc::broad_phase_update(*static_cast<rbc::BroadPhaseState *>(h)); }
    uint32_t ref_bp_get_pairs(void *h, uint32_t *out, uint32_t cap)
    {
        const auto &pairs = static_cast<rbc::BroadPhaseState *>(h)->pairs;
        const uint32_t n = static_cast<uint32_t>(pairs.size());
        for (uint32_t i = 0; i < n && i < cap; ++i)
        {
            out[2 * i] = pairs[i].id_a;
            out[2 * i + 1] = pairs[i].id_b;
        }
        return n;
    }
    void ref_bp_get_fat_aabb(void *h, uint32_t handle, double *aabb)
    {
        const auto &o = static_cast<rbc::BroadPhaseState *>(h)->objects.at(handle);
        put3(aabb, o.fat_aabb.min);
        put3(aabb + 3, o.fat_aabb.max);
    }
}
