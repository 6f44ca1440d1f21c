/* rbps_gpu_world.hpp - rbps::World on the GPU: a C++ drop-in over the C ABI.
 *
 * Replaces rbps::World (include/rbps/API/World.hpp:87-213) for code written
 * against it: the same construction World(timestep, substeps), the same
 * create_body / create_collider / create_{prismatic,revolute,fixed}_joint
 * calls taking the reference's own parameter structs (BodyParams,
 * BodyAPI.hpp:22-31; ColliderParams with any rbc::Shape, ColliderAPI.hpp:
 * 17-27; Prismatic/Revolute/FixedJointParams, JointAPI.hpp:24-69), the same
 * step(), and the state read back through public SoA fields indexed by
 * bodies.index_of(id) (ID == slot, as in the reference without removals).
 * Include it where World.hpp was included and compile against the
 * reference's headers (for the parameter structs and shapes) and link
 * librbps_b200.so.
 *
 * How it maps onto the device:
 *   - creation calls only record descriptors; the device world is built at
 *     the first step() (one world of one rbps_batch; hull, heightmap and
 *     mesh data are copied then, so the caller's ConvexHullData / HeightmapData
 *     / MeshData need to outlive only that first step);
 *   - step() is rbps_batch_step(1) followed by a read-back of every body's
 *     pose and velocities into `bodies` and of the last substep's contact
 *     count into `contacts.n_contacts`;
 *   - writes to bodies.position / orientation / linear_velocity /
 *     angular_velocity / force between steps are detected (bitwise) and
 *     uploaded before the next step;
 *   - a creation call after the first step, or a change of torque, mass,
 *     inertia, type, timestep or substeps, rebuilds the device world from
 *     the current state.  A rebuild restarts the broadphase's persistent
 *     state and the joints' accumulated multipliers, so the reference's
 *     trajectory is reproduced bit for bit (FP64) only for worlds built
 *     before their first step.
 * Errors are thrown as rbps_gpu::Error with the library's RBPS_ERR_* code
 * (the reference has no status codes on this path; a collider or joint
 * naming a body that does not exist is rejected here).  Not thread-safe,
 * like the reference's World. */
#ifndef RBPS_GPU_WORLD_HPP
#define RBPS_GPU_WORLD_HPP

#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>

#include "rbps/API/BodyAPI.hpp"
#include "rbps/API/ColliderAPI.hpp"
#include "rbps/API/JointAPI.hpp"
#include "rbps_gpu.h"

namespace rbps_gpu
{
    using m3d::quat;
    using m3d::scalar;
    using m3d::smat3;
    using m3d::vec3;

    /* A failed library call: code is the RBPS_ERR_* status. */
    struct Error : std::runtime_error
    {
        int code;
        Error(int c, const std::string &msg) : std::runtime_error(msg), code(c) {}
    };

    inline void check(int rc, const char *what)
    {
        if (rc == RBPS_OK)
            return;
        char buf[1024] = {0};
        rbps_last_error(buf, sizeof(buf));
        throw Error(rc, std::string(what) + ": " + buf);
    }

    /* Device execution options (the reference has none): FP64 in the
     * reference's sequential order reproduces it bit for bit. */
    struct Options
    {
        int32_t precision = RBPS_PRECISION_FP64;
        int32_t solve_mode = RBPS_SOLVE_REFERENCE_ORDER;
        int32_t device = 0;
        void *stream = nullptr;          /* cudaStream_t; NULL = the library's own */
        uint32_t max_pairs_per_world = 0; /* 0 = automatic */
    };

    /* The fields of rbps::BodyCollection (Body.hpp:52-69) that callers
     * read and write, one entry per body, indexed by index_of(id). */
    struct Bodies
    {
        std::vector<vec3> force, torque, position, linear_velocity, angular_velocity;
        std::vector<quat> orientation;
        std::vector<scalar> mass, inverse_mass;
        std::vector<rbps::BodyType> type;
        std::vector<smat3> inertia_tensor, inverse_inertia_tensor;

        uint32_t count() const { return (uint32_t)position.size(); }
        /* ID == slot (the reference's ids and packed indices agree while no
         * body is removed); -1 for an id never issued. */
        int32_t index_of(uint32_t id) const { return id < count() ? (int32_t)id : -1; }
    };

    /* ColliderCollection's count / index_of; `desc` holds what was created. */
    struct Colliders
    {
        std::vector<rbps_collider_desc> desc;
        uint32_t count() const { return (uint32_t)desc.size(); }
        int32_t index_of(uint32_t id) const { return id < count() ? (int32_t)id : -1; }
    };

    struct Joints
    {
        std::vector<rbps_joint_desc> desc;
        uint32_t count() const { return (uint32_t)desc.size(); }
    };

    /* ContactList's size after a step: the contact points of the last
     * substep (the reference clears and refills the list every substep). */
    struct Contacts
    {
        uint32_t n_contacts = 0;
    };

    class World
    {
    public:
        scalar timestep = 1.0 / 60.0; /* World::timestep (World.hpp:97) */
        int substeps = 20;            /* World::substeps (World.hpp:98) */
        Bodies bodies;
        Colliders colliders;
        Joints joints;
        Contacts contacts;

        World() : World(1.0 / 60.0, 20) {}
        World(scalar timestep_, int substeps_, const Options &opt = Options())
            : timestep(timestep_), substeps(substeps_), opt_(opt)
        {
        }
        ~World() { release(); }
        World(const World &) = delete;
        World &operator=(const World &) = delete;

        /* rbps::create_body (BodyAPI.hpp:53-81): gravity baked into the
         * force as (0, -9.8f * mass, 0). */
        uint32_t create_body(const rbps::BodyParams &p)
        {
            const bool stat = p.type == rbps::STATIC;
            bodies.force.push_back(vec3{0, -9.8f * p.mass, 0});
            bodies.torque.push_back(vec3(0));
            bodies.mass.push_back(p.mass);
            bodies.inverse_mass.push_back(stat ? scalar(0) : scalar(1) / p.mass);
            bodies.type.push_back(p.type);
            bodies.position.push_back(p.position);
            bodies.orientation.push_back(p.orientation);
            bodies.linear_velocity.push_back(p.linear_velocity);
            bodies.angular_velocity.push_back(p.angular_velocity);
            bodies.inertia_tensor.push_back(p.inertia_tensor);
            bodies.inverse_inertia_tensor.push_back(stat ? smat3{} : p.inertia_tensor.inverse());
            structure_changed_ = true;
            return bodies.count() - 1;
        }

        /* rbps::create_collider (ColliderAPI.hpp:58-83) for any rbc::Shape. */
        uint32_t create_collider(const rbps::ColliderParams &p)
        {
            if (bodies.index_of(p.body_id) < 0)
                throw Error(RBPS_ERR_INVALID, "create_collider: body " + std::to_string(p.body_id) +
                                                  " does not exist");
            rbps_collider_desc d;
            rbps_collider_desc_default(&d);
            d.body_id = p.body_id;
            d.is_static = p.is_static ? 1 : 0;
            d.local_pos[0] = p.local_pos.x;
            d.local_pos[1] = p.local_pos.y;
            d.local_pos[2] = p.local_pos.z;
            d.local_rot[0] = p.local_rot.w;
            d.local_rot[1] = p.local_rot.x;
            d.local_rot[2] = p.local_rot.y;
            d.local_rot[3] = p.local_rot.z;
            d.restitution = p.restitution;
            d.static_friction = p.static_friction;
            d.dynamic_friction = p.dynamic_friction;
            shape_of(p.shape, d);
            colliders.desc.push_back(d);
            structure_changed_ = true;
            return colliders.count() - 1;
        }

        /* rbps::create_prismatic_joint (JointAPI.hpp:24-37). */
        uint32_t create_prismatic_joint(const rbps::PrismaticJointParams &p)
        {
            rbps_joint_desc d = joint_common(RBPS_JOINT_PRISMATIC, p.body_1, p.body_2, p.r_1, p.r_2);
            put3(d.axis, p.moving_axis);
            d.actuation = (int32_t)p.actuation_type;
            d.compliance = p.compliance;
            d.damping = p.damping;
            d.limited = p.limited ? 1 : 0;
            d.lower_limit = p.lower_limit;
            d.upper_limit = p.upper_limit;
            return add_joint(d);
        }

        /* rbps::create_revolute_joint (JointAPI.hpp:43-57). */
        uint32_t create_revolute_joint(const rbps::RevoluteJointParams &p)
        {
            rbps_joint_desc d = joint_common(RBPS_JOINT_REVOLUTE, p.body_1, p.body_2, p.r_1, p.r_2);
            put3(d.axis, p.aligned_axis);
            put3(d.limit_axis, p.limit_axis);
            d.actuation = (int32_t)p.actuation_type;
            d.compliance = p.compliance;
            d.damping = p.damping;
            d.limited = p.limited ? 1 : 0;
            d.lower_limit = p.lower_limit;
            d.upper_limit = p.upper_limit;
            return add_joint(d);
        }

        /* rbps::create_fixed_joint (JointAPI.hpp:63-69). */
        uint32_t create_fixed_joint(const rbps::FixedJointParams &p)
        {
            return add_joint(joint_common(RBPS_JOINT_FIXED, p.body_1, p.body_2, p.r_1, p.r_2));
        }

        /* World::step (World.hpp:192-212): one frame of `substeps` substeps. */
        void step()
        {
            if (bodies.count() == 0) // nothing to simulate (World.hpp:192-212 on an empty world)
            {
                contacts.n_contacts = 0;
                return;
            }
            prepare();
            check(rbps_batch_step(b_, 1), "rbps_batch_step");
            pull();
        }

        /* The underlying batch (one world), built on demand; for callers
         * that move on to the batched API. */
        rbps_batch *batch()
        {
            prepare();
            return b_;
        }

    private:
        Options opt_;
        rbps_batch *b_ = nullptr;
        bool structure_changed_ = true;
        scalar built_timestep_ = 0;
        int built_substeps_ = 0;
        // state as last exchanged with the device (bitwise change detection)
        Bodies synced_;
        // hull / heightmap / mesh colliders: the caller's data, registered at build
        std::vector<const rbc::ConvexHullData *> hull_src_;
        std::vector<const rbc::HeightmapData *> hmap_src_;
        std::vector<const rbc::MeshData *> mesh_src_;

        static void put3(double *o, const vec3 &v)
        {
            o[0] = v.x;
            o[1] = v.y;
            o[2] = v.z;
        }

        template <class T>
        static uint32_t index_in(std::vector<const T *> &v, const T *p)
        {
            for (size_t i = 0; i < v.size(); ++i)
                if (v[i] == p)
                    return (uint32_t)i;
            v.push_back(p);
            return (uint32_t)(v.size() - 1);
        }

        // rbc::Shape (ShapeTypes.hpp:67-69) -> shape kind + params; data
        // shapes keep their source pointer until the build copies it
        void shape_of(const rbc::Shape &s, rbps_collider_desc &d)
        {
            std::visit(
                [&](const auto &sh) {
                    using S = std::decay_t<decltype(sh)>;
                    for (double &x : d.params)
                        x = 0.0;
                    if constexpr (std::is_same_v<S, rbc::Sphere>)
                    {
                        d.shape = RBPS_SHAPE_SPHERE;
                        d.params[0] = sh.radius;
                    }
                    else if constexpr (std::is_same_v<S, rbc::Box>)
                    {
                        d.shape = RBPS_SHAPE_BOX;
                        put3(d.params, sh.half_extents);
                    }
                    else if constexpr (std::is_same_v<S, rbc::Ellipsoid>)
                    {
                        d.shape = RBPS_SHAPE_ELLIPSOID;
                        put3(d.params, sh.half_extents);
                    }
                    else if constexpr (std::is_same_v<S, rbc::Capsule>)
                    {
                        d.shape = RBPS_SHAPE_CAPSULE;
                        d.params[0] = sh.half_height;
                        d.params[1] = sh.radius;
                    }
                    else if constexpr (std::is_same_v<S, rbc::Cylinder>)
                    {
                        d.shape = RBPS_SHAPE_CYLINDER;
                        d.params[0] = sh.half_height;
                        d.params[1] = sh.base_radius;
                    }
                    else if constexpr (std::is_same_v<S, rbc::Cone>)
                    {
                        d.shape = RBPS_SHAPE_CONE;
                        d.params[0] = sh.half_height;
                        d.params[1] = sh.base_radius;
                    }
                    else if constexpr (std::is_same_v<S, rbc::Plane>)
                    {
                        d.shape = RBPS_SHAPE_PLANE;
                        put3(d.params, sh.normal);
                        d.params[3] = sh.d;
                    }
                    else if constexpr (std::is_same_v<S, rbc::ConvexHull>)
                    {
                        if (!sh.data)
                            throw Error(RBPS_ERR_INVALID, "create_collider: ConvexHull without data");
                        d.shape = RBPS_SHAPE_CONVEX_HULL;
                        d.hull = index_in(hull_src_, sh.data);
                    }
                    else if constexpr (std::is_same_v<S, rbc::Heightmap>)
                    {
                        if (!sh.data)
                            throw Error(RBPS_ERR_INVALID, "create_collider: Heightmap without data");
                        d.shape = RBPS_SHAPE_HEIGHTMAP;
                        d.hull = index_in(hmap_src_, sh.data);
                    }
                    else
                    {
                        static_assert(std::is_same_v<S, rbc::Mesh>, "a shape of rbc::Shape is not mapped");
                        if (!sh.data)
                            throw Error(RBPS_ERR_INVALID, "create_collider: Mesh without data");
                        d.shape = RBPS_SHAPE_MESH;
                        d.hull = index_in(mesh_src_, sh.data);
                    }
                },
                s.v);
        }

        rbps_joint_desc joint_common(int32_t type, size_t b1, size_t b2, const vec3 &r1, const vec3 &r2)
        {
            if (bodies.index_of((uint32_t)b1) < 0 || bodies.index_of((uint32_t)b2) < 0 || b1 > UINT32_MAX ||
                b2 > UINT32_MAX)
                throw Error(RBPS_ERR_INVALID, "create_*_joint: joint bodies do not exist");
            rbps_joint_desc d;
            rbps_joint_desc_default(&d, type);
            d.body_1 = (uint32_t)b1;
            d.body_2 = (uint32_t)b2;
            put3(d.r_1, r1);
            put3(d.r_2, r2);
            return d;
        }

        uint32_t add_joint(const rbps_joint_desc &d)
        {
            joints.desc.push_back(d);
            structure_changed_ = true;
            return joints.count() - 1;
        }

        void release()
        {
            if (b_)
                rbps_batch_destroy(b_);
            b_ = nullptr;
        }

        template <class V>
        static bool same(const std::vector<V> &a, const std::vector<V> &b)
        {
            return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(V)) == 0);
        }

        // (Re)creates the device world from the recorded descriptors and the
        // current body state.
        void build()
        {
            release();
            rbps_batch_desc bd;
            rbps_batch_desc_default(&bd);
            bd.n_worlds = 1;
            bd.timestep = timestep;
            bd.substeps = substeps;
            bd.precision = opt_.precision;
            bd.solve_mode = opt_.solve_mode;
            bd.device = opt_.device;
            bd.stream = opt_.stream;
            bd.max_pairs_per_world = opt_.max_pairs_per_world;
            check(rbps_batch_create(&bd, &b_), "rbps_batch_create");
            std::vector<uint32_t> hull_id, hmap_id, mesh_id;
            for (const rbc::ConvexHullData *h : hull_src_)
            {
                if (!h->face_indices || !h->face_count)
                    throw Error(RBPS_ERR_INVALID, "ConvexHull data without triangles");
                std::vector<double> v(3 * (size_t)h->vert_count);
                for (uint32_t i = 0; i < h->vert_count; ++i)
                    put3(&v[3 * (size_t)i], h->vertices[i]);
                uint32_t id = 0;
                check(rbps_hull_create(b_, v.data(), h->vert_count, h->face_indices, h->face_count, &id),
                      "rbps_hull_create");
                hull_id.push_back(id);
            }
            for (const rbc::HeightmapData *h : hmap_src_)
            {
                double scale[3], origin[3];
                put3(scale, h->scale);
                put3(origin, h->origin);
                uint32_t id = 0;
                check(rbps_heightmap_create(b_, h->heights, h->rows, h->cols, scale, origin, &id),
                      "rbps_heightmap_create");
                hmap_id.push_back(id);
            }
            for (const rbc::MeshData *m : mesh_src_)
            {
                std::vector<double> v(3 * (size_t)m->vert_count);
                for (uint32_t i = 0; i < m->vert_count; ++i)
                    put3(&v[3 * (size_t)i], m->vertices[i]);
                uint32_t id = 0;
                check(rbps_mesh_create(b_, v.data(), m->vert_count, m->indices, m->face_count, &id),
                      "rbps_mesh_create");
                mesh_id.push_back(id);
            }
            for (uint32_t i = 0; i < bodies.count(); ++i)
            {
                rbps_body_desc d;
                rbps_body_desc_default(&d);
                d.type = bodies.type[i] == rbps::STATIC ? RBPS_BODY_STATIC : RBPS_BODY_DYNAMIC;
                d.mass = bodies.mass[i];
                const smat3 &I = bodies.inertia_tensor[i];
                const double inert[6] = {I.xx, I.yy, I.zz, I.xy, I.xz, I.yz};
                std::memcpy(d.inertia, inert, sizeof(inert));
                put3(d.position, bodies.position[i]);
                const quat &q = bodies.orientation[i];
                d.orientation[0] = q.w;
                d.orientation[1] = q.x;
                d.orientation[2] = q.y;
                d.orientation[3] = q.z;
                put3(d.linear_velocity, bodies.linear_velocity[i]);
                put3(d.angular_velocity, bodies.angular_velocity[i]);
                uint32_t id = 0;
                check(rbps_world_add_body(b_, 0, &d, &id), "rbps_world_add_body");
                double f[3], t[3];
                put3(f, bodies.force[i]);
                put3(t, bodies.torque[i]);
                check(rbps_world_set_body_force(b_, 0, id, f, t), "rbps_world_set_body_force");
            }
            for (rbps_collider_desc d : colliders.desc)
            {
                if (d.shape == RBPS_SHAPE_CONVEX_HULL)
                    d.hull = hull_id[d.hull];
                else if (d.shape == RBPS_SHAPE_HEIGHTMAP)
                    d.hull = hmap_id[d.hull];
                else if (d.shape == RBPS_SHAPE_MESH)
                    d.hull = mesh_id[d.hull];
                check(rbps_world_add_collider(b_, 0, &d, nullptr), "rbps_world_add_collider");
            }
            for (const rbps_joint_desc &d : joints.desc)
                check(rbps_world_add_joint(b_, 0, &d, nullptr), "rbps_world_add_joint");
            check(rbps_batch_commit(b_), "rbps_batch_commit");
            built_timestep_ = timestep;
            built_substeps_ = substeps;
            structure_changed_ = false;
            synced_ = bodies;
        }

        // Uploads the body state and forces the caller changed since the
        // last exchange.
        void push()
        {
            const size_t n = bodies.count();
            if (!same(bodies.position, synced_.position) || !same(bodies.orientation, synced_.orientation) ||
                !same(bodies.linear_velocity, synced_.linear_velocity) ||
                !same(bodies.angular_velocity, synced_.angular_velocity))
            {
                std::vector<double> p(3 * n), q(4 * n), v(3 * n), w(3 * n);
                for (size_t i = 0; i < n; ++i)
                {
                    put3(&p[3 * i], bodies.position[i]);
                    const quat &o = bodies.orientation[i];
                    q[4 * i] = o.w;
                    q[4 * i + 1] = o.x;
                    q[4 * i + 2] = o.y;
                    q[4 * i + 3] = o.z;
                    put3(&v[3 * i], bodies.linear_velocity[i]);
                    put3(&w[3 * i], bodies.angular_velocity[i]);
                }
                rbps_state_view sv{p.data(), q.data(), v.data(), w.data()};
                check(rbps_batch_set_state(b_, 0, &sv), "rbps_batch_set_state");
            }
            if (!same(bodies.force, synced_.force))
            {
                std::vector<double> f(3 * n);
                for (size_t i = 0; i < n; ++i)
                    put3(&f[3 * i], bodies.force[i]);
                check(rbps_batch_set_forces_all(b_, f.data()), "rbps_batch_set_forces_all");
            }
            synced_ = bodies;
        }

        // Builds the device world when its structure or a build-time field
        // changed, else uploads the caller's edits.
        void prepare()
        {
            const bool rebuild = !b_ || structure_changed_ || timestep != built_timestep_ ||
                                 substeps != built_substeps_ || !same(bodies.torque, synced_.torque) ||
                                 !same(bodies.mass, synced_.mass) || !same(bodies.type, synced_.type) ||
                                 !same(bodies.inertia_tensor, synced_.inertia_tensor);
            if (rebuild)
                build();
            else
                push();
        }

        // Reads every body's pose and velocities and the contact count back.
        void pull()
        {
            const size_t n = bodies.count();
            std::vector<double> p(3 * n), q(4 * n), v(3 * n), w(3 * n);
            rbps_state_view sv{p.data(), q.data(), v.data(), w.data()};
            check(rbps_batch_get_state(b_, 0, &sv), "rbps_batch_get_state");
            for (size_t i = 0; i < n; ++i)
            {
                bodies.position[i] = vec3{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
                bodies.orientation[i] = quat{q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
                bodies.linear_velocity[i] = vec3{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
                bodies.angular_velocity[i] = vec3{w[3 * i], w[3 * i + 1], w[3 * i + 2]};
            }
            rbps_stats st;
            check(rbps_batch_get_stats(b_, &st), "rbps_batch_get_stats");
            contacts.n_contacts = (uint32_t)st.contacts;
            synced_ = bodies;
        }
    };
} // namespace rbps_gpu

#endif /* RBPS_GPU_WORLD_HPP */
