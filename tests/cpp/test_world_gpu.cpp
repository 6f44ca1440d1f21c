// test_world_gpu.cpp - the reference World's behaviour tests run through the
// C++ drop-in rbps_gpu::World, beside the reference's own rbps::World.
//
// Every scenario of the reference's tests/rbps/API/test_world.cpp (lines
// 22-255: construction, creation, empty and collider-free steps, free fall,
// a static body, a sphere landing on and not tunnelling through a static
// box, two spheres colliding, momentum, contact-list lifetime) is built
// twice from the same calls -- once in rbps::World (the reference, compiled
// from its own sources into the oracle library) and once in rbps_gpu::World
// (FP64, reference order, on the GPU) -- and stepped in lockstep.  After
// every step the bodies' positions, orientations and velocities must be
// bitwise equal, and each scenario's own assertion must hold on the GPU
// world.  Two more scenarios exercise what those tests do not: every shape
// of rbc::Shape that the device collides (plane, box, sphere, capsule,
// cylinder, cone, ellipsoid, convex hull) and the three joint types with
// axes, anchors, limits, compliance and damping.
//
// Test infrastructure: built by oracle/Makefile (target `world_test`)
// against the reference's headers, run by tests/test_world_cpp_gpu.py.
// Prints one line per scenario and exits non-zero on any failure.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rbps/API/World.hpp"
#include "rbps_gpu_world.hpp"

using m3d::quat;
using m3d::scalar;
using m3d::smat3;
using m3d::vec3;

namespace
{
    int g_failures = 0;

#define CHECK(c)                                                                                   \
    do                                                                                             \
    {                                                                                              \
        if (!(c))                                                                                  \
        {                                                                                          \
            std::printf("    check failed: %s (line %d)\n", #c, __LINE__);                         \
            ++g_failures;                                                                          \
        }                                                                                          \
    } while (0)

    // The two worlds of one scenario, built by the same calls.
    struct Twin
    {
        rbps::World ref;
        rbps_gpu::World gpu;
        int steps = 0;
        int mismatches = 0;

        Twin() = default;
        Twin(scalar ts, int ss) : ref(ts, ss), gpu(ts, ss) {}

        template <class F>
        uint32_t both(F f)
        {
            const uint32_t a = f(ref), b = f(gpu);
            CHECK(a == b);
            return b;
        }

        static bool same_bits(const void *a, const void *b, size_t n) { return std::memcmp(a, b, n) == 0; }

        // bitwise state equality of every body after the step just taken
        void compare()
        {
            const uint32_t n = gpu.bodies.count();
            if (n != (uint32_t)ref.bodies.position.size())
            {
                std::printf("    step %d: body counts differ\n", steps);
                ++mismatches;
                return;
            }
            for (uint32_t i = 0; i < n; ++i)
            {
                const bool ok = same_bits(&ref.bodies.position[i], &gpu.bodies.position[i], sizeof(vec3)) &&
                                same_bits(&ref.bodies.orientation[i], &gpu.bodies.orientation[i], sizeof(quat)) &&
                                same_bits(&ref.bodies.linear_velocity[i], &gpu.bodies.linear_velocity[i],
                                          sizeof(vec3)) &&
                                same_bits(&ref.bodies.angular_velocity[i], &gpu.bodies.angular_velocity[i],
                                          sizeof(vec3));
                if (!ok)
                {
                    ++g_failures;
                    if (mismatches < 3)
                        std::printf("    step %d body %u: ref (%.17g %.17g %.17g) gpu (%.17g %.17g %.17g)\n", steps,
                                    i, ref.bodies.position[i].x, ref.bodies.position[i].y, ref.bodies.position[i].z,
                                    gpu.bodies.position[i].x, gpu.bodies.position[i].y, gpu.bodies.position[i].z);
                    ++mismatches;
                }
            }
        }

        void step(int n = 1)
        {
            for (int k = 0; k < n; ++k)
            {
                ref.step();
                gpu.step();
                ++steps;
                compare();
            }
        }
    };

    // The reference tests' helpers (their header is not in the reference
    // tree): a dynamic sphere of radius r and mass m (solid-sphere inertia)
    // and a static box of half-extent 2 ("ground center at -3, top at -1").
    template <class W>
    uint32_t add_dynamic_sphere(W &w, vec3 pos, scalar r = 0.5, scalar mass = 1.0, vec3 vel = vec3(0.0))
    {
        rbps::BodyParams bp;
        bp.type = rbps::DYNAMIC;
        bp.mass = mass;
        const scalar i = 0.4 * mass * r * r;
        bp.inertia_tensor = smat3{i, i, i, 0, 0, 0};
        bp.position = pos;
        bp.linear_velocity = vel;
        const uint32_t id = w.create_body(bp);
        rbps::ColliderParams cp;
        cp.shape = rbc::Sphere{r};
        cp.body_id = id;
        w.create_collider(cp);
        return id;
    }

    template <class W>
    uint32_t add_static_box(W &w, vec3 pos)
    {
        rbps::BodyParams bp;
        bp.type = rbps::STATIC;
        bp.position = pos;
        const uint32_t id = w.create_body(bp);
        rbps::ColliderParams cp;
        cp.shape = rbc::Box{vec3{2.0, 2.0, 2.0}};
        cp.body_id = id;
        cp.is_static = true;
        w.create_collider(cp);
        return id;
    }

    vec3 pos_of(const rbps_gpu::World &w, uint32_t id) { return w.bodies.position[w.bodies.index_of(id)]; }
    vec3 vel_of(const rbps_gpu::World &w, uint32_t id) { return w.bodies.linear_velocity[w.bodies.index_of(id)]; }

    // ------------------------------------------------- test_world.cpp:22-90
    void parameterized_construction()
    {
        Twin t(1.0 / 120.0, 10);
        CHECK(std::fabs(t.gpu.timestep - 1.0 / 120.0) < 1e-9);
        CHECK(t.gpu.substeps == 10);
    }

    void create_body_returns_valid_id()
    {
        Twin t;
        const uint32_t id = t.both([](auto &w) {
            rbps::BodyParams bp;
            bp.position = vec3{0, 0, 0};
            bp.mass = 1.0;
            bp.type = rbps::DYNAMIC;
            return w.create_body(bp);
        });
        CHECK(t.gpu.bodies.index_of(id) >= 0);
        CHECK(std::fabs(pos_of(t.gpu, id).y) < 1e-6);
    }

    void create_multiple_bodies()
    {
        Twin t;
        const uint32_t a = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{0, 2, 0}); });
        const uint32_t b = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{0, -2, 0}); });
        CHECK(a != b);
        CHECK(t.gpu.bodies.count() == 2);
        CHECK(t.gpu.colliders.count() == 2);
        t.step(3);
    }

    void step_empty_world()
    {
        Twin t;
        t.step(2);
        CHECK(t.gpu.contacts.n_contacts == 0);
    }

    void step_single_body_no_collider()
    {
        Twin t;
        t.both([](auto &w) {
            rbps::BodyParams bp;
            bp.position = vec3{0, 10, 0};
            bp.linear_velocity = vec3{0, 0, 0};
            bp.mass = 1.0;
            bp.type = rbps::DYNAMIC;
            return w.create_body(bp);
        });
        t.step(1);
        CHECK(t.gpu.contacts.n_contacts == 0);
    }

    // ------------------------------------------------ test_world.cpp:96-255
    void free_fall_moves_body_downward()
    {
        Twin t(1.0 / 60.0, 20);
        const uint32_t id = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{0, 10, 0}); });
        const scalar y0 = pos_of(t.gpu, id).y;
        t.step(1);
        CHECK(pos_of(t.gpu, id).y < y0);
    }

    void free_fall_velocity_increases()
    {
        Twin t(1.0 / 60.0, 20);
        const uint32_t id = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{0, 10, 0}); });
        t.step(1);
        const scalar vy1 = vel_of(t.gpu, id).y;
        t.step(1);
        CHECK(vel_of(t.gpu, id).y < vy1);
    }

    void static_body_does_not_move()
    {
        Twin t;
        const uint32_t id = t.both([](auto &w) { return add_static_box(w, vec3{0, 0, 0}); });
        const vec3 p0 = pos_of(t.gpu, id);
        t.step(10);
        const vec3 p1 = pos_of(t.gpu, id);
        CHECK(std::fabs(p1.x - p0.x) < 1e-6 && std::fabs(p1.y - p0.y) < 1e-6 && std::fabs(p1.z - p0.z) < 1e-6);
    }

    void sphere_lands_on_ground()
    {
        Twin t(1.0 / 60.0, 20);
        t.both([](auto &w) { return add_static_box(w, vec3{0, -3, 0}); });
        const uint32_t id = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{0, 1, 0}, 0.5); });
        t.step(180);
        const vec3 v = vel_of(t.gpu, id);
        CHECK(std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z) < 2.0);
        CHECK(pos_of(t.gpu, id).y > -4.0);
    }

    void sphere_does_not_tunnel_through_ground()
    {
        Twin t(1.0 / 60.0, 25);
        t.both([](auto &w) { return add_static_box(w, vec3{0, -3, 0}); });
        const uint32_t id = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{0, 2, 0}, 0.5); });
        t.step(300);
        CHECK(pos_of(t.gpu, id).y > -5.0);
    }

    void two_spheres_collide_and_separate()
    {
        Twin t(1.0 / 60.0, 20);
        const uint32_t a = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{-2, 0, 0}, 0.5, 1.0, vec3{5, 0, 0}); });
        const uint32_t b = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{2, 0, 0}, 0.5, 1.0, vec3{-5, 0, 0}); });
        t.step(30);
        CHECK(vel_of(t.gpu, a).x < 0.0 || vel_of(t.gpu, b).x > 0.0);
    }

    void collision_conserves_momentum_approximately()
    {
        Twin t(1.0 / 60.0, 20);
        const uint32_t a = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{-2, 0, 0}, 0.5, 1.0, vec3{3, 0, 0}); });
        const uint32_t b = t.both([](auto &w) { return add_dynamic_sphere(w, vec3{2, 0, 0}, 0.5, 1.0, vec3{0, 0, 0}); });
        auto px = [&]() {
            const auto &B = t.gpu.bodies;
            return B.linear_velocity[B.index_of(a)].x * B.mass[B.index_of(a)] +
                   B.linear_velocity[B.index_of(b)].x * B.mass[B.index_of(b)];
        };
        const scalar before = px();
        t.step(60);
        CHECK(std::fabs(px() - before) <= std::fabs(before) * 0.2 + 0.1);
    }

    void contacts_cleared_each_frame()
    {
        Twin t(1.0 / 60.0, 20);
        t.both([](auto &w) { return add_static_box(w, vec3{0, -1, 0}); });
        t.both([](auto &w) { return add_dynamic_sphere(w, vec3{0, 0, 0}, 0.5); });
        t.step(10);
        CHECK(t.gpu.contacts.n_contacts <= 16);
        CHECK(t.gpu.contacts.n_contacts == t.ref.contacts.n_contacts);
    }

    void no_contacts_when_bodies_separated()
    {
        Twin t;
        t.both([](auto &w) { return add_dynamic_sphere(w, vec3{0, 100, 0}); });
        t.both([](auto &w) { return add_dynamic_sphere(w, vec3{100, 0, 0}); });
        t.step(1);
        CHECK(t.gpu.contacts.n_contacts == 0);
    }

    // ----------------------------------------------- beyond test_world.cpp
    // A unit cube as a convex hull: 8 vertices, 12 outward CCW triangles.
    const vec3 kCubeVerts[8] = {{-0.3, -0.3, -0.3}, {0.3, -0.3, -0.3}, {0.3, 0.3, -0.3}, {-0.3, 0.3, -0.3},
                                {-0.3, -0.3, 0.3},  {0.3, -0.3, 0.3},  {0.3, 0.3, 0.3},  {-0.3, 0.3, 0.3}};
    const uint32_t kCubeTris[36] = {0, 3, 2, 0, 2, 1, 4, 5, 6, 4, 6, 7, 0, 1, 5, 0, 5, 4,
                                    3, 7, 6, 3, 6, 2, 0, 4, 7, 0, 7, 3, 1, 2, 6, 1, 6, 5};

    template <class W>
    uint32_t add_shape(W &w, const rbc::Shape &s, vec3 pos, quat rot, scalar mass, smat3 inertia)
    {
        rbps::BodyParams bp;
        bp.mass = mass;
        bp.inertia_tensor = inertia;
        bp.position = pos;
        bp.orientation = rot;
        const uint32_t id = w.create_body(bp);
        rbps::ColliderParams cp;
        cp.shape = s;
        cp.body_id = id;
        cp.restitution = 0.2;
        cp.static_friction = 0.6;
        cp.dynamic_friction = 0.4;
        w.create_collider(cp);
        return id;
    }

    void every_shape_on_a_plane()
    {
        static rbc::ConvexHullData *cube = rbc::convex_hull_data_create(kCubeVerts, 8, kCubeTris, 12);
        Twin t(1.0 / 60.0, 10);
        t.both([](auto &w) {
            rbps::BodyParams g;
            g.type = rbps::STATIC;
            const uint32_t id = w.create_body(g);
            rbps::ColliderParams cp;
            cp.shape = rbc::Plane{};
            cp.body_id = id;
            cp.is_static = true;
            return w.create_collider(cp);
        });
        const quat tilt = m3d::normalize(quat{0.95, 0.2, 0.1, 0.15});
        const smat3 I{0.05, 0.05, 0.05, 0, 0, 0};
        const scalar x0 = -3.0;
        t.both([&](auto &w) { return add_shape(w, rbc::Box{vec3{0.3, 0.2, 0.25}}, vec3{x0, 0.8, 0}, tilt, 1.0, I); });
        t.both([&](auto &w) { return add_shape(w, rbc::Sphere{0.3}, vec3{x0 + 1, 0.9, 0}, tilt, 1.0, I); });
        t.both([&](auto &w) { return add_shape(w, rbc::Capsule{0.3, 0.15}, vec3{x0 + 2, 1.0, 0}, tilt, 1.0, I); });
        t.both([&](auto &w) { return add_shape(w, rbc::Cylinder{0.25, 0.2}, vec3{x0 + 3, 0.9, 0}, tilt, 1.0, I); });
        t.both([&](auto &w) { return add_shape(w, rbc::Cone{0.25, 0.25}, vec3{x0 + 4, 0.9, 0}, tilt, 1.0, I); });
        t.both([&](auto &w) {
            return add_shape(w, rbc::Ellipsoid{vec3{0.3, 0.2, 0.25}}, vec3{x0 + 5, 0.9, 0}, tilt, 1.0, I);
        });
        t.both([&](auto &w) { return add_shape(w, rbc::ConvexHull{cube}, vec3{x0 + 6, 0.9, 0}, tilt, 1.0, I); });
        // a stack across two of them: box on box and hull on box
        t.both([&](auto &w) { return add_shape(w, rbc::Box{vec3{0.25, 0.2, 0.25}}, vec3{x0, 1.5, 0.05}, quat{}, 1.0, I); });
        t.both([&](auto &w) { return add_shape(w, rbc::ConvexHull{cube}, vec3{x0, 2.3, 0.0}, tilt, 1.0, I); });
        t.step(90);
        for (uint32_t i = 1; i < t.gpu.bodies.count(); ++i)
        {
            CHECK(t.gpu.bodies.position[i].y > 0.0);
            CHECK(t.gpu.bodies.position[i].y < 3.0);
        }
        CHECK(t.gpu.contacts.n_contacts == t.ref.contacts.n_contacts);
        CHECK(t.gpu.contacts.n_contacts > 0);
    }

    void joints_with_every_parameter()
    {
        Twin t(1.0 / 60.0, 20);
        const smat3 I{0.02, 0.03, 0.02, 0, 0, 0};
        t.both([](auto &w) {
            rbps::BodyParams a;
            a.type = rbps::STATIC;
            a.position = vec3{0, 5, 0};
            return w.create_body(a);
        });
        for (int k = 0; k < 4; ++k)
            t.both([&](auto &w) {
                rbps::BodyParams b;
                b.mass = 1.0 + 0.5 * k;
                b.inertia_tensor = I;
                b.position = vec3{0.6 * (k + 1), 5.0 - 0.1 * k, 0.05 * k};
                b.linear_velocity = vec3{0.1 * k, 0, -0.2};
                b.angular_velocity = vec3{0, 0.3, 0.1 * k};
                return w.create_body(b);
            });
        t.both([](auto &w) {
            rbps::RevoluteJointParams r;
            r.body_1 = 0;
            r.body_2 = 1;
            r.aligned_axis = vec3{0, 0, 1};
            r.limit_axis = vec3{1, 0, 0};
            r.r_1 = vec3{0.3, 0, 0};
            r.r_2 = vec3{-0.3, 0, 0};
            r.compliance = 1e-6;
            return w.create_revolute_joint(r);
        });
        t.both([](auto &w) {
            rbps::RevoluteJointParams r;
            r.body_1 = 1;
            r.body_2 = 2;
            r.aligned_axis = vec3{0, 0, 1};
            r.limit_axis = vec3{1, 0, 0};
            r.r_1 = vec3{0.3, 0, 0};
            r.r_2 = vec3{-0.3, 0, 0};
            r.limited = true;
            r.lower_limit = -0.6;
            r.upper_limit = 0.6;
            return w.create_revolute_joint(r);
        });
        t.both([](auto &w) {
            rbps::PrismaticJointParams p;
            p.body_1 = 2;
            p.body_2 = 3;
            p.moving_axis = vec3{1, 0, 0};
            p.r_1 = vec3{0.3, 0, 0};
            p.r_2 = vec3{-0.3, 0, 0};
            p.limited = true;
            p.lower_limit = -0.1;
            p.upper_limit = 0.1;
            p.damping = 0.5;
            return w.create_prismatic_joint(p);
        });
        t.both([](auto &w) {
            rbps::FixedJointParams f;
            f.body_1 = 3;
            f.body_2 = 4;
            f.r_1 = vec3{0.3, 0, 0};
            f.r_2 = vec3{-0.3, 0, 0};
            return w.create_fixed_joint(f);
        });
        CHECK(t.gpu.joints.count() == 4);
        t.step(60);
        CHECK(t.gpu.bodies.position[4].y < 5.0); // the chain swings down
    }

    struct Case
    {
        const char *name;
        void (*fn)();
    };
} // namespace

int main()
{
    const Case cases[] = {{"world_parameterized_construction", parameterized_construction},
                          {"world_create_body_returns_valid_id", create_body_returns_valid_id},
                          {"world_create_multiple_bodies", create_multiple_bodies},
                          {"world_step_empty_world", step_empty_world},
                          {"world_step_single_body_no_collider", step_single_body_no_collider},
                          {"world_free_fall_moves_body_downward", free_fall_moves_body_downward},
                          {"world_free_fall_velocity_increases", free_fall_velocity_increases},
                          {"world_static_body_does_not_move", static_body_does_not_move},
                          {"world_sphere_lands_on_ground", sphere_lands_on_ground},
                          {"world_sphere_does_not_tunnel_through_ground", sphere_does_not_tunnel_through_ground},
                          {"world_two_spheres_collide_and_separate", two_spheres_collide_and_separate},
                          {"world_collision_conserves_momentum_approximately",
                           collision_conserves_momentum_approximately},
                          {"world_contacts_cleared_each_frame", contacts_cleared_each_frame},
                          {"world_no_contacts_when_bodies_separated", no_contacts_when_bodies_separated},
                          {"every_shape_on_a_plane", every_shape_on_a_plane},
                          {"joints_with_every_parameter", joints_with_every_parameter}};
    int failed = 0;
    for (const Case &c : cases)
    {
        const int before = g_failures;
        try
        {
            c.fn();
        }
        catch (const rbps_gpu::Error &e)
        {
            std::printf("    rbps_gpu::Error %d: %s\n", e.code, e.what());
            ++g_failures;
        }
        const bool ok = g_failures == before;
        failed += ok ? 0 : 1;
        std::printf("%s %s\n", ok ? "PASS" : "FAIL", c.name);
    }
    std::printf("%d of %zu scenarios failed\n", failed, sizeof(cases) / sizeof(cases[0]));
    return failed ? 1 : 0;
}
