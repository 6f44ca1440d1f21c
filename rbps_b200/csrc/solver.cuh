// solver.cuh - body integration and the XPBD contact / joint rows.
//
// Device restatement, with the reference's operation order, of
//   Body.cpp:11-109        integrate, velocity update, impulse appliers,
//                          generalised inverse masses
//   Contact.cpp:35-289     position-level normal + friction, velocity-level
//                          restitution + dynamic friction
//   Constraint.cpp:5-106   compliant XPBD rows
//   Joint.cpp:18-267       joint errors and damping
// The world-space inverse inertia is a pure function of the body's current
// orientation at every point the reference reads it (every read follows an
// update_inertia_tensor_world of the same body with no orientation change
// in between), so it is recomputed from the orientation here instead of
// being stored.
#pragma once
#include "math.cuh"

// How the per-row contact relaxation routines are compiled: inline by
// default, so the two bodies a pair relaxes stay in registers across its
// rows; -DRBPS_SOLVER_OUTLINE makes them separate functions (smaller kernel
// code, bodies passed through the stack).
#ifdef RBPS_SOLVER_OUTLINE
#define RBPS_SOLVER_CALL __noinline__
#else
#define RBPS_SOLVER_CALL __forceinline__
#endif

namespace rbps_gpu
{
    template <class T> struct alignas(4 * sizeof(T)) V4
    {
        T x, y, z, w;
    };
    template <class T> struct alignas(4 * sizeof(T)) Q4
    {
        T w, x, y, z;
    };
    template <class T> struct alignas(8 * sizeof(T)) S8
    {
        T xx, yy, zz, xy, xz, yz, p0, p1;
    };

    template <class T> __device__ __forceinline__ vec3<T> v3(const V4<T> &a) { return {a.x, a.y, a.z}; }
    template <class T> __device__ __forceinline__ V4<T> v4(const vec3<T> &a, T w = T(0)) { return {a.x, a.y, a.z, w}; }
    template <class T> __device__ __forceinline__ quat<T> q4(const Q4<T> &a) { return {a.w, a.x, a.y, a.z}; }
    template <class T> __device__ __forceinline__ Q4<T> q4s(const quat<T> &a) { return {a.w, a.x, a.y, a.z}; }
    template <class T> __device__ __forceinline__ smat3<T> s3(const S8<T> &a) { return {a.xx, a.yy, a.zz, a.xy, a.xz, a.yz}; }

    enum : uint8_t
    {
        kStatic = 0,
        kDynamic = 1
    };

    // Body SoA of one batch (global body index).  T = solver scalar,
    // P = position scalar (double in the FP32_POS64 mode).
    template <class T, class P>
    struct Bodies
    {
        V4<P> *pos;      // position
        Q4<T> *rot;      // orientation
        V4<T> *lin;      // linear velocity; w = inverse mass
        V4<T> *ang;      // angular velocity
        V4<P> *prev_pos;
        Q4<T> *prev_rot;
        V4<T> *force;
        V4<T> *torque;
        S8<T> *inertia;     // body-frame inertia tensor
        S8<T> *inv_inertia; // body-frame inverse inertia tensor
        uint8_t *type;

        __device__ __forceinline__ bool is_static(uint32_t i) const { return type[i] == kStatic; }
        __device__ __forceinline__ vec3<T> x(uint32_t i) const { return vec3<T>(v3(pos[i])); }
        __device__ __forceinline__ quat<T> q(uint32_t i) const { return q4(rot[i]); }
        __device__ __forceinline__ T inv_mass(uint32_t i) const { return lin[i].w; }
        __device__ __forceinline__ smat3<T> inv_inertia_world(uint32_t i) const
        {
            return world_tensor(q(i), s3(inv_inertia[i]));
        }
        __device__ __forceinline__ void set_q(uint32_t i, const quat<T> &v) const { rot[i] = q4s(v); }
        __device__ __forceinline__ void set_x(uint32_t i, const vec3<T> &v) const
        {
            pos[i] = V4<P>{P(v.x), P(v.y), P(v.z), P(0)};
        }
    };

    // ------------------------------------------------------- Body.cpp
    // update_position_and_orientation for one dynamic body (Body.cpp:18-39)
    template <class T, class P>
    __device__ void integrate_body(const Bodies<T, P> &B, uint32_t i, T dt)
    {
        if (B.is_static(i))
            return;
        const quat<T> q0 = B.q(i);
        const mat3<T> R = mat3_cast(q0);
        const smat3<T> Iw = sym_of(mul(R, s3(B.inertia[i])) * R.transpose());
        const smat3<T> Iinvw = sym_of(mul(R, s3(B.inv_inertia[i])) * R.transpose());
        B.prev_pos[i] = B.pos[i];
        V4<T> l = B.lin[i];
        vec3<T> v = v3(l);
        v += v3(B.force[i]) * l.w * dt;
        B.lin[i] = v4(v, l.w);
        vec3<T> x = B.x(i);
        x += v * dt;
        B.set_x(i, x);
        B.prev_rot[i] = B.rot[i];
        vec3<T> w = v3(B.ang[i]);
        w += (Iinvw * dt) * (v3(B.torque[i]) - cross(w, Iw * w));
        B.ang[i] = v4(w);
        const vec3<T> os = w * (T(0.5) * dt);
        const quat<T> r(T(0.0), os.x, os.y, os.z);
        B.set_q(i, normalize(q0 + r * q0));
    }

    // integrate_body of body i of S, written to body j of D: the pose and
    // velocities go to D (a static body is copied as it is), the previous
    // pose to D's previous-pose arrays, and the type is copied.  The same
    // operations in the same order as integrate_body; a team that keeps its
    // world in shared memory loads and integrates each body in one pass.
    template <class T, class P>
    __device__ void integrate_body_into(const Bodies<T, P> &S, uint32_t i, const Bodies<T, P> &D, uint32_t j, T dt)
    {
        const uint8_t ty = S.type[i];
        const V4<P> p0 = S.pos[i];
        const Q4<T> r0 = S.rot[i];
        const V4<T> l = S.lin[i];
        const V4<T> a0 = S.ang[i];
        D.type[j] = ty;
        if (ty == kStatic)
        {
            D.pos[j] = p0;
            D.rot[j] = r0;
            D.lin[j] = l;
            D.ang[j] = a0;
            D.prev_pos[j] = S.prev_pos[i];
            D.prev_rot[j] = S.prev_rot[i];
            return;
        }
        const quat<T> q0 = q4(r0);
        const mat3<T> R = mat3_cast(q0);
        const smat3<T> Iw = sym_of(mul(R, s3(S.inertia[i])) * R.transpose());
        const smat3<T> Iinvw = sym_of(mul(R, s3(S.inv_inertia[i])) * R.transpose());
        D.prev_pos[j] = p0;
        vec3<T> v = v3(l);
        v += v3(S.force[i]) * l.w * dt;
        D.lin[j] = v4(v, l.w);
        vec3<T> x = vec3<T>(v3(p0));
        x += v * dt;
        D.pos[j] = V4<P>{P(x.x), P(x.y), P(x.z), P(0)};
        D.prev_rot[j] = r0;
        vec3<T> w = v3(a0);
        w += (Iinvw * dt) * (v3(S.torque[i]) - cross(w, Iw * w));
        D.ang[j] = v4(w);
        const vec3<T> os = w * (T(0.5) * dt);
        const quat<T> r(T(0.0), os.x, os.y, os.z);
        D.rot[j] = q4s(normalize(q0 + r * q0));
    }

    // update_velocities for one body (Body.cpp:41-57)
    template <class T, class P>
    __device__ void update_velocity_body(const Bodies<T, P> &B, uint32_t i, T inv_dt)
    {
        if (B.is_static(i))
            return;
        const T im = B.lin[i].w;
        const vec3<T> v = (B.x(i) - vec3<T>(v3(B.prev_pos[i]))) * inv_dt;
        B.lin[i] = v4(v, im);
        const quat<T> dq = B.q(i) * conjugate(q4(B.prev_rot[i]));
        vec3<T> w = vec3<T>(dq.x, dq.y, dq.z) * (T(2) * inv_dt);
        w = dq.w >= T(0) ? w : -w;
        B.ang[i] = v4(w);
    }

    // ------------------------------------------------------- register-resident bodies
    // The two bodies of a pair are loaded once per candidate (all its contact
    // rows) or per joint (all its rows), relaxed in registers and stored
    // once: every row reads the state the previous row wrote, exactly as the
    // reference's in-place updates do, without a memory round trip on the
    // serial critical path.
    template <class T, class P>
    struct BodyR
    {
        vec3<T> x, v, w, xp;
        quat<T> q, qp;
        smat3<T> Iinv; // body-frame inverse inertia
        T inv_mass;
        bool stat;
    };

    template <class T, class P>
    __device__ __forceinline__ void load_body(const Bodies<T, P> &B, uint32_t i, BodyR<T, P> &b, bool prev)
    {
        b.stat = B.is_static(i);
        b.x = B.x(i);
        b.q = B.q(i);
        const V4<T> l = B.lin[i];
        b.v = v3(l);
        b.inv_mass = l.w;
        b.w = v3(B.ang[i]);
        b.Iinv = s3(B.inv_inertia[i]);
        if (prev)
        {
            b.xp = vec3<T>(v3(B.prev_pos[i]));
            b.qp = q4(B.prev_rot[i]);
        }
    }

    template <class T, class P>
    __device__ __forceinline__ void store_pose(const Bodies<T, P> &B, uint32_t i, const BodyR<T, P> &b)
    {
        if (b.stat)
            return;
        B.set_x(i, b.x);
        B.set_q(i, b.q);
    }

    template <class T, class P>
    __device__ __forceinline__ void store_vel(const Bodies<T, P> &B, uint32_t i, const BodyR<T, P> &b)
    {
        if (b.stat)
            return;
        B.lin[i] = v4(b.v, b.inv_mass);
        B.ang[i] = v4(b.w);
    }

    // get_positional_generalized_inverse_mass (Body.cpp:94-101); Iw receives
    // the refreshed world inverse inertia for the impulse appliers.
    template <class T, class P>
    __device__ __forceinline__ T pos_w(const BodyR<T, P> &b, const vec3<T> &r, const vec3<T> &n, smat3<T> &Iw)
    {
        if (b.stat)
            return T(0.0);
        Iw = world_tensor(b.q, b.Iinv);
        const vec3<T> c = cross(r, n);
        return b.inv_mass + dot(c, Iw * c);
    }

    // get_rotational_generalized_inverse_mass (Body.cpp:103-109)
    template <class T, class P>
    __device__ __forceinline__ T rot_w(const BodyR<T, P> &b, const vec3<T> &n, smat3<T> &Iw)
    {
        if (b.stat)
            return T(0.0);
        Iw = world_tensor(b.q, b.Iinv);
        return dot(n, Iw * n);
    }

    // apply_positional_constraint_impulse (Body.cpp:59-68)
    template <class T, class P>
    __device__ __forceinline__ void pos_impulse(BodyR<T, P> &b, const smat3<T> &Iw, const vec3<T> &J, const vec3<T> &r)
    {
        if (b.stat)
            return;
        b.x += J * b.inv_mass;
        const vec3<T> rv = Iw * cross(r, J) * T(0.5);
        const quat<T> rq(T(0.0), rv.x, rv.y, rv.z);
        b.q = normalize(b.q + rq * b.q);
    }

    // apply_rotational_constraint_impulse (Body.cpp:70-77)
    template <class T, class P>
    __device__ __forceinline__ void rot_impulse(BodyR<T, P> &b, const smat3<T> &Iw, const vec3<T> &J)
    {
        if (b.stat)
            return;
        const vec3<T> rv = Iw * J * T(0.5);
        const quat<T> rq(T(0.0), rv.x, rv.y, rv.z);
        b.q = normalize(b.q + rq * b.q);
    }

    // apply_positional_velocity_constraint_impulse (Body.cpp:79-85)
    template <class T, class P>
    __device__ __forceinline__ void pos_vel_impulse(BodyR<T, P> &b, const smat3<T> &Iw, const vec3<T> &J,
                                                    const vec3<T> &r)
    {
        if (b.stat)
            return;
        b.v += J * b.inv_mass;
        b.w += Iw * cross(r, J);
    }

    // apply_rotational_velocity_constraint_impulse (Body.cpp:87-92)
    template <class T, class P>
    __device__ __forceinline__ void rot_vel_impulse(BodyR<T, P> &b, const smat3<T> &Iw, const vec3<T> &J)
    {
        if (b.stat)
            return;
        b.w += Iw * J;
    }

    // ------------------------------------------------------- contacts
    template <class T, class P>
    struct ContactPt
    {
        V4<T> ra;      // r_a_local
        V4<T> rb;      // r_b_local
        V4<P> pa;      // point_on_a
        V4<P> pb;      // point_on_b
        T lam_n, lam_t, vrel, depth;
        int coll;      // collision flag
        int pad_[3];
    };

    // Narrowphase output of one candidate pair: up to four ContactList rows
    // sharing normal, bodies and material mix.
    template <class T, class P>
    struct CandContacts
    {
        V4<T> normal;
        V4<T> mat; // restitution, static friction, dynamic friction
        int n;
        int pad_[3];
        ContactPt<T, P> pt[4];
    };

    // apply_constraint_position_level + solve_normal_constraint +
    // solve_tangent_constraint (Contact.cpp:35-195) for one contact row.
    template <class T, class P>
    __device__ RBPS_SOLVER_CALL void contact_position(BodyR<T, P> &A, BodyR<T, P> &Bb, const vec3<T> &n, T static_friction,
                                     ContactPt<T, P> &c, T inv_h)
    {
        const vec3<T> ra_l = v3(c.ra), rb_l = v3(c.rb);
        const vec3<T> p_a = A.x + rotate(A.q, ra_l);
        const vec3<T> p_b = Bb.x + rotate(Bb.q, rb_l);
        c.pa = V4<P>{P(p_a.x), P(p_a.y), P(p_a.z), P(0)};
        c.pb = V4<P>{P(p_b.x), P(p_b.y), P(p_b.z), P(0)};
        const T d = dot(p_a - p_b, n);
        if (d <= T(0.0))
        {
            c.coll = 0;
            return;
        }
        c.coll = 1;
        const vec3<T> r_a = p_a - A.x;
        const vec3<T> r_b = p_b - Bb.x;
        {
            const vec3<T> v_rel = (A.v + cross(A.w, r_a)) - (Bb.v + cross(Bb.w, r_b));
            c.vrel = dot(v_rel, n);
        }
        {
            smat3<T> Ia, Ib;
            const T w_a = pos_w(A, r_a, n, Ia);
            const T w_b = pos_w(Bb, r_b, n, Ib);
            const T denom = w_a + w_b;
            if (!(denom < T(kEpsilon)))
            {
                const T dl = div_guarded(-d, denom);
                c.lam_n += dl;
                if (c.lam_n > T(0.0))
                    c.lam_n = T(0.0);
                const vec3<T> imp = dl * n;
                pos_impulse(A, Ia, imp, r_a);
                pos_impulse(Bb, Ib, -imp, r_b);
            }
        }
        {
            const vec3<T> ra_wc = rotate(A.q, ra_l);
            const vec3<T> rb_wc = rotate(Bb.q, rb_l);
            const vec3<T> pa_cur = A.x + ra_wc;
            const vec3<T> pb_cur = Bb.x + rb_wc;
            c.pa = V4<P>{P(pa_cur.x), P(pa_cur.y), P(pa_cur.z), P(0)};
            c.pb = V4<P>{P(pb_cur.x), P(pb_cur.y), P(pb_cur.z), P(0)};
            const vec3<T> prev_pa = A.xp + rotate(A.qp, ra_l);
            const vec3<T> prev_pb = Bb.xp + rotate(Bb.qp, rb_l);
            const vec3<T> dp = (pa_cur - prev_pa) - (pb_cur - prev_pb);
            const vec3<T> dpt = dp - dot(dp, n) * n;
            const T slip = length(dpt);
            if (slip < T(kEpsilon))
                return;
            const vec3<T> t = normalize(dpt);
            smat3<T> Ia, Ib;
            const T w_a = pos_w(A, ra_wc, t, Ia);
            const T w_b = pos_w(Bb, rb_wc, t, Ib);
            const T denom = w_a + w_b;
            if (denom < T(kEpsilon))
                return;
            const T dl = div_guarded(-slip, denom);
            const T old = c.lam_t;
            c.lam_t += dl;
            const T cone = static_friction * c.lam_n;
            if (c.lam_t < cone)
                c.lam_t = cone;
            const T actual = c.lam_t - old;
            if (rabs(actual) < T(kEpsilon))
                return;
            const vec3<T> imp = actual * t;
            pos_impulse(A, Ia, imp, ra_wc);
            pos_impulse(Bb, Ib, -imp, rb_wc);
        }
    }

    // apply_constraint_velocity_level (Contact.cpp:206-289) for one row.
    template <class T, class P>
    __device__ RBPS_SOLVER_CALL void contact_velocity(BodyR<T, P> &A, BodyR<T, P> &Bb, const vec3<T> &n, T restitution,
                                     T dynamic_friction, const ContactPt<T, P> &c, T h)
    {
        if (!c.coll)
            return;
        const vec3<T> r_a = vec3<T>(v3(c.pa)) - A.x;
        const vec3<T> r_b = vec3<T>(v3(c.pb)) - Bb.x;
        const vec3<T> v_rel = (A.v + cross(A.w, r_a)) - (Bb.v + cross(Bb.w, r_b));
        const T v_n = dot(v_rel, n);
        const vec3<T> v_t = v_rel - n * v_n;
        const T v_t_mag = length(v_t);
        T e = restitution;
        if (rabs(c.vrel) <= T(2.0 * 9.8) * h)
            e = T(0.0);
        const T v_n_target = rmin(-e * c.vrel, T(0.0));
        const T dv_n = v_n_target - v_n;
        T dv_t = T(0.0);
        if (v_t_mag > T(kEpsilon))
        {
            const T limit = div_guarded(dynamic_friction * rabs(c.lam_n), h);
            dv_t = -rmin(limit, v_t_mag);
        }
        smat3<T> Ia, Ib;
        const T w_a_n = pos_w(A, r_a, n, Ia);
        const T w_b_n = pos_w(Bb, r_b, n, Ib);
        const T denom_n = w_a_n + w_b_n;
        if (denom_n > T(kEpsilon) && rabs(dv_n) > T(kEpsilon))
        {
            const vec3<T> imp = div_guarded(dv_n, denom_n) * n;
            pos_vel_impulse(A, Ia, imp, r_a);
            pos_vel_impulse(Bb, Ib, -imp, r_b);
        }
        if (v_t_mag > T(kEpsilon) && rabs(dv_t) > T(kEpsilon))
        {
            const vec3<T> t = v_t * div_guarded(T(1.0), v_t_mag);
            const T w_a_t = pos_w(A, r_a, t, Ia);
            const T w_b_t = pos_w(Bb, r_b, t, Ib);
            const T denom_t = w_a_t + w_b_t;
            if (denom_t > T(kEpsilon))
            {
                const vec3<T> imp = div_guarded(dv_t, denom_t) * t;
                pos_vel_impulse(A, Ia, imp, r_a);
                pos_vel_impulse(Bb, Ib, -imp, r_b);
            }
        }
    }

    // ------------------------------------------------------- joints
    enum : int
    {
        kRowPositional = 0,
        kRowRotational = 1
    };
    enum : int
    {
        kPrismatic = 0,
        kRevolute = 1,
        kFixed = 2,
        kSpherical = 3
    };
    enum : int
    {
        kActFree = 0,
        kActPosition = 1,
        kActSpeed = 2
    };

    // One compliant constraint row (Constraint.hpp CONSTRAINT_FIELDS).
    template <class T>
    struct Row
    {
        V4<T> dir;   // direction, w = magnitude
        V4<T> r1;    // w = compliance
        V4<T> r2;    // w = lambda
        uint32_t b1, b2;
        int type;
        int pad_;
    };

    // One joint (Joint.hpp JOINT_FIELDS); rows are row0 .. row0+count-1.
    template <class T>
    struct Joint
    {
        V4<T> r1, r2, axis, limit_axis;
        T lower, upper, target_pos, target_speed, damping;
        // sin / cos of the half limit angles, from the host libm: the
        // clamped angle of an active limit is exactly lower or upper, so
        // from_axis_angle(n, phi) needs only these (quat.hpp:111-117).
        T sin_lo, cos_lo, sin_hi, cos_hi;
        uint32_t b1, b2, row0;
        int type, act, limited, count;
    };

    // set_value (Constraint.cpp:5-12).  The reference keeps the direction
    // whenever |value| > EPSILON, but normalize() returns the zero vector
    // below |value|^2 < EPSILON, so an error in (1e-9, 3.2e-5) gets a zero
    // direction and a rotational row then divides by w1 + w2 = 0.  Double
    // precision reproduces that exactly; in float the alignment noise
    // (~1e-7) lands in that band every substep, so the FP32 instantiation
    // divides by the magnitude directly.
    template <class T>
    __device__ __forceinline__ void row_set_value(Row<T> &r, const vec3<T> &value)
    {
        const T mag = length(value);
        vec3<T> d(T(1.0), T(0.0), T(0.0));
        if (mag > T(kEpsilon))
        {
            if constexpr (sizeof(T) == 8)
                d = normalize(value);
            else
                d = value * div_guarded(T(1), mag);
        }
        r.dir = V4<T>{d.x, d.y, d.z, mag};
    }

    // The ball joint's rows (no reference counterpart) take the direction
    // value / |value| whenever |value| > EPSILON, in every precision, so they
    // stay clear of the zero-direction band of set_value above.
    template <class T>
    __device__ __forceinline__ void row_set_value_div(Row<T> &r, const vec3<T> &value)
    {
        const T mag = length(value);
        vec3<T> d(T(1.0), T(0.0), T(0.0));
        if (mag > T(kEpsilon))
            d = value * div_guarded(T(1.0), mag);
        r.dir = V4<T>{d.x, d.y, d.z, mag};
    }

    // compute_delta_lambda (Constraint.cpp:14-18)
    template <class T>
    __device__ __forceinline__ T row_delta_lambda(const Row<T> &r, T w1, T w2, T inv_h)
    {
        const T alpha = r.r1.w * inv_h * inv_h;
        return (-r.dir.w - alpha * r.r2.w) / (w1 + w2 + alpha);
    }

    // compute_{rotational,positional}_constraint_impulse (Constraint.cpp:20-46)
    template <class T, class P>
    __device__ void solve_row(BodyR<T, P> &b1, BodyR<T, P> &b2, Row<T> &r, T inv_h)
    {
        const vec3<T> dir = v3(r.dir);
        smat3<T> I1, I2;
        if (r.type == kRowRotational)
        {
            const T w1 = rot_w(b1, dir, I1);
            const T w2 = rot_w(b2, dir, I2);
            const T dl = row_delta_lambda(r, w1, w2, inv_h);
            r.r2.w += dl;
            const vec3<T> imp = dl * dir;
            rot_impulse(b1, I1, imp);
            rot_impulse(b2, I2, -imp);
        }
        else
        {
            const vec3<T> r1 = rotate(b1.q, v3(r.r1));
            const vec3<T> r2 = rotate(b2.q, v3(r.r2));
            const T w1 = pos_w(b1, r1, dir, I1);
            const T w2 = pos_w(b2, r2, dir, I2);
            const T dl = row_delta_lambda(r, w1, w2, inv_h);
            r.r2.w += dl;
            const vec3<T> imp = dl * dir;
            pos_impulse(b1, I1, imp, r1);
            pos_impulse(b2, I2, -imp, r2);
        }
    }

    // compute_{prismatic,revolute,fixed}_joint_errors (Joint.cpp:18-182)
    template <class T, class P>
    __device__ void joint_errors(const Bodies<T, P> &B, Joint<T> &j, Row<T> *rows, T h)
    {
        const uint32_t b1 = j.b1, b2 = j.b2;
        const quat<T> q1 = B.q(b1), q2 = B.q(b2);
        if (j.type == kRevolute)
        {
            const vec3<T> a1 = rotate(q1, v3(j.axis));
            const vec3<T> a2 = rotate(q2, v3(j.axis));
            row_set_value(rows[0], cross(a1, a2));
            const vec3<T> r1w = rotate(q1, v3(j.r1));
            const vec3<T> r2w = rotate(q2, v3(j.r2));
            const vec3<T> p1 = B.x(b1) + r1w;
            const vec3<T> p2 = B.x(b2) + r2w;
            row_set_value(rows[1], p1 - p2);
            const vec3<T> b1l = rotate(q1, v3(j.limit_axis));
            const vec3<T> b2l = rotate(q2, v3(j.limit_axis));
            vec3<T> err_limit(T(0.0), T(0.0), T(0.0));
            if (j.limited)
            {
                // compute_angle_limit_correction (Joint.cpp:73-90)
                const T phi = atan2(dot(cross(b1l, b2l), a1), dot(b1l, b2l));
                if (phi < j.lower || phi > j.upper)
                {
                    const bool lo = phi < j.lower; // clamp(phi, lower, upper)
                    const T s = lo ? j.sin_lo : j.sin_hi;
                    const T c = lo ? j.cos_lo : j.cos_hi;
                    const vec3<T> nn = normalize(a1);
                    const quat<T> rq(c, nn.x * s, nn.y * s, nn.z * s);
                    const vec3<T> n1 = rotate(rq, b1l);
                    err_limit = cross(n1, b2l);
                }
            }
            row_set_value(rows[2], -err_limit);
            vec3<T> err_drive(T(0.0), T(0.0), T(0.0));
            if (j.act != kActFree)
            {
                if (j.act == kActSpeed)
                    j.target_pos += j.target_speed * h;
                const T theta = j.target_pos + T(3.14159265358979323846);
                const T ct = cos(theta), st = sin(theta);
                const vec3<T> bt = b1l * ct + cross(a1, b1l) * st + a1 * (dot(a1, b1l)) * (T(1) - ct);
                err_drive = cross(bt, b2l);
            }
            row_set_value(rows[3], err_drive);
        }
        else if (j.type == kPrismatic)
        {
            const quat<T> dq = q1 * conjugate(q2);
            row_set_value(rows[0], vec3<T>(dq.x, dq.y, dq.z) * T(2.0));
            const vec3<T> r1w = rotate(q1, v3(j.r1));
            const vec3<T> r2w = rotate(q2, v3(j.r2));
            const vec3<T> p1 = B.x(b1) + r1w;
            const vec3<T> p2 = B.x(b2) + r2w;
            const vec3<T> dp = p1 - p2;
            const vec3<T> axis = rotate(q1, v3(j.axis));
            const T pos = dot(dp, axis);
            T overshoot = T(0);
            if (j.limited)
            {
                const T cl = rclamp(pos, j.lower, j.upper);
                overshoot = pos - cl;
            }
            row_set_value(rows[1], dp - axis * pos + axis * overshoot);
            vec3<T> err_drive(T(0.0), T(0.0), T(0.0));
            if (j.act != kActFree)
            {
                if (j.act == kActSpeed)
                    j.target_pos += j.target_speed * h;
                const vec3<T> ddp = p2 - p1;
                const T curr = dot(ddp, axis);
                err_drive = (j.target_pos - curr) * axis;
            }
            row_set_value(rows[2], err_drive);
        }
        else if (j.type == kSpherical)
        {
            // a ball joint evaluates its rows when they are solved
            // (solve_joint_rows), not here
        }
        else
        {
            const quat<T> dq = q1 * conjugate(q2);
            row_set_value(rows[0], vec3<T>(dq.x, dq.y, dq.z) * T(2.0));
            const vec3<T> r1w = rotate(q1, v3(j.r1));
            const vec3<T> r2w = rotate(q2, v3(j.r2));
            const vec3<T> p1 = B.x(b1) + r1w;
            const vec3<T> p2 = B.x(b2) + r2w;
            row_set_value(rows[1], p1 - p2);
        }
    }

    // Ball joint (RBPS_JOINT_SPHERICAL; no reference counterpart), both rows
    // evaluated on the current poses right before each is solved, as XPBD
    // does (Mueller et al. 2020, Alg. 2), with lambda restarted every
    // substep.  The reference instead sets every joint row's error before
    // solving any (World.hpp:168-173); on a hanging chain those stale errors
    // over-correct and the chain diverges within a few steps.
    //   row 0: attachment p1 - p2, as the revolute joint's (Joint.cpp:107-111)
    //   row 1: swing cone -- the swing angle phi between the bodies' axes
    //          about n = normalize(a1 x a2), limited to [lower, upper] =
    //          [-cone, cone] as compute_angle_limit_correction does
    //          (Joint.cpp:73-90), whose from_axis_angle normalizes n again
    template <class T, class P>
    __device__ __forceinline__ void solve_ball_joint(BodyR<T, P> &b1, BodyR<T, P> &b2, const Joint<T> &j,
                                                     Row<T> *rows, T inv_h)
    {
        {
            const vec3<T> p1 = b1.x + rotate(b1.q, v3(j.r1));
            const vec3<T> p2 = b2.x + rotate(b2.q, v3(j.r2));
            rows[0].r2.w = T(0.0);
            row_set_value_div(rows[0], p1 - p2);
            solve_row(b1, b2, rows[0], inv_h);
        }
        vec3<T> err_limit(T(0.0), T(0.0), T(0.0));
        if (j.limited)
        {
            const vec3<T> a1 = rotate(b1.q, v3(j.axis));
            const vec3<T> a2 = rotate(b2.q, v3(j.axis));
            const vec3<T> c = cross(a1, a2);
            const T phi = atan2(length(c), dot(a1, a2));
            if (phi < j.lower || phi > j.upper)
            {
                const bool lo = phi < j.lower;
                const T s = lo ? j.sin_lo : j.sin_hi;
                const T co = lo ? j.cos_lo : j.cos_hi;
                const vec3<T> nn = normalize(normalize(c));
                const quat<T> rq(co, nn.x * s, nn.y * s, nn.z * s);
                err_limit = cross(rotate(rq, a1), a2);
            }
        }
        rows[1].r2.w = T(0.0);
        row_set_value_div(rows[1], -err_limit);
        solve_row(b1, b2, rows[1], inv_h);
    }

    // All rows of one joint, in row order, its two bodies held in registers.
    template <class T, class P>
    __device__ __noinline__ void solve_joint_rows(const Bodies<T, P> &B, const Joint<T> &j, Row<T> *rows, T inv_h)
    {
        BodyR<T, P> b1, b2;
        load_body(B, j.b1, b1, false);
        load_body(B, j.b2, b2, false);
        if (j.type == kSpherical)
            solve_ball_joint(b1, b2, j, rows, inv_h);
        else
            for (int r = 0; r < j.count; ++r)
                solve_row(b1, b2, rows[r], inv_h);
        store_pose(B, j.b1, b1);
        store_pose(B, j.b2, b2);
    }

    // apply_{prismatic,revolute}_joint_damping (Joint.cpp:184-220)
    template <class T, class P>
    __device__ __noinline__ void joint_damping(const Bodies<T, P> &B, const Joint<T> &j, T h)
    {
        BodyR<T, P> b1, b2;
        load_body(B, j.b1, b1, false);
        load_body(B, j.b2, b2, false);
        if (j.type == kRevolute)
        {
            const vec3<T> dw = (b2.w - b1.w) * rmin(j.damping * h, T(1.0));
            if (length_sq(dw) < T(kEpsilon))
                return;
            const vec3<T> n = normalize(dw);
            smat3<T> I1, I2;
            const T w1 = rot_w(b1, n, I1);
            const T w2 = rot_w(b2, n, I2);
            const vec3<T> imp = dw / (w1 + w2);
            rot_vel_impulse(b1, I1, imp);
            rot_vel_impulse(b2, I2, -imp);
        }
        else if (j.type == kPrismatic)
        {
            const vec3<T> dv = (b2.v - b1.v) * rmin(j.damping * h, T(1.0));
            if (length_sq(dv) < T(kEpsilon))
                return;
            const vec3<T> r1 = rotate(b1.q, v3(j.r1));
            const vec3<T> r2 = rotate(b2.q, v3(j.r2));
            const vec3<T> n = normalize(dv);
            smat3<T> I1, I2;
            const T w1 = pos_w(b1, r1, n, I1);
            const T w2 = pos_w(b2, r2, n, I2);
            const vec3<T> imp = dv / (w1 + w2);
            pos_vel_impulse(b1, I1, imp, r1);
            pos_vel_impulse(b2, I2, -imp, r2);
        }
        else
            return;
        store_vel(B, j.b1, b1);
        store_vel(B, j.b2, b2);
    }
} // namespace rbps_gpu
