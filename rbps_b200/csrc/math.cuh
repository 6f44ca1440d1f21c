// math.cuh - vector / quaternion / 3x3 math for the device engine.
//
// Templated on the scalar type T (double for the FP64 reference-order mode,
// float for the FP32 modes).  Every expression keeps the operand order of
// the reference's math3d headers so that, compiled without FMA contraction
// (-fmad=false for the FP64 translation unit), the FP64 instantiation rounds
// exactly as the reference does on x86-64:
//   vec3 ops / dot / cross / normalize : include/math3d/vec3.hpp:21-204
//   quat product / normalize / rotate  : include/math3d/quat.hpp:84-204
//   mat3 / mat3_cast / smat3           : include/math3d/mat3.hpp:35-315
#pragma once
#include <cstdint>

#define RBPS_HD __host__ __device__ __forceinline__

namespace rbps_gpu
{
    // m3d::EPSILON (core.hpp:49) and the 1-ulp normalisation shortcut
    // threshold used by quat normalize (quat.hpp:157).
    constexpr double kEpsilon = 1e-9;
    constexpr double kQuatUlp = 2.107342e-08;

    // std::abs / std::sqrt; 1/sqrt as two correctly rounded operations
    // (no reciprocal-square-root approximation), as the reference computes it.
    RBPS_HD double rabs(double x) { return fabs(x); }
    RBPS_HD float rabs(float x) { return fabsf(x); }
    RBPS_HD double sqrt_t(double x) { return sqrt(x); }
    RBPS_HD float sqrt_t(float x) { return sqrtf(x); }
    // x / y where y is known to be at least EPSILON (1e-9) in magnitude: in
    // double correctly rounded, as the reference divides; in float on the
    // device the hardware's approximate division (within 2 ulp; it differs
    // in kind from IEEE division only for |y| above 2^126 or denormal, which
    // such a y never is).  The FP32 solver rows divide only through here.
    RBPS_HD double div_guarded(double x, double y) { return x / y; }
    RBPS_HD float div_guarded(float x, float y)
    {
#ifdef __CUDA_ARCH__
        return __fdividef(x, y);
#else
        return x / y;
#endif
    }
    // 1 / sqrt(x) for x >= EPSILON (the normalisations guard it).
    RBPS_HD double inv_sqrt(double x) { return 1.0 / sqrt(x); }
    RBPS_HD float inv_sqrt(float x) { return div_guarded(1.0f, sqrtf(x)); }
    // Squared-length threshold below which a cross product of two unit axes
    // counts as degenerate (parallel edges).  The reference uses EPSILON^2 in
    // double (BoxBox.hpp:45, CapsuleBox.hpp:112); in float the rounding noise
    // of a cross product of nearly parallel unit vectors is ~1e-14, so the
    // FP32 instantiation uses sin^2(1e-5 rad) instead of normalising noise
    // into a separating axis.
    template <class T> RBPS_HD T axis_eps_sq();
    template <> RBPS_HD double axis_eps_sq<double>() { return kEpsilon * kEpsilon; }
    template <> RBPS_HD float axis_eps_sq<float>() { return 1e-10f; }

    // std::min / std::max semantics (operand order matters for -0 and NaN).
    template <class T> RBPS_HD T rmin(T a, T b) { return (b < a) ? b : a; }
    template <class T> RBPS_HD T rmax(T a, T b) { return (a < b) ? b : a; }
    // m3d::clamp (core.hpp:58-62) == std::clamp for ordered values.
    template <class T> RBPS_HD T rclamp(T v, T lo, T hi) { return (v < lo) ? lo : ((v > hi) ? hi : v); }

    template <class T>
    struct vec3
    {
        T x, y, z;
        RBPS_HD vec3() : x(0), y(0), z(0) {}
        RBPS_HD vec3(T a, T b, T c) : x(a), y(b), z(c) {}
        RBPS_HD explicit vec3(T d) : x(d), y(d), z(d) {}
        template <class U>
        RBPS_HD explicit vec3(const vec3<U> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
        RBPS_HD vec3 operator+(const vec3 &r) const { return {x + r.x, y + r.y, z + r.z}; }
        RBPS_HD vec3 operator-(const vec3 &r) const { return {x - r.x, y - r.y, z - r.z}; }
        RBPS_HD vec3 operator*(T s) const { return {x * s, y * s, z * s}; }
        RBPS_HD vec3 operator/(T s) const
        {
            const T inv = T(1.0) / s;
            return {x * inv, y * inv, z * inv};
        }
        RBPS_HD vec3 operator-() const { return {-x, -y, -z}; }
        RBPS_HD vec3 &operator+=(const vec3 &r)
        {
            x += r.x; y += r.y; z += r.z;
            return *this;
        }
        RBPS_HD vec3 &operator-=(const vec3 &r)
        {
            x -= r.x; y -= r.y; z -= r.z;
            return *this;
        }
        RBPS_HD T operator[](int i) const { return (i == 0) ? x : (i == 1) ? y : z; }
    };

    // scalar * vec3 (vec3.hpp:125): components are v.x*s (operand order kept).
    template <class T> RBPS_HD vec3<T> operator*(T s, const vec3<T> &v) { return {v.x * s, v.y * s, v.z * s}; }

    template <class T> RBPS_HD T dot(const vec3<T> &a, const vec3<T> &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    template <class T> RBPS_HD vec3<T> cross(const vec3<T> &a, const vec3<T> &b)
    {
        return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    }
    template <class T> RBPS_HD T length_sq(const vec3<T> &v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
    template <class T> RBPS_HD T length(const vec3<T> &v) { return sqrt_t(length_sq(v)); }
    template <class T> RBPS_HD vec3<T> normalize(const vec3<T> &v)
    {
        const T len_sq = length_sq(v);
        if (len_sq < T(kEpsilon))
            return {T(0), T(0), T(0)};
        const T inv_len = inv_sqrt(len_sq);
        return v * inv_len;
    }

    template <class T>
    struct quat
    {
        T w, x, y, z;
        RBPS_HD quat() : w(1), x(0), y(0), z(0) {}
        RBPS_HD quat(T a, T b, T c, T d) : w(a), x(b), y(c), z(d) {}
        template <class U>
        RBPS_HD explicit quat(const quat<U> &o) : w(T(o.w)), x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
        // Hamilton product (quat.hpp:84-92)
        RBPS_HD quat operator*(const quat &r) const
        {
            quat res;
            res.w = w * r.w - x * r.x - y * r.y - z * r.z;
            res.x = w * r.x + x * r.w + y * r.z - z * r.y;
            res.y = w * r.y + y * r.w + z * r.x - x * r.z;
            res.z = w * r.z + z * r.w + x * r.y - y * r.x;
            return res;
        }
        RBPS_HD quat operator*(T s) const { return {w * s, x * s, y * s, z * s}; }
        RBPS_HD quat operator+(const quat &r) const { return {w + r.w, x + r.x, y + r.y, z + r.z}; }
    };

    // quat.hpp:153-171, including the first-order Pade shortcut
    template <class T> RBPS_HD quat<T> normalize(const quat<T> &q)
    {
        const T mag_sq = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
        if (rabs(T(1.0) - mag_sq) < T(kQuatUlp))
            return q * div_guarded(T(2.0), T(1.0) + mag_sq);
        if (mag_sq < T(kEpsilon))
            return {T(1), T(0), T(0), T(0)};
        return q * inv_sqrt(mag_sq);
    }
    template <class T> RBPS_HD quat<T> conjugate(const quat<T> &q) { return {q.w, -q.x, -q.y, -q.z}; }

    // quat.hpp:188-199: v + 2(s (u x v) + u x (u x v))
    template <class T> RBPS_HD vec3<T> rotate(const quat<T> &q, const vec3<T> &v)
    {
        const vec3<T> u(q.x, q.y, q.z);
        const T s = q.w;
        const vec3<T> uv = cross(u, v);
        const vec3<T> uuv = cross(u, uv);
        return v + ((uv * s) + uuv) * T(2.0);
    }

    // Column-major 3x3 (mat3.hpp:35-166).
    template <class T>
    struct mat3
    {
        vec3<T> c[3];
        RBPS_HD vec3<T> operator*(const vec3<T> &v) const
        {
            return {c[0].x * v.x + c[1].x * v.y + c[2].x * v.z,
                    c[0].y * v.x + c[1].y * v.y + c[2].y * v.z,
                    c[0].z * v.x + c[1].z * v.y + c[2].z * v.z};
        }
        RBPS_HD mat3 operator*(const mat3 &r) const
        {
            mat3 res;
            for (int k = 0; k < 3; ++k)
                res.c[k] = (*this) * r.c[k];
            return res;
        }
        RBPS_HD mat3 transpose() const
        {
            mat3 t;
            t.c[0] = {c[0].x, c[1].x, c[2].x};
            t.c[1] = {c[0].y, c[1].y, c[2].y};
            t.c[2] = {c[0].z, c[1].z, c[2].z};
            return t;
        }
    };

    // mat3.hpp:166-178
    template <class T> RBPS_HD mat3<T> mat3_cast(const quat<T> &q)
    {
        const T x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
        const T xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
        const T yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
        const T wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
        mat3<T> m;
        m.c[0] = {T(1) - (yy + zz), xy + wz, xz - wy};
        m.c[1] = {xy - wz, T(1) - (xx + zz), yz + wx};
        m.c[2] = {xz + wy, yz - wx, T(1) - (xx + yy)};
        return m;
    }

    // Symmetric 3x3 {xx,yy,zz,xy,xz,yz} (mat3.hpp:196-286).
    template <class T>
    struct smat3
    {
        T xx, yy, zz, xy, xz, yz;
        RBPS_HD vec3<T> operator*(const vec3<T> &v) const
        {
            return {xx * v.x + xy * v.y + xz * v.z,
                    xy * v.x + yy * v.y + yz * v.z,
                    xz * v.x + yz * v.y + zz * v.z};
        }
        RBPS_HD smat3 operator*(T s) const { return {xx * s, yy * s, zz * s, xy * s, xz * s, yz * s}; }
    };

    // smat3(const mat3&) symmetrising constructor (mat3.hpp:220-224)
    template <class T> RBPS_HD smat3<T> sym_of(const mat3<T> &m)
    {
        return {m.c[0].x, m.c[1].y, m.c[2].z,
                T(0.5) * (m.c[1].x + m.c[0].y),
                T(0.5) * (m.c[2].x + m.c[0].z),
                T(0.5) * (m.c[2].y + m.c[1].z)};
    }

    // mat3 * smat3 (mat3.hpp:305-313)
    template <class T> RBPS_HD mat3<T> mul(const mat3<T> &l, const smat3<T> &r)
    {
        mat3<T> res;
        res.c[0] = l * vec3<T>{r.xx, r.xy, r.xz};
        res.c[1] = l * vec3<T>{r.xy, r.yy, r.yz};
        res.c[2] = l * vec3<T>{r.xz, r.yz, r.zz};
        return res;
    }

    // update_inertia_tensor_world (Body.cpp:11-16): smat3(R * I * R^T)
    template <class T> RBPS_HD smat3<T> world_tensor(const quat<T> &q, const smat3<T> &local)
    {
        const mat3<T> R = mat3_cast(q);
        return sym_of(mul(R, local) * R.transpose());
    }

    // m3d::tf (tf.hpp:29-78)
    template <class T>
    struct tf
    {
        vec3<T> pos;
        quat<T> rot;
        RBPS_HD vec3<T> transform_point(const vec3<T> &p) const { return pos + rotate(rot, p); }
        RBPS_HD vec3<T> rotate_vector(const vec3<T> &d) const { return rotate(rot, d); }
        RBPS_HD vec3<T> inverse_rotate_vector(const vec3<T> &d) const { return rotate(conjugate(rot), d); }
    };

    // Double-precision AABB (rbc/AABB.hpp:19-59).
    struct aabb
    {
        vec3<double> mn, mx;
    };
    RBPS_HD bool aabb_overlap(const aabb &a, const aabb &b)
    {
        return (a.mn.x <= b.mx.x && a.mx.x >= b.mn.x) &&
               (a.mn.y <= b.mx.y && a.mx.y >= b.mn.y) &&
               (a.mn.z <= b.mx.z && a.mx.z >= b.mn.z);
    }
    RBPS_HD aabb aabb_expand(const aabb &a, double m)
    {
        const vec3<double> e(m, m, m);
        return {a.mn - e, a.mx + e};
    }
    // BroadPhase.cpp:11-17
    RBPS_HD bool aabb_contained(const aabb &t, const aabb &f)
    {
        return t.mn.x >= f.mn.x && t.mx.x <= f.mx.x &&
               t.mn.y >= f.mn.y && t.mx.y <= f.mx.y &&
               t.mn.z >= f.mn.z && t.mx.z <= f.mx.z;
    }
} // namespace rbps_gpu
