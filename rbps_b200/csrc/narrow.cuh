// narrow.cuh - shapes, AABBs and the analytic narrowphase on the device.
//
// One thread evaluates one candidate pair.  Each routine restates the
// reference's pair test with the same operand order (so the FP64
// instantiation reproduces the reference bit for bit) and the same
// normal / point conventions:
//   SphereSphere  rbc/analytic/SphereSphere.hpp:24-51
//   SphereBox     rbc/analytic/SphereBox.hpp:31-115
//   SphereCapsule rbc/analytic/SphereCapsule.hpp:24-71
//   CapsuleCapsule rbc/analytic/CapsuleCapsule.hpp:24-104
//   CapsuleBox    rbc/analytic/CapsuleBox.hpp:28-226
//   BoxBox        rbc/analytic/BoxBox.hpp:29-402
//   X-Plane       rbc/analytic/PlaneCollision.hpp:40-394
//   symmetric dispatch (normal flip) rbc/Dispatcher.hpp:103-116
#pragma once
#include <cmath>
#include "math.cuh"

namespace rbps_gpu
{
    enum ShapeKind : int
    {
        kSphere = 0,
        kBox = 1,
        kEllipsoid = 2,
        kCapsule = 3,
        kCylinder = 4,
        kCone = 5,
        kPlane = 6,
        kHeightmap = 7,
        kMesh = 8,
        kHull = 9
    };

    // Shapes whose pairs (other than with a plane) go through GJK / EPA
    // (gjk_convex_v, Dispatcher.hpp:40-60): the generic convex path.
    RBPS_HD bool gjk_kind(int k) { return k == kHull || k == kEllipsoid || k == kCylinder || k == kCone; }

    // Local support points (Ellipsoid.hpp, Cylinder.hpp, Cone.hpp support()).
    template <class T> RBPS_HD vec3<T> support_ellipsoid(const vec3<T> &a, const vec3<T> &d)
    {
        const vec3<T> scaled(a.x * a.x * d.x, a.y * a.y * d.y, a.z * a.z * d.z);
        const T denom = sqrt_t(a.x * a.x * d.x * d.x + a.y * a.y * d.y * d.y + a.z * a.z * d.z * d.z);
        if (denom < T(kEpsilon))
            return vec3<T>(a.x, T(0.0), T(0.0));
        const T inv = T(1.0) / denom; // vec3::operator/ multiplies by the reciprocal
        return vec3<T>(scaled.x * inv, scaled.y * inv, scaled.z * inv);
    }
    template <class T> RBPS_HD vec3<T> support_cylinder(T hh, T r, const vec3<T> &d)
    {
        const T sy = (d.y >= T(0.0)) ? hh : -hh;
        const T d_radial = sqrt_t(d.x * d.x + d.z * d.z);
        if (d_radial < T(kEpsilon))
            return vec3<T>(r, sy, T(0.0));
        const T scale = r / d_radial;
        return vec3<T>(d.x * scale, sy, d.z * scale);
    }
    template <class T> RBPS_HD vec3<T> support_cone(T hh, T r, const vec3<T> &d)
    {
        const T d_radial = sqrt_t(d.x * d.x + d.z * d.z);
        if (d_radial < T(kEpsilon))
            return (d.y >= T(0.0)) ? vec3<T>(T(0.0), hh, T(0.0)) : vec3<T>(r, -hh, T(0.0));
        const T apex_dot = d.y * hh;
        const T base_edge_dot = d_radial * r - d.y * hh;
        if (apex_dot >= base_edge_dot)
            return vec3<T>(T(0.0), hh, T(0.0));
        const T scale = r / d_radial;
        return vec3<T>(d.x * scale, -hh, d.z * scale);
    }
    // the three above by shape kind (params: ellipsoid semi-axes; cylinder
    // and cone half_height, base_radius)
    template <class T> RBPS_HD vec3<T> support_round(int kind, const double *p, const vec3<T> &d)
    {
        if (kind == kEllipsoid)
            return support_ellipsoid(vec3<T>(T(p[0]), T(p[1]), T(p[2])), d);
        if (kind == kCylinder)
            return support_cylinder(T(p[0]), T(p[1]), d);
        return support_cone(T(p[0]), T(p[1]), d);
    }

    // Hull geometry of one batch: vertices (double, local frame) per hull.
    // Bases of one hull's polygon / adjacency tables (ConvexHullData,
    // ConvexHull.hpp:60-98) in HullSetDev::u32 and poly_n; np = polygons
    // (0: no tables, the manifold is one EPA point).
    struct HullDesc
    {
        uint32_t np;
        uint32_t po, pi, pn;     // polygon offsets (np + 1), indices, first normal
        uint32_t v2p_o, v2p_i;   // vertex -> polygons (offsets: vertices + 1)
        uint32_t v2n_o, v2n_i;   // vertex -> neighbours
        uint32_t p2p_o, p2p_i;   // polygon -> polygons (offsets: np + 1)
    };

    // One heightmap (HeightmapData, Heightmap.hpp): rows x cols float
    // samples at heights[off ..], grid spacing / height scale, the (0, 0)
    // vertex, and the precomputed world height range.
    struct HmDesc
    {
        uint32_t rows, cols, off, pad_;
        double scale[3], origin[3];
        double min_h, max_h;
    };

    // One triangle mesh (MeshData, Mesh.hpp): vertices [v0, v0 + nv), faces
    // [f0, f0 + nf) of the batch arrays, its local AABB.
    struct MeshDesc
    {
        uint32_t v0, nv, f0, nf;
        double aabb[6];
    };

    struct HullSetDev
    {
        const double *verts;      // 3 per vertex
        const uint32_t *v_off;    // n_hulls + 1
        const double *local_aabb; // 6 per hull
        const HullDesc *desc;     // per hull
        const uint32_t *u32;      // all index tables
        const double *poly_n;     // 3 per polygon
        const float *hm_heights;  // heightmap samples (ShapeDev::hull = heightmap id)
        const HmDesc *hm_desc;    // per heightmap
        const MeshDesc *mesh;     // per triangle mesh (ShapeDev::hull = mesh id)
        const double *mesh_v;     // local vertices, 3 per vertex
        const uint32_t *mesh_i;   // 3 vertex indices per face (mesh-relative)
        const double *mesh_n;     // unit face normals, 3 per face
    };

    struct ShapeDev
    {
        int kind;
        int hull;
        double p[4];
    };

    template <class T>
    struct Manifold
    {
        vec3<T> normal;
        vec3<T> pos[4];
        T depth[4];
        int n;
    };

    // ------------------------------------------------------------ AABBs
    // compute_aabb per shape, always in double (the broadphase runs in double
    // in every precision mode so its pair set can match the reference).
    RBPS_HD aabb compute_aabb(const ShapeDev &s, const tf<double> &t, const HullSetDev &hs)
    {
        if (s.kind == kSphere) // Sphere.hpp:83-87
        {
            const vec3<double> r(s.p[0], s.p[0], s.p[0]);
            return {t.pos - r, t.pos + r};
        }
        if (s.kind == kBox) // Box.hpp:101-112
        {
            const mat3<double> R = mat3_cast(t.rot);
            const vec3<double> h(s.p[0], s.p[1], s.p[2]);
            const vec3<double> e(rabs(R.c[0].x) * h.x + rabs(R.c[1].x) * h.y + rabs(R.c[2].x) * h.z,
                                 rabs(R.c[0].y) * h.x + rabs(R.c[1].y) * h.y + rabs(R.c[2].y) * h.z,
                                 rabs(R.c[0].z) * h.x + rabs(R.c[1].z) * h.y + rabs(R.c[2].z) * h.z);
            return {t.pos - e, t.pos + e};
        }
        if (s.kind == kCapsule) // Capsule.hpp:129-139
        {
            const vec3<double> axis = t.rotate_vector(vec3<double>(0.0, s.p[0], 0.0));
            const vec3<double> p1 = t.pos + axis;
            const vec3<double> p2 = t.pos - axis;
            const vec3<double> r(s.p[1], s.p[1], s.p[1]);
            return {vec3<double>(rmin(p1.x, p2.x), rmin(p1.y, p2.y), rmin(p1.z, p2.z)) - r,
                    vec3<double>(rmax(p1.x, p2.x), rmax(p1.y, p2.y), rmax(p1.z, p2.z)) + r};
        }
        if (s.kind == kHull) // ConvexHull.hpp:484-499
        {
            const double *la = hs.local_aabb + 6 * s.hull;
            const vec3<double> lmn(la[0], la[1], la[2]), lmx(la[3], la[4], la[5]);
            const vec3<double> centre = (lmn + lmx) * 0.5;
            const vec3<double> half = (lmx - lmn) * 0.5;
            const mat3<double> R = mat3_cast(t.rot);
            const vec3<double> wc = t.pos + t.rotate_vector(centre);
            const vec3<double> e(rabs(R.c[0].x) * half.x + rabs(R.c[1].x) * half.y + rabs(R.c[2].x) * half.z,
                                 rabs(R.c[0].y) * half.x + rabs(R.c[1].y) * half.y + rabs(R.c[2].y) * half.z,
                                 rabs(R.c[0].z) * half.x + rabs(R.c[1].z) * half.y + rabs(R.c[2].z) * half.z);
            return {wc - e, wc + e};
        }
        if (s.kind == kEllipsoid) // Ellipsoid.hpp compute_aabb
        {
            const mat3<double> R = mat3_cast(t.rot);
            const vec3<double> a(s.p[0], s.p[1], s.p[2]);
            const vec3<double> e(
                sqrt_t(R.c[0].x * R.c[0].x * a.x * a.x + R.c[1].x * R.c[1].x * a.y * a.y + R.c[2].x * R.c[2].x * a.z * a.z),
                sqrt_t(R.c[0].y * R.c[0].y * a.x * a.x + R.c[1].y * R.c[1].y * a.y * a.y + R.c[2].y * R.c[2].y * a.z * a.z),
                sqrt_t(R.c[0].z * R.c[0].z * a.x * a.x + R.c[1].z * R.c[1].z * a.y * a.y + R.c[2].z * R.c[2].z * a.z * a.z));
            return {t.pos - e, t.pos + e};
        }
        if (s.kind == kCylinder || s.kind == kCone) // Cylinder.hpp / Cone.hpp compute_aabb
        {
            const vec3<double> axes[6] = {vec3<double>(1, 0, 0), vec3<double>(-1, 0, 0), vec3<double>(0, 1, 0),
                                          vec3<double>(0, -1, 0), vec3<double>(0, 0, 1), vec3<double>(0, 0, -1)};
            vec3<double> mn = t.pos, mx = t.pos;
            for (int k = 0; k < 6; ++k)
            {
                const vec3<double> ld = t.inverse_rotate_vector(axes[k]);
                const vec3<double> ws = t.pos + t.rotate_vector(support_round<double>(s.kind, s.p, ld));
                mn = vec3<double>(rmin(mn.x, ws.x), rmin(mn.y, ws.y), rmin(mn.z, ws.z));
                mx = vec3<double>(rmax(mx.x, ws.x), rmax(mx.y, ws.y), rmax(mx.z, ws.z));
            }
            return {mn, mx};
        }
        if (s.kind == kMesh) // Mesh.hpp compute_aabb
        {
            const double *la = hs.mesh[s.hull].aabb;
            const vec3<double> lmn(la[0], la[1], la[2]), lmx(la[3], la[4], la[5]);
            const vec3<double> centre = (lmn + lmx) * 0.5;
            const vec3<double> half = (lmx - lmn) * 0.5;
            const mat3<double> R = mat3_cast(t.rot);
            const vec3<double> wc = t.pos + t.rotate_vector(centre);
            const vec3<double> e(rabs(R.c[0].x) * half.x + rabs(R.c[1].x) * half.y + rabs(R.c[2].x) * half.z,
                                 rabs(R.c[0].y) * half.x + rabs(R.c[1].y) * half.y + rabs(R.c[2].y) * half.z,
                                 rabs(R.c[0].z) * half.x + rabs(R.c[1].z) * half.y + rabs(R.c[2].z) * half.z);
            return {wc - e, wc + e};
        }
        if (s.kind == kHeightmap) // Heightmap.hpp compute_aabb (world frame, tf unused)
        {
            const HmDesc &h = hs.hm_desc[s.hull];
            return {vec3<double>(h.origin[0], h.min_h, h.origin[2]),
                    vec3<double>(h.origin[0] + double(h.cols - 1) * h.scale[0], h.max_h,
                                 h.origin[2] + double(h.rows - 1) * h.scale[2])};
        }
        // Plane (Plane.hpp:46-50): infinite; planes never enter the SAP.
        const double inf = HUGE_VAL;
        return {vec3<double>(-inf, -inf, -inf), vec3<double>(inf, inf, inf)};
    }

    // ---------------------------------------------------------- supports
    template <class T> __device__ __forceinline__ vec3<T> support_sphere(T r, const vec3<T> &d)
    {
        return normalize(d) * r; // Sphere.hpp:47-50
    }

    template <class T> __device__ __forceinline__ void capsule_endpoints(T hh, const tf<T> &t, vec3<T> &p1, vec3<T> &p2)
    {
        const vec3<T> axis = t.rotate_vector(vec3<T>(T(0), hh, T(0))); // Capsule.hpp:43-49
        p1 = t.pos + axis;
        p2 = t.pos - axis;
    }

    // ------------------------------------------------------ Sphere-Sphere
    template <class T>
    __device__ bool sphere_sphere(T ra, const tf<T> &ta, T rb, const tf<T> &tb, Manifold<T> &m)
    {
        const vec3<T> delta = tb.pos - ta.pos;
        const T dist = length(delta);
        const T rsum = ra + rb;
        if (dist >= rsum)
            return false;
        m.normal = (dist > T(kEpsilon)) ? delta / dist : vec3<T>(T(1), T(0), T(0));
        m.n = 1;
        m.depth[0] = rsum - dist;
        m.pos[0] = ta.pos + m.normal * ra;
        return true;
    }

    // -------------------------------------------------------- Sphere-Box
    template <class T>
    __device__ bool sphere_box(T r, const tf<T> &ts, const vec3<T> &h, const tf<T> &tb, Manifold<T> &out)
    {
        const vec3<T> lc = tb.inverse_rotate_vector(ts.pos - tb.pos);
        const vec3<T> closest(rclamp(lc.x, -h.x, h.x), rclamp(lc.y, -h.y, h.y), rclamp(lc.z, -h.z, h.z));
        const vec3<T> ld = lc - closest;
        const T dist = length(ld);
        if (dist > T(kEpsilon))
        {
            if (dist >= r)
                return false;
            out.n = 1;
            out.normal = -tb.rotate_vector(ld / dist);
            out.depth[0] = r - dist;
            out.pos[0] = tb.transform_point(closest);
            return true;
        }
        const T px = h.x - rabs(lc.x);
        const T py = h.y - rabs(lc.y);
        const T pz = h.z - rabs(lc.z);
        vec3<T> ln;
        if (px <= py && px <= pz)
            ln = vec3<T>(lc.x > T(0) ? T(1.0) : T(-1.0), T(0), T(0));
        else if (py <= px && py <= pz)
            ln = vec3<T>(T(0), lc.y > T(0) ? T(1.0) : T(-1.0), T(0));
        else
            ln = vec3<T>(T(0), T(0), lc.z > T(0) ? T(1.0) : T(-1.0));
        out.n = 1;
        out.normal = -tb.rotate_vector(ln);
        out.depth[0] = r + rmin(px, rmin(py, pz));
        const vec3<T> fp(ln.x != T(0) ? ln.x * h.x : rclamp(lc.x, -h.x, h.x),
                         ln.y != T(0) ? ln.y * h.y : rclamp(lc.y, -h.y, h.y),
                         ln.z != T(0) ? ln.z * h.z : rclamp(lc.z, -h.z, h.z));
        out.pos[0] = tb.transform_point(fp);
        return true;
    }

    // ---------------------------------------------------- Sphere-Capsule
    template <class T>
    __device__ bool sphere_capsule(T rs, const tf<T> &ts, T hh, T rc, const tf<T> &tc, Manifold<T> &m)
    {
        vec3<T> p1, p2;
        capsule_endpoints(hh, tc, p1, p2);
        const vec3<T> d = p2 - p1;
        const T len2 = length_sq(d);
        T t = T(0);
        if (len2 > T(kEpsilon))
            t = rclamp(dot(ts.pos - p1, d) / len2, T(0), T(1));
        const vec3<T> closest = p1 + d * t;
        const vec3<T> delta = ts.pos - closest;
        const T dist = length(delta);
        const T rsum = rs + rc;
        if (dist >= rsum)
            return false;
        m.n = 1;
        m.normal = (dist > T(kEpsilon)) ? (-delta) / dist : vec3<T>(T(1), T(0), T(0));
        m.depth[0] = rsum - dist;
        m.pos[0] = closest - m.normal * rc;
        return true;
    }

    // --------------------------------------------------- Capsule-Capsule
    template <class T>
    __device__ bool capsule_capsule(T hha, T ra, const tf<T> &ta, T hhb, T rb, const tf<T> &tb, Manifold<T> &m)
    {
        vec3<T> p1, p2, q1, q2;
        capsule_endpoints(hha, ta, p1, p2);
        capsule_endpoints(hhb, tb, q1, q2);
        const vec3<T> d1 = p2 - p1;
        const vec3<T> d2 = q2 - q1;
        const vec3<T> r = p1 - q1;
        const T A = length_sq(d1);
        const T E = length_sq(d2);
        const T F = dot(d2, r);
        T s = T(0), t = T(0);
        const T B = dot(d1, d2);
        const T denom = A * E - B * B;
        const bool parallel = denom < T(kEpsilon * kEpsilon);
        if (parallel)
        {
            if (A > T(kEpsilon))
                s = rclamp((-dot(d1, r)) / A, T(0), T(1));
            if (E > T(kEpsilon))
                t = rclamp(dot(d2, -r) / E, T(0), T(1));
        }
        else
        {
            const T C = dot(d1, r);
            s = rclamp((B * F - C * E) / denom, T(0), T(1));
            t = (B * s + F) / E;
            if (t < T(0))
            {
                t = T(0);
                s = rclamp((-C) / A, T(0), T(1));
            }
            else if (t > T(1))
            {
                t = T(1);
                s = rclamp((B - C) / A, T(0), T(1));
            }
        }
        const vec3<T> ca = p1 + d1 * s;
        const vec3<T> cb = q1 + d2 * t;
        const vec3<T> delta = ca - cb;
        const T dist = length(delta);
        const T rsum = ra + rb;
        if (dist >= rsum)
            return false;
        const vec3<T> normal = (dist > T(kEpsilon)) ? delta / dist : vec3<T>(T(1), T(0), T(0));
        m.normal = normal;
        m.pos[0] = cb + normal * rb;
        m.depth[0] = rsum - dist;
        if (!parallel)
        {
            m.n = 1;
        }
        else
        {
            // the reference's placeholder second point (CapsuleCapsule.hpp:84-100)
            m.n = 2;
            m.pos[1] = q1 + normal * rb;
            m.depth[1] = rsum - dist;
        }
        return true;
    }

    // ------------------------------------------------------- Capsule-Box
    template <class T>
    __device__ __forceinline__ bool clip_line(T p, T q, T &tmin, T &tmax)
    {
        if (rabs(p) < T(kEpsilon))
            return q >= T(0);
        const T t = q / p;
        if (p > T(0))
        {
            if (t < tmax)
                tmax = t;
        }
        else
        {
            if (t > tmin)
                tmin = t;
        }
        return tmin <= tmax;
    }

    template <class T>
    __device__ bool capsule_box(T hh, T rad, const tf<T> &tc, const vec3<T> &he, const tf<T> &tb, Manifold<T> &m)
    {
        vec3<T> p1, p2;
        capsule_endpoints(hh, tc, p1, p2);
        const vec3<T> d = p2 - p1;
        const vec3<T> l = d * T(0.5);
        const vec3<T> c = p1 + l;
        const vec3<T> ax[3] = {tb.rotate_vector(vec3<T>(T(1), T(0), T(0))),
                               tb.rotate_vector(vec3<T>(T(0), T(1), T(0))),
                               tb.rotate_vector(vec3<T>(T(0), T(0), T(1)))};
        const T e[3] = {he.x, he.y, he.z};
        const vec3<T> diff = c - tb.pos;
        T best_depth = sizeof(T) == 8 ? T(1.7976931348623157e308) : T(3.40282347e38f);
        vec3<T> best_normal(T(1), T(0), T(0));
        int best_feat = -1;
        for (int i = 0; i < 3; ++i)
        {
            const vec3<T> axis = ax[i];
            const T r_box = e[i];
            const T r_cap = rabs(dot(l, axis)) + rad;
            const T dist = rabs(dot(diff, axis));
            const T overlap = r_box + r_cap - dist;
            if (overlap < T(0))
                return false;
            if (overlap < best_depth)
            {
                best_depth = overlap;
                best_normal = (dot(diff, axis) >= T(0)) ? axis : -axis;
                best_feat = i;
            }
        }
        for (int i = 0; i < 3; ++i)
        {
            vec3<T> axis = cross(ax[i], l);
            const T len_sq = length_sq(axis);
            if (len_sq < axis_eps_sq<T>())
                continue;
            axis = axis / sqrt_t(len_sq);
            const T r_box = e[0] * rabs(dot(ax[0], axis)) + e[1] * rabs(dot(ax[1], axis)) + e[2] * rabs(dot(ax[2], axis));
            const T r_cap = rad;
            const T dist = rabs(dot(diff, axis));
            const T overlap = r_box + r_cap - dist;
            if (overlap < T(0))
                return false;
            if (overlap < best_depth)
            {
                best_depth = overlap;
                best_normal = (dot(diff, axis) >= T(0)) ? axis : -axis;
                best_feat = i + 3;
            }
        }
        m.normal = -best_normal;
        m.n = 0;
        if (best_feat < 3)
        {
            T t0 = T(0), t1 = T(1);
            const int iA = (best_feat + 1) % 3;
            const int iB = (best_feat + 2) % 3;
            const vec3<T> p1_rel = p1 - tb.pos;
            const T pA = dot(d, ax[iA]), valA = dot(p1_rel, ax[iA]);
            if (!clip_line(pA, e[iA] - valA, t0, t1))
                return true;
            if (!clip_line(-pA, e[iA] + valA, t0, t1))
                return true;
            const T pB = dot(d, ax[iB]), valB = dot(p1_rel, ax[iB]);
            if (!clip_line(pB, e[iB] - valB, t0, t1))
                return true;
            if (!clip_line(-pB, e[iB] + valB, t0, t1))
                return true;
            const vec3<T> pt0 = p1 + d * t0;
            const T depth0 = rad + e[best_feat] - dot(pt0 - tb.pos, best_normal);
            if (depth0 > T(0))
            {
                m.pos[m.n] = pt0 - best_normal * rad;
                m.depth[m.n] = depth0;
                m.n++;
            }
            if (t1 - t0 > T(kEpsilon))
            {
                const vec3<T> pt1 = p1 + d * t1;
                const T depth1 = rad + e[best_feat] - dot(pt1 - tb.pos, best_normal);
                if (depth1 > T(0))
                {
                    m.pos[m.n] = pt1 - best_normal * rad;
                    m.depth[m.n] = depth1;
                    m.n++;
                }
            }
        }
        else
        {
            const int edge_axis = best_feat - 3;
            const vec3<T> v = ax[edge_axis];
            const vec3<T> support_box = tb.pos +
                                        ax[0] * ((dot(ax[0], best_normal) >= T(0)) ? e[0] : -e[0]) +
                                        ax[1] * ((dot(ax[1], best_normal) >= T(0)) ? e[1] : -e[1]) +
                                        ax[2] * ((dot(ax[2], best_normal) >= T(0)) ? e[2] : -e[2]);
            const vec3<T> r = p1 - support_box;
            const T a = length_sq(d);
            const T b = dot(d, v);
            const T f = dot(v, r);
            const T c_dot = dot(d, r);
            const T denom = a - b * b;
            const T t = (denom > T(kEpsilon)) ? rclamp((b * f - c_dot) / denom, T(0), T(1)) : T(0.5);
            const vec3<T> pt = p1 + d * t;
            m.n = 1;
            m.pos[0] = pt - best_normal * rad;
            m.depth[0] = best_depth;
        }
        if (m.n == 0)
        {
            m.n = 1;
            m.pos[0] = c - best_normal * rad;
            m.depth[0] = best_depth;
        }
        return true;
    }

    // ----------------------------------------------------------- Box-Box
    template <class T>
    __device__ __forceinline__ T obb_radius(const vec3<T> &h, const vec3<T> ax[3], const vec3<T> &axis)
    {
        return rabs(dot(ax[0], axis)) * h.x + rabs(dot(ax[1], axis)) * h.y + rabs(dot(ax[2], axis)) * h.z;
    }

    template <class T>
    __device__ __forceinline__ bool test_axis(const vec3<T> &axis, const vec3<T> &ha, const vec3<T> axA[3],
                                              const vec3<T> &hb, const vec3<T> axB[3], const vec3<T> &cd,
                                              T &best_depth, vec3<T> &best_normal, int feat, int &best_feat, T bias)
    {
        const T len_sq = length_sq(axis);
        if (len_sq < axis_eps_sq<T>())
            return true;
        const vec3<T> na = axis / sqrt_t(len_sq);
        const T rA = obb_radius(ha, axA, na);
        const T rB = obb_radius(hb, axB, na);
        const T dist = rabs(dot(cd, na));
        const T overlap = rA + rB - dist;
        if (overlap < T(0))
            return false;
        if ((overlap + bias) < best_depth)
        {
            best_depth = overlap + bias;
            best_normal = (dot(cd, na) >= T(0)) ? na : -na;
            best_feat = feat;
        }
        return true;
    }

    // get_best_face (BoxBox.hpp:69-101)
    template <class T>
    __device__ __forceinline__ void best_face(const vec3<T> &h, const tf<T> &t, const vec3<T> ax[3],
                                              const vec3<T> &dir, vec3<T> corners[4], vec3<T> &out_n)
    {
        const T half[3] = {h.x, h.y, h.z};
        int best = 0;
        T best_dot = rabs(dot(ax[0], dir));
        for (int i = 1; i < 3; ++i)
        {
            const T d = rabs(dot(ax[i], dir));
            if (d > best_dot)
            {
                best_dot = d;
                best = i;
            }
        }
        const T sign = (dot(ax[best], dir) >= T(0)) ? T(1.0) : T(-1.0);
        out_n = ax[best] * sign;
        const vec3<T> fc = t.pos + out_n * half[best];
        const int u = (best + 1) % 3;
        const int v = (best + 2) % 3;
        corners[0] = fc + ax[u] * half[u] + ax[v] * half[v];
        corners[1] = fc - ax[u] * half[u] + ax[v] * half[v];
        corners[2] = fc - ax[u] * half[u] - ax[v] * half[v];
        corners[3] = fc + ax[u] * half[u] - ax[v] * half[v];
    }

    template <class T>
    __device__ __forceinline__ int clip_poly(const vec3<T> *poly, int n, const vec3<T> &pn, const vec3<T> &pp, vec3<T> *out)
    {
        int on = 0;
        for (int i = 0; i < n; ++i)
        {
            const vec3<T> A = poly[i];
            const vec3<T> B = poly[(i + 1) % n];
            const T dA = dot(A - pp, pn);
            const T dB = dot(B - pp, pn);
            if (dA >= T(0))
                out[on++] = A;
            if ((dA > T(0)) != (dB > T(0)))
            {
                const T t = dA / (dA - dB);
                out[on++] = A + (B - A) * t;
            }
        }
        return on;
    }

    // reduce_to_4 of BoxBox.hpp:130-231
    template <class T>
    __device__ int reduce_to_4_box(const vec3<T> *pts, const T *dep, int n, vec3<T> *op, T *od)
    {
        if (n <= 4)
        {
            for (int i = 0; i < n; ++i)
            {
                op[i] = pts[i];
                od[i] = dep[i];
            }
            return n;
        }
        int i0 = 0;
        for (int i = 1; i < n; ++i)
            if (dep[i] > dep[i0])
                i0 = i;
        int i1 = (i0 == 0) ? 1 : 0;
        T best = T(-1.0);
        for (int i = 0; i < n; ++i)
        {
            if (i == i0)
                continue;
            const T d = length_sq(pts[i] - pts[i0]);
            if (d > best)
            {
                best = d;
                i1 = i;
            }
        }
        int i2 = -1;
        best = T(-1.0);
        const vec3<T> seg = pts[i1] - pts[i0];
        for (int i = 0; i < n; ++i)
        {
            if (i == i0 || i == i1)
                continue;
            const T d = length_sq(cross(pts[i] - pts[i0], seg));
            if (d > best)
            {
                best = d;
                i2 = i;
            }
        }
        if (i2 < 0)
        {
            i2 = 0;
            while (i2 == i0 || i2 == i1)
                ++i2;
        }
        int i3 = -1;
        T min_dot = T(1.0);
        const vec3<T> tri_n = cross(pts[i2] - pts[i0], seg);
        for (int i = 0; i < n; ++i)
        {
            if (i == i0 || i == i1 || i == i2)
                continue;
            const T d = dot(cross(pts[i] - pts[i0], seg), tri_n);
            if (d < min_dot)
            {
                min_dot = d;
                i3 = i;
            }
        }
        if (i3 < 0 || min_dot >= T(0))
        {
            best = T(-1.0);
            for (int i = 0; i < n; ++i)
            {
                if (i == i0 || i == i1 || i == i2)
                    continue;
                const T d = length_sq(pts[i] - pts[i2]);
                if (d > best)
                {
                    best = d;
                    i3 = i;
                }
            }
        }
        if (i3 < 0)
        {
            i3 = 0;
            while (i3 == i0 || i3 == i1 || i3 == i2)
                ++i3;
        }
        op[0] = pts[i0]; od[0] = dep[i0];
        op[1] = pts[i1]; od[1] = dep[i1];
        op[2] = pts[i2]; od[2] = dep[i2];
        op[3] = pts[i3]; od[3] = dep[i3];
        return 4;
    }

    template <class T>
    __device__ bool box_box(const vec3<T> &ha, const tf<T> &ta, const vec3<T> &hb, const tf<T> &tb, Manifold<T> &m)
    {
        const vec3<T> cd = tb.pos - ta.pos;
        const vec3<T> ax[3] = {ta.rotate_vector(vec3<T>(T(1), T(0), T(0))),
                               ta.rotate_vector(vec3<T>(T(0), T(1), T(0))),
                               ta.rotate_vector(vec3<T>(T(0), T(0), T(1)))};
        const vec3<T> bx[3] = {tb.rotate_vector(vec3<T>(T(1), T(0), T(0))),
                               tb.rotate_vector(vec3<T>(T(0), T(1), T(0))),
                               tb.rotate_vector(vec3<T>(T(0), T(0), T(1)))};
        T best_depth = sizeof(T) == 8 ? T(1.7976931348623157e308) : T(3.40282347e38f);
        vec3<T> best_normal(T(1), T(0), T(0));
        int best_feat = 0, feat = 0;
        for (int i = 0; i < 3; ++i, ++feat)
            if (!test_axis(ax[i], ha, ax, hb, bx, cd, best_depth, best_normal, feat, best_feat, T(0)))
                return false;
        for (int i = 0; i < 3; ++i, ++feat)
            if (!test_axis(bx[i], ha, ax, hb, bx, cd, best_depth, best_normal, feat, best_feat, T(0)))
                return false;
        const T edge_bias = T(0.001f); // float literal in the reference (BoxBox.hpp:263)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j, ++feat)
                if (!test_axis(cross(ax[i], bx[j]), ha, ax, hb, bx, cd, best_depth, best_normal, feat, best_feat, edge_bias))
                    return false;
        if (best_feat >= 6)
            best_depth -= edge_bias;
        m.normal = best_normal;
        m.n = 0;
        if (best_feat < 6)
        {
            const bool ref_is_A = best_feat < 3;
            const vec3<T> &ref_h = ref_is_A ? ha : hb;
            const tf<T> &ref_t = ref_is_A ? ta : tb;
            const vec3<T> *ref_ax = ref_is_A ? ax : bx;
            const vec3<T> &inc_h = ref_is_A ? hb : ha;
            const tf<T> &inc_t = ref_is_A ? tb : ta;
            const vec3<T> *inc_ax = ref_is_A ? bx : ax;
            const vec3<T> target = ref_is_A ? best_normal : -best_normal;
            vec3<T> rc[4], rn, ic[4], in_;
            best_face(ref_h, ref_t, ref_ax, target, rc, rn);
            best_face(inc_h, inc_t, inc_ax, -target, ic, in_);
            vec3<T> buf0[16], buf1[16];
            int cnt = 4;
            for (int i = 0; i < 4; ++i)
                buf0[i] = ic[i];
            const vec3<T> ref_center = (rc[0] + rc[1] + rc[2] + rc[3]) * T(0.25f);
            for (int i = 0; i < 4; ++i)
            {
                const vec3<T> edge = rc[(i + 1) % 4] - rc[i];
                vec3<T> side_n = normalize(cross(rn, edge));
                if (dot(side_n, ref_center - rc[i]) < T(0.0f))
                    side_n = -side_n;
                cnt = clip_poly(buf0, cnt, side_n, rc[i], buf1);
                if (cnt == 0)
                    break;
                for (int k = 0; k < cnt; ++k)
                    buf0[k] = buf1[k];
            }
            if (cnt == 0)
                return false;
            const T ref_d = dot(rc[0], rn);
            vec3<T> kp[16];
            T kd[16];
            int kn = 0;
            for (int i = 0; i < cnt; ++i)
            {
                const T sd = dot(buf0[i], rn) - ref_d;
                if (sd <= T(kEpsilon))
                {
                    kp[kn] = buf0[i] - rn * (sd * T(0.5f));
                    kd[kn] = -sd;
                    ++kn;
                }
            }
            if (kn == 0)
                return false;
            m.n = reduce_to_4_box(kp, kd, kn, m.pos, m.depth);
        }
        else
        {
            const int ei = (best_feat - 6) / 3;
            const int ej = (best_feat - 6) % 3;
            const T extA[3] = {ha.x, ha.y, ha.z};
            const T extB[3] = {hb.x, hb.y, hb.z};
            const vec3<T> nb = -best_normal;
            const vec3<T> pa = ta.pos + ta.rotate_vector(vec3<T>(
                                            (dot(ax[0], best_normal) >= T(0) ? T(1.0) : T(-1.0)) * (ei == 0 ? T(0.0) : extA[0]),
                                            (dot(ax[1], best_normal) >= T(0) ? T(1.0) : T(-1.0)) * (ei == 1 ? T(0.0) : extA[1]),
                                            (dot(ax[2], best_normal) >= T(0) ? T(1.0) : T(-1.0)) * (ei == 2 ? T(0.0) : extA[2])));
            const vec3<T> pb = tb.pos + tb.rotate_vector(vec3<T>(
                                            (dot(bx[0], nb) >= T(0) ? T(1.0) : T(-1.0)) * (ej == 0 ? T(0.0) : extB[0]),
                                            (dot(bx[1], nb) >= T(0) ? T(1.0) : T(-1.0)) * (ej == 1 ? T(0.0) : extB[1]),
                                            (dot(bx[2], nb) >= T(0) ? T(1.0) : T(-1.0)) * (ej == 2 ? T(0.0) : extB[2])));
            const vec3<T> d1 = ax[ei], d2 = bx[ej];
            const vec3<T> r = pa - pb;
            const T b_dot = dot(d1, d2);
            const T c_dot = dot(d1, r);
            const T f_dot = dot(d2, r);
            const T denom = T(1.0f) - b_dot * b_dot;
            T s = T(0.0f), t = T(0.0f);
            if (denom > T(kEpsilon))
                s = (b_dot * f_dot - c_dot) / denom;
            const T ea = extA[ei];
            const T eb = extB[ej];
            if (s < -ea || s > ea)
                s = rclamp(s, -ea, ea);
            t = s * b_dot + f_dot;
            if (t < -eb || t > eb)
            {
                t = rclamp(t, -eb, eb);
                s = rclamp(t * b_dot - c_dot, -ea, ea);
            }
            m.n = 1;
            m.pos[0] = (pa + d1 * s + pb + d2 * t) * T(0.5f);
            m.depth[0] = best_depth;
        }
        return true;
    }

    // -------------------------------------------------------- X vs Plane
    // world normal / offset of a plane (Plane.hpp:38-45)
    template <class T>
    __device__ __forceinline__ void plane_world(const ShapeDev &pl, const tf<T> &tp, vec3<T> &wn, T &wd)
    {
        wn = tp.rotate_vector(vec3<T>(T(pl.p[0]), T(pl.p[1]), T(pl.p[2])));
        wd = T(pl.p[3]) + dot(wn, tp.pos);
    }

    // convex_vs_plane for Sphere (PlaneCollision.hpp:40-61)
    template <class T>
    __device__ bool sphere_plane(T r, const tf<T> &ts, const ShapeDev &pl, const tf<T> &tp, Manifold<T> &out)
    {
        vec3<T> wn;
        T wd;
        plane_world(pl, tp, wn, wd);
        const vec3<T> ld = ts.inverse_rotate_vector(-wn);
        const vec3<T> ls = support_sphere(r, ld);
        const vec3<T> ws = ts.pos + ts.rotate_vector(ls);
        const T sd = dot(ws, wn) - wd;
        if (sd >= T(0))
            return false;
        out.normal = -wn;
        out.n = 1;
        out.depth[0] = -sd;
        out.pos[0] = ws;
        return true;
    }

    // convex_vs_plane for Ellipsoid and Cone (PlaneCollision.hpp:40-61,
    // RBC_PLANE_SPEC): the support point along -n, one contact.
    template <class T>
    __device__ bool round_plane(const ShapeDev &s, const tf<T> &ts, const ShapeDev &pl, const tf<T> &tp,
                                Manifold<T> &out)
    {
        vec3<T> wn;
        T wd;
        plane_world(pl, tp, wn, wd);
        const vec3<T> ld = ts.inverse_rotate_vector(-wn);
        const vec3<T> ls = support_round<T>(s.kind, s.p, ld);
        const vec3<T> ws = ts.pos + ts.rotate_vector(ls);
        const T sd = dot(ws, wn) - wd;
        if (sd >= T(0))
            return false;
        out.normal = -wn;
        out.n = 1;
        out.depth[0] = -sd;
        out.pos[0] = ws;
        return true;
    }

    // Cylinder vs Plane (PlaneCollision.hpp:416-536): the four cardinal rim
    // points of the facing cap when the axis is within 10 degrees of the
    // normal, else one rim point per cap, each kept when its distance is at
    // most 1e-4f.
    template <class T>
    __device__ bool cylinder_plane(T hh, T r, const tf<T> &ta, const ShapeDev &pl, const tf<T> &tp, Manifold<T> &out)
    {
        vec3<T> wn;
        T wd;
        plane_world(pl, tp, wn, wd);
        const vec3<T> axis = ta.rotate_vector(vec3<T>(T(0), T(1), T(0)));
        const T cos_theta = dot(axis, wn);
        const vec3<T> lneg = ta.inverse_rotate_vector(-wn);
        const vec3<T> sl = support_cylinder(hh, r, lneg);
        const vec3<T> sw = ta.transform_point(sl);
        const T sdist = dot(sw, wn) - wd;
        const T eps = T(1e-4f);
        if (sdist > eps)
            return false;
        out.normal = -wn;
        out.n = 0;
        const T abs_cos = rabs(cos_theta);
        if (abs_cos >= T(0.985f))
        {
            const T cap_sign = (cos_theta < T(0.0f)) ? T(1.0f) : T(-1.0f);
            const vec3<T> cap = ta.pos + axis * (cap_sign * hh);
            vec3<T> r1 = cross(axis, vec3<T>(T(1), T(0), T(0)));
            if (dot(r1, r1) < T(1e-6f))
                r1 = cross(axis, vec3<T>(T(0), T(0), T(1)));
            r1 = normalize(r1);
            const vec3<T> r2 = normalize(cross(axis, r1));
            const vec3<T> rim[4] = {cap + r1 * r, cap - r1 * r, cap + r2 * r, cap - r2 * r};
            for (int i = 0; i < 4; ++i)
            {
                const T dist = dot(rim[i], wn) - wd;
                if (dist <= eps)
                {
                    out.pos[out.n] = rim[i];
                    out.depth[out.n] = -dist;
                    out.n++;
                }
            }
        }
        else
        {
            const T radial_len = sqrt_t(sl.x * sl.x + sl.z * sl.z);
            vec3<T> radial_world(T(0), T(0), T(0));
            if (radial_len > T(kEpsilon))
                radial_world = ta.rotate_vector(vec3<T>(sl.x / radial_len * r, T(0.0f), sl.z / radial_len * r));
            const vec3<T> pts[2] = {ta.pos + axis * hh + radial_world, ta.pos - axis * hh + radial_world};
            for (int i = 0; i < 2; ++i)
            {
                const T dist = dot(pts[i], wn) - wd;
                if (dist <= eps)
                {
                    out.pos[out.n] = pts[i];
                    out.depth[out.n] = -dist;
                    out.n++;
                }
            }
        }
        return out.n > 0;
    }

    // Box vs Plane (PlaneCollision.hpp:289-337)
    template <class T>
    __device__ bool box_plane(const vec3<T> &h, const tf<T> &ta, const ShapeDev &pl, const tf<T> &tp, Manifold<T> &out)
    {
        vec3<T> wn;
        T wd;
        plane_world(pl, tp, wn, wd);
        const vec3<T> u[3] = {ta.rotate_vector(vec3<T>(T(1), T(0), T(0))),
                              ta.rotate_vector(vec3<T>(T(0), T(1), T(0))),
                              ta.rotate_vector(vec3<T>(T(0), T(0), T(1)))};
        const T eps = T(1e-4f);
        const T r = h.x * rabs(dot(u[0], wn)) + h.y * rabs(dot(u[1], wn)) + h.z * rabs(dot(u[2], wn));
        const T cdist = dot(ta.pos, wn) - wd;
        if (cdist - r > eps)
            return false;
        out.normal = -wn;
        out.n = 0;
        for (int sx = -1; sx <= 1; sx += 2)
            for (int sy = -1; sy <= 1; sy += 2)
                for (int sz = -1; sz <= 1; sz += 2)
                {
                    const vec3<T> corner = ta.pos + (T(sx) * h.x) * u[0] + (T(sy) * h.y) * u[1] + (T(sz) * h.z) * u[2];
                    const T dist = dot(corner, wn) - wd;
                    if (dist <= eps && out.n < 4)
                    {
                        out.pos[out.n] = corner;
                        out.depth[out.n] = -dist;
                        out.n++;
                    }
                }
        return out.n > 0;
    }

    // Capsule vs Plane (PlaneCollision.hpp:344-389)
    template <class T>
    __device__ bool capsule_plane(T hh, T rad, const tf<T> &ta, const ShapeDev &pl, const tf<T> &tp, Manifold<T> &out)
    {
        vec3<T> wn;
        T wd;
        plane_world(pl, tp, wn, wd);
        vec3<T> p1, p2;
        capsule_endpoints(hh, ta, p1, p2);
        const T d1 = dot(p1, wn) - wd;
        const T d2 = dot(p2, wn) - wd;
        out.n = 0;
        out.normal = -wn;
        const T eps = T(1e-4);
        const vec3<T> ro = wn * rad;
        const T thr = rad + eps;
        if (d1 <= thr)
        {
            out.pos[out.n] = p1 - ro;
            out.depth[out.n] = rad - d1;
            out.n++;
        }
        if (d2 <= thr)
        {
            out.pos[out.n] = p2 - ro;
            out.depth[out.n] = rad - d2;
            out.n++;
        }
        return out.n > 0;
    }

    // Hull vertex support (ConvexHull.hpp:457-473): first maximum wins.
    template <class T>
    __device__ __forceinline__ vec3<T> support_hull(const HullSetDev &hs, int hull, const vec3<T> &dir)
    {
        const uint32_t b = hs.v_off[hull], e = hs.v_off[hull + 1];
        if (b == e)
            return vec3<T>();
        const double *v = hs.verts + 3 * b;
        vec3<T> best{T(v[0]), T(v[1]), T(v[2])};
        T best_d = dot(best, dir);
        for (uint32_t i = 1; i < e - b; ++i)
        {
            const vec3<T> p{T(v[3 * i]), T(v[3 * i + 1]), T(v[3 * i + 2])};
            const T d = dot(p, dir);
            if (d > best_d)
            {
                best_d = d;
                best = p;
            }
        }
        return best;
    }

    // ConvexHull vs Plane (PlaneCollision.hpp:90-285): vertex gather within
    // 1e-4f of the plane, then the 4-point area reduction.
    template <class T>
    __device__ bool hull_plane(const HullSetDev &hs, int hull, const tf<T> &ta, const ShapeDev &pl, const tf<T> &tp,
                               Manifold<T> &out)
    {
        const uint32_t vb = hs.v_off[hull], ve = hs.v_off[hull + 1];
        if (vb == ve)
            return false;
        vec3<T> wn;
        T wd;
        plane_world(pl, tp, wn, wd);
        const vec3<T> ln = ta.inverse_rotate_vector(wn);
        const T ld = wd - dot(ta.pos, wn);
        const T eps = T(1e-4f);
        const vec3<T> deepest = support_hull(hs, hull, -ln);
        if (dot(deepest, ln) - ld > eps)
            return false;
        vec3<T> tp_pos[32];
        T tp_dep[32];
        int tc = 0;
        const double *v = hs.verts + 3 * vb;
        for (uint32_t i = 0; i < ve - vb; ++i)
        {
            const vec3<T> lv{T(v[3 * i]), T(v[3 * i + 1]), T(v[3 * i + 2])};
            const T dist = dot(lv, ln) - ld;
            if (dist <= eps && tc < 32)
            {
                tp_pos[tc] = lv;
                tp_dep[tc] = -dist;
                tc++;
            }
        }
        if (tc == 0)
            return false;
        out.normal = -wn;
        out.n = 0;
        if (tc <= 4)
        {
            for (int i = 0; i < tc; ++i)
            {
                out.pos[i] = ta.transform_point(tp_pos[i]);
                out.depth[i] = tp_dep[i];
            }
            out.n = tc;
            return true;
        }
        int idx[4] = {-1, -1, -1, -1};
        {
            T best = T(-1e18f);
            for (int i = 0; i < tc; ++i)
                if (tp_dep[i] > best)
                {
                    best = tp_dep[i];
                    idx[0] = i;
                }
        }
        {
            const vec3<T> p0 = tp_pos[idx[0]];
            T best = T(-1e18f);
            for (int i = 0; i < tc; ++i)
            {
                if (i == idx[0])
                    continue;
                const vec3<T> d = tp_pos[i] - p0;
                const T d2 = dot(d, d);
                if (d2 > best)
                {
                    best = d2;
                    idx[1] = i;
                }
            }
        }
        {
            const vec3<T> p0 = tp_pos[idx[0]];
            const vec3<T> edge = tp_pos[idx[1]] - p0;
            T best = T(-1e18f);
            for (int i = 0; i < tc; ++i)
            {
                if (i == idx[0] || i == idx[1])
                    continue;
                const vec3<T> c = cross(edge, tp_pos[i] - p0);
                const T d2 = dot(c, c);
                if (d2 > best)
                {
                    best = d2;
                    idx[2] = i;
                }
            }
        }
        {
            const vec3<T> p0 = tp_pos[idx[0]], p1 = tp_pos[idx[1]], p2 = tp_pos[idx[2]];
            const vec3<T> e01 = p1 - p0, e12 = p2 - p1, e20 = p0 - p2;
            T best = T(-1e18f);
            for (int i = 0; i < tc; ++i)
            {
                if (i == idx[0] || i == idx[1] || i == idx[2])
                    continue;
                const vec3<T> x = tp_pos[i];
                const T a0 = dot(cross(e01, x - p0), ln);
                const T a1 = dot(cross(e12, x - p1), ln);
                const T a2 = dot(cross(e20, x - p2), ln);
                T score = a0;
                if (a1 > score)
                    score = a1;
                if (a2 > score)
                    score = a2;
                if (score > best)
                {
                    best = score;
                    idx[3] = i;
                }
            }
        }
        const int emit = (idx[3] >= 0) ? 4 : 3;
        for (int i = 0; i < emit; ++i)
        {
            out.pos[i] = ta.transform_point(tp_pos[idx[i]]);
            out.depth[i] = tp_dep[idx[i]];
        }
        out.n = emit;
        return out.n > 0;
    }

    // Pair kinds after canonical ordering; GJK pairs are reported to the
    // caller (they are evaluated by the warp-cooperative GJK/EPA kernel).
    enum PairResult : int
    {
        kMiss = 0,
        kHit = 1,
        kNeedsGjk = 2
    };

    // dispatch (Dispatcher.hpp:212-217) over the analytic table.
    // ------------------------------------------------------- Heightmaps
    // Triangle helpers (TriangleUtils.hpp) and the sphere / capsule / box vs
    // heightmap tests (HeightmapCollision.hpp): every cell under the shape's
    // AABB, two triangles per cell, the deepest single contact kept.
    template <class T>
    __device__ vec3<T> tri_closest(const vec3<T> &P, const vec3<T> &A, const vec3<T> &B, const vec3<T> &C)
    {
        const vec3<T> AB = B - A, AC = C - A, AP = P - A;
        const T d1 = dot(AB, AP), d2 = dot(AC, AP);
        if (d1 <= T(0.0) && d2 <= T(0.0))
            return A;
        const vec3<T> BP = P - B;
        const T d3 = dot(AB, BP), d4 = dot(AC, BP);
        if (d3 >= T(0.0) && d4 <= d3)
            return B;
        const T vc = d1 * d4 - d3 * d2;
        if (vc <= T(0.0) && d1 >= T(0.0) && d3 <= T(0.0))
            return A + AB * (d1 / (d1 - d3));
        const vec3<T> CP = P - C;
        const T d5 = dot(AB, CP), d6 = dot(AC, CP);
        if (d6 >= T(0.0) && d5 <= d6)
            return C;
        const T vb = d5 * d2 - d1 * d6;
        if (vb <= T(0.0) && d2 >= T(0.0) && d6 <= T(0.0))
            return A + AC * (d2 / (d2 - d6));
        const T va = d3 * d6 - d5 * d4;
        if (va <= T(0.0) && (d4 - d3) >= T(0.0) && (d5 - d6) >= T(0.0))
        {
            const T w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
            return B + (C - B) * w;
        }
        const T denom = T(1.0) / (va + vb + vc);
        const T v = vb * denom, w = vc * denom;
        return A + AB * v + AC * w;
    }

    template <class T>
    __device__ T tri_seg_seg_sq(const vec3<T> &p1, const vec3<T> &p2, const vec3<T> &q1, const vec3<T> &q2)
    {
        const vec3<T> d1 = p2 - p1, d2 = q2 - q1, r = p1 - q1;
        const T a = length_sq(d1), e = length_sq(d2), f = dot(d2, r);
        T s, t;
        if (a < T(kEpsilon) && e < T(kEpsilon))
            s = t = T(0.0);
        else if (a < T(kEpsilon))
        {
            s = T(0.0);
            t = rclamp(f / e, T(0), T(1));
        }
        else
        {
            const T c = dot(d1, r);
            if (e < T(kEpsilon))
            {
                t = T(0.0);
                s = rclamp(-c / a, T(0), T(1));
            }
            else
            {
                const T b = dot(d1, d2);
                const T denom = a * e - b * b;
                s = denom > T(kEpsilon) ? rclamp((b * f - c * e) / denom, T(0), T(1)) : T(0.0);
                t = (b * s + f) / e;
                if (t < T(0.0))
                {
                    t = T(0.0);
                    s = rclamp(-c / a, T(0), T(1));
                }
                else if (t > T(1.0))
                {
                    t = T(1.0);
                    s = rclamp((b - c) / a, T(0), T(1));
                }
            }
        }
        return length_sq((p1 + d1 * s) - (q1 + d2 * t));
    }

    template <class T>
    __device__ T tri_seg_sq(const vec3<T> &P, const vec3<T> &Q, const vec3<T> &A, const vec3<T> &B, const vec3<T> &C)
    {
        T best = length_sq(P - tri_closest(P, A, B, C));
        best = rmin(best, length_sq(Q - tri_closest(Q, A, B, C)));
        best = rmin(best, tri_seg_seg_sq(P, Q, A, B));
        best = rmin(best, tri_seg_seg_sq(P, Q, B, C));
        best = rmin(best, tri_seg_seg_sq(P, Q, C, A));
        return best;
    }

    // kind: 0 sphere (p0 = centre, r), 1 capsule (segment p0-p1, r), 2 box
    // (tb, half-extents h); one triangle, one point, normal from the
    // triangle toward the shape.
    template <class T>
    __device__ bool tri_contact(int kind, const vec3<T> &p0, const vec3<T> &p1, T r, const tf<T> &tb, const vec3<T> &h,
                                const vec3<T> &A, const vec3<T> &B, const vec3<T> &C, const vec3<T> &n,
                                Manifold<T> &m)
    {
        if (kind == 0) // tri::sphere_vs_triangle
        {
            const vec3<T> closest = tri_closest(p0, A, B, C);
            const vec3<T> delta = p0 - closest;
            const T dist2 = length_sq(delta);
            if (dist2 > r * r)
                return false;
            const T dist = sqrt_t(dist2);
            if (dist > T(kEpsilon))
            {
                const T inv = T(1.0) / dist;
                m.normal = vec3<T>(delta.x * inv, delta.y * inv, delta.z * inv);
                m.depth[0] = r - dist;
                m.pos[0] = closest;
            }
            else
            {
                const T side = dot(n, p0 - A);
                m.normal = (side >= T(0.0)) ? n : -n;
                m.depth[0] = r + rabs(side);
                m.pos[0] = p0 - m.normal * r;
            }
            m.n = 1;
            return true;
        }
        if (kind == 1) // tri::capsule_vs_triangle
        {
            const T d1 = dot(n, p0 - A), d2 = dot(n, p1 - A);
            if (d1 > r && d2 > r)
                return false;
            if (d1 < -r && d2 < -r)
                return false;
            const T sq = tri_seg_sq(p0, p1, A, B, C);
            if (sq > r * r)
                return false;
            const T dist = sqrt_t(sq);
            const vec3<T> cp1 = tri_closest(p0, A, B, C), cp2 = tri_closest(p1, A, B, C);
            const T d1sq = length_sq(p0 - cp1), d2sq = length_sq(p1 - cp2);
            const vec3<T> &rs = (d1sq <= d2sq) ? p0 : p1;
            const vec3<T> &rt = (d1sq <= d2sq) ? cp1 : cp2;
            const vec3<T> delta = rs - rt;
            if (dist > T(kEpsilon))
            {
                const T inv = T(1.0) / dist;
                m.normal = vec3<T>(delta.x * inv, delta.y * inv, delta.z * inv);
                m.depth[0] = r - dist;
            }
            else
            {
                m.normal = n;
                m.depth[0] = r;
            }
            m.pos[0] = rt;
            m.n = 1;
            return true;
        }
        // box vs one heightmap triangle (HeightmapCollision.hpp, Box)
        const T centre_dist = dot(tb.pos - A, n);
        const vec3<T> ln = tb.inverse_rotate_vector(n);
        const T box_r = rabs(ln.x) * h.x + rabs(ln.y) * h.y + rabs(ln.z) * h.z;
        if (centre_dist > box_r)
            return false;
        const vec3<T> proj = tb.pos - n * centre_dist;
        const vec3<T> closest = tri_closest(proj, A, B, C);
        if (length(proj - closest) > box_r)
            return false;
        const T depth = box_r - centre_dist;
        if (depth <= T(0.0))
            return false;
        m.normal = n;
        m.n = 1;
        m.pos[0] = closest;
        m.depth[0] = depth;
        return true;
    }

    // heightmap_test (HeightmapCollision.hpp): shape `kind` (see
    // tri_contact) with world AABB [qmn, qmx] against heightmap `id`.
    template <class T>
    __device__ bool heightmap_contact(const HullSetDev &hs, uint32_t id, int kind, const vec3<T> &p0,
                                      const vec3<T> &p1, T r, const tf<T> &tb, const vec3<T> &h,
                                      const vec3<T> &qmn, const vec3<T> &qmx, Manifold<T> &out)
    {
        const HmDesc &hd = hs.hm_desc[id];
        const float *H = hs.hm_heights + hd.off;
        const T ox = T(hd.origin[0]), oy = T(hd.origin[1]), oz = T(hd.origin[2]);
        const T sx = T(hd.scale[0]), sy = T(hd.scale[1]), sz = T(hd.scale[2]);
        const int r0 = max(0, int((qmn.z - oz) / sz));
        const int r1 = min(int(hd.rows) - 2, int((qmx.z - oz) / sz));
        const int c0 = max(0, int((qmn.x - ox) / sx));
        const int c1 = min(int(hd.cols) - 2, int((qmx.x - ox) / sx));
        auto vtx = [&](int row, int col) {
            return vec3<T>(ox + T(col) * sx, T(H[(uint32_t)row * hd.cols + (uint32_t)col]) * sy + oy, oz + T(row) * sz);
        };
        bool hit = false;
        T best = T(0.0);
        for (int rr = r0; rr <= r1; ++rr)
            for (int cc = c0; cc <= c1; ++cc)
            {
                const vec3<T> V00 = vtx(rr, cc), V10 = vtx(rr + 1, cc), V01 = vtx(rr, cc + 1), V11 = vtx(rr + 1, cc + 1);
                for (int k = 0; k < 2; ++k)
                {
                    const vec3<T> A = k ? V10 : V00, B = k ? V11 : V10, C = V01;
                    const vec3<T> n = normalize(cross(B - A, C - A));
                    Manifold<T> cand;
                    cand.n = 0;
                    if (tri_contact(kind, p0, p1, r, tb, h, A, B, C, n, cand) && cand.depth[0] > best)
                    {
                        best = cand.depth[0];
                        out = cand;
                        hit = true;
                    }
                }
            }
        return hit;
    }

    // Sphere / Capsule / Box (shape a) against heightmap hm; other shapes
    // against a heightmap find no contact (the primary CollisionAlgorithm of
    // a non-convex pair, Dispatcher.hpp:40-60).
    template <class T>
    __device__ bool shape_heightmap(const ShapeDev &sa, const tf<T> &ta, const ShapeDev &hm, const HullSetDev &hs,
                                    Manifold<T> &m)
    {
        const vec3<T> zero(T(0), T(0), T(0));
        if (sa.kind == kSphere) // compute_aabb(Sphere)
        {
            const T r = T(sa.p[0]);
            const vec3<T> rr(r, r, r);
            return heightmap_contact(hs, uint32_t(hm.hull), 0, ta.pos, zero, r, ta, zero, ta.pos - rr, ta.pos + rr, m);
        }
        if (sa.kind == kCapsule) // capsule_endpoints + compute_aabb(Capsule)
        {
            const T hh = T(sa.p[0]), r = T(sa.p[1]);
            vec3<T> p1, p2;
            capsule_endpoints(hh, ta, p1, p2);
            const vec3<T> axis = ta.rotate_vector(vec3<T>(T(0.0), hh, T(0.0)));
            const vec3<T> a1 = ta.pos + axis, a2 = ta.pos - axis;
            const vec3<T> rr(r, r, r);
            const vec3<T> qmn = vec3<T>(rmin(a1.x, a2.x), rmin(a1.y, a2.y), rmin(a1.z, a2.z)) - rr;
            const vec3<T> qmx = vec3<T>(rmax(a1.x, a2.x), rmax(a1.y, a2.y), rmax(a1.z, a2.z)) + rr;
            return heightmap_contact(hs, uint32_t(hm.hull), 1, p1, p2, r, ta, zero, qmn, qmx, m);
        }
        if (sa.kind == kBox) // compute_aabb(Box)
        {
            const vec3<T> h(T(sa.p[0]), T(sa.p[1]), T(sa.p[2]));
            const mat3<T> R = mat3_cast(ta.rot);
            const vec3<T> e(rabs(R.c[0].x) * h.x + rabs(R.c[1].x) * h.y + rabs(R.c[2].x) * h.z,
                            rabs(R.c[0].y) * h.x + rabs(R.c[1].y) * h.y + rabs(R.c[2].y) * h.z,
                            rabs(R.c[0].z) * h.x + rabs(R.c[1].z) * h.y + rabs(R.c[2].z) * h.z);
            return heightmap_contact(hs, uint32_t(hm.hull), 2, zero, zero, T(0), ta, h, ta.pos - e, ta.pos + e, m);
        }
        return false;
    }

    // ------------------------------------------------------------ Meshes
    // mesh_world_triangle (MeshCollision.hpp): face f of mesh `id` in world
    // space under tm, with its rotated precomputed normal.
    template <class T>
    __device__ __forceinline__ void mesh_triangle(const HullSetDev &hs, const MeshDesc &md, uint32_t f, const tf<T> &tm,
                                                  vec3<T> &A, vec3<T> &B, vec3<T> &C, vec3<T> &n)
    {
        const uint32_t *ix = hs.mesh_i + 3 * (size_t)(md.f0 + f);
        auto v = [&](uint32_t k) {
            const double *p = hs.mesh_v + 3 * (size_t)(md.v0 + k);
            return vec3<T>(T(p[0]), T(p[1]), T(p[2]));
        };
        A = tm.pos + tm.rotate_vector(v(ix[0]));
        B = tm.pos + tm.rotate_vector(v(ix[1]));
        C = tm.pos + tm.rotate_vector(v(ix[2]));
        const double *fn = hs.mesh_n + 3 * (size_t)(md.f0 + f);
        n = tm.rotate_vector(vec3<T>(T(fn[0]), T(fn[1]), T(fn[2])));
    }

    // mesh_test_all with the sphere / capsule / box per-triangle tests
    // (kind 0 / 1 / 2; the box test is the mesh's own: depth = box_r -
    // edge distance, kept when positive), deepest contact of all faces.
    template <class T>
    __device__ bool mesh_contact(const HullSetDev &hs, uint32_t id, const tf<T> &tm, int kind, const vec3<T> &p0,
                                 const vec3<T> &p1, T r, const tf<T> &tb, const vec3<T> &h, Manifold<T> &out)
    {
        const MeshDesc &md = hs.mesh[id];
        bool hit = false;
        T best = T(0.0);
        for (uint32_t f = 0; f < md.nf; ++f)
        {
            vec3<T> A, B, C, n;
            mesh_triangle(hs, md, f, tm, A, B, C, n);
            Manifold<T> cand;
            cand.n = 0;
            bool ok;
            if (kind == 2)
            {
                const T centre_dist = dot(tb.pos - A, n);
                const vec3<T> ln = tb.inverse_rotate_vector(n);
                const T box_r = rabs(ln.x) * h.x + rabs(ln.y) * h.y + rabs(ln.z) * h.z;
                ok = false;
                if (centre_dist <= box_r)
                {
                    const vec3<T> proj = tb.pos - n * centre_dist;
                    const vec3<T> closest = tri_closest(proj, A, B, C);
                    const T edge_d = length(proj - closest);
                    if (edge_d <= box_r)
                    {
                        cand.normal = n;
                        cand.n = 1;
                        cand.depth[0] = box_r - edge_d;
                        cand.pos[0] = closest;
                        ok = cand.depth[0] > T(0.0);
                    }
                }
            }
            else
                ok = tri_contact(kind, p0, p1, r, tb, h, A, B, C, n, cand);
            if (ok && cand.depth[0] > best)
            {
                best = cand.depth[0];
                out = cand;
                hit = true;
            }
        }
        return hit;
    }

    // Mesh vs Mesh (MeshCollision.hpp): every vertex of every face of A as a
    // sphere of radius 0 against all faces of B, the deepest kept.
    template <class T>
    __device__ bool mesh_mesh(const HullSetDev &hs, uint32_t ia, const tf<T> &ta, uint32_t ib, const tf<T> &tb,
                              Manifold<T> &out)
    {
        const MeshDesc &ma = hs.mesh[ia];
        bool hit = false;
        T best = T(0.0);
        Manifold<T> cand;
        cand.n = 0;
        const vec3<T> zero(T(0), T(0), T(0));
        for (uint32_t f = 0; f < ma.nf; ++f)
        {
            vec3<T> A, B, C, n;
            mesh_triangle(hs, ma, f, ta, A, B, C, n);
            const vec3<T> verts[3] = {A, B, C};
            for (int k = 0; k < 3; ++k)
                if (mesh_contact(hs, ib, tb, 0, verts[k], zero, T(0.0), tb, zero, cand) && cand.depth[0] > best)
                {
                    best = cand.depth[0];
                    out = cand;
                    hit = true;
                }
        }
        return hit;
    }

    // Sphere / Capsule / Box (shape a) or a mesh against mesh `mesh`; other
    // shapes find no contact (the primary algorithm of a non-convex pair).
    template <class T>
    __device__ bool shape_mesh(const ShapeDev &sa, const tf<T> &ta, const ShapeDev &mesh, const tf<T> &tm,
                               const HullSetDev &hs, Manifold<T> &m)
    {
        const vec3<T> zero(T(0), T(0), T(0));
        const uint32_t id = uint32_t(mesh.hull);
        if (sa.kind == kSphere)
            return mesh_contact(hs, id, tm, 0, ta.pos, zero, T(sa.p[0]), ta, zero, m);
        if (sa.kind == kCapsule)
        {
            vec3<T> p1, p2;
            capsule_endpoints(T(sa.p[0]), ta, p1, p2);
            return mesh_contact(hs, id, tm, 1, p1, p2, T(sa.p[1]), ta, zero, m);
        }
        if (sa.kind == kBox)
            return mesh_contact(hs, id, tm, 2, zero, zero, T(0), ta, vec3<T>(T(sa.p[0]), T(sa.p[1]), T(sa.p[2])), m);
        if (sa.kind == kMesh)
            return mesh_mesh(hs, uint32_t(sa.hull), ta, id, tm, m);
        return false;
    }

    // convex_vs_plane for a mesh (RBC_PLANE_SPEC(Mesh)): the support vertex
    // along -n (first of the largest dot products, Mesh.hpp support).
    template <class T>
    __device__ bool mesh_plane(const HullSetDev &hs, uint32_t id, const tf<T> &ts, const ShapeDev &pl, const tf<T> &tp,
                               Manifold<T> &out)
    {
        vec3<T> wn;
        T wd;
        plane_world(pl, tp, wn, wd);
        const vec3<T> ld = ts.inverse_rotate_vector(-wn);
        const MeshDesc &md = hs.mesh[id];
        vec3<T> ls(T(0), T(0), T(0));
        if (md.nv)
        {
            const double *V = hs.mesh_v + 3 * (size_t)md.v0;
            ls = vec3<T>(T(V[0]), T(V[1]), T(V[2]));
            T bd = dot(ls, ld);
            for (uint32_t i = 1; i < md.nv; ++i)
            {
                const vec3<T> p{T(V[3 * i]), T(V[3 * i + 1]), T(V[3 * i + 2])};
                const T d = dot(p, ld);
                if (d > bd)
                {
                    bd = d;
                    ls = p;
                }
            }
        }
        const vec3<T> ws = ts.pos + ts.rotate_vector(ls);
        const T sd = dot(ws, wn) - wd;
        if (sd >= T(0))
            return false;
        out.normal = -wn;
        out.n = 1;
        out.depth[0] = -sd;
        out.pos[0] = ws;
        return true;
    }

    // Sel selects the routines compiled in: kSelAll every pair; kSelNoBoxBox
    // all but box-box; kSelBoxBox box-box only; kSelCommon the pairs of
    // spheres, boxes, capsules and planes but box-box (the caller guarantees
    // the kinds), so a kernel carries only the code, registers and local
    // buffers of the routines it can meet.
    constexpr int kSelAll = 0, kSelNoBoxBox = 1, kSelBoxBox = 2, kSelCommon = 3;

    template <class T, int Sel = kSelAll>
    __device__ __forceinline__ int dispatch_pair(const ShapeDev &sa, const tf<T> &ta, const ShapeDev &sb,
                                                 const tf<T> &tb, const HullSetDev &hs, Manifold<T> &m)
    {
        if constexpr (Sel == kSelBoxBox)
            return box_box(vec3<T>(T(sa.p[0]), T(sa.p[1]), T(sa.p[2])), ta, vec3<T>(T(sb.p[0]), T(sb.p[1]), T(sb.p[2])),
                           tb, m)
                       ? kHit
                       : kMiss;
        constexpr bool kAny = Sel != kSelCommon; // kinds beyond the four common ones
        const int ka = sa.kind, kb = sb.kind;
        bool hit = false;
        bool flip = false;
        if (kb == kPlane)
        {
            if (ka == kSphere)
                hit = sphere_plane(T(sa.p[0]), ta, sb, tb, m);
            else if (ka == kBox)
                hit = box_plane(vec3<T>(T(sa.p[0]), T(sa.p[1]), T(sa.p[2])), ta, sb, tb, m);
            else if (ka == kCapsule)
                hit = capsule_plane(T(sa.p[0]), T(sa.p[1]), ta, sb, tb, m);
            else if (!kAny)
            {
                // no other kind reaches a kSelCommon kernel
            }
            else if (ka == kHull)
                hit = hull_plane(hs, sa.hull, ta, sb, tb, m);
            else if (ka == kCylinder)
                hit = cylinder_plane(T(sa.p[0]), T(sa.p[1]), ta, sb, tb, m);
            else if (ka == kEllipsoid || ka == kCone)
                hit = round_plane(sa, ta, sb, tb, m);
            else if (ka == kMesh)
                hit = mesh_plane(hs, uint32_t(sa.hull), ta, sb, tb, m);
            return hit ? kHit : kMiss;
        }
        if (ka == kPlane)
        {
            if (kb == kSphere)
                hit = sphere_plane(T(sb.p[0]), tb, sa, ta, m);
            else if (kb == kBox)
                hit = box_plane(vec3<T>(T(sb.p[0]), T(sb.p[1]), T(sb.p[2])), tb, sa, ta, m);
            else if (kb == kCapsule)
                hit = capsule_plane(T(sb.p[0]), T(sb.p[1]), tb, sa, ta, m);
            else if (!kAny)
            {
                // no other kind reaches a kSelCommon kernel
            }
            else if (kb == kHull)
                hit = hull_plane(hs, sb.hull, tb, sa, ta, m);
            else if (kb == kCylinder)
                hit = cylinder_plane(T(sb.p[0]), T(sb.p[1]), tb, sa, ta, m);
            else if (kb == kEllipsoid || kb == kCone)
                hit = round_plane(sb, tb, sa, ta, m);
            else if (kb == kMesh)
                hit = mesh_plane(hs, uint32_t(sb.hull), tb, sa, ta, m);
            if (hit)
                m.normal = -m.normal;
            return hit ? kHit : kMiss;
        }
        if (kAny && (ka == kMesh || kb == kMesh))
        {
            if (ka == kHeightmap || kb == kHeightmap)
                return kMiss; // no Mesh / Heightmap algorithm: the primary one finds nothing
            if (kb == kMesh)
                hit = shape_mesh(sa, ta, sb, tb, hs, m);
            else
            {
                hit = shape_mesh(sb, tb, sa, ta, hs, m); // CollisionAlgorithmSym
                if (hit)
                    m.normal = -m.normal;
            }
            return hit ? kHit : kMiss;
        }
        if (kAny && (ka == kHeightmap || kb == kHeightmap))
        {
            if (kb == kHeightmap)
                hit = shape_heightmap(sa, ta, sb, hs, m);
            else
            {
                hit = shape_heightmap(sb, tb, sa, hs, m); // CollisionAlgorithmSym
                if (hit)
                    m.normal = -m.normal;
            }
            return hit ? kHit : kMiss;
        }
        if (kAny && (gjk_kind(ka) || gjk_kind(kb)))
            return kNeedsGjk;
        if (ka == kSphere && kb == kSphere)
            hit = sphere_sphere(T(sa.p[0]), ta, T(sb.p[0]), tb, m);
        else if (ka == kSphere && kb == kBox)
            hit = sphere_box(T(sa.p[0]), ta, vec3<T>(T(sb.p[0]), T(sb.p[1]), T(sb.p[2])), tb, m);
        else if (ka == kBox && kb == kSphere)
        {
            hit = sphere_box(T(sb.p[0]), tb, vec3<T>(T(sa.p[0]), T(sa.p[1]), T(sa.p[2])), ta, m);
            flip = true;
        }
        else if (Sel == kSelAll && ka == kBox && kb == kBox)
            hit = box_box(vec3<T>(T(sa.p[0]), T(sa.p[1]), T(sa.p[2])), ta, vec3<T>(T(sb.p[0]), T(sb.p[1]), T(sb.p[2])), tb, m);
        else if (ka == kSphere && kb == kCapsule)
            hit = sphere_capsule(T(sa.p[0]), ta, T(sb.p[0]), T(sb.p[1]), tb, m);
        else if (ka == kCapsule && kb == kSphere)
        {
            hit = sphere_capsule(T(sb.p[0]), tb, T(sa.p[0]), T(sa.p[1]), ta, m);
            flip = true;
        }
        else if (ka == kCapsule && kb == kCapsule)
            hit = capsule_capsule(T(sa.p[0]), T(sa.p[1]), ta, T(sb.p[0]), T(sb.p[1]), tb, m);
        else if (ka == kCapsule && kb == kBox)
            hit = capsule_box(T(sa.p[0]), T(sa.p[1]), ta, vec3<T>(T(sb.p[0]), T(sb.p[1]), T(sb.p[2])), tb, m);
        else if (ka == kBox && kb == kCapsule)
        {
            hit = capsule_box(T(sb.p[0]), T(sb.p[1]), tb, vec3<T>(T(sa.p[0]), T(sa.p[1]), T(sa.p[2])), ta, m);
            flip = true;
        }
        if (hit && flip)
            m.normal = -m.normal;
        return hit ? kHit : kMiss;
    }
} // namespace rbps_gpu
