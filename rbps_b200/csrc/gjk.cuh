// gjk.cuh - GJK, EPA and the convex contact manifold on the device: the
// narrowphase of every convex pair without an analytic routine (a convex
// hull against a sphere, box, capsule or hull), as rbc::gjk_epa_manifold
// runs it (ContactManifoldGenerator.cpp:415-440).
//
// Same operation order as the reference, so the FP64 instantiation gives the
// same bits:
//   * GJK (GJK.cpp:18-97) over the simplex of Simplex.hpp: four vertex slots
//     addressed through an order array, a new vertex taking the first slot
//     no live entry uses (DoSimplex.cpp:6-16), and the line / triangle /
//     tetrahedron cases of Line.cpp, Triangle.cpp, Tetrahedron.cpp;
//   * EPA (EPA.cpp:141-378): at most 256 faces and 128 vertices, faces never
//     freed, the seed-coplanar shortcut, horizon edges cancelled in both
//     directions with order-preserving erase, the barycentric witness on A;
//   * the manifold (ContactManifoldGenerator.cpp:176-413): for two hulls
//     with polygon tables the reference / incident polygon clip
//     (Clipping.cpp:37-101) or the edge-edge closest points
//     (Clipping.cpp:103-128); one EPA point otherwise; reduce_to_4
//     (ContactManifoldGenerator.hpp:88-154).
// One warp runs one pair: the scans over hull vertices, EPA faces and
// horizon edges are split across its lanes, and the polytope, edge list and
// clipping buffers live in the warp's shared-memory workspace (two views
// of one region: the polytope while EPA runs, the clipping buffers after).
#pragma once
#include <cfloat>
#include <cstdint>

#include "narrow.cuh"

namespace rbps_gpu
{
    // A workspace limit of the GJK path was hit: the device error word gets
    // RBPS_ERR_INTERNAL with site 20 + k (the pair reports no contact).
    __device__ __forceinline__ void set_gjk_error(int *err, int k)
    {
        if (err && atomicCAS(err, 0, -6) == 0)
        {
            err[1] = 20 + k;
            err[2] = 0;
        }
    }

    template <class T> __device__ __forceinline__ T big_value();
    template <> __device__ __forceinline__ double big_value<double>() { return DBL_MAX; }
    template <> __device__ __forceinline__ float big_value<float>() { return FLT_MAX; }

    constexpr int kEpaMaxFaces = 256;
    constexpr int kEpaMaxVerts = 128;
    constexpr int kEpaMaxIter = 128;
    constexpr int kGjkMaxIter = 128;
    constexpr int kEpaMaxEdges = 3 * kEpaMaxFaces;
    constexpr int kClipMaxPoly = 64;                     // polygon vertices / neighbour planes handled
    constexpr int kClipCap = (kClipMaxPoly * 2) * 2 + 8; // (inc_n + planes) * 2 + 8 at the limits

    template <class T>
    struct SVert
    {
        vec3<T> w0, w1, w;
    };

    template <class T>
    struct EpaFace
    {
        vec3<T> n;
        T d;
        uint8_t v[3];
        uint8_t obsolete;
    };

    // The clipping buffers of the hull-hull manifold alone: the second view
    // of a warp's shared workspace, over the EPA polytope it no longer needs.
    template <class T>
    struct GjkClipWork
    {
        vec3<T> inc[kClipMaxPoly], ref[kClipMaxPoly];
        vec3<T> pl_n[kClipMaxPoly], pl_p[kClipMaxPoly];
        vec3<T> buf_a[kClipCap + 4], buf_b[kClipCap + 4];
        vec3<T> keep[kClipCap + 4];
        T keep_d[kClipCap + 4];
    };

    // The EPA polytope of one warp's evaluation (first view of its workspace).
    template <class T>
    struct GjkEpaWork
    {
        SVert<T> verts[kEpaMaxVerts];
        EpaFace<T> faces[kEpaMaxFaces];
        uint8_t edges[2 * kEpaMaxEdges];
    };

    // Bytes of one warp's shared workspace: the two views overlap.
    template <class T>
    constexpr size_t gjk_warp_bytes()
    {
        return ((sizeof(GjkEpaWork<T>) > sizeof(GjkClipWork<T>) ? sizeof(GjkEpaWork<T>) : sizeof(GjkClipWork<T>)) +
                15) / 16 * 16;
    }

    // One convex shape in world space (shape_support, ShapeTypes.hpp:130-133,
    // through the transform as MinkowskiDiff::support_a/b, MinkowskiDiff.hpp).
    template <class T>
    struct ConvexShape
    {
        const ShapeDev *s;
        tf<T> t;
    };

    template <class T>
    __device__ vec3<T> local_support(const ShapeDev &s, const HullSetDev &hs, const vec3<T> &d)
    {
        switch (s.kind)
        {
        case kSphere: // Sphere.hpp:48-51
            return normalize(d) * T(s.p[0]);
        case kBox: // Box.hpp:49-55
            return vec3<T>(d.x > T(0) ? T(s.p[0]) : -T(s.p[0]), d.y > T(0) ? T(s.p[1]) : -T(s.p[1]),
                           d.z > T(0) ? T(s.p[2]) : -T(s.p[2]));
        case kCapsule: // Capsule.hpp:72-79
        {
            const vec3<T> endpoint(T(0.0), d.y >= T(0.0) ? T(s.p[0]) : -T(s.p[0]), T(0.0));
            const T len = length(d);
            if (len < T(kEpsilon))
                return endpoint;
            return endpoint + (d / len) * T(s.p[1]);
        }
        case kEllipsoid:
        case kCylinder:
        case kCone:
            return support_round<T>(s.kind, s.p, d);
        default: // ConvexHull.hpp:457-472
        {
            const uint32_t v0 = hs.v_off[s.hull], v1 = hs.v_off[s.hull + 1];
            if (v1 == v0)
                return vec3<T>();
            const double *V = hs.verts;
            vec3<T> best{T(V[3 * v0]), T(V[3 * v0 + 1]), T(V[3 * v0 + 2])};
            T best_d = dot(best, d);
            for (uint32_t i = v0 + 1; i < v1; ++i)
            {
                const vec3<T> p{T(V[3 * i]), T(V[3 * i + 1]), T(V[3 * i + 2])};
                const T dd = dot(p, d);
                if (dd > best_d)
                {
                    best_d = dd;
                    best = p;
                }
            }
            return best;
        }
        }
    }

    template <class T>
    __device__ __forceinline__ vec3<T> world_support(const ConvexShape<T> &c, const HullSetDev &hs, const vec3<T> &dir)
    {
        return c.t.transform_point(local_support(*c.s, hs, c.t.inverse_rotate_vector(dir)));
    }

    // ------------------------------------------------------------ one warp per pair
    // In the warp forms below every lane of the warp runs the same control
    // flow on the same values (scalar state is computed redundantly, so it
    // is bit-identical on every lane); the loops over hull vertices, EPA
    // faces, vertices and horizon edges are split across the lanes and
    // joined by warp reductions that keep the serial scans' tie rules.
    // Shared memory is written by one lane (or each lane its own entries)
    // between __syncwarp()s.
    constexpr unsigned kWarpAll = 0xffffffffu;

    // Support of a hull: the first vertex (lowest index) of maximal dot
    // product, as the serial scan's strict `>` keeps (ConvexHull.hpp:457-472);
    // a NaN first dot keeps vertex 0 as the serial scan does.  Other shapes
    // are closed forms, the same on every lane.
    template <class T>
    __device__ vec3<T> warp_local_support(const ShapeDev &s, const HullSetDev &hs, const vec3<T> &d)
    {
        if (s.kind != kHull)
            return local_support(s, hs, d);
        const uint32_t v0 = hs.v_off[s.hull], v1 = hs.v_off[s.hull + 1];
        if (v1 == v0)
            return vec3<T>();
        const double *V = hs.verts;
        const uint32_t lane = threadIdx.x & 31u;
        T best_d = T(0);
        uint32_t best_i = ~0u;
        for (uint32_t i = v0 + lane; i < v1; i += 32)
        {
            const vec3<T> p{T(V[3 * i]), T(V[3 * i + 1]), T(V[3 * i + 2])};
            const T dd = dot(p, d);
            if (dd == dd && (best_i == ~0u || dd > best_d))
            {
                best_d = dd;
                best_i = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            const T od = __shfl_xor_sync(kWarpAll, best_d, o);
            const uint32_t oi = __shfl_xor_sync(kWarpAll, best_i, o);
            if (oi != ~0u && (best_i == ~0u || od > best_d || (od == best_d && oi < best_i)))
            {
                best_d = od;
                best_i = oi;
            }
        }
        const vec3<T> p0{T(V[3 * v0]), T(V[3 * v0 + 1]), T(V[3 * v0 + 2])};
        const T d0 = dot(p0, d);
        if (d0 != d0 || best_i == ~0u)
            return p0;
        return vec3<T>{T(V[3 * best_i]), T(V[3 * best_i + 1]), T(V[3 * best_i + 2])};
    }

    template <bool Warp, class T>
    __device__ __forceinline__ vec3<T> support_of(const ConvexShape<T> &c, const HullSetDev &hs, const vec3<T> &dir)
    {
        if constexpr (Warp)
            return c.t.transform_point(warp_local_support(*c.s, hs, c.t.inverse_rotate_vector(dir)));
        else
            return world_support(c, hs, dir);
    }

    // ------------------------------------------------------------ GJK
    template <class T>
    struct Simplex
    {
        SVert<T> st[4];
        int vi[4]; // slot of each live vertex, newest first
        int rank;
    };

    template <class T>
    __device__ __forceinline__ vec3<T> triple_cross(const vec3<T> &a, const vec3<T> &b, const vec3<T> &c)
    {
        return cross(cross(a, b), c);
    }

    template <class T>
    __device__ void simplex_add(Simplex<T> &s, const SVert<T> &v)
    {
        int slot = 0;
        for (int i = 0; i < 4; ++i)
        {
            bool used = false;
            for (int j = 0; j < s.rank; ++j)
                if (s.vi[j] == i)
                {
                    used = true;
                    break;
                }
            if (!used)
            {
                slot = i;
                break;
            }
        }
        s.st[slot] = v;
        const int n = s.rank < 3 ? s.rank : 3;
        for (int i = n; i > 0; --i)
            s.vi[i] = s.vi[i - 1];
        s.vi[0] = slot;
        if (s.rank < 4)
            ++s.rank;
    }

    template <class T>
    __device__ void do_simplex_2(Simplex<T> &s, vec3<T> &dir)
    {
        const vec3<T> a = s.st[s.vi[0]].w, b = s.st[s.vi[1]].w;
        const vec3<T> ao = -a, ab = b - a;
        if (dot(ab, ao) >= T(0.0))
        {
            s.rank = 2;
            dir = triple_cross(ab, ao, ab);
            if (length_sq(dir) < T(1e-6))
            {
                const T ax = rabs(ab.x), ay = rabs(ab.y), az = rabs(ab.z);
                const vec3<T> axis = (ax <= ay && ax <= az) ? vec3<T>(T(1), T(0), T(0))
                                     : (ay <= az ? vec3<T>(T(0), T(1), T(0)) : vec3<T>(T(0), T(0), T(1)));
                dir = cross(ab, axis);
                if (length_sq(dir) < T(1e-6))
                    dir = cross(ab, vec3<T>(T(0), T(0), T(1)));
            }
        }
        else
        {
            s.rank = 1;
            dir = ao;
        }
    }

    template <class T>
    __device__ void do_simplex_3(Simplex<T> &s, vec3<T> &dir)
    {
        const vec3<T> a = s.st[s.vi[0]].w, b = s.st[s.vi[1]].w, c = s.st[s.vi[2]].w;
        const vec3<T> ao = -a, ab = b - a, ac = c - a;
        const vec3<T> abc = cross(ab, ac);
        if (dot(cross(abc, ac), ao) >= T(0.0))
        {
            if (dot(ac, ao) >= T(0.0))
            {
                s.vi[1] = s.vi[2];
                s.rank = 2;
                dir = triple_cross(ac, ao, ac);
            }
            else if (dot(ab, ao) >= T(0.0))
            {
                s.rank = 2;
                dir = triple_cross(ab, ao, ab);
            }
            else
            {
                s.rank = 1;
                dir = ao;
            }
        }
        else if (dot(cross(ab, abc), ao) >= T(0.0))
        {
            if (dot(ab, ao) >= T(0.0))
            {
                s.rank = 2;
                dir = triple_cross(ab, ao, ab);
            }
            else
            {
                s.rank = 1;
                dir = ao;
            }
        }
        else if (dot(abc, ao) >= T(0.0))
        {
            s.rank = 3;
            dir = abc;
        }
        else
        {
            const int tmp = s.vi[1];
            s.vi[1] = s.vi[2];
            s.vi[2] = tmp;
            s.rank = 3;
            dir = -abc;
        }
    }

    // Keeps the listed vertices (slots of a, b, c, d by letter) in order.
    template <class T>
    __device__ __forceinline__ void keep(Simplex<T> &s, int r, int x0, int x1 = 0, int x2 = 0)
    {
        s.vi[0] = x0;
        if (r > 1)
            s.vi[1] = x1;
        if (r > 2)
            s.vi[2] = x2;
        s.rank = r;
    }

    // Returns true when the origin is inside the tetrahedron.
    template <class T>
    __device__ bool do_simplex_4(Simplex<T> &s, vec3<T> &dir)
    {
        const int va = s.vi[0], vb = s.vi[1], vc = s.vi[2], vd = s.vi[3];
        const vec3<T> a = s.st[va].w, b = s.st[vb].w, c = s.st[vc].w, d = s.st[vd].w;
        const vec3<T> ao = -a, ab = b - a, ac = c - a, ad = d - a;
        const vec3<T> abc = cross(ab, ac), acd = cross(ac, ad), adb = cross(ad, ab);
        const T kInside = T(1e-10);
        unsigned info = 0;
        if (dot(abc, ao) > kInside)
            info |= 1u;
        if (dot(acd, ao) > kInside)
            info |= 2u;
        if (dot(adb, ao) > kInside)
            info |= 4u;
        switch (info)
        {
        case 0:
            return true;
        case 1:
            if (dot(cross(abc, ac), ao) >= T(0.0))
            {
                if (dot(ac, ao) >= T(0.0)) { keep(s, 2, va, vc); dir = triple_cross(ac, ao, ac); }
                else if (dot(ab, ao) >= T(0.0)) { keep(s, 2, va, vb); dir = triple_cross(ab, ao, ab); }
                else { keep(s, 1, va); dir = ao; }
            }
            else if (dot(cross(ab, abc), ao) >= T(0.0))
            {
                if (dot(ab, ao) >= T(0.0)) { keep(s, 2, va, vb); dir = triple_cross(ab, ao, ab); }
                else { keep(s, 1, va); dir = ao; }
            }
            else { keep(s, 3, va, vb, vc); dir = abc; }
            break;
        case 2:
            if (dot(cross(acd, ad), ao) >= T(0.0))
            {
                if (dot(ad, ao) >= T(0.0)) { keep(s, 2, va, vd); dir = triple_cross(ad, ao, ad); }
                else if (dot(ac, ao) >= T(0.0)) { keep(s, 2, va, vc); dir = triple_cross(ac, ao, ac); }
                else { keep(s, 1, va); dir = ao; }
            }
            else if (dot(cross(ac, acd), ao) >= T(0.0))
            {
                if (dot(ac, ao) >= T(0.0)) { keep(s, 2, va, vc); dir = triple_cross(ac, ao, ac); }
                else { keep(s, 1, va); dir = ao; }
            }
            else { keep(s, 3, va, vc, vd); dir = acd; }
            break;
        case 3:
            if (dot(ac, ao) >= T(0.0)) { keep(s, 2, va, vc); dir = triple_cross(ac, ao, ac); }
            else { keep(s, 1, va); dir = ao; }
            break;
        case 4:
            if (dot(cross(adb, ab), ao) >= T(0.0))
            {
                if (dot(ab, ao) >= T(0.0)) { keep(s, 2, va, vb); dir = triple_cross(ab, ao, ab); }
                else if (dot(ad, ao) >= T(0.0)) { keep(s, 2, va, vd); dir = triple_cross(ad, ao, ad); }
                else { keep(s, 1, va); dir = ao; }
            }
            else if (dot(cross(ad, adb), ao) >= T(0.0))
            {
                if (dot(ad, ao) >= T(0.0)) { keep(s, 2, va, vd); dir = triple_cross(ad, ao, ad); }
                else { keep(s, 1, va); dir = ao; }
            }
            else { keep(s, 3, va, vd, vb); dir = adb; }
            break;
        case 5:
            if (dot(ab, ao) >= T(0.0)) { keep(s, 2, va, vb); dir = triple_cross(ab, ao, ab); }
            else { keep(s, 1, va); dir = ao; }
            break;
        case 6:
            if (dot(ad, ao) >= T(0.0)) { keep(s, 2, va, vd); dir = triple_cross(ad, ao, ad); }
            else { keep(s, 1, va); dir = ao; }
            break;
        default:
            keep(s, 1, va);
            dir = ao;
            break;
        }
        return false;
    }

    enum
    {
        kGjkValid = 0,
        kGjkInside = 1,
        kGjkFailed = 2
    };

    // Warp = true: every lane of a warp runs it (support_of the warp form).
    template <class T, bool Warp = false>
    __device__ int gjk_evaluate(const ConvexShape<T> &A, const ConvexShape<T> &B, const HullSetDev &hs,
                                const vec3<T> &guess, Simplex<T> &s)
    {
        s.rank = 0;
        for (int i = 0; i < 4; ++i)
            s.vi[i] = i;
        vec3<T> dir = length_sq(guess) > T(kEpsilon) ? guess : vec3<T>(T(1.0), T(0.0), T(0.0));
        SVert<T> v0;
        v0.w0 = support_of<Warp>(A, hs, dir);
        v0.w1 = support_of<Warp>(B, hs, -dir);
        v0.w = v0.w0 - v0.w1;
        simplex_add(s, v0);
        dir = -v0.w;
        for (int it = 0; it < kGjkMaxIter; ++it)
        {
            SVert<T> nx;
            nx.w0 = support_of<Warp>(A, hs, dir);
            nx.w1 = support_of<Warp>(B, hs, -dir);
            nx.w = nx.w0 - nx.w1;
            if (dot(nx.w, dir) < T(0.0))
                return kGjkValid;
            simplex_add(s, nx);
            bool inside = false;
            if (s.rank == 2)
                do_simplex_2(s, dir);
            else if (s.rank == 3)
                do_simplex_3(s, dir);
            else if (s.rank == 4)
                inside = do_simplex_4(s, dir);
            if (inside)
                return kGjkInside;
        }
        return kGjkFailed;
    }

    // ------------------------------------------------------------ EPA
    enum
    {
        kEpaValid = 0,
        kEpaFailed = 1,
        kEpaOutOfFaces = 2,
        kEpaOutOfVertices = 3,
        kEpaNonLinear = 4
    };

    // compute_face_normal (EPA.cpp:19-67)
    template <class T>
    __device__ bool epa_face_normal(EpaFace<T> &f, const SVert<T> *V, int n_all)
    {
        const vec3<T> a = V[f.v[0]].w, b = V[f.v[1]].w, c = V[f.v[2]].w;
        vec3<T> n = cross(b - a, c - a);
        const T n_len = length(n);
        if (n_len < T(kEpsilon))
            return false;
        n = n / n_len;
        T d = dot(n, a);
        const T kCop = T(1e-12);
        if (d < -kCop)
        {
            n = -n;
            d = -d;
        }
        else if (d <= kCop)
        {
            bool fixed = false;
            for (int i = 0; i < n_all; ++i)
            {
                const T t = dot(n, V[i].w);
                if (t > kCop)
                {
                    n = -n;
                    d = T(0.0);
                    fixed = true;
                    break;
                }
                if (t < -kCop)
                {
                    d = T(0.0);
                    fixed = true;
                    break;
                }
            }
            if (!fixed)
                return false;
        }
        f.n = n;
        f.d = d;
        f.obsolete = 0;
        return true;
    }

    template <class T>
    struct EpaResult
    {
        vec3<T> normal;
        T depth;
        vec3<T> contact;
    };

    // ------------------------------------------------------------ manifold
    template <class T>
    __device__ __forceinline__ vec3<T> hull_vertex(const HullSetDev &hs, uint32_t hull, uint32_t i)
    {
        const double *p = hs.verts + 3 * (size_t)(hs.v_off[hull] + i);
        return vec3<T>(T(p[0]), T(p[1]), T(p[2]));
    }

    template <class T>
    __device__ __forceinline__ vec3<T> hull_poly_normal(const HullSetDev &hs, const HullDesc &h, uint32_t p)
    {
        const double *n = hs.poly_n + 3 * (size_t)(h.pn + p);
        return vec3<T>(T(n[0]), T(n[1]), T(n[2]));
    }

    // support_vertex_index (ContactManifoldGenerator.cpp:25-38)
    template <class T>
    __device__ uint32_t support_vertex_index(const HullSetDev &hs, uint32_t hull, const tf<T> &t, const vec3<T> &wd)
    {
        const vec3<T> ld = t.inverse_rotate_vector(wd);
        const uint32_t nv = hs.v_off[hull + 1] - hs.v_off[hull];
        uint32_t best = 0;
        T best_d = dot(hull_vertex<T>(hs, hull, 0), ld);
        for (uint32_t i = 1; i < nv; ++i)
        {
            const T d = dot(hull_vertex<T>(hs, hull, i), ld);
            if (d > best_d)
            {
                best_d = d;
                best = i;
            }
        }
        return best;
    }

    // pick_best_polygon (ContactManifoldGenerator.cpp:40-60)
    template <class T>
    __device__ uint32_t pick_best_polygon(const HullSetDev &hs, const HullDesc &h, const tf<T> &t, uint32_t sv,
                                          const vec3<T> &wd, T &align)
    {
        const uint32_t *off = hs.u32 + h.v2p_o, *idx = hs.u32 + h.v2p_i;
        const uint32_t s = off[sv], e = off[sv + 1];
        uint32_t best = (s < e) ? idx[s] : 0u;
        T best_d = -big_value<T>();
        for (uint32_t i = s; i < e; ++i)
        {
            const uint32_t p = idx[i];
            const T d = dot(t.rotate_vector(hull_poly_normal<T>(hs, h, p)), wd);
            if (d > best_d)
            {
                best_d = d;
                best = p;
            }
        }
        align = best_d;
        return best;
    }

    // pick_best_edge_pair (ContactManifoldGenerator.cpp:68-126)
    template <class T>
    __device__ bool pick_best_edge_pair(const HullSetDev &hs, uint32_t ha, const HullDesc &da, const tf<T> &ta,
                                        uint32_t sa, uint32_t hb, const HullDesc &db, const tf<T> &tb, uint32_t sb,
                                        const vec3<T> &wn, uint32_t e[4], vec3<T> &out_n, T &align)
    {
        const vec3<T> wsa = ta.transform_point(hull_vertex<T>(hs, ha, sa));
        const vec3<T> wsb = tb.transform_point(hull_vertex<T>(hs, hb, sb));
        const uint32_t *ao = hs.u32 + da.v2n_o, *ai = hs.u32 + da.v2n_i;
        const uint32_t *bo = hs.u32 + db.v2n_o, *bi = hs.u32 + db.v2n_i;
        const uint32_t na_s = ao[sa], na_e = ao[sa + 1], nb_s = bo[sb], nb_e = bo[sb + 1];
        if (na_s >= na_e || nb_s >= nb_e)
            return false;
        T best_d = -big_value<T>();
        bool found = false;
        for (uint32_t i = na_s; i < na_e; ++i)
        {
            const uint32_t na = ai[i];
            const vec3<T> ea = wsa - ta.transform_point(hull_vertex<T>(hs, ha, na));
            for (uint32_t j = nb_s; j < nb_e; ++j)
            {
                const uint32_t nb = bi[j];
                const vec3<T> eb = wsb - tb.transform_point(hull_vertex<T>(hs, hb, nb));
                const vec3<T> c = cross(ea, eb);
                const T c_len = length(c);
                if (c_len < T(kEpsilon))
                    continue;
                const vec3<T> cn = c / c_len;
                const T d_pos = dot(cn, wn);
                if (d_pos > best_d)
                {
                    best_d = d_pos;
                    e[0] = sa; e[1] = na; e[2] = sb; e[3] = nb;
                    out_n = cn;
                    found = true;
                }
                const T d_neg = -d_pos;
                if (d_neg > best_d)
                {
                    best_d = d_neg;
                    e[0] = sa; e[1] = na; e[2] = sb; e[3] = nb;
                    out_n = -cn;
                    found = true;
                }
            }
        }
        align = best_d;
        return found;
    }

    // skew_line_closest_points (Clipping.cpp:103-128)
    template <class T>
    __device__ bool skew_closest(const vec3<T> &p1, const vec3<T> &d1, const vec3<T> &p2, const vec3<T> &d2,
                                 vec3<T> &l1, vec3<T> &l2)
    {
        const T n1 = d1.x * d2.x + d1.y * d2.y + d1.z * d2.z;
        const T n2 = d2.x * d2.x + d2.y * d2.y + d2.z * d2.z;
        const T m1 = -d1.x * d1.x - d1.y * d1.y - d1.z * d1.z;
        const T m2 = -d2.x * d1.x - d2.y * d1.y - d2.z * d1.z;
        const T r1 = -d1.x * p2.x + d1.x * p1.x - d1.y * p2.y + d1.y * p1.y - d1.z * p2.z + d1.z * p1.z;
        const T r2 = -d2.x * p2.x + d2.x * p1.x - d2.y * p2.y + d2.y * p1.y - d2.z * p2.z + d2.z * p1.z;
        const T denom = (n1 * m2) - (n2 * m1);
        if (rabs(denom) < T(kEpsilon))
            return false;
        const T n = ((r1 * m2) - (r2 * m1)) / denom;
        const T m = ((n1 * r2) - (n2 * r1)) / denom;
        l1 = p1 + d1 * m;
        l2 = p2 + d2 * n;
        return true;
    }

    // sutherland_hodgman (Clipping.cpp:37-101) from `in` through the planes,
    // ping-ponging between a and b; returns min(count, cap) points in *res.
    template <class T>
    __device__ int sutherland_hodgman(const vec3<T> *in, int n_in, const vec3<T> *pn, const vec3<T> *pp, int n_planes,
                                      bool remove_only, vec3<T> *a, vec3<T> *b, int cap, const vec3<T> **res,
                                      int *err)
    {
        *res = a;
        if (n_in <= 0 || n_planes <= 0 || cap <= 0)
            return 0;
        int na = n_in;
        for (int i = 0; i < n_in; ++i)
            a[i] = in[i];
        for (int p = 0; p < n_planes; ++p)
        {
            if (na == 0)
                break;
            const vec3<T> N = pn[p], P = pp[p];
            const T dplane = -dot(N, P);
            int nb = 0;
            vec3<T> start = a[na - 1];
            for (int j = 0; j < na; ++j)
            {
                const vec3<T> end = a[j];
                const bool start_in = dot(start, N) + dplane >= T(0.0);
                const bool end_in = dot(end, N) + dplane >= T(0.0);
                if (nb + 2 > kClipCap + 4)
                {
                    set_gjk_error(err, 2);
                    return 0;
                }
                if (remove_only)
                {
                    if (end_in)
                        b[nb++] = end;
                }
                else
                {
                    // plane_edge_intersection (Clipping.cpp:15-33)
                    bool cut_ok = false;
                    vec3<T> cut;
                    if (start_in != end_in)
                    {
                        const vec3<T> ab = end - start;
                        const T ab_p = dot(N, ab);
                        if (!(rabs(ab_p) <= T(1e-6)))
                        {
                            const vec3<T> p_co = N * (-dplane);
                            T fac = -dot(N, start - p_co) / ab_p;
                            if (fac < T(0.0))
                                fac = T(0.0);
                            if (fac > T(1.0))
                                fac = T(1.0);
                            cut = start + ab * fac;
                            cut_ok = true;
                        }
                    }
                    if (start_in && end_in)
                        b[nb++] = end;
                    else if (start_in && !end_in)
                    {
                        if (cut_ok)
                            b[nb++] = cut;
                    }
                    else if (!start_in && end_in)
                    {
                        if (cut_ok)
                            b[nb++] = cut;
                        b[nb++] = end;
                    }
                }
                start = end;
            }
            vec3<T> *t = a;
            a = b;
            b = t;
            na = nb;
        }
        *res = a;
        return na < cap ? na : cap;
    }

    // reduce_to_4 (ContactManifoldGenerator.hpp:88-154)
    template <class T>
    __device__ int reduce_to_4(const vec3<T> *pts, const T *dep, int n, Manifold<T> &m)
    {
        if (n <= 4)
        {
            for (int i = 0; i < n; ++i)
            {
                m.pos[i] = pts[i];
                m.depth[i] = dep[i];
            }
            return n;
        }
        int i0 = 0;
        for (int i = 1; i < n; ++i)
            if (dep[i] > dep[i0])
                i0 = i;
        int i1 = (i0 == 0) ? 1 : 0;
        T best = length_sq(pts[i1] - pts[i0]);
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
        best = T(0.0);
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
            for (int i = 0; i < n; ++i)
                if (i != i0 && i != i1)
                {
                    i2 = i;
                    break;
                }
        int i3 = -1;
        best = T(0.0);
        if (i2 >= 0)
        {
            const vec3<T> tri_n = cross(pts[i1] - pts[i0], pts[i2] - pts[i0]);
            for (int i = 0; i < n; ++i)
            {
                if (i == i0 || i == i1 || i == i2)
                    continue;
                const T d = rabs(dot(pts[i] - pts[i0], tri_n));
                if (d > best)
                {
                    best = d;
                    i3 = i;
                }
            }
            if (i3 < 0)
                for (int i = 0; i < n; ++i)
                    if (i != i0 && i != i1 && i != i2)
                    {
                        i3 = i;
                        break;
                    }
        }
        m.pos[0] = pts[i0];
        m.depth[0] = dep[i0];
        m.pos[1] = pts[i1];
        m.depth[1] = dep[i1];
        if (i2 >= 0)
        {
            m.pos[2] = pts[i2];
            m.depth[2] = dep[i2];
        }
        if (i3 >= 0)
        {
            m.pos[3] = pts[i3];
            m.depth[3] = dep[i3];
            return 4;
        }
        return (i2 >= 0) ? 3 : 2;
    }

    template <class T>
    __device__ __forceinline__ void single_point(Manifold<T> &m, const vec3<T> &n, const vec3<T> &p, T d)
    {
        m.normal = n;
        m.n = 1;
        m.pos[0] = p;
        m.depth[0] = d;
    }

    // manifold_convex_convex (ContactManifoldGenerator.cpp:176-379) for two
    // hulls with polygon tables.
    // WS: the clipping buffers (GjkClipWork, the second view of a warp's
    // shared workspace).
    template <class T, class WS>
    __device__ void manifold_hull_hull(const EpaResult<T> &r, const HullSetDev &hs, uint32_t ha, const tf<T> &ta,
                                       uint32_t hb, const tf<T> &tb, WS &ws, Manifold<T> &m, int *err)
    {
        m.normal = r.normal;
        m.n = 0;
        const HullDesc da = hs.desc[ha], db = hs.desc[hb];
        const vec3<T> inv_normal = -r.normal;
        const uint32_t sa = support_vertex_index(hs, ha, ta, r.normal);
        const uint32_t sb = support_vertex_index(hs, hb, tb, inv_normal);
        T align_a, align_b;
        const uint32_t poly_a = pick_best_polygon(hs, da, ta, sa, r.normal, align_a);
        const uint32_t poly_b = pick_best_polygon(hs, db, tb, sb, inv_normal, align_b);
        uint32_t e[4] = {0, 0, 0, 0};
        vec3<T> edge_n(T(0), T(0), T(0));
        T align_e = -big_value<T>();
        const bool has_edge = pick_best_edge_pair(hs, ha, da, ta, sa, hb, db, tb, sb, r.normal, e, edge_n, align_e);
        const T EPS = T(1e-4);
        if (has_edge && align_e > align_a + EPS && align_e > align_b + EPS)
        {
            const vec3<T> p1 = ta.transform_point(hull_vertex<T>(hs, ha, e[0]));
            const vec3<T> d1 = ta.transform_point(hull_vertex<T>(hs, ha, e[1])) - p1;
            const vec3<T> p2 = tb.transform_point(hull_vertex<T>(hs, hb, e[2]));
            const vec3<T> d2 = tb.transform_point(hull_vertex<T>(hs, hb, e[3])) - p2;
            vec3<T> l1, l2;
            if (skew_closest(p1, d1, p2, d2, l1, l2))
                single_point(m, r.normal, (l1 + l2) * T(0.5), r.depth);
            else
                single_point(m, r.normal, r.contact, r.depth);
            return;
        }
        const bool ref_is_a = align_a > align_b;
        const HullDesc &dref = ref_is_a ? da : db;
        const HullDesc &dinc = ref_is_a ? db : da;
        const uint32_t href = ref_is_a ? ha : hb, hinc = ref_is_a ? hb : ha;
        const tf<T> &tref = ref_is_a ? ta : tb;
        const tf<T> &tinc = ref_is_a ? tb : ta;
        const uint32_t ref_poly = ref_is_a ? poly_a : poly_b;
        const uint32_t inc_poly = ref_is_a ? poly_b : poly_a;
        const vec3<T> ref_n = tref.rotate_vector(hull_poly_normal<T>(hs, dref, ref_poly));
        const uint32_t *inc_off = hs.u32 + dinc.po, *inc_idx = hs.u32 + dinc.pi;
        const uint32_t inc_s = inc_off[inc_poly], inc_e = inc_off[inc_poly + 1];
        const int inc_n = (int)(inc_e - inc_s);
        if (inc_n < 3)
        {
            single_point(m, r.normal, r.contact, r.depth);
            return;
        }
        const uint32_t *ref_off = hs.u32 + dref.po, *ref_idx = hs.u32 + dref.pi;
        const uint32_t ref_s = ref_off[ref_poly], ref_e = ref_off[ref_poly + 1];
        const uint32_t *p2o = hs.u32 + dref.p2p_o, *p2i = hs.u32 + dref.p2p_i;
        const uint32_t n_s = p2o[ref_poly], n_e = p2o[ref_poly + 1];
        if (inc_n > kClipMaxPoly || (int)(ref_e - ref_s) > kClipMaxPoly || (int)(n_e - n_s) > kClipMaxPoly)
        {
            set_gjk_error(err, 3); // polygon beyond the workspace: no contact
            return;
        }
        for (int i = 0; i < inc_n; ++i)
            ws.inc[i] = tinc.transform_point(hull_vertex<T>(hs, hinc, inc_idx[inc_s + i]));
        for (uint32_t i = 0; i < ref_e - ref_s; ++i)
            ws.ref[i] = tref.transform_point(hull_vertex<T>(hs, href, ref_idx[ref_s + i]));
        const vec3<T> ref_pt = ws.ref[0];
        const int n_planes = (int)(n_e - n_s);
        for (int i = 0; i < n_planes; ++i)
        {
            const uint32_t nbp = p2i[n_s + i];
            const uint32_t first_v = ref_idx[ref_off[nbp]];
            ws.pl_p[i] = tref.transform_point(hull_vertex<T>(hs, href, first_v));
            ws.pl_n[i] = -tref.rotate_vector(hull_poly_normal<T>(hs, dref, nbp));
        }
        const int clip_cap = (inc_n + n_planes) * 2 + 8;
        const vec3<T> *clipped = ws.inc;
        int n_clipped = inc_n;
        if (n_planes > 0)
            n_clipped = sutherland_hodgman(ws.inc, inc_n, ws.pl_n, ws.pl_p, n_planes, false, ws.buf_a, ws.buf_b,
                                           clip_cap, &clipped, err);
        // the ref-plane pass reads `clipped` (one of buf_a / buf_b or inc)
        // and writes into ws.keep / buf ping-pong: copy it first
        for (int i = 0; i < n_clipped; ++i)
            ws.keep[i] = clipped[i];
        const vec3<T> rpn = -ref_n;
        const vec3<T> *fin = ws.buf_a;
        const int n_final = sutherland_hodgman(ws.keep, n_clipped, &rpn, &ref_pt, 1, true, ws.buf_a, ws.buf_b,
                                               clip_cap + 4, &fin, err);
        int n_keep = 0;
        for (int i = 0; i < n_final; ++i)
        {
            const vec3<T> p = fin[i];
            const T d_to_plane = dot(p - ref_pt, ref_n);
            const vec3<T> diff = ref_n * d_to_plane;
            const T pen = ref_is_a ? dot(diff, r.normal) : -dot(diff, r.normal);
            if (pen <= T(0.0))
            {
                ws.keep[n_keep] = p;
                ws.keep_d[n_keep] = -pen;
                ++n_keep;
            }
        }
        if (n_keep == 0)
        {
            single_point(m, r.normal, r.contact, r.depth);
            return;
        }
        m.n = reduce_to_4(ws.keep, ws.keep_d, n_keep, m);
    }

    // ------------------------------------------------------------ EPA on a warp
    // add_edge (EPA.cpp:71-84) on a warp: the first stored edge equal to
    // (a, b) in either direction is found by a ballot over 32 entries at a
    // time and erased with the later entries moved down in order; otherwise
    // (a, b) is appended.  Every lane calls it with the same arguments.
    __device__ __forceinline__ void warp_add_edge(uint8_t *E, int &ne, uint8_t a, uint8_t b)
    {
        const int lane = (int)(threadIdx.x & 31u);
        int hit = -1;
        for (int base = 0; base < ne && hit < 0; base += 32)
        {
            const int i = base + lane;
            const bool match = i < ne && ((E[2 * i] == a && E[2 * i + 1] == b) || (E[2 * i] == b && E[2 * i + 1] == a));
            const unsigned m = __ballot_sync(kWarpAll, match);
            if (m)
                hit = base + __ffs(m) - 1;
        }
        if (hit >= 0)
        {
            for (int base = hit; base + 1 < ne; base += 32)
            {
                const int k = base + lane;
                uint8_t x0 = 0, x1 = 0;
                if (k + 1 < ne)
                {
                    x0 = E[2 * k + 2];
                    x1 = E[2 * k + 3];
                }
                __syncwarp();
                if (k + 1 < ne)
                {
                    E[2 * k] = x0;
                    E[2 * k + 1] = x1;
                }
                __syncwarp();
            }
            --ne;
        }
        else
        {
            if (lane == 0)
            {
                E[2 * ne] = a;
                E[2 * ne + 1] = b;
            }
            ++ne;
        }
        __syncwarp();
    }

    // epa_evaluate on one warp, the polytope in the warp's shared workspace.
    // The same steps in the same order as the serial form (EPA.cpp:141-378):
    // the nearest live face is a warp argmin keeping the lowest index on
    // ties (the serial scan's strict `<`); the faces that see the new vertex
    // are tested 32 at a time and their edges added in face order; the new
    // faces are built 32 at a time and packed in edge order, a degenerate
    // one leaving no slot, with OutOfFaces where the serial loop would meet
    // 256 faces.  Every lane returns the same result.
    template <class T>
    __device__ int epa_evaluate_warp(const Simplex<T> &seed, const ConvexShape<T> &A, const ConvexShape<T> &B,
                                     const HullSetDev &hs, GjkEpaWork<T> &ws, EpaResult<T> &out, int *err)
    {
        const uint32_t lane = threadIdx.x & 31u;
        out.normal = vec3<T>(T(0), T(0), T(0));
        out.depth = T(0.0);
        out.contact = vec3<T>(T(0), T(0), T(0));
        if (seed.rank != 4)
            return kEpaNonLinear;
        SVert<T> *V = ws.verts;
        EpaFace<T> *F = ws.faces;
        __syncwarp();
        if (lane == 0)
            for (int i = 0; i < 4; ++i)
                V[i] = seed.st[seed.vi[i]];
        __syncwarp();
        int nv = 4, nf = 0;
        {
            const vec3<T> va = V[0].w, vb = V[1].w, vc = V[2].w, vd = V[3].w;
            const T e2 = T(kEpsilon) * T(kEpsilon);
            vec3<T> pn = cross(vb - va, vc - va);
            if (length_sq(pn) < e2)
                pn = cross(vb - va, vd - va);
            if (length_sq(pn) < e2)
                pn = cross(vc - va, vd - va);
            if (length_sq(pn) > e2)
            {
                pn = normalize(pn);
                const T dist_d = rabs(dot(vd - va, pn));
                if (dist_d < T(1e-5))
                {
                    const vec3<T> sp = support_of<true>(A, hs, pn) - support_of<true>(B, hs, -pn);
                    const vec3<T> sn = support_of<true>(A, hs, -pn) - support_of<true>(B, hs, pn);
                    const T dist_pos = dot(sp - va, pn);
                    const T dist_neg = dot(sn - va, -pn);
                    if (dist_pos < T(1e-4) || dist_neg < T(1e-4))
                    {
                        out.normal = (dist_pos <= dist_neg) ? pn : -pn;
                        out.depth = T(0.0);
                        out.contact = (V[0].w0 + V[1].w0 + V[2].w0 + V[3].w0) * T(0.25);
                        return kEpaValid;
                    }
                }
            }
        }
        {
            // initial tetrahedron faces (A,B,C), (A,C,D), (A,D,B), (B,C,D): lane k builds face k
            const uint8_t init[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 2, 3}};
            EpaFace<T> f;
            bool ok = true;
            if (lane < 4)
            {
                f.v[0] = init[lane][0];
                f.v[1] = init[lane][1];
                f.v[2] = init[lane][2];
                f.obsolete = 0;
                ok = epa_face_normal(f, V, nv);
            }
            if (__ballot_sync(kWarpAll, !ok))
                return kEpaNonLinear;
            if (lane < 4)
                F[lane] = f;
            nf = 4;
            __syncwarp();
        }
        int ne = 0;
        for (int it = 0; it < kEpaMaxIter; ++it)
        {
            T min_d = big_value<T>();
            int ci = -1;
            for (int i = (int)lane; i < nf; i += 32)
                if (!F[i].obsolete && F[i].d < min_d)
                {
                    min_d = F[i].d;
                    ci = i;
                }
            for (int o = 16; o > 0; o >>= 1)
            {
                const T od = __shfl_xor_sync(kWarpAll, min_d, o);
                const int oi = __shfl_xor_sync(kWarpAll, ci, o);
                if (oi >= 0 && (ci < 0 || od < min_d || (od == min_d && oi < ci)))
                {
                    min_d = od;
                    ci = oi;
                }
            }
            if (ci < 0)
                return kEpaFailed;
            const EpaFace<T> cf = F[ci];
            const vec3<T> dir = cf.n;
            SVert<T> w;
            w.w0 = support_of<true>(A, hs, dir);
            w.w1 = support_of<true>(B, hs, -dir);
            w.w = w.w0 - w.w1;
            const T d_proj = dot(w.w, dir);
            if (d_proj - min_d < T(1e-6))
            {
                out.normal = cf.n;
                out.depth = min_d;
                const vec3<T> q = cf.n * min_d;
                const vec3<T> p0 = V[cf.v[0]].w, p1 = V[cf.v[1]].w, p2 = V[cf.v[2]].w;
                const vec3<T> e0 = p1 - p0, e1 = p2 - p0, r = q - p0;
                const T d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1);
                const T d20 = dot(r, e0), d21 = dot(r, e1);
                const T denom = d00 * d11 - d01 * d01;
                if (rabs(denom) < T(kEpsilon))
                    out.contact = V[cf.v[0]].w0;
                else
                {
                    const T v_w = (d11 * d20 - d01 * d21) / denom;
                    const T w_w = (d00 * d21 - d01 * d20) / denom;
                    const T u_w = T(1.0) - v_w - w_w;
                    out.contact = V[cf.v[0]].w0 * u_w + V[cf.v[1]].w0 * v_w + V[cf.v[2]].w0 * w_w;
                }
                return kEpaValid;
            }
            bool dup = false;
            for (int i = (int)lane; i < nv; i += 32)
                dup = dup || length_sq(V[i].w - w.w) < T(kEpsilon) * T(kEpsilon);
            if (__any_sync(kWarpAll, dup))
            {
                out.normal = cf.n;
                out.depth = min_d;
                out.contact = V[cf.v[0]].w0;
                return kEpaValid;
            }
            if (nv >= kEpaMaxVerts)
                return kEpaOutOfVertices;
            const uint8_t wi = (uint8_t)nv;
            if (lane == 0)
                V[nv] = w;
            ++nv;
            __syncwarp();
            // the horizon: faces that see w, their edges in face order
            ne = 0;
            for (int base = 0; base < nf; base += 32)
            {
                const int i = base + (int)lane;
                bool vis = false;
                if (i < nf && !F[i].obsolete)
                {
                    const EpaFace<T> &f = F[i];
                    const vec3<T> centroid = (V[f.v[0]].w + V[f.v[1]].w + V[f.v[2]].w) * (T(1.0) / T(3.0));
                    vis = dot(f.n, w.w - centroid) > T(0.0);
                }
                unsigned m = __ballot_sync(kWarpAll, vis);
                if (vis)
                    F[i].obsolete = 1;
                while (m)
                {
                    const int fi = base + __ffs(m) - 1;
                    m &= m - 1;
                    if (ne + 3 > kEpaMaxEdges)
                    {
                        if (lane == 0)
                            set_gjk_error(err, 1);
                        return kEpaFailed;
                    }
                    const uint8_t a = F[fi].v[0], b = F[fi].v[1], c = F[fi].v[2];
                    warp_add_edge(ws.edges, ne, a, b);
                    warp_add_edge(ws.edges, ne, b, c);
                    warp_add_edge(ws.edges, ne, c, a);
                }
            }
            __syncwarp();
            // new faces on the horizon edges, packed in edge order
            for (int base = 0; base < ne; base += 32)
            {
                const int e = base + (int)lane;
                EpaFace<T> f;
                bool ok = false;
                if (e < ne)
                {
                    f.v[0] = ws.edges[2 * e];
                    f.v[1] = ws.edges[2 * e + 1];
                    f.v[2] = wi;
                    f.obsolete = 0;
                    ok = epa_face_normal(f, V, nv);
                }
                const unsigned okm = __ballot_sync(kWarpAll, ok);
                const int before = nf + __popc(okm & ((1u << lane) - 1u));
                if (__any_sync(kWarpAll, e < ne && before >= kEpaMaxFaces))
                    return kEpaOutOfFaces;
                if (ok)
                    F[before] = f;
                nf += __popc(okm);
            }
            __syncwarp();
        }
        return kEpaFailed;
    }

    // gjk_epa_manifold on one warp: every lane calls it with the same pair
    // and `ws` the warp's shared workspace (gjk_warp_bytes<T>()).  The
    // return value is the same on every lane; the manifold is complete on
    // lane 0 (a hull-hull manifold is clipped by lane 0 alone, in the
    // workspace's second view).
    template <class T>
    __device__ bool gjk_epa_manifold_warp(const ShapeDev &sa, const tf<T> &ta, const ShapeDev &sb, const tf<T> &tb,
                                          const HullSetDev &hs, unsigned char *ws, Manifold<T> &m, int *err)
    {
        const ConvexShape<T> A{&sa, ta}, B{&sb, tb};
        vec3<T> guess = tb.pos - ta.pos;
        if (length_sq(guess) < T(kEpsilon))
            guess = vec3<T>(T(1.0), T(0.0), T(0.0));
        Simplex<T> s;
        if (gjk_evaluate<T, true>(A, B, hs, guess, s) != kGjkInside)
            return false;
        EpaResult<T> r;
        if (epa_evaluate_warp(s, A, B, hs, *reinterpret_cast<GjkEpaWork<T> *>(ws), r, err) != kEpaValid)
            return false;
        m.normal = r.normal;
        m.n = 0;
        const bool adj_a = sa.kind == kHull && hs.desc[sa.hull].np > 0;
        const bool adj_b = sb.kind == kHull && hs.desc[sb.hull].np > 0;
        __syncwarp(); // the polytope is dead: the clipping view may overwrite it
        if (adj_a && adj_b)
        {
            if ((threadIdx.x & 31u) == 0)
                manifold_hull_hull(r, hs, (uint32_t)sa.hull, ta, (uint32_t)sb.hull, tb,
                                   *reinterpret_cast<GjkClipWork<T> *>(ws), m, err);
        }
        else
            single_point(m, r.normal, r.contact, r.depth);
        __syncwarp();
        return true;
    }
} // namespace rbps_gpu
