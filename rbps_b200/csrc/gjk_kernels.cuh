// gjk_kernels.cuh - the kernels that run GJK / EPA / the convex manifold:
// the per-substep pass over the queued hull pairs of a batch, and the
// stand-alone pair query behind rbps_batch_collide.  They are compiled in
// their own translation units (gjk_f64.cu, gjk_f32.cu) with -fmad=false, so
// the double-precision GJK arithmetic rounds like the reference in every
// engine precision while the FP32 engine keeps FMA contraction.
#pragma once
#include "engine_impl.cuh"

namespace rbps_gpu
{
    // The queued GJK pairs of this substep, one per thread, each thread on
    // its own workspace (gridDim * blockDim <= gjk_slots).
    template <class T, class P>
    __global__ void __launch_bounds__(128) k_gjk(const Engine<T, P> E)
    {
        const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
        const uint32_t nth = gridDim.x * blockDim.x;
        const uint32_t n = min(*E.gjk_count, E.gjk_cap);
        GjkWork<double> &ws = reinterpret_cast<GjkWork<double> *>(E.gjk_ws)[tid];
        for (uint32_t i = tid; i < n; i += nth)
        {
            const uint2 e = E.gjk_list[i];
            gjk_candidate(E, e.x, e.y, ws);
        }
    }

    template <class T, class P>
    cudaError_t launch_gjk(const Engine<T, P> &e, cudaStream_t stream)
    {
        if (!e.gjk_list)
            return cudaSuccess;
        k_gjk<T, P><<<e.gjk_slots / 128, 128, 0, stream>>>(e);
        return cudaGetLastError();
    }

    // rbc::dispatch (Dispatcher.hpp:208-213) on independent shape pairs, one
    // thread per pair; transforms are 7 doubles (position, quaternion wxyz).
    template <class T, class P>
    __device__ void collide_one(const ShapeDev *sa, const double *ta, const ShapeDev *sb, const double *tb,
                                const HullSetDev &hulls, uint32_t i, CollideOut *out, GjkWork<double> &ws, int *err)
    {
        auto load_tf_d = [](const double *p) {
            tf<double> t;
            t.pos = vec3<double>(p[0], p[1], p[2]);
            t.rot = quat<double>(p[3], p[4], p[5], p[6]);
            return t;
        };
        auto load_tf = [](const double *p) {
            tf<T> t;
            t.pos = vec3<T>(T(p[0]), T(p[1]), T(p[2]));
            t.rot = quat<T>(T(p[3]), T(p[4]), T(p[5]), T(p[6]));
            return t;
        };
        const tf<T> a = load_tf(ta + 7 * (size_t)i), b = load_tf(tb + 7 * (size_t)i);
        Manifold<T> m;
        m.n = 0;
        int res = dispatch_pair(sa[i], a, sb[i], b, hulls, m);
        if (res == kNeedsGjk)
        {
            const tf<double> ad = load_tf_d(ta + 7 * (size_t)i), bd = load_tf_d(tb + 7 * (size_t)i);
            Manifold<double> md;
            md.n = 0;
            const bool hit = gjk_epa_manifold(sa[i], ad, sb[i], bd, hulls, ws, md, err);
            m = manifold_cast<T>(md);
            res = hit ? kHit : kMiss;
        }
        CollideOut o;
        o.status = res;
        o.n_points = res == kHit ? m.n : 0;
        o.normal[0] = o.normal[1] = o.normal[2] = 0.0;
        for (int k = 0; k < 4; ++k)
        {
            o.depth[k] = 0.0;
            o.position[k][0] = o.position[k][1] = o.position[k][2] = 0.0;
        }
        if (res == kHit)
        {
            o.normal[0] = double(m.normal.x);
            o.normal[1] = double(m.normal.y);
            o.normal[2] = double(m.normal.z);
            for (int k = 0; k < m.n && k < 4; ++k)
            {
                o.position[k][0] = double(m.pos[k].x);
                o.position[k][1] = double(m.pos[k].y);
                o.position[k][2] = double(m.pos[k].z);
                o.depth[k] = double(m.depth[k]);
            }
        }
        out[i] = o;
    }

    template <class T, class P>
    __global__ void k_collide(const ShapeDev *sa, const double *ta, const ShapeDev *sb, const double *tb,
                              const HullSetDev hulls, uint32_t n, CollideOut *out, void *gjk_ws, int *err)
    {
        const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
        for (uint32_t i = tid; i < n; i += gridDim.x * blockDim.x)
            collide_one<T, P>(sa, ta, sb, tb, hulls, i, out, reinterpret_cast<GjkWork<double> *>(gjk_ws)[tid], err);
    }

    template <class T, class P>
    size_t gjk_work_bytes()
    {
        return sizeof(GjkWork<double>);
    }

    // threads = workspaces in gjk_ws (a multiple of 128)
    template <class T, class P>
    cudaError_t launch_collide(const ShapeDev *sa, const double *ta, const ShapeDev *sb, const double *tb,
                               const HullSetDev &hulls, uint32_t n, CollideOut *out, void *gjk_ws, uint32_t threads,
                               int *err, cudaStream_t stream)
    {
        if (n)
            k_collide<T, P><<<threads / 128, 128, 0, stream>>>(sa, ta, sb, tb, hulls, n, out, gjk_ws, err);
        return cudaGetLastError();
    }
} // namespace rbps_gpu

#define RBPS_INSTANTIATE_GJK(T, P)                                                                             \
    template cudaError_t rbps_gpu::launch_gjk<T, P>(const rbps_gpu::Engine<T, P> &, cudaStream_t);              \
    template cudaError_t rbps_gpu::launch_collide<T, P>(const rbps_gpu::ShapeDev *, const double *,               \
                                                       const rbps_gpu::ShapeDev *, const double *,               \
                                                       const rbps_gpu::HullSetDev &, uint32_t,                   \
                                                       rbps_gpu::CollideOut *, void *, uint32_t, int *,          \
                                                       cudaStream_t);                                            \
    template size_t rbps_gpu::gjk_work_bytes<T, P>();
