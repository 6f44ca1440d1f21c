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
    // Warps per CTA of the GJK kernels; each warp owns gjk_warp_bytes of the
    // CTA's dynamic shared memory.
    constexpr int kGjkWarps = 4;
    constexpr size_t kGjkWarpBytes = gjk_warp_bytes<double>();
    constexpr size_t kGjkSmem = kGjkWarps * kGjkWarpBytes;

    // Opens a GJK kernel to its shared workspaces (once per device and kernel).
    template <class K>
    cudaError_t gjk_smem_attr(K kernel)
    {
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGjkSmem);
    }

    // The queued GJK pairs of this substep, one warp per pair, the warp's
    // polytope and clipping buffers in shared memory.
    template <class T, class P>
    __global__ void __launch_bounds__(kGjkWarps * 32) k_gjk(const Engine<T, P> E)
    {
        extern __shared__ __align__(16) unsigned char gjk_smem[];
        unsigned char *ws = gjk_smem + (threadIdx.x >> 5) * kGjkWarpBytes;
        const uint32_t warp = blockIdx.x * kGjkWarps + (threadIdx.x >> 5);
        const uint32_t n_warps = gridDim.x * kGjkWarps;
        const uint32_t n = min(*E.gjk_count, E.gjk_cap);
        for (uint32_t i = warp; i < n; i += n_warps)
        {
            const uint2 e = E.gjk_list[i];
            gjk_candidate_warp(E, e.x, e.y, ws);
        }
    }

    template <class T, class P>
    cudaError_t launch_gjk(const Engine<T, P> &e, cudaStream_t stream)
    {
        if (!e.gjk_list)
            return cudaSuccess;
        k_gjk<T, P><<<e.gjk_slots, kGjkWarps * 32, kGjkSmem, stream>>>(e);
        return cudaGetLastError();
    }

    // Sizes the GJK pass: CTAs of kGjkWarps warps that the device keeps
    // resident at once (the grid loops over the queued pairs).
    template <class T, class P>
    cudaError_t prepare_gjk(int sm_count, uint32_t *ctas)
    {
        cudaError_t rc = gjk_smem_attr(k_gjk<T, P>);
        int per_sm = 0;
        if (rc == cudaSuccess)
            rc = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gjk<T, P>, kGjkWarps * 32, kGjkSmem);
        *ctas = (uint32_t)(per_sm > 0 ? per_sm : 1) * (uint32_t)sm_count;
        return rc;
    }

    // rbc::dispatch (Dispatcher.hpp:208-213) on independent shape pairs, one
    // warp per pair: every lane runs the analytic routines alike (the same
    // result on every lane) and, for a pair without one, GJK / EPA / the
    // manifold together on the warp's shared workspace; lane 0 writes the
    // result.  Transforms are 7 doubles (position, quaternion wxyz).
    template <class T, class P>
    __device__ void collide_one_warp(const ShapeDev *sa, const double *ta, const ShapeDev *sb, const double *tb,
                                     const HullSetDev &hulls, uint32_t i, CollideOut *out, unsigned char *ws, int *err)
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
            const bool hit = gjk_epa_manifold_warp(sa[i], ad, sb[i], bd, hulls, ws, md, err);
            m = manifold_cast<T>(md);
            res = hit ? kHit : kMiss;
        }
        if ((threadIdx.x & 31u) != 0)
            return;
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
    __global__ void __launch_bounds__(kGjkWarps * 32) k_collide(const ShapeDev *sa, const double *ta,
                                                                 const ShapeDev *sb, const double *tb,
                                                                 const HullSetDev hulls, uint32_t n, CollideOut *out,
                                                                 int *err)
    {
        extern __shared__ __align__(16) unsigned char gjk_smem[];
        unsigned char *ws = gjk_smem + (threadIdx.x >> 5) * kGjkWarpBytes;
        const uint32_t warp = blockIdx.x * kGjkWarps + (threadIdx.x >> 5);
        for (uint32_t i = warp; i < n; i += gridDim.x * kGjkWarps)
            collide_one_warp<T, P>(sa, ta, sb, tb, hulls, i, out, ws, err);
    }

    template <class T, class P>
    cudaError_t launch_collide(const ShapeDev *sa, const double *ta, const ShapeDev *sb, const double *tb,
                               const HullSetDev &hulls, uint32_t n, CollideOut *out, int *err, cudaStream_t stream)
    {
        if (!n)
            return cudaSuccess;
        cudaError_t rc = gjk_smem_attr(k_collide<T, P>);
        if (rc != cudaSuccess)
            return rc;
        const uint32_t ctas = (uint32_t)std::min<size_t>(((size_t)n + kGjkWarps - 1) / kGjkWarps, 4096);
        k_collide<T, P><<<ctas, kGjkWarps * 32, kGjkSmem, stream>>>(sa, ta, sb, tb, hulls, n, out, err);
        return cudaGetLastError();
    }
} // namespace rbps_gpu

#define RBPS_INSTANTIATE_GJK(T, P)                                                                             \
    template cudaError_t rbps_gpu::launch_gjk<T, P>(const rbps_gpu::Engine<T, P> &, cudaStream_t);              \
    template cudaError_t rbps_gpu::launch_collide<T, P>(const rbps_gpu::ShapeDev *, const double *,               \
                                                       const rbps_gpu::ShapeDev *, const double *,               \
                                                       const rbps_gpu::HullSetDev &, uint32_t,                   \
                                                       rbps_gpu::CollideOut *, int *, cudaStream_t);             \
    template cudaError_t rbps_gpu::prepare_gjk<T, P>(int, uint32_t *);
