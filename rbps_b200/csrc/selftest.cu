// selftest.cu - self-checking entry points for the team primitives (scan,
// stable radix sort) used by every phase of the step, run on one CTA
// (BlockTeam) or a cooperative grid (GridTeam).  The caller compares the
// results with a host reference; the kernels only touch the buffers
// allocated here, sized by the same rules as the engine's scratch.
#include <algorithm>
#include <vector>

#include "engine_impl.cuh"
#include "rbps_gpu.h"

using namespace rbps_gpu;

int rbps_internal_fail(int code, const char *msg);

namespace
{
    template <class Team>
    __global__ void __launch_bounds__(256) k_sort(uint32_t *k, uint32_t *v, uint32_t *kt, uint32_t *vt, uint32_t n,
                                                  int bits, uint32_t *counts, uint32_t *ts)
    {
        __shared__ BlockShared sh;
        Team tm;
        team_radix_sort(tm, k, v, kt, vt, n, bits, counts, ts, sh);
    }

    template <class Team>
    __global__ void __launch_bounds__(256) k_scan(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *ts,
                                                  uint32_t *total)
    {
        __shared__ BlockShared sh;
        Team tm;
        const uint32_t t = team_excl_scan(tm, in, out, n, ts, sh);
        if (tm.leader())
            *total = t;
    }

    struct Bufs
    {
        std::vector<void *> p;
        ~Bufs()
        {
            for (void *x : p)
                cudaFree(x);
        }
        uint32_t *get(size_t words)
        {
            void *x = nullptr;
            if (cudaMalloc(&x, std::max<size_t>(words, 1) * 4) != cudaSuccess)
                return nullptr;
            cudaMemset(x, 0, std::max<size_t>(words, 1) * 4);
            p.push_back(x);
            return (uint32_t *)x;
        }
    };

    int launch(const void *fn, bool grid, int block, void **args, size_t n)
    {
        int g = 1;
        if (grid)
        {
            int dev = 0, sms = 0, occ = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, 0);
            g = (int)std::max<size_t>(1, std::min<size_t>((n + block - 1) / block, (size_t)occ * sms));
            if (cudaLaunchCooperativeKernel(fn, dim3(g), dim3(block), args, 0, 0) != cudaSuccess)
                return rbps_internal_fail(RBPS_ERR_CUDA, "selftest: cooperative launch failed");
        }
        else if (cudaLaunchKernel(fn, dim3(1), dim3(block), args, 0, 0) != cudaSuccess)
            return rbps_internal_fail(RBPS_ERR_CUDA, "selftest: launch failed");
        if (cudaDeviceSynchronize() != cudaSuccess)
            return rbps_internal_fail(RBPS_ERR_CUDA, "selftest: kernel failed");
        return RBPS_OK;
    }
} // namespace

// Stable radix sort of keys[0..n) by their low `bits` bits with values
// 0..n-1; grid != 0 runs it on a cooperative grid, else on one CTA.
extern "C" RBPS_API int rbps_selftest_sort(const uint32_t *keys, uint32_t n, int32_t bits, int32_t grid,
                                           int32_t block, uint32_t *keys_out, uint32_t *vals_out)
{
    if (block < 32 || block > 256 || block % 32 || bits < 1 || bits > 32)
        return rbps_internal_fail(RBPS_ERR_INVALID, "selftest_sort: bad block or bits");
    Bufs B;
    const size_t nt = (n + block - 1) / block + 1, counts = 256 * nt, ts = (counts + block - 1) / block + nt + 4;
    uint32_t *k = B.get(n), *v = B.get(n), *kt = B.get(n), *vt = B.get(n), *c = B.get(counts), *t = B.get(ts);
    if (!k || !v || !kt || !vt || !c || !t)
        return rbps_internal_fail(RBPS_ERR_CUDA, "selftest_sort: allocation failed");
    std::vector<uint32_t> iota(n);
    for (uint32_t i = 0; i < n; ++i)
        iota[i] = i;
    cudaMemcpy(k, keys, n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(v, iota.data(), n * 4, cudaMemcpyHostToDevice);
    void *args[] = {&k, &v, &kt, &vt, &n, &bits, &c, &t};
    const int rc = grid ? launch((const void *)k_sort<GridTeam>, true, block, args, n)
                        : launch((const void *)k_sort<BlockTeam>, false, block, args, n);
    if (rc)
        return rc;
    cudaMemcpy(keys_out, k, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(vals_out, v, n * 4, cudaMemcpyDeviceToHost);
    return RBPS_OK;
}

// Exclusive scan of in[0..n); *total receives the sum.
extern "C" RBPS_API int rbps_selftest_scan(const uint32_t *in, uint32_t n, int32_t grid, int32_t block,
                                           uint32_t *out, uint32_t *total)
{
    if (block < 32 || block > 256 || block % 32)
        return rbps_internal_fail(RBPS_ERR_INVALID, "selftest_scan: bad block");
    Bufs B;
    const size_t ts = (n + block - 1) / block + 4;
    uint32_t *di = B.get(n), *dout = B.get(n), *t = B.get(ts), *tot = B.get(1);
    if (!di || !dout || !t || !tot)
        return rbps_internal_fail(RBPS_ERR_CUDA, "selftest_scan: allocation failed");
    cudaMemcpy(di, in, n * 4, cudaMemcpyHostToDevice);
    void *args[] = {&di, &dout, &n, &t, &tot};
    const int rc = grid ? launch((const void *)k_scan<GridTeam>, true, block, args, n)
                        : launch((const void *)k_scan<BlockTeam>, false, block, args, n);
    if (rc)
        return rc;
    cudaMemcpy(out, dout, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(total, tot, 4, cudaMemcpyDeviceToHost);
    return RBPS_OK;
}
