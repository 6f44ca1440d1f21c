// team.cuh - cooperative primitives over a "team" of CTAs.
//
// A world is stepped by one team.  Small worlds of a batch use a team of one
// CTA (BlockTeam, barrier = __syncthreads) and many worlds run concurrently
// on the GPU; a large single world uses a team spanning the whole
// cooperative grid (GridTeam, barrier = grid sync).  Every phase of the step
// is written once against this interface.
//
// Primitives: flat loops (team rank / size), tile loops (cta / ncta), an
// exclusive scan and a stable LSD radix sort of (u32 key, u32 value) over
// global-memory arrays.  Tiles are blockDim.x items; every thread of a CTA
// runs every tile iteration of its CTA, so block barriers inside tile loops
// are uniform.  The primitives are compiled as separate (non-inlined)
// functions so their code does not depend on the kernel that calls them.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>

namespace rbps_gpu
{
    namespace cg = cooperative_groups;

    struct BlockTeam
    {
        __device__ __forceinline__ uint32_t cta() const { return 0; }
        __device__ __forceinline__ uint32_t ncta() const { return 1; }
        __device__ __forceinline__ uint32_t rank() const { return threadIdx.x; }
        __device__ __forceinline__ uint32_t size() const { return blockDim.x; }
        __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }
        __device__ __forceinline__ void sync() const { __syncthreads(); }
    };

    struct GridTeam
    {
        __device__ __forceinline__ uint32_t cta() const { return blockIdx.x; }
        __device__ __forceinline__ uint32_t ncta() const { return gridDim.x; }
        __device__ __forceinline__ uint32_t rank() const { return blockIdx.x * blockDim.x + threadIdx.x; }
        __device__ __forceinline__ uint32_t size() const { return gridDim.x * blockDim.x; }
        __device__ __forceinline__ bool leader() const { return blockIdx.x == 0 && threadIdx.x == 0; }
        __device__ __forceinline__ void sync() const { cg::this_grid().sync(); }
    };

    // One warp of a CTA as a team (barrier = __syncwarp); the phases that
    // need only flat loops and barriers run unchanged on it.
    struct WarpTeam
    {
        __device__ __forceinline__ uint32_t cta() const { return 0; }
        __device__ __forceinline__ uint32_t ncta() const { return 1; }
        __device__ __forceinline__ uint32_t rank() const { return threadIdx.x & 31u; }
        __device__ __forceinline__ uint32_t size() const { return 32; }
        __device__ __forceinline__ bool leader() const { return (threadIdx.x & 31u) == 0; }
        __device__ __forceinline__ void sync() const { __syncwarp(); }
    };

    // Two warps of a 128-thread CTA as a team: threads [64 h, 64 h + 64) for
    // half h, barrier = the named barrier 1 + h over its 64 threads (0 is
    // __syncthreads', which the halves do not use).
    struct PairTeam
    {
        __device__ __forceinline__ uint32_t cta() const { return 0; }
        __device__ __forceinline__ uint32_t ncta() const { return 1; }
        __device__ __forceinline__ uint32_t rank() const { return threadIdx.x & 63u; }
        __device__ __forceinline__ uint32_t size() const { return 64; }
        __device__ __forceinline__ bool leader() const { return (threadIdx.x & 63u) == 0; }
        __device__ __forceinline__ uint32_t half() const { return threadIdx.x >> 6; }
        __device__ __forceinline__ void sync() const
        {
            asm volatile("bar.sync %0, 64;" ::"r"(1 + (threadIdx.x >> 6)) : "memory");
        }
    };

    constexpr int kMaxWarps = 32;

    // Shared scratch of the block primitives (one per CTA).
    // Shared scratch of a block scan (all a kernel needs that only scans).
    struct ScanShared
    {
        uint32_t warp[kMaxWarps];
        uint32_t bcast[4];
    };

    // Shared scratch of the block scans and the radix sort's ranking passes.
    struct BlockShared : ScanShared
    {
        uint32_t hist[256];
        uint32_t wdig[8 * 256]; // per-warp digit counts, <= 8 warps per tile rank pass
    };

    __device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
    __device__ __forceinline__ uint32_t warp_id() { return threadIdx.x >> 5; }

    __device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
    {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
            if (lane_id() >= (uint32_t)o)
                v += n;
        }
        return v;
    }

    // Exclusive block scan of one value per thread; *total gets the sum.
    // Contains two __syncthreads; every thread of the block must call it.
    __device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, ScanShared &sh, uint32_t *total)
    {
        const uint32_t inc = warp_incl_scan(v);
        const uint32_t nw = (blockDim.x + 31) >> 5;
        if (lane_id() == 31)
            sh.warp[warp_id()] = inc;
        __syncthreads();
        if (warp_id() == 0)
        {
            const uint32_t x = lane_id() < nw ? sh.warp[lane_id()] : 0u;
            const uint32_t xi = warp_incl_scan(x);
            if (lane_id() < nw)
                sh.warp[lane_id()] = xi - x;
            if (lane_id() == 31)
                sh.bcast[0] = xi;
        }
        __syncthreads();
        const uint32_t res = sh.warp[warp_id()] + inc - v;
        *total = sh.bcast[0];
        __syncthreads();
        return res;
    }

    // Exclusive scan of in[0..n) into out (may alias in) by the team.
    // tile_sums needs ceil(n / blockDim.x) + 1 words of global scratch.
    // Returns the total to every thread.  Ends with a team barrier.
    template <class Team>
    __device__ __noinline__ uint32_t team_excl_scan(const Team &tm, const uint32_t *in, uint32_t *out, uint32_t n,
                                       uint32_t *tile_sums, BlockShared &sh)
    {
        const uint32_t B = blockDim.x;
        const uint32_t ntiles = (n + B - 1) / B;
        for (uint32_t t = tm.cta(); t < ntiles; t += tm.ncta())
        {
            const uint32_t i = t * B + threadIdx.x;
            uint32_t tot;
            block_excl_scan(i < n ? in[i] : 0u, sh, &tot);
            if (threadIdx.x == 0)
                tile_sums[t] = tot;
        }
        tm.sync();
        if (tm.cta() == 0)
        {
            uint32_t carry = 0;
            for (uint32_t base = 0; base < ntiles; base += B)
            {
                const uint32_t i = base + threadIdx.x;
                const uint32_t v = i < ntiles ? tile_sums[i] : 0u;
                uint32_t tot;
                const uint32_t ex = block_excl_scan(v, sh, &tot);
                if (i < ntiles)
                    tile_sums[i] = ex + carry;
                carry += tot;
            }
            if (threadIdx.x == 0)
                tile_sums[ntiles] = carry;
        }
        tm.sync();
        for (uint32_t t = tm.cta(); t < ntiles; t += tm.ncta())
        {
            const uint32_t i = t * B + threadIdx.x;
            const uint32_t v = i < n ? in[i] : 0u;
            uint32_t tot;
            const uint32_t ex = block_excl_scan(v, sh, &tot);
            if (i < n)
                out[i] = ex + tile_sums[t];
        }
        const uint32_t total = ntiles ? tile_sums[ntiles] : 0u;
        tm.sync();
        return total;
    }

    // One stable counting pass on 8-bit digit `shift` of keys: (k0,v0) -> (k1,v1).
    // counts needs 256 * ntiles words, tile_sums ntiles*256/B + 2 words.
    template <class Team>
    __device__ __noinline__ void radix_pass(const Team &tm, const uint32_t *k0, const uint32_t *v0, uint32_t *k1, uint32_t *v1,
                               uint32_t n, int shift, uint32_t *counts, uint32_t *tile_sums, BlockShared &sh)
    {
        const uint32_t B = blockDim.x;
        const uint32_t ntiles = (n + B - 1) / B;
        // A: digit histogram per tile, digit-major layout counts[d * ntiles + t]
        for (uint32_t t = tm.cta(); t < ntiles; t += tm.ncta())
        {
            for (uint32_t d = threadIdx.x; d < 256; d += B)
                sh.hist[d] = 0;
            __syncthreads();
            const uint32_t i = t * B + threadIdx.x;
            if (i < n)
                atomicAdd(&sh.hist[(k0[i] >> shift) & 255u], 1u);
            __syncthreads();
            for (uint32_t d = threadIdx.x; d < 256; d += B)
                counts[d * ntiles + t] = sh.hist[d];
            __syncthreads();
        }
        tm.sync();
        team_excl_scan(tm, counts, counts, 256 * ntiles, tile_sums, sh);
        // B: stable scatter; rank inside the tile from warp match masks
        const uint32_t nw = (B + 31) >> 5;
        for (uint32_t t = tm.cta(); t < ntiles; t += tm.ncta())
        {
            for (uint32_t x = threadIdx.x; x < nw * 256; x += B)
                sh.wdig[x] = 0;
            __syncthreads();
            const uint32_t i = t * B + threadIdx.x;
            const bool live = i < n;
            const uint32_t key = live ? k0[i] : 0u;
            const uint32_t d = live ? ((key >> shift) & 255u) : 256u;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            const uint32_t lt = (1u << lane_id()) - 1u;
            const uint32_t lane_rank = __popc(peers & lt);
            if (live && lane_rank == 0)
                sh.wdig[warp_id() * 256 + d] = __popc(peers);
            __syncthreads();
            // exclusive prefix over warps, per digit
            for (uint32_t dd = threadIdx.x; dd < 256; dd += B)
            {
                uint32_t run = 0;
                for (uint32_t w = 0; w < nw; ++w)
                {
                    const uint32_t c = sh.wdig[w * 256 + dd];
                    sh.wdig[w * 256 + dd] = run;
                    run += c;
                }
            }
            __syncthreads();
            if (live)
            {
                const uint32_t dst = counts[d * ntiles + t] + sh.wdig[warp_id() * 256 + d] + lane_rank;
                if (dst < n) // a corrupted count must never write outside the buffer
                {
                    k1[dst] = key;
                    v1[dst] = v0[i];
                }
            }
            __syncthreads();
        }
        tm.sync();
    }

    // Stable sort of (keys, vals)[0..n) by the low `bits` bits of the key.
    // The result is left in (keys, vals); (kt, vt) are ping-pong buffers.
    template <class Team>
    __device__ __noinline__ void team_radix_sort(const Team &tm, uint32_t *keys, uint32_t *vals, uint32_t *kt, uint32_t *vt,
                                    uint32_t n, int bits, uint32_t *counts, uint32_t *tile_sums, BlockShared &sh)
    {
        if (n <= 1)
            return;
        const int passes = (bits + 7) / 8;
        uint32_t *a_k = keys, *a_v = vals, *b_k = kt, *b_v = vt;
        for (int p = 0; p < passes; ++p)
        {
            radix_pass(tm, a_k, a_v, b_k, b_v, n, 8 * p, counts, tile_sums, sh);
            uint32_t *tk = a_k, *tv = a_v;
            a_k = b_k; a_v = b_v; b_k = tk; b_v = tv;
        }
        if (a_k != keys)
        {
            for (uint32_t i = tm.rank(); i < n; i += tm.size())
            {
                keys[i] = a_k[i];
                vals[i] = a_v[i];
            }
            tm.sync();
        }
    }
    // A sort staged in shared memory: a CTA team with `smem` (kSmemSortWords
    // words) and at least 128 threads copies up to kSmemSortMax (key, value)
    // pairs in, runs the same stable radix sort on the shared copies and
    // copies the result back -- the same permutation as sorting in place,
    // without a global-memory round trip per pass step.  Other teams and
    // larger inputs sort in place.
    constexpr uint32_t kSmemSortMax = 1536;
    constexpr uint32_t kSmemSortCounts = 256 * (kSmemSortMax / 128);
    constexpr uint32_t kSmemSortWords = 4 * kSmemSortMax + kSmemSortCounts + 64;

    template <class Team>
    __device__ __forceinline__ void team_sort_staged(const Team &tm, uint32_t *keys, uint32_t *vals, uint32_t *kt,
                                                     uint32_t *vt, uint32_t n, int bits, uint32_t *counts,
                                                     uint32_t *tile_sums, BlockShared &sh, uint32_t *)
    {
        team_radix_sort(tm, keys, vals, kt, vt, n, bits, counts, tile_sums, sh);
    }

    __device__ __forceinline__ void team_sort_staged(const BlockTeam &tm, uint32_t *keys, uint32_t *vals, uint32_t *kt,
                                                     uint32_t *vt, uint32_t n, int bits, uint32_t *counts,
                                                     uint32_t *tile_sums, BlockShared &sh, uint32_t *smem)
    {
        if (!smem || n > kSmemSortMax || blockDim.x < 128 || n <= 1)
        {
            team_radix_sort(tm, keys, vals, kt, vt, n, bits, counts, tile_sums, sh);
            return;
        }
        uint32_t *ak = smem, *av = smem + kSmemSortMax;
        uint32_t *bk = smem + 2 * kSmemSortMax, *bv = smem + 3 * kSmemSortMax;
        uint32_t *sc = smem + 4 * kSmemSortMax, *st = sc + kSmemSortCounts;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        {
            ak[i] = keys[i];
            av[i] = vals[i];
        }
        __syncthreads();
        team_radix_sort(tm, ak, av, bk, bv, n, bits, sc, st, sh);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        {
            keys[i] = ak[i];
            vals[i] = av[i];
        }
        __syncthreads();
    }
} // namespace rbps_gpu
