// sap_static.cu - allocation-free SAP pair query.
//
// Some callers cannot allocate device memory once they are running: real-time
// control loops (cudaMalloc can block and synchronise the whole device),
// hosts that own a fixed device-memory budget and forbid allocations after
// start-up, and code that interleaves with other work on a stream and cannot
// afford an implicit synchronisation.  rbps_sap_pairs_static gives them the
// SAP sort + sweep with no allocation at all: the caller passes device
// buffers for the inputs and outputs, and the working memory is the
// file-scope array g_sap_scratch below, which every GPU that loads this
// library holds until the process exits.
//
// Limits: at most kStaticMaxObjects objects and kStaticMaxPairs pairs per
// call (the scratch is sized for exactly that).  Every call uses the same
// array, so calls whose kernels overlap on the GPU (different streams
// without ordering between them) race and corrupt each other; order them on
// one stream.  The array keeps the previous call's contents; the kernel
// rewrites everything it reads except the error word, which it clears first.
#include <mutex>

#include "engine_impl.cuh"
#include "rbps_gpu.h"

using namespace rbps_gpu;

int rbps_internal_fail(int code, const char *msg);

namespace
{
    constexpr uint32_t kStaticMaxObjects = 8192;
    constexpr uint32_t kStaticMaxPairs = 65536;
    constexpr uint32_t kStaticBlock = 256;
    // *n_pairs sentinels: more pairs than kStaticMaxPairs, and a failed
    // internal consistency check of the sort (endpoint ids or key order)
    constexpr uint32_t kStaticOverflow = 0xFFFFFFFFu;
    constexpr uint32_t kStaticCheckFailed = 0xFFFFFFFEu;
    constexpr uint32_t kNep = 2 * kStaticMaxObjects + 1;
    constexpr uint32_t kPc = kStaticMaxPairs + 1;
    constexpr uint32_t kTiles = ((kNep > kPc ? kNep : kPc) + kStaticBlock - 1) / kStaticBlock + 1;
    constexpr uint32_t kCounts = 256 * kTiles;
    constexpr uint32_t kTileSums = (kCounts + kStaticBlock - 1) / kStaticBlock + kTiles + 4;

    // word offsets inside the scratch array
    constexpr uint32_t oKey = 0;
    constexpr uint32_t oId = oKey + kNep;
    constexpr uint32_t oPos = oId + kNep;
    constexpr uint32_t oK2 = oPos + kNep;
    constexpr uint32_t oV2 = oK2 + kNep;
    constexpr uint32_t oCnt = oV2 + kNep;
    constexpr uint32_t oCounts = oCnt + kNep;
    constexpr uint32_t oTileSums = oCounts + kCounts;
    constexpr uint32_t oPrA = oTileSums + kTileSums;
    constexpr uint32_t oPrB = oPrA + kPc;
    constexpr uint32_t oPk = oPrB + kPc;
    constexpr uint32_t oPv = oPk + kPc;
    constexpr uint32_t oPk2 = oPv + kPc;
    constexpr uint32_t oPv2 = oPk2 + kPc;
    constexpr uint32_t oMisc = oPv2 + kPc;
    constexpr uint32_t oErr = oMisc + kMiscWords;
    constexpr uint32_t kScratchWords = oErr + 4;

    // The working memory of rbps_sap_pairs_static (about 2.3 MB per GPU).
    static __device__ __align__(256) uint32_t g_sap_scratch[kScratchWords];

    struct StaticScr
    {
        uint32_t *ep_k2, *ep_v2, *counts, *tile_sums, *cnt, *pr_a, *pr_b, *pk, *pv, *pk2, *pv2, *misc;
    };

    // fat: 6 doubles per object {min.x,min.y,min.z,max.x,max.y,max.z};
    // user_ids: 1 per object; pairs: (id_a, id_b) with id_a < id_b in the
    // reference emission order; *n_pairs = pairs found, kStaticOverflow when
    // they exceeded kStaticMaxPairs, kStaticCheckFailed when a consistency
    // check of the sort failed.
    __global__ void __launch_bounds__(kStaticBlock) k_sap_static(uint32_t *scratch, const double *fat_in,
                                                                 const uint32_t *user_ids, uint32_t n,
                                                                 uint32_t *pairs, uint32_t pair_cap,
                                                                 uint32_t *n_pairs)
    {
        __shared__ BlockShared sh;
        BlockTeam tm;
        int *err = (int *)(scratch + oErr);
        if (threadIdx.x == 0)
            *err = 0;
        uint32_t *key = scratch + oKey, *id = scratch + oId, *pos = scratch + oPos;
        // endpoints in insertion order (min, max per object), as a freshly
        // filled BroadPhaseState holds them (BroadPhase.cpp:30-46)
        const FatBox *fat = reinterpret_cast<const FatBox *>(fat_in);
        for (uint32_t o = threadIdx.x; o < n; o += blockDim.x)
        {
            const FatBox f = fat[o];
            key[2 * o] = order_key(__double2float_rn(f.mn[0]));
            key[2 * o + 1] = order_key(__double2float_rn(f.mx[0]));
            id[2 * o] = 2 * o;
            id[2 * o + 1] = 2 * o + 1;
        }
        __syncthreads();
        StaticScr S{scratch + oK2, scratch + oV2, scratch + oCounts, scratch + oTileSums, scratch + oCnt,
                    scratch + oPrA, scratch + oPrB, scratch + oPk, scratch + oPv, scratch + oPk2,
                    scratch + oPv2, scratch + oMisc};
        const uint32_t total = sap_sort_sweep(tm, fat, key, id, pos, n, 2 * n, kStaticMaxPairs, err, S, sh);
        // sap_sort_sweep ends with a block barrier, so every thread reads the
        // same error word here.  On any error the pairs buffer is left as it
        // was: the pairs kept before an overflow are neither a prefix of the
        // emission order nor complete.
        const int e = *err;
        if (e == 0)
            for (uint32_t k = threadIdx.x; k < total && k < pair_cap; k += blockDim.x)
            {
                const uint32_t r = S.pv[k];
                const uint32_t ua = user_ids[S.pr_a[r]], ub = user_ids[S.pr_b[r]];
                pairs[2 * k] = ua < ub ? ua : ub;
                pairs[2 * k + 1] = ua < ub ? ub : ua;
            }
        if (threadIdx.x == 0)
            *n_pairs = e == 0 ? total : e == RBPS_ERR_CAPACITY ? kStaticOverflow : kStaticCheckFailed;
    }

    // Device address of g_sap_scratch, looked up once per device.  A
    // cudaDeviceReset unloads the module, and the array may come back at
    // another address: the cached address is then stale, so the entry point
    // must not be called on a device after a reset of that device in the
    // same process.
    constexpr int kMaxDevices = 64;
    uint32_t *g_scratch_ptr[kMaxDevices] = {};
    std::mutex g_setup_mutex;

    int scratch_for_current_device(uint32_t **out)
    {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
            return rbps_internal_fail(RBPS_ERR_CUDA, "rbps_sap_pairs_static: no current CUDA device");
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev])
        {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_sap_scratch);
            if (e != cudaSuccess || !p)
                return rbps_internal_fail(RBPS_ERR_CUDA, "rbps_sap_pairs_static: cudaGetSymbolAddress failed");
            g_scratch_ptr[dev] = static_cast<uint32_t *>(p);
        }
        *out = g_scratch_ptr[dev];
        return RBPS_OK;
    }
} // namespace

extern "C" int rbps_sap_pairs_static(const double *fat_aabbs, const uint32_t *user_ids, uint32_t n_objects,
                                     uint32_t *pairs, uint32_t pair_cap, uint32_t *n_pairs, void *stream)
{
    if (n_objects > kStaticMaxObjects)
        return rbps_internal_fail(RBPS_ERR_INVALID,
                                  "rbps_sap_pairs_static: more than 8192 objects (the static scratch limit)");
    if ((n_objects && (!fat_aabbs || !user_ids)) || !n_pairs || (pair_cap && !pairs))
        return rbps_internal_fail(RBPS_ERR_INVALID, "rbps_sap_pairs_static: null buffer");
    uint32_t *scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc)
        return rc;
    k_sap_static<<<1, kStaticBlock, 0, (cudaStream_t)stream>>>(scratch, fat_aabbs, user_ids, n_objects, pairs,
                                                               pair_cap, n_pairs);
    if (cudaGetLastError() != cudaSuccess)
        return rbps_internal_fail(RBPS_ERR_CUDA, "rbps_sap_pairs_static: launch failed");
    return RBPS_OK;
}
