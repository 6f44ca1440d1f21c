// bp_api.cu - standalone GPU drop-in for the rbc SAP broadphase API
// (rbc/BroadPhase.hpp:151-260, BroadPhase.cpp:160-245).
//
// Object bookkeeping (insert / remove / move / move_swept, free-list slot
// reuse, endpoint append and removal) follows the reference on the host;
// rbps_bp_update uploads the SAP state and runs the device sort + sweep
// (sap_sort_sweep, shared with the batched engine), then reads back the
// pairs in the reference emission order and the new endpoint order.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "engine_impl.cuh"
#include "rbps_gpu.h"

using namespace rbps_gpu;

extern int rbps_internal_fail(int code, const char *msg);

namespace
{
    struct BpScr
    {
        uint32_t *ep_k2, *ep_v2, *counts, *tile_sums, *cnt, *pr_a, *pr_b, *pk, *pv, *pk2, *pv2, *misc;
    };

    template <class Team>
    __global__ void __launch_bounds__(256) k_bp_update(FatBox *fat, uint32_t *ep_key, uint32_t *ep_id,
                                                       uint32_t *ep_pos, uint32_t nbp, uint32_t id_limit,
                                                       uint32_t pair_cap, int *error, BpScr S)
    {
        __shared__ BlockShared sh;
        Team tm;
        const uint32_t n = sap_sort_sweep(tm, fat, ep_key, ep_id, ep_pos, nbp, id_limit, pair_cap, error, S, sh);
        if (tm.leader())
            S.misc[kMiscFlags + 5] = n;
    }

    uint32_t okey(float f)
    {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        if ((u & 0x7fffffffu) == 0u)
            u = 0u;
        return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    }

    thread_local std::string bp_err;
    int bfail(int code, const char *m)
    {
        bp_err = m;
        return rbps_internal_fail(code, m);
    }
} // namespace

struct rbps_bp
{
    double margin, threshold;
    struct Obj
    {
        double fat[6];
        double tight[6];
        uint32_t user_id;
        bool alive;
    };
    std::vector<Obj> objects;
    std::vector<uint32_t> free_list;
    std::vector<uint32_t> order;   // endpoint ids (slot*2 + is_max) in list order
    std::vector<float> value;      // float value per endpoint id
    std::vector<uint32_t> pairs;   // last update, (id_a, id_b) pairs
    bool dirty = false;
    // device
    size_t cap_obj = 0, cap_pairs = 0;
    FatBox *d_fat = nullptr;
    uint32_t *d_key = nullptr, *d_id = nullptr, *d_pos = nullptr;
    int *d_err = nullptr;
    std::vector<void *> scratch;
    BpScr S{};
    int occ = 0, sms = 0;
    int single_cta = 0;  // run sort + sweep on one CTA (small broadphases)
    int block = 256;

    void free_dev()
    {
        for (void *p : scratch)
            cudaFree(p);
        scratch.clear();
        cudaFree(d_fat);
        cudaFree(d_key);
        cudaFree(d_id);
        cudaFree(d_pos);
        cudaFree(d_err);
        d_fat = nullptr;
        d_key = d_id = d_pos = nullptr;
        d_err = nullptr;
        cap_obj = cap_pairs = 0;
    }
    ~rbps_bp() { free_dev(); }
};

static void set_fat(rbps_bp::Obj &o, const aabb &f)
{
    o.fat[0] = f.mn.x; o.fat[1] = f.mn.y; o.fat[2] = f.mn.z;
    o.fat[3] = f.mx.x; o.fat[4] = f.mx.y; o.fat[5] = f.mx.z;
}

static aabb from6(const double *a) { return {vec3<double>(a[0], a[1], a[2]), vec3<double>(a[3], a[4], a[5])}; }

extern "C" int rbps_bp_create(double fat_margin, double reinsert_threshold, rbps_bp **out)
{
    if (!out)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_create: null output");
    auto *bp = new rbps_bp();
    bp->margin = fat_margin;
    bp->threshold = reinsert_threshold;
    *out = bp;
    return RBPS_OK;
}

extern "C" int rbps_bp_destroy(rbps_bp *bp)
{
    delete bp;
    return RBPS_OK;
}

extern "C" int rbps_bp_insert(rbps_bp *bp, uint32_t user_id, const double a[6], uint32_t *handle)
{
    if (!bp || !a)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_insert: null argument");
    uint32_t slot;
    if (!bp->free_list.empty())
    {
        slot = bp->free_list.back();
        bp->free_list.pop_back();
    }
    else
    {
        slot = (uint32_t)bp->objects.size();
        bp->objects.emplace_back();
        bp->value.resize(2 * bp->objects.size());
    }
    rbps_bp::Obj &o = bp->objects[slot];
    std::memcpy(o.tight, a, sizeof(o.tight));
    set_fat(o, aabb_expand(from6(a), bp->margin));
    o.user_id = user_id;
    o.alive = true;
    bp->value[2 * slot] = (float)o.fat[0];
    bp->value[2 * slot + 1] = (float)o.fat[3];
    bp->order.push_back(2 * slot);
    bp->order.push_back(2 * slot + 1);
    bp->dirty = true;
    if (handle)
        *handle = slot;
    return RBPS_OK;
}

extern "C" int rbps_bp_remove(rbps_bp *bp, uint32_t h)
{
    if (!bp || h >= bp->objects.size() || !bp->objects[h].alive)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_remove: invalid handle");
    bp->objects[h].alive = false;
    bp->order.erase(std::remove_if(bp->order.begin(), bp->order.end(), [h](uint32_t id) { return (id >> 1) == h; }),
                    bp->order.end());
    bp->free_list.push_back(h);
    return RBPS_OK;
}

extern "C" int rbps_bp_move(rbps_bp *bp, uint32_t h, const double a[6])
{
    if (!bp || !a || h >= bp->objects.size() || !bp->objects[h].alive)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_move: invalid handle");
    rbps_bp::Obj &o = bp->objects[h];
    std::memcpy(o.tight, a, sizeof(o.tight));
    if (aabb_contained(from6(a), from6(o.fat)))
        return RBPS_OK;
    set_fat(o, aabb_expand(from6(a), bp->margin + bp->threshold));
    bp->value[2 * h] = (float)o.fat[0];
    bp->value[2 * h + 1] = (float)o.fat[3];
    bp->dirty = true;
    return RBPS_OK;
}

extern "C" int rbps_bp_move_swept(rbps_bp *bp, uint32_t h, const double a[6], const double v[3], double dt)
{
    if (!bp || !a || !v)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_move_swept: null argument");
    const double m = bp->margin;
    const vec3<double> dv = vec3<double>(v[0], v[1], v[2]) * dt;
    const vec3<double> emn(m + (dv.x < 0 ? -dv.x : 0.0), m + (dv.y < 0 ? -dv.y : 0.0), m + (dv.z < 0 ? -dv.z : 0.0));
    const vec3<double> emx(m + (dv.x > 0 ? dv.x : 0.0), m + (dv.y > 0 ? dv.y : 0.0), m + (dv.z > 0 ? dv.z : 0.0));
    const aabb t = from6(a);
    const vec3<double> mn = t.mn - emn, mx = t.mx + emx;
    const double s[6] = {mn.x, mn.y, mn.z, mx.x, mx.y, mx.z};
    return rbps_bp_move(bp, h, s);
}

static int bp_grow(rbps_bp *bp, size_t nobj, size_t npairs)
{
    if (nobj <= bp->cap_obj && npairs <= bp->cap_pairs)
        return RBPS_OK;
    const size_t co = std::max(nobj, std::max<size_t>(2 * bp->cap_obj, 64));
    const size_t cp = std::max(npairs, std::max<size_t>(2 * bp->cap_pairs, 1024));
    bp->free_dev();
    const size_t nep = 2 * co + 1, B = (size_t)bp->block;
    const size_t nt = std::max((nep + B - 1) / B, (cp + B - 1) / B) + 1;
    const size_t counts = 256 * nt, tsums = std::max((counts + B - 1) / B, nt) + 4;
    auto al = [&](void **p, size_t bytes) -> int {
        if (cudaMalloc(p, bytes) != cudaSuccess)
            return bfail(RBPS_ERR_CUDA, "rbps_bp: device allocation failed");
        cudaMemset(*p, 0, bytes);
        return RBPS_OK;
    };
    int rc;
    if ((rc = al((void **)&bp->d_fat, co * sizeof(FatBox))) || (rc = al((void **)&bp->d_key, nep * 4)) ||
        (rc = al((void **)&bp->d_id, nep * 4)) || (rc = al((void **)&bp->d_pos, nep * 4)) ||
        (rc = al((void **)&bp->d_err, 64)))
        return rc;
    uint32_t **fields[] = {&bp->S.ep_k2, &bp->S.ep_v2, &bp->S.counts, &bp->S.tile_sums, &bp->S.cnt, &bp->S.pr_a,
                           &bp->S.pr_b, &bp->S.pk, &bp->S.pv, &bp->S.pk2, &bp->S.pv2, &bp->S.misc};
    const size_t sizes[] = {nep, nep, counts, tsums, nep, cp, cp, cp, cp, cp, cp, (size_t)kMiscWords};
    for (int i = 0; i < 12; ++i)
    {
        void *p;
        if ((rc = al(&p, sizes[i] * 4)))
            return rc;
        bp->scratch.push_back(p);
        *fields[i] = (uint32_t *)p;
    }
    bp->cap_obj = co;
    bp->cap_pairs = cp;
    return RBPS_OK;
}

extern "C" int rbps_bp_update(rbps_bp *bp)
{
    if (!bp)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_update: null state");
    bp->pairs.clear();
    const uint32_t nep = (uint32_t)bp->order.size(), nbp = nep / 2;
    bp->dirty = false;
    if (nep == 0)
        return RBPS_OK;
    if (!bp->sms)
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&bp->sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bp->occ, k_bp_update<GridTeam>, 256, 0);
        if (bp->occ < 1)
            return bfail(RBPS_ERR_CUDA, "rbps_bp_update: kernel cannot be resident");
    }
    size_t want_pairs = std::max<size_t>(1024, 8 * (size_t)nbp);
    for (int attempt = 0; attempt < 2; ++attempt)
    {
        int rc = bp_grow(bp, bp->objects.size(), want_pairs);
        if (rc)
            return rc;
        const size_t no = bp->objects.size();
        std::vector<FatBox> fat(no);
        for (size_t i = 0; i < no; ++i)
        {
            std::memcpy(fat[i].mn, bp->objects[i].fat, 3 * sizeof(double));
            std::memcpy(fat[i].mx, bp->objects[i].fat + 3, 3 * sizeof(double));
        }
        std::vector<uint32_t> keys(nep);
        for (uint32_t i = 0; i < nep; ++i)
            keys[i] = okey(bp->value[bp->order[i]]);
        if (cudaMemcpy(bp->d_fat, fat.data(), no * sizeof(FatBox), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(bp->d_key, keys.data(), nep * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(bp->d_id, bp->order.data(), nep * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(bp->d_err, 0, 4) != cudaSuccess)
            return bfail(RBPS_ERR_CUDA, "rbps_bp_update: upload failed");
        const int grid = (int)std::max<size_t>(1, std::min<size_t>((nep + 1023) / 1024, (size_t)bp->occ * bp->sms));
        uint32_t cap = (uint32_t)bp->cap_pairs;
        uint32_t id_limit = (uint32_t)(2 * no);
        void *args[] = {&bp->d_fat, &bp->d_key, &bp->d_id, &bp->d_pos, (void *)&nbp, &id_limit, &cap, &bp->d_err,
                        &bp->S};
        cudaError_t e = bp->single_cta
                            ? cudaLaunchKernel((const void *)k_bp_update<BlockTeam>, dim3(1), dim3(bp->block), args, 0, 0)
                            : cudaLaunchCooperativeKernel((const void *)k_bp_update<GridTeam>, dim3(grid), dim3(256),
                                                          args, 0, 0);
        if (e != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
            return bfail(RBPS_ERR_CUDA, "rbps_bp_update: kernel failed");
        uint32_t misc[8];
        int err = 0;
        cudaMemcpy(misc, bp->S.misc, sizeof(misc), cudaMemcpyDeviceToHost);
        cudaMemcpy(&err, bp->d_err, 4, cudaMemcpyDeviceToHost);
        // the endpoint order is now sorted (the sort is stable and idempotent)
        cudaMemcpy(bp->order.data(), bp->d_id, nep * 4, cudaMemcpyDeviceToHost);
        if (err == RBPS_ERR_CAPACITY && attempt == 0)
        {
            want_pairs = misc[kMiscFlags + 4];
            continue;
        }
        if (err)
            return bfail(err, "rbps_bp_update: device error");
        const uint32_t n = misc[kMiscFlags + 5];
        std::vector<uint32_t> pv(n), pa(n), pb(n);
        cudaMemcpy(pv.data(), bp->S.pv, n * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(pa.data(), bp->S.pr_a, n * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(pb.data(), bp->S.pr_b, n * 4, cudaMemcpyDeviceToHost);
        bp->pairs.resize(2 * (size_t)n);
        for (uint32_t k = 0; k < n; ++k)
        {
            const uint32_t ua = bp->objects[pa[pv[k]]].user_id, ub = bp->objects[pb[pv[k]]].user_id;
            bp->pairs[2 * k] = ua < ub ? ua : ub;
            bp->pairs[2 * k + 1] = ua < ub ? ub : ua;
        }
        return RBPS_OK;
    }
    return bfail(RBPS_ERR_CAPACITY, "rbps_bp_update: pair capacity");
}

extern "C" int rbps_bp_get_pairs(rbps_bp *bp, uint32_t *pairs, uint32_t cap, uint32_t *n_out)
{
    if (!bp)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_get_pairs: null state");
    const uint32_t n = (uint32_t)(bp->pairs.size() / 2);
    if (n_out)
        *n_out = n;
    if (pairs)
        std::memcpy(pairs, bp->pairs.data(), std::min(n, cap) * 2 * sizeof(uint32_t));
    return RBPS_OK;
}

extern "C" int rbps_bp_get_fat_aabb(rbps_bp *bp, uint32_t h, double a[6])
{
    if (!bp || h >= bp->objects.size() || !a)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_get_fat_aabb: invalid handle");
    std::memcpy(a, bp->objects[h].fat, 6 * sizeof(double));
    return RBPS_OK;
}

extern "C" int rbps_bp_configure(rbps_bp *bp, int32_t single_cta, int32_t block_threads)
{
    if (!bp || block_threads < 32 || block_threads > 256 || block_threads % 32)
        return bfail(RBPS_ERR_INVALID, "rbps_bp_configure: block_threads must be 32..256, a multiple of 32");
    bp->single_cta = single_cta != 0;
    if (bp->block != block_threads)
    {
        bp->free_dev();
        bp->block = block_threads;
    }
    return RBPS_OK;
}
