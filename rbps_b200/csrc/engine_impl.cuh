// engine_impl.cuh - one world step (World::step, World.hpp:192-212) executed
// by a team of CTAs, and the kernels that run it over a batch.
//
// Frame (once per step):
//   1. SAP object update: tight AABB, velocity sweep, fat-AABB escape test,
//      endpoint key refresh        (CollisionPipeline.cpp:14-53,
//                                   BroadPhase.hpp:228-249, BroadPhase.cpp:211-232)
//   2. stable radix sort of the endpoints by their float key, seeded with
//      the previous frame's order (== the reference's insertion sort,
//      BroadPhase.cpp:80-94)
//   3. sweep: for every opening endpoint, the objects whose interval is
//      open there, 3-D fat-AABB test; pairs ordered by (opening position of
//      the later object, opening position of the earlier one), which is the
//      order bp_sweep emits them (BroadPhase.cpp:104-152)
//   4. narrowphase candidates: filtered SAP pairs, then the static
//      plane-vs-collider list (CollisionPipeline.cpp:110-198)
//   5. colored mode only: Jones-Plassmann colouring of the candidates by
//      shared dynamic bodies
// Substeps (World.hpp:203-211): narrowphase + contact emission, integrate,
// position solve (contacts, joint errors, joint rows), velocity update,
// velocity solve (contacts, joint damping).
#pragma once
#include "engine_types.cuh"
#include "gjk.cuh"
#include "team.cuh"
#include <type_traits>

namespace rbps_gpu
{
    __device__ __forceinline__ uint32_t order_key(float f)
    {
        uint32_t u = __float_as_uint(f);
        if ((u & 0x7fffffffu) == 0u)
            u = 0u; // -0.0f and +0.0f compare equal in the reference's sort
        return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    }

    constexpr int kErrInternal = -6;
    constexpr int kErrState = -5; // RBPS_ERR_STATE

    __device__ __forceinline__ void set_error(int *err, int code)
    {
        atomicCAS(err, 0, code);
    }

    // First failing consistency check: err[0] = code, err[1] = site,
    // err[2] = offending value (the host reports them in the error message).
    __device__ __forceinline__ void set_error_at(int *err, int code, int site, uint32_t value)
    {
        if (atomicCAS(err, 0, code) == 0)
        {
            err[1] = site;
            err[2] = (int)value;
        }
    }

    __device__ __forceinline__ uint32_t hash32(uint32_t x)
    {
        x ^= x >> 16;
        x *= 0x7feb352dU;
        x ^= x >> 15;
        x *= 0x846ca68bU;
        x ^= x >> 16;
        return x;
    }

    template <class T, class P>
    struct Scr
    {
        uint32_t *ep_k2, *ep_v2, *counts, *tile_sums, *cnt, *pr_a, *pr_b, *pk, *pv, *pk2, *pv2, *cflag;
        Cand *cand;
        CandContacts<T, P> *cc;
        uint32_t *color;
        unsigned long long *bmask, *bprio, *claim;
        uint32_t *corder, *misc, *act, *alist;
        float4 *yz;
    };

    template <class T, class P>
    __device__ __forceinline__ Scr<T, P> scratch_ptrs(char *base, const ScratchLayout &L)
    {
        Scr<T, P> s;
        s.ep_k2 = (uint32_t *)(base + L.ep_k2);
        s.ep_v2 = (uint32_t *)(base + L.ep_v2);
        s.counts = (uint32_t *)(base + L.counts);
        s.tile_sums = (uint32_t *)(base + L.tile_sums);
        s.cnt = (uint32_t *)(base + L.cnt);
        s.pr_a = (uint32_t *)(base + L.pr_a);
        s.pr_b = (uint32_t *)(base + L.pr_b);
        s.pk = (uint32_t *)(base + L.pk);
        s.pv = (uint32_t *)(base + L.pv);
        s.pk2 = (uint32_t *)(base + L.pk2);
        s.pv2 = (uint32_t *)(base + L.pv2);
        s.cflag = (uint32_t *)(base + L.cflag);
        s.cand = (Cand *)(base + L.cand);
        s.cc = (CandContacts<T, P> *)(base + L.cc);
        s.color = (uint32_t *)(base + L.color);
        s.bmask = (unsigned long long *)(base + L.bmask);
        s.bprio = (unsigned long long *)(base + L.bprio);
        s.claim = (unsigned long long *)(base + L.claim);
        s.yz = (float4 *)(base + L.yz);
        s.corder = (uint32_t *)(base + L.corder);
        s.misc = (uint32_t *)(base + L.misc);
        s.act = (uint32_t *)(base + L.act);
        s.alist = (uint32_t *)(base + L.alist);
        return s;
    }

    // collider_world_tf (Collider.hpp:73-80) in the solver scalar
    template <class T, class P>
    __device__ __forceinline__ tf<T> collider_tf(const Engine<T, P> &E, uint32_t gc, uint32_t gb)
    {
        const vec3<T> bp = E.B.x(gb);
        const quat<T> br = E.B.q(gb);
        const V4<double> lp = E.c_lpos[gc];
        const Q4<double> lr = E.c_lrot[gc];
        tf<T> t;
        t.pos = bp + rotate(br, vec3<T>(T(lp.x), T(lp.y), T(lp.z)));
        t.rot = br * quat<T>(T(lr.w), T(lr.x), T(lr.y), T(lr.z));
        return t;
    }

    // Radius of a sphere about the collider's origin that holds the shape;
    // 0 for the unbounded or table-driven kinds (plane, heightmap, mesh).
    template <class T>
    __device__ __forceinline__ T shape_bound(const ShapeDev &s, const HullSetDev &hs)
    {
        const T a = T(s.p[0]), b = T(s.p[1]), c = T(s.p[2]);
        switch (s.kind)
        {
        case kSphere: return a;
        case kBox: return sqrt(a * a + b * b + c * c);
        case kCapsule: return a + b;
        case kEllipsoid: return rmax(a, rmax(b, c));
        case kCylinder:
        case kCone: return sqrt(a * a + b * b);
        case kHull:
        {
            const double *la = hs.local_aabb + 6 * s.hull;
            const T x = rmax(rabs(T(la[0])), rabs(T(la[3]))), y = rmax(rabs(T(la[1])), rabs(T(la[4])));
            const T z = rmax(rabs(T(la[2])), rabs(T(la[5])));
            return sqrt(x * x + y * y + z * z);
        }
        default: return T(0);
        }
    }

    // True when the two shapes are certainly apart: their bounding spheres
    // (or a bounding sphere and a plane) are separated by more than
    // kBoundMargin, far beyond any contact tolerance of the narrowphase
    // (the largest is the 1e-4 of the box-plane corner test), so GJK would
    // report no contact.  The test only skips work: the contact rows are the
    // same (none), bit for bit.
    constexpr double kBoundMargin = 1e-2;

    template <class T>
    __device__ __forceinline__ bool bounds_separate(const ShapeDev &sa, const tf<T> &ta, const ShapeDev &sb,
                                                    const tf<T> &tb, const HullSetDev &hs)
    {
        if (sa.kind == kPlane || sb.kind == kPlane)
        {
            const bool a_plane = sa.kind == kPlane;
            const ShapeDev &pl = a_plane ? sa : sb;
            const ShapeDev &ot = a_plane ? sb : sa;
            const tf<T> &tp = a_plane ? ta : tb;
            const tf<T> &to = a_plane ? tb : ta;
            const T r = shape_bound<T>(ot, hs);
            if (!(r > T(0)))
                return false;
            const vec3<T> n = rotate(tp.rot, vec3<T>(T(pl.p[0]), T(pl.p[1]), T(pl.p[2])));
            const T len = length(n);
            if (!(len > T(0.5)))
                return false;
            const T dist = dot(n, to.pos - tp.pos) / len - T(pl.p[3]);
            return dist > r + T(kBoundMargin);
        }
        const T ra = shape_bound<T>(sa, hs), rb = shape_bound<T>(sb, hs);
        if (!(ra > T(0)) || !(rb > T(0)))
            return false;
        const T reach = ra + rb + T(kBoundMargin);
        return length_sq(ta.pos - tb.pos) > reach * reach;
    }

    template <class T, class P>
    __device__ __forceinline__ tf<double> collider_tf_d(const Engine<T, P> &E, uint32_t gc, uint32_t gb)
    {
        const V4<P> bpv = E.B.pos[gb];
        const Q4<T> brv = E.B.rot[gb];
        const vec3<double> bp(double(bpv.x), double(bpv.y), double(bpv.z));
        const quat<double> br(double(brv.w), double(brv.x), double(brv.y), double(brv.z));
        const V4<double> lp = E.c_lpos[gc];
        const Q4<double> lr = E.c_lrot[gc];
        tf<double> t;
        t.pos = bp + rotate(br, vec3<double>(lp.x, lp.y, lp.z));
        t.rot = br * quat<double>(lr.w, lr.x, lr.y, lr.z);
        return t;
    }

    __device__ __forceinline__ aabb load_fat(const FatBox &f)
    {
        return {vec3<double>(f.mn[0], f.mn[1], f.mn[2]), vec3<double>(f.mx[0], f.mx[1], f.mx[2])};
    }

    __device__ __forceinline__ bool fat_overlap(const FatBox &a, const FatBox &b)
    {
        return (a.mn[0] <= b.mx[0] && a.mx[0] >= b.mn[0]) &&
               (a.mn[1] <= b.mx[1] && a.mx[1] >= b.mn[1]) &&
               (a.mn[2] <= b.mx[2] && a.mx[2] >= b.mn[2]);
    }

    // The y / z part of fat_overlap on float copies rounded outward
    // (mn down, mx up): false only where fat_overlap is false too.
    __device__ __forceinline__ bool yz_may_overlap(const float4 &a, const float4 &b)
    {
        return a.x <= b.y && a.y >= b.x && a.z <= b.w && a.w >= b.z;
    }

    // ------------------------------------------------------------ broadphase
    // Sub-phase timer of the broadphase: the CTA's thread 0 adds the cycles
    // since t to slot s of prof (null when profiling is off) and restarts t.
    __device__ __forceinline__ void sub_mark(unsigned long long *prof, int s, long long &t)
    {
        if (prof && threadIdx.x == 0)
        {
            const long long now = clock64();
            prof[s] += (unsigned long long)(now - t);
            t = now;
        }
    }

    // One-CTA fast path of the endpoint sort, in the staging area `smem`
    // (kSmemSortWords words).  moved[i] (shared) flags the previous
    // positions whose keys the frame's object update rewrote.  When the
    // other endpoints (R) are still in key order, the stable sort of the
    // whole array -- keys ordered, equal keys in previous order -- is the
    // merge of R with the moved endpoints (M) by (key, previous position):
    // R is sorted that way already, M is ranked by counting, and each
    // endpoint's final position is its rank in its own list plus the count
    // of the other list's endpoints before it (a binary search).  ep_key,
    // ep_id and ep_pos are then written once.  Returns false with nothing
    // written when M exceeds kMergeMax or R is out of order (the first frame
    // after a commit, whose endpoints are in insertion order, and any array
    // that is not the last sort's output); the caller then sorts in full.
    // Every thread of the CTA must call it; it ends with a block barrier.
    constexpr uint32_t kMergeMax = 512;
    static_assert(3 * kSmemSortMax + 6 * kMergeMax <= kSmemSortWords, "the merge's lists fit the staging area");

    static __device__ __noinline__ bool merge_moved_endpoints(uint32_t *ep_key, uint32_t *ep_id, uint32_t *ep_pos, uint32_t nep,
                                                       uint32_t id_limit, const uint32_t *moved, uint32_t *smem,
                                                       ScanShared &sh, int *error)
    {
        uint32_t *rk = smem, *rp = smem + kSmemSortMax, *rid = smem + 2 * kSmemSortMax;
        uint32_t *mk = smem + 3 * kSmemSortMax, *mp = mk + kMergeMax, *mid = mp + kMergeMax;
        uint32_t *smk = mid + kMergeMax, *smp = smk + kMergeMax, *mfin = smp + kMergeMax;
        const uint32_t B = blockDim.x, t = threadIdx.x;
        // each thread a contiguous run of positions, so M and R keep order
        const uint32_t per = (nep + B - 1) / B;
        const uint32_t i0 = min(nep, t * per), i1 = min(nep, i0 + per);
        uint32_t mine = 0;
        for (uint32_t i = i0; i < i1; ++i)
            mine += moved[i] ? 1u : 0u;
        if (t == 0)
            sh.bcast[2] = 0u; // R out of order (published by the scan's barriers)
        uint32_t m;
        uint32_t mi = block_excl_scan(mine, sh, &m);
        if (m > kMergeMax)
            return false;
        for (uint32_t i = i0; i < i1; ++i)
        {
            const uint32_t key = ep_key[i], id = ep_id[i];
            if (moved[i])
            {
                mk[mi] = key;
                mp[mi] = i;
                mid[mi] = id;
                ++mi;
            }
            else
            {
                const uint32_t r = i - mi;
                rk[r] = key;
                rp[r] = i;
                rid[r] = id;
            }
        }
        __syncthreads();
        const uint32_t nr = nep - m;
        for (uint32_t r = t; r + 1 < nr; r += B)
            if (rk[r] > rk[r + 1])
                sh.bcast[2] = 1u;
        for (uint32_t u = t; u < m; u += B)
        {
            const uint32_t k = mk[u], p = mp[u];
            uint32_t rank = 0;
            for (uint32_t v = 0; v < m; ++v)
                rank += (mk[v] < k || (mk[v] == k && v < u)) ? 1u : 0u; // v < u <=> mp[v] < p
            uint32_t lo = 0, hi = nr;
            while (lo < hi)
            {
                const uint32_t h = (lo + hi) >> 1;
                if (rk[h] < k || (rk[h] == k && rp[h] < p))
                    lo = h + 1;
                else
                    hi = h;
            }
            smk[rank] = k;
            smp[rank] = p;
            mfin[u] = rank + lo;
        }
        __syncthreads();
        const bool bad = sh.bcast[2] != 0u;
        __syncthreads(); // everyone has read the flag before the caller reuses sh
        if (bad)
            return false;
        if (m == 0)
            return true; // nothing moved and the order holds: the arrays stand
        for (uint32_t r = t; r < nr; r += B)
        {
            const uint32_t k = rk[r], p = rp[r];
            uint32_t lo = 0, hi = m;
            while (lo < hi)
            {
                const uint32_t h = (lo + hi) >> 1;
                if (smk[h] < k || (smk[h] == k && smp[h] < p))
                    lo = h + 1;
                else
                    hi = h;
            }
            const uint32_t f = r + lo, id = rid[r];
            ep_key[f] = k;
            ep_id[f] = id;
            if (id < id_limit)
                ep_pos[id] = f;
            else
                set_error_at(error, kErrInternal, 1, id);
        }
        for (uint32_t u = t; u < m; u += B)
        {
            const uint32_t f = mfin[u], id = mid[u];
            ep_key[f] = mk[u];
            ep_id[f] = id;
            if (id < id_limit)
                ep_pos[id] = f;
            else
                set_error_at(error, kErrInternal, 1, id);
        }
        __syncthreads();
        return true;
    }

    // One-CTA fast path of the sweep, in the staging area `smem`: a single
    // pass over the overlap runs that leaves the pairs in the reference's
    // emission order without sorting them.  That order is by the position j
    // of the later opening endpoint, then by the position i of the earlier
    // one (BroadPhase.cpp:104-152).  The pass counts each j's pairs (hist),
    // appends every hit (i, j) to a staging list (warp-aggregated slots, so
    // the list has no particular order) and stores each opening endpoint's
    // own count in S.cnt.  A scan of hist gives each j its first slot, a
    // scatter groups the list by j, and an entry's final slot is its group's
    // first plus the number of the group's entries with a smaller i.  The
    // first min(total, pair_cap) pairs are written to S.pr_a / S.pr_b (pk =
    // j, pv = identity).  Returns the pair count, or ~0u when the hits do not
    // fit the staging lists ((kSmemSortWords - 2 nep) / 2 entries each: 3,104
    // at the largest nep); S.cnt is complete then, and the caller emits and
    // sorts in global memory.  Every thread of the CTA must call it.  prof:
    // sub-timers (sweep, pair order), or null.
    template <class SC>
    __device__ __noinline__ uint32_t sweep_staged(const FatBox *fat, const uint32_t *ep_id, const uint32_t *ep_pos,
                                                  uint32_t nep, uint32_t id_limit, uint32_t pair_cap, int *error,
                                                  const SC &S, ScanShared &sh, uint32_t *smem,
                                                  unsigned long long *prof)
    {
        long long tclk = prof ? clock64() : 0;
        // hist and fill per endpoint, then the two hit lists in what is left
        const uint32_t cap = (kSmemSortWords - 2 * nep) / 2;
        uint32_t *hist = smem, *fill = smem + nep;
        uint32_t *lst = smem + 2 * nep, *grp = lst + cap;
        const uint32_t B = blockDim.x, t = threadIdx.x, lane = t & 31u;
        for (uint32_t i = t; i < nep; i += B)
        {
            hist[i] = 0u;
            fill[i] = 0u;
        }
        if (t == 0)
            sh.bcast[3] = 0u;
        __syncthreads();
        for (uint32_t i = t; i < nep; i += B)
        {
            const uint32_t id = ep_id[i];
            uint32_t c = 0;
            if (!(id & 1u) && id < id_limit)
            {
                const FatBox fa = fat[id >> 1];
                const uint32_t end = min(ep_pos[id + 1], nep);
                for (uint32_t j = i + 1; j < end; ++j)
                {
                    const uint32_t id2 = ep_id[j];
                    const bool hit = !(id2 & 1u) && id2 < id_limit && fat_overlap(fa, fat[id2 >> 1]);
                    // one list reservation per warp step, for the lanes that hit
                    const uint32_t act = __activemask();
                    const uint32_t hm = __ballot_sync(act, hit);
                    if (hm)
                    {
                        const uint32_t leader = __ffs(hm) - 1;
                        uint32_t s = 0;
                        if (lane == leader)
                            s = atomicAdd(&sh.bcast[3], (uint32_t)__popc(hm));
                        s = __shfl_sync(act, s, leader) + __popc(hm & ((1u << lane) - 1u));
                        if (hit)
                        {
                            if (s < cap)
                                lst[s] = (i << 16) | j;
                            atomicAdd(&hist[j], 1u);
                            ++c;
                        }
                    }
                }
            }
            S.cnt[i] = c;
        }
        __syncthreads();
        sub_mark(prof, kPhSweep, tclk);
        const uint32_t total = sh.bcast[3];
        if (total > cap)
            return ~0u;
        // first slot of each j
        const uint32_t per = (nep + B - 1) / B;
        const uint32_t i0 = min(nep, t * per), i1 = min(nep, i0 + per);
        uint32_t mine = 0;
        for (uint32_t i = i0; i < i1; ++i)
            mine += hist[i];
        uint32_t sum;
        uint32_t run = block_excl_scan(mine, sh, &sum);
        for (uint32_t i = i0; i < i1; ++i)
        {
            const uint32_t h = hist[i];
            hist[i] = run;
            run += h;
        }
        if (t == 0 && sum != total)
            set_error_at(error, kErrInternal, 6, total); // the two counts of one pass must agree
        __syncthreads();
        for (uint32_t s = t; s < total; s += B)
        {
            const uint32_t v = lst[s], j = v & 0xffffu;
            const uint32_t g = hist[j] + atomicAdd(&fill[j], 1u);
            if (g < total)
                grp[g] = v;
        }
        __syncthreads();
        const uint32_t n_out = min(total, pair_cap);
        for (uint32_t s = t; s < total; s += B)
        {
            const uint32_t v = grp[s], i = v >> 16, j = v & 0xffffu;
            if (i >= nep || j >= nep)
            {
                set_error_at(error, kErrInternal, 6, v); // a slot the scatter left unwritten
                continue;
            }
            const uint32_t g0 = hist[j], g1 = min(total, g0 + fill[j]);
            uint32_t f = g0;
            for (uint32_t u = g0; u < g1; ++u)
                f += (grp[u] >> 16) < i ? 1u : 0u;
            if (f < n_out)
            {
                S.pr_a[f] = ep_id[i] >> 1;
                S.pr_b[f] = ep_id[j] >> 1;
                S.pk[f] = j;
                S.pv[f] = f;
            }
        }
        __syncthreads();
        sub_mark(prof, kPhPairOrder, tclk);
        return total;
    }

    // Sort + sweep of one SAP state (BroadPhase.cpp:80-152).  On return
    // S.pk / S.pv hold the pairs in the reference emission order (pv indexes
    // the raw object pairs S.pr_a / S.pr_b); returns the pair count.
    // id_limit bounds the endpoint ids (2 * object slots; slots of removed
    // objects leave gaps in the standalone broadphase).  A one-CTA team
    // with the shared staging area sort_smem takes the fast paths above:
    // the merge of the endpoints flagged in `moved` (shared, one word per
    // endpoint position; null to sort in full) and the single-pass sweep.
    template <class Team, class SC>
    __device__ __noinline__ uint32_t sap_sort_sweep(const Team &tm, const FatBox *fat, uint32_t *ep_key, uint32_t *ep_id,
                                       uint32_t *ep_pos, uint32_t nbp, uint32_t id_limit, uint32_t pair_cap,
                                       int *error, const SC &S, BlockShared &sh, uint32_t *sort_smem = nullptr,
                                       float4 *yz = nullptr, const uint32_t *moved = nullptr,
                                       unsigned long long *prof = nullptr)
    {
        const uint32_t nep = 2 * nbp;
        long long tclk = prof ? clock64() : 0;
        constexpr bool kBlock = std::is_same<Team, BlockTeam>::value;
        const bool staged = kBlock && sort_smem != nullptr && nep <= kSmemSortMax && blockDim.x >= 128;
        bool merged = false;
        if constexpr (kBlock)
            if (staged && moved)
                merged = merge_moved_endpoints(ep_key, ep_id, ep_pos, nep, id_limit, moved, sort_smem, sh, error);
        // stable sort of the endpoints, previous order as the tie-break
        if (!merged)
            team_sort_staged(tm, ep_key, ep_id, S.ep_k2, S.ep_v2, nep, 32, S.counts, S.tile_sums, sh, sort_smem);
        // inverse permutation (the merge wrote it already)
        for (uint32_t i = tm.rank(); i < nep; i += tm.size())
        {
            if (!merged)
            {
                const uint32_t id = ep_id[i];
                if (id < id_limit)
                    ep_pos[id] = i;
                else
                    set_error_at(error, kErrInternal, 1, id);
            }
            if (i + 1 < nep && ep_key[i] > ep_key[i + 1])
                set_error_at(error, kErrInternal, 4, i); // the endpoint sort must leave the keys ordered
        }
        sub_mark(prof, kPhEndpointSort, tclk);
        // A grid team's sweep reads every object of an overlap run; most fail
        // on y or z.  With yz, it first tests 16-byte float extents rounded
        // outward and reads the 48-byte double box only where they overlap,
        // so the pairs are exactly those of fat_overlap.
        const bool pre = tm.ncta() > 1 && yz != nullptr;
        if (pre)
            for (uint32_t o = tm.rank(); o < nbp; o += tm.size())
            {
                const FatBox f = fat[o];
                yz[o] = make_float4(__double2float_rd(f.mn[1]), __double2float_ru(f.mx[1]),
                                    __double2float_rd(f.mn[2]), __double2float_ru(f.mx[2]));
            }
        tm.sync();
        bool counted = false;
        if constexpr (kBlock)
            if (staged)
            {
                const uint32_t n =
                    sweep_staged(fat, ep_id, ep_pos, nep, id_limit, pair_cap, error, S, sh, sort_smem, prof);
                if (prof && threadIdx.x == 0)
                    tclk = clock64();
                if (n != ~0u)
                {
                    if (tm.leader())
                        S.misc[kMiscFlags + 4] = n; // unclamped pair count
                    uint32_t total = n;
                    if (total > pair_cap)
                    {
                        if (tm.leader())
                            set_error(error, -2);
                        total = pair_cap;
                    }
                    for (uint32_t k = tm.rank(); k + 1 < total; k += tm.size())
                        if (S.pk[k] > S.pk[k + 1])
                            set_error_at(error, kErrInternal, 5, k); // pairs must leave in key order
                    tm.sync();
                    return total;
                }
                counted = true; // too many pairs to stage: S.cnt holds the counts
            }
        // count the pairs each opening endpoint emits.  A team spread over
        // the cooperative grid (one large world) gives each opening endpoint
        // a warp that tests 32 endpoints of its overlap run at a time: the
        // runs are long there (hundreds of endpoints) and uneven, so one
        // thread per endpoint would leave most lanes waiting on a few.
        const bool by_warp = tm.ncta() > 1;
        const uint32_t lane = threadIdx.x & 31u;
        if (by_warp && !counted)
        {
            for (uint32_t i = tm.rank() >> 5; i < nep; i += tm.size() >> 5)
            {
                const uint32_t id = ep_id[i]; // the same for the whole warp
                uint32_t c = 0;
                if (!(id & 1u) && id < id_limit)
                {
                    const FatBox fa = fat[id >> 1];
                    const float4 fq = pre ? yz[id >> 1] : float4{};
                    const uint32_t end = min(ep_pos[id + 1], nep);
                    for (uint32_t j0 = i + 1; j0 < end; j0 += 32)
                    {
                        const uint32_t j = j0 + lane;
                        bool hit = false;
                        if (j < end)
                        {
                            const uint32_t id2 = ep_id[j];
                            hit = !(id2 & 1u) && id2 < id_limit && (!pre || yz_may_overlap(fq, yz[id2 >> 1])) &&
                                  fat_overlap(fa, fat[id2 >> 1]);
                        }
                        c += __popc(__ballot_sync(0xffffffffu, hit));
                    }
                }
                if (lane == 0)
                    S.cnt[i] = c;
            }
        }
        else if (!counted)
            for (uint32_t i = tm.rank(); i < nep; i += tm.size())
            {
                const uint32_t id = ep_id[i];
                uint32_t c = 0;
                if (!(id & 1u) && id < id_limit)
                {
                    const FatBox fa = fat[id >> 1];
                    const uint32_t end = min(ep_pos[id + 1], nep);
                    for (uint32_t j = i + 1; j < end; ++j)
                    {
                        const uint32_t id2 = ep_id[j];
                        if (!(id2 & 1u) && id2 < id_limit && fat_overlap(fa, fat[id2 >> 1]))
                            ++c;
                    }
                }
                S.cnt[i] = c;
            }
        tm.sync();
        uint32_t total = team_excl_scan(tm, S.cnt, S.cnt, nep, S.tile_sums, sh);
        if (tm.leader())
            S.misc[kMiscFlags + 4] = total; // unclamped pair count
        if (total > pair_cap)
        {
            if (tm.leader())
                set_error(error, -2);
            total = pair_cap;
        }
        // emit (earlier-opening object, later object, later opening position)
        if (by_warp)
        {
            for (uint32_t i = tm.rank() >> 5; i < nep; i += tm.size() >> 5)
            {
                const uint32_t id = ep_id[i];
                if ((id & 1u) || id >= id_limit)
                    continue;
                uint32_t k = S.cnt[i];
                const FatBox fa = fat[id >> 1];
                const float4 fq = pre ? yz[id >> 1] : float4{};
                const uint32_t end = min(ep_pos[id + 1], nep);
                for (uint32_t j0 = i + 1; j0 < end && k < total; j0 += 32)
                {
                    const uint32_t j = j0 + lane;
                    uint32_t id2 = 0;
                    bool hit = false;
                    if (j < end)
                    {
                        id2 = ep_id[j];
                        hit = !(id2 & 1u) && id2 < id_limit && (!pre || yz_may_overlap(fq, yz[id2 >> 1])) &&
                              fat_overlap(fa, fat[id2 >> 1]);
                    }
                    const uint32_t m = __ballot_sync(0xffffffffu, hit);
                    const uint32_t kk = k + __popc(m & ((1u << lane) - 1u));
                    if (hit && kk < total)
                    {
                        S.pr_a[kk] = id >> 1;
                        S.pr_b[kk] = id2 >> 1;
                        S.pk[kk] = j;
                        S.pv[kk] = kk;
                    }
                    k += __popc(m);
                }
            }
        }
        else
            for (uint32_t i = tm.rank(); i < nep; i += tm.size())
            {
                const uint32_t id = ep_id[i];
                if ((id & 1u) || id >= id_limit)
                    continue;
                uint32_t k = S.cnt[i];
                const FatBox fa = fat[id >> 1];
                const uint32_t end = min(ep_pos[id + 1], nep);
                for (uint32_t j = i + 1; j < end && k < total; ++j)
                {
                    const uint32_t id2 = ep_id[j];
                    if (!(id2 & 1u) && id2 < id_limit && fat_overlap(fa, fat[id2 >> 1]))
                    {
                        S.pr_a[k] = id >> 1;
                        S.pr_b[k] = id2 >> 1;
                        S.pk[k] = j;
                        S.pv[k] = k;
                        ++k;
                    }
                }
            }
        tm.sync();
        sub_mark(prof, kPhSweep, tclk);
        // reference emission order: stable sort by the later opening position
        const int bits = nep > 1 ? 32 - __clz(nep - 1) : 1;
        team_sort_staged(tm, S.pk, S.pv, S.pk2, S.pv2, total, bits, S.counts, S.tile_sums, sh, sort_smem);
        for (uint32_t k = tm.rank(); k + 1 < total; k += tm.size())
            if (S.pk[k] > S.pk[k + 1])
                set_error_at(error, kErrInternal, 5, k); // pair sort must leave the keys ordered
        tm.sync(); // the caller rewrites S.pk next
        sub_mark(prof, kPhPairOrder, tclk);
        return total;
    }

    // prof: the world's phase-timer slots for the sort / sweep / pair-order
    // sub-timers (one-CTA teams; null otherwise).
    template <class T, class P, class Team>
    __device__ uint32_t broadphase(const Engine<T, P> &E, const Team &tm, const WorldDev &W, const Scr<T, P> &S,
                                   BlockShared &sh, uint32_t *sort_smem = nullptr, unsigned long long *prof = nullptr)
    {
        const uint32_t nbp = W.n_bp;
        const uint32_t eb = 2 * W.bp_off;
        FatBox *fat = E.fat + W.bp_off;
        uint32_t *ep_key = E.ep_key + eb;
        uint32_t *ep_id = E.ep_id + eb;
        uint32_t *ep_pos = E.ep_pos + eb;
        const uint32_t nep = 2 * nbp;
        // a one-CTA team with a staging area flags the endpoint positions
        // whose keys it rewrites, for the sort's merge fast path
        uint32_t *moved = nullptr;
        if constexpr (std::is_same<Team, BlockTeam>::value)
            if (sort_smem && nep <= kSmemSortMax)
            {
                moved = sh.wdig;
                for (uint32_t i = tm.rank(); i < nep; i += tm.size())
                    moved[i] = 0u;
                tm.sync();
            }

        // object update (update_broad_phase_aabbs + broad_phase_move_swept)
        for (uint32_t o = tm.rank(); o < nbp; o += tm.size())
        {
            const uint32_t lc = E.bp_coll[W.bp_off + o];
            const uint32_t gc = W.coll_off + lc;
            if (E.c_static[gc])
                continue;
            const uint32_t gb = W.body_off + E.c_body[gc];
            const tf<double> t = collider_tf_d(E, gc, gb);
            aabb tight = compute_aabb(E.shape[gc], t, E.hulls);
            if (E.use_vel_exp)
            {
                const V4<T> lv = E.B.lin[gb];
                const vec3<double> dv = vec3<double>(double(lv.x), double(lv.y), double(lv.z)) * E.dt_frame;
                const double m = E.fat_margin;
                const vec3<double> emn(m + (dv.x < 0 ? -dv.x : 0.0), m + (dv.y < 0 ? -dv.y : 0.0), m + (dv.z < 0 ? -dv.z : 0.0));
                const vec3<double> emx(m + (dv.x > 0 ? dv.x : 0.0), m + (dv.y > 0 ? dv.y : 0.0), m + (dv.z > 0 ? dv.z : 0.0));
                tight = aabb{tight.mn - emn, tight.mx + emx};
            }
            const aabb f0 = load_fat(fat[o]);
            if (aabb_contained(tight, f0))
                continue;
            const aabb f1 = aabb_expand(tight, E.fat_margin + E.reinsert_threshold);
            FatBox fb;
            fb.mn[0] = f1.mn.x; fb.mn[1] = f1.mn.y; fb.mn[2] = f1.mn.z;
            fb.mx[0] = f1.mx.x; fb.mx[1] = f1.mx.y; fb.mx[2] = f1.mx.z;
            fat[o] = fb;
            const uint32_t p0 = ep_pos[2 * o], p1 = ep_pos[2 * o + 1];
            ep_key[p0] = order_key(__double2float_rn(f1.mn.x));
            ep_key[p1] = order_key(__double2float_rn(f1.mx.x));
            if (moved)
            {
                if (p0 < nep)
                    moved[p0] = 1u;
                if (p1 < nep)
                    moved[p1] = 1u;
            }
        }
        tm.sync();
        return sap_sort_sweep(tm, fat, ep_key, ep_id, ep_pos, nbp, nep, W.pair_cap, E.error, S, sh, sort_smem,
                              W.n_bodies > kGridWorldBodies ? S.yz : nullptr, moved, prof);
    }

    // Filtered SAP pairs followed by the plane candidates; returns the count.
    template <class T, class P, class Team>
    __device__ uint32_t build_candidates(const Engine<T, P> &E, const Team &tm, const WorldDev &W, const Scr<T, P> &S,
                                         uint32_t n_pairs, BlockShared &sh)
    {
        // SAP pair (lo, hi) user ids, filters of run_narrow_phase (CollisionPipeline.cpp:121-133)
        for (uint32_t k = tm.rank(); k < n_pairs; k += tm.size())
        {
            const uint32_t r = S.pv[k];
            const uint32_t oa = r < n_pairs ? S.pr_a[r] : ~0u;
            const uint32_t ob = r < n_pairs ? S.pr_b[r] : ~0u;
            if (oa >= W.n_bp || ob >= W.n_bp)
            {
                // corrupt pair record: report it and drop the pair
                set_error_at(E.error, kErrInternal, 2, r);
                S.pk[k] = 0;
                S.pk2[k] = 0;
                S.cflag[k] = 0;
                continue;
            }
            const uint32_t ua = E.bp_coll[W.bp_off + oa];
            const uint32_t ub = E.bp_coll[W.bp_off + ob];
            const uint32_t lo = ua < ub ? ua : ub;
            const uint32_t hi = ua < ub ? ub : ua;
            S.pk[k] = lo;
            S.pk2[k] = hi;
            const uint32_t ga = W.coll_off + lo, gb = W.coll_off + hi;
            const bool keep = !(E.c_static[ga] && E.c_static[gb]) && (E.c_body[ga] != E.c_body[gb]);
            S.cflag[k] = keep ? 1u : 0u;
            if (E.dump_pairs && W.dump_slot != ~0u && k < E.dump_pair_cap)
            {
                uint32_t *dp = E.dump_pairs + (size_t)W.dump_slot * 2 * E.dump_pair_cap;
                dp[2 * k] = lo;
                dp[2 * k + 1] = hi;
            }
        }
        tm.sync();
        const uint32_t n_sap = team_excl_scan(tm, S.cflag, S.cflag, n_pairs, S.tile_sums, sh);
        for (uint32_t k = tm.rank(); k < n_pairs; k += tm.size())
        {
            const uint32_t lo = S.pk[k], hi = S.pk2[k];
            const uint32_t ga = W.coll_off + lo, gb = W.coll_off + hi;
            const bool keep = lo != hi && !(E.c_static[ga] && E.c_static[gb]) && (E.c_body[ga] != E.c_body[gb]);
            if (keep && S.cflag[k] < n_pairs)
                S.cand[S.cflag[k]] = Cand{lo, hi, E.c_body[ga], E.c_body[gb]};
        }
        for (uint32_t q = tm.rank(); q < W.n_pc; q += tm.size())
        {
            const uint2 pc = E.plane_cand[W.pc_off + q];
            S.cand[n_sap + q] = Cand{pc.x, pc.y, E.c_body[W.coll_off + pc.x], E.c_body[W.coll_off + pc.y]};
        }
        tm.sync();
        return n_sap + W.n_pc;
    }

    // Colouring of the candidates that produced contact rows in this substep
    // (the others have nothing to relax), in rounds:
    // * up to kGridWorldBodies bodies, Jones-Plassmann: a candidate takes the
    //   lowest colour free on both of its dynamic bodies once it holds the
    //   highest priority among the uncoloured candidates sharing them.  A
    //   body gets at most one colour a round, so a body with d contacts takes
    //   d rounds or more;
    // * larger worlds, claims: every uncoloured candidate picks one colour
    //   free on both bodies (hashed among the lowest few) and claims that
    //   (body, colour) slot on each; the highest claim on both slots wins.
    //   Many contacts of one body are coloured per round: on tangled chains
    //   (contacts up to 53 per body) 8 rounds instead of more than 96.
    // Both are deterministic (priorities are hashes of the candidate index).
    // Candidates whose bodies have used all 64 colours, or still uncoloured
    // after kMaxColorRounds, go to the serial colour; idle candidates get
    // kColorIdle and are not bucketed.  Returns the number of regular
    // colours; corder / colour offsets are filled.
    // Second-level colours for the overflow bucket [coff[64], coff[65]) of
    // corder: the team leader colours its candidates first-fit in order on
    // a second set of body masks (bprio, free after the Jones-Plassmann
    // rounds), and the bucket is reordered by those colours, so that the
    // solves can relax it colour by colour (kMiscC2Off) instead of on one
    // thread; entry 64 keeps what still does not fit.  The bucket comes
    // after every first-level colour, so the Gauss-Seidel order stays a
    // sequence of conflict-free sets.
    template <class T, class P, class Team>
    __device__ void color_overflow(const Engine<T, P> &E, const Team &tm, const WorldDev &W, const Scr<T, P> &S)
    {
        uint32_t *misc = S.misc;
        const uint32_t s0 = misc[kMiscCOff + kColorSerial], s1 = misc[kMiscCOff + kColorSerial + 1];
        uint32_t *cnt = misc + kMiscC2Count, *off = misc + kMiscC2Off;
        for (uint32_t k = tm.rank(); k < 66; k += tm.size())
            cnt[k] = 0u;
        if (s1 > s0)
        {
            for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
                S.bprio[b] = 0ull;
            for (uint32_t q = s0 + tm.rank(); q < s1; q += tm.size())
                S.alist[q - s0] = S.corder[q];
        }
        tm.sync();
        if (tm.leader())
        {
            const uint8_t *type = E.B.type + W.body_off;
            constexpr uint32_t kAhead = 8; // candidates loaded ahead of the mask updates
            const uint32_t ns = s1 - s0;
            for (uint32_t q0 = 0; q0 < ns; q0 += kAhead)
            {
                uint32_t cs[kAhead];
                Cand cd[kAhead];
                bool da[kAhead], db[kAhead];
#pragma unroll
                for (uint32_t k = 0; k < kAhead; ++k)
                    if (q0 + k < ns)
                    {
                        cs[k] = S.alist[q0 + k];
                        cd[k] = S.cand[cs[k]];
                        da[k] = type[cd[k].ba] == kDynamic;
                        db[k] = type[cd[k].bb] == kDynamic;
                    }
#pragma unroll
                for (uint32_t k = 0; k < kAhead; ++k)
                    if (q0 + k < ns)
                    {
                        const unsigned long long used =
                            (da[k] ? S.bprio[cd[k].ba] : 0ull) | (db[k] ? S.bprio[cd[k].bb] : 0ull);
                        uint32_t col = kColorSerial;
                        if (used != ~0ull)
                        {
                            col = (uint32_t)(__ffsll((long long)~used) - 1);
                            const unsigned long long bit = 1ull << col;
                            if (da[k])
                                S.bprio[cd[k].ba] |= bit;
                            if (db[k])
                                S.bprio[cd[k].bb] |= bit;
                        }
                        S.act[cs[k]] = col;
                        cnt[col] += 1u;
                    }
            }
            uint32_t run = s0;
            for (uint32_t k = 0; k <= kColorSerial; ++k)
            {
                const uint32_t n = cnt[k];
                off[k] = run;
                cnt[k] = run; // fill cursor
                run += n;
            }
            off[kColorSerial + 1] = run;
        }
        tm.sync();
        for (uint32_t q = tm.rank(); q < s1 - s0; q += tm.size())
        {
            const uint32_t c = S.alist[q];
            S.corder[atomicAdd(&cnt[S.act[c]], 1u)] = c;
        }
        tm.sync();
    }

    template <class T, class P, class Team>
    __device__ uint32_t color_active(const Engine<T, P> &E, const Team &tm, const WorldDev &W, const Scr<T, P> &S,
                                     uint32_t n_cand, BlockShared &sh)
    {
        uint32_t *misc = S.misc;
        // compact the active candidates into alist
        for (uint32_t c = tm.rank(); c < n_cand; c += tm.size())
            S.act[c] = S.cc[c].n > 0 ? 1u : 0u;
        for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
        {
            S.bmask[b] = 0ull;
            S.bprio[b] = 0ull;
        }
        const bool by_claim = W.n_bodies > kGridWorldBodies;
        if (by_claim)
            for (uint32_t x = tm.rank(); x < W.n_bodies * 64u; x += tm.size())
                S.claim[x] = 0ull;
        for (uint32_t x = tm.rank(); x < kMaxColorRounds + 2 * 66; x += tm.size())
            misc[kMiscCCount + x] = 0u;
        tm.sync();
        const uint32_t n_act = team_excl_scan(tm, S.act, S.act, n_cand, S.tile_sums, sh);
        for (uint32_t c = tm.rank(); c < n_cand; c += tm.size())
        {
            if (S.cc[c].n > 0)
                S.alist[S.act[c]] = c;
            S.color[c] = S.cc[c].n > 0 ? 0xffffffffu : kColorIdle;
        }
        tm.sync();
        const uint8_t *type = E.B.type + W.body_off;
        uint32_t round = 1;
        if (by_claim)
        {
            // uncoloured contacts per body (bprio's words reused as counters)
            uint32_t *ucnt = (uint32_t *)S.bprio;
            for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
            {
                const Cand cd = S.cand[S.alist[q]];
                if (type[cd.ba] == kDynamic)
                    atomicAdd(&ucnt[cd.ba], 1u);
                if (type[cd.bb] == kDynamic)
                    atomicAdd(&ucnt[cd.bb], 1u);
            }
            tm.sync();
            for (; round <= kMaxColorRounds && n_act; ++round)
            {
                // each uncoloured candidate claims one colour free on both
                // bodies, drawn from the lowest max(1, u / 2) free colours (u:
                // the larger uncoloured count of its bodies), so a body's
                // candidates spread over several colours in one round
                for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
                {
                    const uint32_t c = S.alist[q];
                    if (S.color[c] != 0xffffffffu)
                        continue;
                    const Cand cd = S.cand[c];
                    const bool da = type[cd.ba] == kDynamic, db = type[cd.bb] == kDynamic;
                    const unsigned long long used = (da ? S.bmask[cd.ba] : 0ull) | (db ? S.bmask[cd.bb] : 0ull);
                    if (used == ~0ull)
                    {
                        S.color[c] = kColorSerial;
                        continue;
                    }
                    unsigned long long f = ~used;
                    const uint32_t u = max(da ? ucnt[cd.ba] : 1u, db ? ucnt[cd.bb] : 1u);
                    const uint32_t span = min((uint32_t)__popcll(f), max(1u, u / 2u));
                    for (uint32_t k = hash32(c * 0x9e3779b1u + round) % span; k; --k)
                        f &= f - 1ull;
                    const uint32_t col = (uint32_t)(__ffsll((long long)f) - 1);
                    S.act[c] = col;
                    const unsigned long long val = ((unsigned long long)round << 56) |
                                                   ((unsigned long long)(hash32(c ^ (round << 24)) & 0xffffffu) << 32) | c;
                    if (da)
                        atomicMax(&S.claim[(size_t)cd.ba * 64u + col], val);
                    if (db)
                        atomicMax(&S.claim[(size_t)cd.bb * 64u + col], val);
                }
                tm.sync();
                // the highest claim on each (body, colour) slot wins it
                uint32_t lost = 0;
                for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
                {
                    const uint32_t c = S.alist[q];
                    if (S.color[c] != 0xffffffffu)
                        continue;
                    const Cand cd = S.cand[c];
                    const bool da = type[cd.ba] == kDynamic, db = type[cd.bb] == kDynamic;
                    const uint32_t col = S.act[c];
                    const unsigned long long val = ((unsigned long long)round << 56) |
                                                   ((unsigned long long)(hash32(c ^ (round << 24)) & 0xffffffu) << 32) | c;
                    const bool won = (!da || S.claim[(size_t)cd.ba * 64u + col] == val) &&
                                     (!db || S.claim[(size_t)cd.bb * 64u + col] == val);
                    if (!won)
                    {
                        ++lost;
                        continue;
                    }
                    S.color[c] = col;
                    const unsigned long long bit = 1ull << col;
                    if (da)
                    {
                        atomicOr(&S.bmask[cd.ba], bit);
                        atomicSub(&ucnt[cd.ba], 1u);
                    }
                    if (db)
                    {
                        atomicOr(&S.bmask[cd.bb], bit);
                        atomicSub(&ucnt[cd.bb], 1u);
                    }
                }
                lost = __reduce_add_sync(0xffffffffu, lost);
                if (lost && lane_id() == 0)
                    atomicAdd(&misc[kMiscLeft + round - 1], lost);
                tm.sync();
                if (misc[kMiscLeft + round - 1] == 0u)
                    break;
            }
        }
        for (; !by_claim && round <= kMaxColorRounds && n_act; ++round)
        {
            for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
            {
                const uint32_t c = S.alist[q];
                if (S.color[c] != 0xffffffffu)
                    continue;
                const Cand cd = S.cand[c];
                const unsigned long long val = ((unsigned long long)round << 56) |
                                               ((unsigned long long)(hash32(c) & 0xffffffu) << 32) | c;
                if (type[cd.ba] == kDynamic)
                    atomicMax(&S.bprio[cd.ba], val);
                if (type[cd.bb] == kDynamic)
                    atomicMax(&S.bprio[cd.bb], val);
            }
            tm.sync();
            for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
            {
                const uint32_t c = S.alist[q];
                if (S.color[c] != 0xffffffffu)
                    continue;
                const Cand cd = S.cand[c];
                const unsigned long long val = ((unsigned long long)round << 56) |
                                               ((unsigned long long)(hash32(c) & 0xffffffu) << 32) | c;
                const bool da = type[cd.ba] == kDynamic, db = type[cd.bb] == kDynamic;
                const bool won = (!da || S.bprio[cd.ba] == val) && (!db || S.bprio[cd.bb] == val);
                if (!won)
                {
                    atomicAdd(&misc[kMiscLeft + round - 1], 1u);
                    continue;
                }
                const unsigned long long used = (da ? S.bmask[cd.ba] : 0ull) | (db ? S.bmask[cd.bb] : 0ull);
                uint32_t col;
                if (used == ~0ull)
                    col = kColorSerial;
                else
                {
                    col = (uint32_t)(__ffsll((long long)~used) - 1);
                    const unsigned long long bit = 1ull << col;
                    if (da)
                        S.bmask[cd.ba] |= bit;
                    if (db)
                        S.bmask[cd.bb] |= bit;
                }
                S.color[c] = col;
            }
            tm.sync();
            if (misc[kMiscLeft + round - 1] == 0u)
                break;
        }
        if (round > kMaxColorRounds)
        {
            for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
                if (S.color[S.alist[q]] == 0xffffffffu)
                    S.color[S.alist[q]] = kColorSerial;
            tm.sync();
        }
        // bucket the active candidates by colour
        for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
            atomicAdd(&misc[kMiscCCount + S.color[S.alist[q]]], 1u);
        tm.sync();
        if (tm.leader())
        {
            uint32_t run = 0, ncol = 0;
            for (uint32_t k = 0; k <= kColorSerial; ++k)
            {
                const uint32_t n = misc[kMiscCCount + k];
                misc[kMiscCOff + k] = run;
                misc[kMiscCCount + k] = run; // becomes the fill cursor
                if (n && k < kColorSerial)
                    ncol = k + 1;
                run += n;
            }
            misc[kMiscCOff + kColorSerial + 1] = run;
            misc[kMiscFlags + 1] = ncol;
        }
        tm.sync();
        for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
        {
            const uint32_t c = S.alist[q];
            const uint32_t slot = atomicAdd(&misc[kMiscCCount + S.color[c]], 1u);
            S.corder[slot] = c;
        }
        tm.sync();
        color_overflow(E, tm, W, S);
        return misc[kMiscFlags + 1];
    }

    // emit_contact (CollisionPipeline.cpp:59-104): a pair's manifold into
    // its contact rows (points on A and B, body-local lever arms, mixed
    // materials).
    template <class T, class P>
    __device__ __forceinline__ void emit_manifold(const Engine<T, P> &E, uint32_t gca, uint32_t gcb, uint32_t gba,
                                                  uint32_t gbb, const Manifold<T> &m, int n, CandContacts<T, P> &out)
    {
        out.n = n;
        if (n == 0)
            return;
        out.normal = v4(m.normal);
        const V4<T> ma = E.c_mat[gca], mb = E.c_mat[gcb];
        out.mat = V4<T>{rmin(ma.x, mb.x), (ma.y + mb.y) * T(0.5), (ma.z + mb.z) * T(0.5), T(0)};
        const vec3<T> xa = E.B.x(gba), xb = E.B.x(gbb);
        const quat<T> qa = conjugate(E.B.q(gba)), qb = conjugate(E.B.q(gbb));
        for (int k = 0; k < n; ++k)
        {
            const T half = m.depth[k] * T(0.5);
            const vec3<T> pa = m.pos[k] + m.normal * half;
            const vec3<T> pb = m.pos[k] - m.normal * half;
            ContactPt<T, P> &c = out.pt[k];
            c.ra = v4(rotate(qa, pa - xa));
            c.rb = v4(rotate(qb, pb - xb));
            c.pa = V4<P>{P(pa.x), P(pa.y), P(pa.z), P(0)};
            c.pb = V4<P>{P(pb.x), P(pb.y), P(pb.z), P(0)};
            c.lam_n = T(0.0);
            c.lam_t = T(0.0);
            c.vrel = T(0.0);
            c.depth = m.depth[k];
            c.coll = 0;
        }
    }

    // Narrowphase of one candidate (the analytic routines); returns
    // kNeedsGjk for a pair the GJK pass handles (its rows are left empty).
    template <class T, class P, int Sel>
    __device__ __forceinline__ int narrow_pair(const Engine<T, P> &E, uint32_t gca, uint32_t gcb, uint32_t gba,
                                               uint32_t gbb, CandContacts<T, P> &out)
    {
        const tf<T> ta = collider_tf(E, gca, gba);
        const tf<T> tb = collider_tf(E, gcb, gbb);
        Manifold<T> m;
        m.n = 0;
        int res = dispatch_pair<T, Sel>(E.shape[gca], ta, E.shape[gcb], tb, E.hulls, m);
        // a pair for the GJK pass whose bounding spheres are apart stays out
        // of the queue (GJK would find it apart); the analytic routines exit
        // early on their own, and the same test in front of them measured
        // slower on the batched workload
        if (res == kNeedsGjk && bounds_separate(E.shape[gca], ta, E.shape[gcb], tb, E.hulls))
            res = kMiss;
        emit_manifold(E, gca, gcb, gba, gbb, m, res == kHit ? m.n : 0, out);
        return res;
    }

    template <class T, class P, int Sel = kSelAll>
    __device__ __forceinline__ int narrow_candidate(const Engine<T, P> &E, const WorldDev &W, const Cand &cd,
                                                    CandContacts<T, P> &out)
    {
        if (cd.ca >= W.n_coll || cd.cb >= W.n_coll || cd.ba >= W.n_bodies || cd.bb >= W.n_bodies)
        {
            set_error_at(E.error, kErrInternal, 3, cd.ca);
            out.n = 0;
            return kMiss;
        }
        return narrow_pair<T, P, Sel>(E, W.coll_off + cd.ca, W.coll_off + cd.cb, W.body_off + cd.ba,
                                      W.body_off + cd.bb, out);
    }

    // A GJK pair found by the narrowphase: queued for k_gjk and counted
    // (WorldStats::n_gjk, summed over the step's substeps).  Every batch
    // with a hull collider has the queue; only hull pairs need GJK.
    template <class T, class P>
    __device__ __forceinline__ void queue_gjk(const Engine<T, P> &E, uint32_t w, uint32_t c, uint32_t &n_gjk)
    {
        ++n_gjk;
        if (E.gjk_list)
        {
            const uint32_t slot = atomicAdd(E.gjk_count, 1u);
            if (slot < E.gjk_cap)
                E.gjk_list[slot] = make_uint2(w, c);
            else
                set_error_at(E.error, -2, 6, slot); // RBPS_ERR_CAPACITY
        }
    }

    // A double manifold in precision T.
    template <class T>
    __device__ __forceinline__ Manifold<T> manifold_cast(const Manifold<double> &d)
    {
        Manifold<T> m;
        m.n = d.n;
        m.normal = vec3<T>(d.normal);
        for (int k = 0; k < 4; ++k)
        {
            m.pos[k] = vec3<T>(d.pos[k]);
            m.depth[k] = T(d.depth[k]);
        }
        return m;
    }

    // GJK / EPA / manifold of one queued pair (world w, candidate c) on one
    // warp: every lane runs GJK / EPA with the warp's shared workspace `ws`;
    // lane 0 writes the contact block.  GJK and EPA run in double in every
    // precision: their tolerances (EPA convergence 1e-6, coplanarity 1e-12)
    // are below float resolution.
    template <class T, class P>
    __device__ void gjk_candidate_warp(const Engine<T, P> &E, uint32_t w, uint32_t c, unsigned char *ws)
    {
        const WorldDev W = E.worlds[w];
        const Cand cd = E.wcand ? E.wcand[w][c] : world_scratch(E, W).cand[c];
        const uint32_t gca = W.coll_off + cd.ca, gcb = W.coll_off + cd.cb;
        const uint32_t gba = W.body_off + cd.ba, gbb = W.body_off + cd.bb;
        const tf<double> ta = collider_tf_d(E, gca, gba);
        const tf<double> tb = collider_tf_d(E, gcb, gbb);
        Manifold<double> m;
        m.n = 0;
        const bool hit = gjk_epa_manifold_warp(E.shape[gca], ta, E.shape[gcb], tb, E.hulls, ws, m, E.error);
        if ((threadIdx.x & 31u) == 0)
        {
            CandContacts<T, P> &out = E.wcc ? E.wcc[w][c] : world_scratch(E, W).cc[c];
            const Manifold<T> mt = manifold_cast<T>(m);
            emit_manifold(E, gca, gcb, gba, gbb, mt, hit ? mt.n : 0, out);
        }
    }

    // All contact rows of one candidate pair (global bodies ba, bb), in list
    // order, with both bodies in registers (load once, relax, store once).
    template <class T, class P>
    __device__ __forceinline__ void solve_pair_position(const Bodies<T, P> &B, T inv_h, uint32_t ba, uint32_t bb,
                                                        CandContacts<T, P> &cc)
    {
        const int n = cc.n;
        if (n == 0)
            return;
        const vec3<T> nrm = v3(cc.normal);
        const T sf = cc.mat.y;
        BodyR<T, P> A, Bb;
        load_body(B, ba, A, true);
        load_body(B, bb, Bb, true);
        for (int k = 0; k < n; ++k)
            contact_position(A, Bb, nrm, sf, cc.pt[k], inv_h);
        store_pose(B, ba, A);
        store_pose(B, bb, Bb);
    }

    template <class T, class P>
    __device__ __forceinline__ void solve_pair_velocity(const Bodies<T, P> &B, T h, uint32_t ba, uint32_t bb,
                                                        const CandContacts<T, P> &cc)
    {
        const int n = cc.n;
        if (n == 0)
            return;
        const vec3<T> nrm = v3(cc.normal);
        BodyR<T, P> A, Bb;
        load_body(B, ba, A, false);
        load_body(B, bb, Bb, false);
        for (int k = 0; k < n; ++k)
            contact_velocity(A, Bb, nrm, cc.mat.x, cc.mat.z, cc.pt[k], h);
        store_vel(B, ba, A);
        store_vel(B, bb, Bb);
    }

    template <class T, class P>
    __device__ __forceinline__ void solve_cand_position(const Engine<T, P> &E, const WorldDev &W, const Cand &cd,
                                                        CandContacts<T, P> &cc)
    {
        solve_pair_position(E.B, E.inv_h, W.body_off + cd.ba, W.body_off + cd.bb, cc);
    }

    template <class T, class P>
    __device__ __forceinline__ void solve_cand_velocity(const Engine<T, P> &E, const WorldDev &W, const Cand &cd,
                                                        const CandContacts<T, P> &cc)
    {
        solve_pair_velocity(E.B, E.h, W.body_off + cd.ba, W.body_off + cd.bb, cc);
    }

    template <class T, class P>
    __device__ __forceinline__ Row<T> *joint_rows(const Engine<T, P> &E, const Joint<T> &j)
    {
        return E.rows + j.row0;
    }

    // Per-world phase timers (diagnostics; off when Engine::prof is null).
    // The team leader adds the SM cycles of each phase, read after the
    // phase's closing barrier, into prof[world * kProfSlots + phase].
    struct PhaseClock
    {
        unsigned long long *p;
        long long t;
        __device__ PhaseClock(unsigned long long *slots, bool frame_start)
        {
            p = slots;
            t = 0;
            if (p)
            {
                t = clock64();
                if (frame_start)
                {
                    unsigned long long g;
                    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(g));
                    p[kProfStartNs] = g;
                    p[kProfCta] = blockIdx.x;
                }
            }
        }
        __device__ void mark(int phase)
        {
            if (!p)
                return;
            const long long now = clock64();
            p[phase] += (unsigned long long)(now - t);
            t = now;
        }
        __device__ void finish()
        {
            if (!p)
                return;
            unsigned long long g;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(g));
            p[kProfEndNs] = g;
        }
    };

    template <class T, class P, class Team>
    __device__ __forceinline__ unsigned long long *prof_slots(const Engine<T, P> &E, const Team &tm, uint32_t w)
    {
        return tm.leader() && E.prof ? E.prof + (size_t)w * kProfSlots : nullptr;
    }

    // The scratch slice of world W (layout from the world's own sizes).
    template <class T, class P>
    __device__ __forceinline__ Scr<T, P> world_scratch(const Engine<T, P> &E, const WorldDev &W)
    {
        return scratch_ptrs<T, P>(E.scratch + W.scr_off,
                                  make_layout(W.n_bp, W.n_bodies, W.pair_cap, W.n_pc, sizeof(CandContacts<T, P>)));
    }

    // Bodies of corder slot q (candidate c): from the packed pair written at
    // colouring when the team keeps its world in shared memory (book), else
    // from the candidate.
    template <class T, class P>
    __device__ __forceinline__ void slot_pair(const Scr<T, P> &S, const uint32_t *book, uint32_t q, uint32_t c,
                                              uint32_t &ba, uint32_t &bb)
    {
        if (book)
        {
            const uint32_t pr = S.act[q];
            ba = pr & 0xffffu;
            bb = pr >> 16;
        }
        else
        {
            const Cand cd = S.cand[c];
            ba = cd.ba;
            bb = cd.bb;
        }
    }

    // Candidate and bodies of colour-ordered slot q: from the team's shared
    // slots when the colouring left them there, else as slot_pair.
    template <class T, class P>
    __device__ __forceinline__ void slot_entry(const Scr<T, P> &S, const uint32_t *book, const uint2 *slots, uint32_t q,
                                               uint32_t &c, uint32_t &ba, uint32_t &bb)
    {
        if (slots)
        {
            const uint2 e = slots[q];
            c = e.x;
            ba = e.y & 0xffffu;
            bb = e.y >> 16;
            return;
        }
        c = S.corder[q];
        slot_pair(S, book, q, c, ba, bb);
    }

    // Asks L2 for every 128-byte line of [p, p + bytes) (prefetch.global.L2).
    __device__ __forceinline__ void prefetch_l2_range(const void *p, size_t bytes)
    {
        const uintptr_t a = reinterpret_cast<uintptr_t>(p);
        for (uintptr_t l = a & ~uintptr_t(127); l < a + bytes; l += 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(l));
    }

    // ------------------------------------------------------------ the step
    // World::step (World.hpp:192-212) as phases.  Every phase ends with a
    // team barrier and keeps its state in the world's scratch slice, so each
    // phase runs as its own kernel: over all small worlds, one CTA per world
    // (every CTA runs the same phase's code at a time), or for one large
    // world on the whole cooperative grid.

    // Frame (once per step): SAP object update, sort, sweep; candidate list.
    template <class T, class P, class Team>
    __device__ void phase_frame(const Engine<T, P> &E, const Team &tm, uint32_t w, BlockShared &sh,
                                uint32_t *sort_smem = nullptr)
    {
        const WorldDev W = E.worlds[w];
        const Scr<T, P> S = world_scratch(E, W);
        PhaseClock clk(prof_slots(E, tm, w), true);
        if (tm.leader())
        {
            S.misc[kMiscNGjk] = 0u;
            S.misc[kMiscMaxColors] = 0u;
            S.misc[kMiscColorValid] = 0u; // a new candidate list: no colouring yet
        }
        const uint32_t n_pairs =
            broadphase(E, tm, W, S, sh, sort_smem, std::is_same<Team, BlockTeam>::value ? prof_slots(E, tm, w) : nullptr);
        clk.mark(kPhBroadphase);
        const uint32_t n_cand = build_candidates(E, tm, W, S, n_pairs, sh);
        if (tm.leader())
        {
            S.misc[kMiscNPairs] = n_pairs;
            S.misc[kMiscNCand] = n_cand;
        }
        tm.sync();
        clk.mark(kPhCandidates);
    }

    // Narrowphase + contacts.clear() / emit (every substep, World.hpp:205-206).
    template <class T, class P, class Team>
    __device__ void phase_narrow(const Engine<T, P> &E, const Team &tm, uint32_t w)
    {
        const WorldDev W = E.worlds[w];
        const Scr<T, P> S = world_scratch(E, W);
        PhaseClock clk(prof_slots(E, tm, w), false);
        const uint32_t n_cand = S.misc[kMiscNCand];
        uint32_t n_gjk = 0;
        for (uint32_t c = tm.rank(); c < n_cand; c += tm.size())
            if (narrow_candidate(E, W, S.cand[c], S.cc[c]) == kNeedsGjk)
                queue_gjk(E, w, c, n_gjk);
        if (n_gjk)
            atomicAdd(S.misc + kMiscNGjk, n_gjk);
        tm.sync();
        clk.mark(kPhNarrow);
    }

    // Colouring of the contacting candidates (colored mode), then integrate
    // (Body.cpp:18-39).
    template <class T, class P, class Team>
    __device__ void phase_color_integrate(const Engine<T, P> &E, const Team &tm, uint32_t w, BlockShared &sh)
    {
        const WorldDev W = E.worlds[w];
        const Scr<T, P> S = world_scratch(E, W);
        PhaseClock clk(prof_slots(E, tm, w), false);
        if (E.solve_mode == 1)
        {
            const uint32_t nc = color_active(E, tm, W, S, S.misc[kMiscNCand], sh);
            if (tm.leader() && nc > S.misc[kMiscMaxColors])
                S.misc[kMiscMaxColors] = nc;
        }
        clk.mark(kPhColor);
        for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
            integrate_body(E.B, W.body_off + b, E.h);
        tm.sync();
        clk.mark(kPhIntegrate);
    }

    // Position solve (World.hpp:168-173): contacts, joint errors, joint rows;
    // then the velocity update (Body.cpp:41-57).  B is the body view the
    // team works on and boff the view index of the world's body 0
    // (W.body_off for the batch arrays, 0 for a shared-memory copy).
    // Relaxes colours [0, n) of a colour-ordered slot list (offsets off),
    // solve(q) per slot, with a team barrier after each colour.  On a grid
    // team the trailing colours of at most one CTA's worth of slots each run
    // on CTA 0 alone, separated by block barriers, and one grid barrier
    // follows them: a colour's slots share no dynamic body, so which threads
    // relax them does not change the result.  solve has one call site, so
    // the same machine code (and FP32 contraction) relaxes a slot either way.
    // Tangled worlds end in dozens of such colours (a body with 60 contacts
    // needs 60 colours, most of them nearly empty), and a grid barrier costs
    // several block barriers.
    template <class Team, class F>
    __device__ __forceinline__ void sweep_colors(const Team &tm, const uint32_t *off, uint32_t n, F &&solve)
    {
        constexpr bool kGrid = std::is_same<Team, GridTeam>::value;
        if constexpr (!kGrid)
        {
            // one CTA or one warp: every colour behind a team barrier (the
            // skip test for empty colours measured 0.4 % slower here)
            for (uint32_t col = 0; col < n; ++col)
            {
                for (uint32_t q = off[col] + tm.rank(); q < off[col + 1]; q += tm.size())
                    solve(q);
                tm.sync();
            }
            return;
        }
        uint32_t tail = n;
        if constexpr (kGrid)
            while (tail > 0 && off[tail] - off[tail - 1] <= blockDim.x)
                --tail;
        for (uint32_t col = 0; col < n; ++col)
        {
            if (off[col + 1] == off[col])
                continue;
            const bool on_cta = kGrid && col >= tail; // uniform over the team
            if (!on_cta || blockIdx.x == 0)
            {
                const uint32_t r = on_cta ? threadIdx.x : tm.rank(), step = on_cta ? blockDim.x : tm.size();
                for (uint32_t q = off[col] + r; q < off[col + 1]; q += step)
                    solve(q);
            }
            if (on_cta)
                __syncthreads();
            else
                tm.sync();
        }
        if (kGrid && tail < n)
            tm.sync();
    }

    template <class T, class P, class Team>
    __device__ void phase_position_on(const Engine<T, P> &E, const Team &tm, uint32_t w, const Bodies<T, P> &B,
                                      uint32_t boff, const uint32_t *book = nullptr, const uint2 *slots = nullptr)
    {
        const WorldDev W = E.worlds[w];
        const Scr<T, P> S = world_scratch(E, W);
        PhaseClock clk(prof_slots(E, tm, w), false);
        const uint32_t shift = W.body_off - boff; // joint body ids are batch-global
        const uint32_t n_cand = S.misc[kMiscNCand];
        if (E.solve_mode != 1)
        {
            if (tm.leader())
            {
                for (uint32_t c = 0; c < n_cand; ++c)
                {
                    const Cand cd = S.cand[c];
                    solve_pair_position(B, E.inv_h, boff + cd.ba, boff + cd.bb, S.cc[c]);
                }
                for (uint32_t j = 0; j < W.n_joints; ++j)
                {
                    Joint<T> jt = E.joints[W.joint_off + j];
                    jt.b1 -= shift;
                    jt.b2 -= shift;
                    joint_errors(B, jt, joint_rows(E, jt), E.h);
                    E.joints[W.joint_off + j].target_pos = jt.target_pos;
                }
                for (uint32_t j = 0; j < W.n_joints; ++j)
                {
                    Joint<T> jt = E.joints[W.joint_off + j];
                    jt.b1 -= shift;
                    jt.b2 -= shift;
                    solve_joint_rows(B, jt, joint_rows(E, jt), E.inv_h);
                }
            }
            tm.sync();
            clk.mark(kPhContactPos); // reference order: contacts and joints in one phase
        }
        else
        {
            const uint32_t *coff = book ? book + 66 : S.misc + kMiscCOff;
            const uint32_t n_colors = book ? book[132] : S.misc[kMiscNColors];
            const bool sl = slots && book && book[133];
            sweep_colors(tm, coff, n_colors, [&](uint32_t q) {
                uint32_t c, ba, bb;
                slot_entry(S, book, sl ? slots : nullptr, q, c, ba, bb);
                solve_pair_position(B, E.inv_h, boff + ba, boff + bb, S.cc[c]);
            });
            if (coff[kColorSerial + 1] > coff[kColorSerial])
            {
                // the overflow bucket: second-level colours (global misc),
                // then on one thread what is left
                const uint32_t *c2 = S.misc + kMiscC2Off;
                uint32_t serial0 = coff[kColorSerial];
                if (!book)
                {
                    sweep_colors(tm, c2, kColorSerial, [&](uint32_t q) {
                        const uint32_t c = S.corder[q];
                        const Cand cd = S.cand[c];
                        solve_pair_position(B, E.inv_h, boff + cd.ba, boff + cd.bb, S.cc[c]);
                    });
                    serial0 = c2[kColorSerial];
                }
                if (tm.leader())
                    for (uint32_t q = serial0; q < coff[kColorSerial + 1]; ++q)
                    {
                        const uint32_t c = sl ? slots[q].x : S.corder[q];
                        const Cand cd = S.cand[c];
                        solve_pair_position(B, E.inv_h, boff + cd.ba, boff + cd.bb, S.cc[c]);
                    }
                tm.sync();
            }
            clk.mark(kPhContactPos);
            if (W.n_joints)
            {
                for (uint32_t j = tm.rank(); j < W.n_joints; j += tm.size())
                {
                    Joint<T> jt = E.joints[W.joint_off + j];
                    jt.b1 -= shift;
                    jt.b2 -= shift;
                    joint_errors(B, jt, joint_rows(E, jt), E.h);
                    E.joints[W.joint_off + j].target_pos = jt.target_pos;
                }
                tm.sync();
                const uint32_t *jco = E.jcolor_off + W.jc_off;
                for (uint32_t jc = 0; jc < W.n_jcolors; ++jc)
                {
                    for (uint32_t q = jco[jc] + tm.rank(); q < jco[jc + 1]; q += tm.size())
                    {
                        Joint<T> jt = E.joints[W.joint_off + E.jorder[q]];
                        jt.b1 -= shift;
                        jt.b2 -= shift;
                        solve_joint_rows(B, jt, joint_rows(E, jt), E.inv_h);
                    }
                    tm.sync();
                }
            }
            clk.mark(kPhJointPos);
        }
        for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
            update_velocity_body(B, boff + b, E.inv_h);
        tm.sync();
        clk.mark(kPhVelUpdate);
    }

    template <class T, class P, class Team>
    __device__ void phase_position(const Engine<T, P> &E, const Team &tm, uint32_t w)
    {
        phase_position_on(E, tm, w, E.B, E.worlds[w].body_off);
    }

    // Velocity solve (World.hpp:176-180): restitution / friction, joint damping.
    template <class T, class P, class Team>
    __device__ void phase_velocity_on(const Engine<T, P> &E, const Team &tm, uint32_t w, const Bodies<T, P> &B,
                                      uint32_t boff, const uint32_t *book = nullptr, const uint2 *slots = nullptr)
    {
        const WorldDev W = E.worlds[w];
        const Scr<T, P> S = world_scratch(E, W);
        PhaseClock clk(prof_slots(E, tm, w), false);
        const uint32_t shift = W.body_off - boff;
        if (E.solve_mode != 1)
        {
            if (tm.leader())
            {
                const uint32_t n_cand = S.misc[kMiscNCand];
                for (uint32_t c = 0; c < n_cand; ++c)
                {
                    const Cand cd = S.cand[c];
                    solve_pair_velocity(B, E.h, boff + cd.ba, boff + cd.bb, S.cc[c]);
                }
                for (uint32_t j = 0; j < W.n_joints; ++j)
                {
                    Joint<T> jt = E.joints[W.joint_off + j];
                    jt.b1 -= shift;
                    jt.b2 -= shift;
                    joint_damping(B, jt, E.h);
                }
            }
            tm.sync();
        }
        else
        {
            const uint32_t *coff = book ? book + 66 : S.misc + kMiscCOff;
            const uint32_t n_colors = book ? book[132] : S.misc[kMiscNColors];
            const bool sl = slots && book && book[133];
            sweep_colors(tm, coff, n_colors, [&](uint32_t q) {
                uint32_t c, ba, bb;
                slot_entry(S, book, sl ? slots : nullptr, q, c, ba, bb);
                solve_pair_velocity(B, E.h, boff + ba, boff + bb, S.cc[c]);
            });
            if (coff[kColorSerial + 1] > coff[kColorSerial])
            {
                const uint32_t *c2 = S.misc + kMiscC2Off;
                uint32_t serial0 = coff[kColorSerial];
                if (!book)
                {
                    sweep_colors(tm, c2, kColorSerial, [&](uint32_t q) {
                        const uint32_t c = S.corder[q];
                        const Cand cd = S.cand[c];
                        solve_pair_velocity(B, E.h, boff + cd.ba, boff + cd.bb, S.cc[c]);
                    });
                    serial0 = c2[kColorSerial];
                }
                if (tm.leader())
                    for (uint32_t q = serial0; q < coff[kColorSerial + 1]; ++q)
                    {
                        const uint32_t c = sl ? slots[q].x : S.corder[q];
                        const Cand cd = S.cand[c];
                        solve_pair_velocity(B, E.h, boff + cd.ba, boff + cd.bb, S.cc[c]);
                    }
                tm.sync();
            }
            const uint32_t *jco = E.jcolor_off + W.jc_off;
            for (uint32_t jc = 0; jc < W.n_jcolors; ++jc)
            {
                for (uint32_t q = jco[jc] + tm.rank(); q < jco[jc + 1]; q += tm.size())
                {
                    Joint<T> jt = E.joints[W.joint_off + E.jorder[q]];
                    jt.b1 -= shift;
                    jt.b2 -= shift;
                    joint_damping(B, jt, E.h);
                }
                tm.sync();
            }
        }
        clk.mark(kPhVelSolve);
    }

    template <class T, class P, class Team>
    __device__ void phase_velocity(const Engine<T, P> &E, const Team &tm, uint32_t w)
    {
        phase_velocity_on(E, tm, w, E.B, E.worlds[w].body_off);
    }

    // Statistics and parity dumps of the last substep.
    template <class T, class P, class Team>
    __device__ void phase_stats(const Engine<T, P> &E, const Team &tm, uint32_t w)
    {
        const WorldDev W = E.worlds[w];
        const Scr<T, P> S = world_scratch(E, W);
        PhaseClock clk(prof_slots(E, tm, w), false);
        const bool colored = E.solve_mode == 1;
        const uint32_t n_cand = S.misc[kMiscNCand];
        uint32_t *ncon = S.misc + kMiscNContacts;
        if (tm.leader())
            *ncon = 0;
        tm.sync();
        uint32_t local = 0;
        for (uint32_t c = tm.rank(); c < n_cand; c += tm.size())
        {
            local += S.cc[c].n;
            if (E.dump_cc && W.dump_slot != ~0u && c < E.dump_cand_cap)
            {
                const size_t o = (size_t)W.dump_slot * E.dump_cand_cap + c;
                E.dump_cand[o] = S.cand[c];
                E.dump_cc[o] = S.cc[c];
                E.dump_color[o] = colored ? S.color[c] : 0u;
            }
        }
        if (local)
            atomicAdd(ncon, local);
        if (E.check_state)
        {
            // failure detection: a non-finite pose or velocity anywhere in
            // the world is reported with the world index (the reference has
            // no such check; its state just propagates the NaN)
            for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
            {
                const uint32_t g = W.body_off + b;
                const V4<P> x = E.B.pos[g];
                const Q4<T> q = E.B.rot[g];
                const V4<T> v = E.B.lin[g], om = E.B.ang[g];
                const bool ok = isfinite(x.x) && isfinite(x.y) && isfinite(x.z) && isfinite(q.w) && isfinite(q.x) &&
                                isfinite(q.y) && isfinite(q.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z) &&
                                isfinite(om.x) && isfinite(om.y) && isfinite(om.z);
                if (!ok)
                    set_error_at(E.error, kErrState, 7, w);
            }
        }
        tm.sync();
        if (tm.leader())
        {
            const uint32_t *coff = S.misc + kMiscCOff;
            WorldStats st;
            st.n_pairs = S.misc[kMiscNPairs];
            st.n_cand = n_cand;
            st.n_contacts = *ncon;
            st.n_colors = S.misc[kMiscMaxColors];
            st.n_serial = colored ? coff[kColorSerial + 1] - coff[kColorSerial] : 0u;
            st.n_gjk = S.misc[kMiscNGjk];
            st.pad_[0] = st.pad_[1] = 0;
            E.stats[w] = st;
        }
        tm.sync();
        clk.mark(kPhStats);
        clk.finish();
    }

    // ------------------------------------------------------------ kernels
    constexpr int kMaxBlock = 256;

    // Persistent CTAs pull small worlds (largest first) from a work counter
    // and run one phase on each.
    template <class F>
    __device__ __forceinline__ void each_small_world(const uint32_t *list, uint32_t n, uint32_t *counter, F &&f)
    {
        __shared__ uint32_t next;
        for (;;)
        {
            if (threadIdx.x == 0)
                next = atomicAdd(counter, 1u);
            __syncthreads();
            const uint32_t q = next;
            __syncthreads();
            if (q >= n)
                break;
            f(list[q]);
        }
    }

    // Resident 256-thread frame CTAs per SM the register allocation must
    // allow.  The count ptxas prints for the kernel leaves out its
    // non-inlined callees (the sort and sweep): unbounded, the kernel
    // launched at 150 registers, one CTA per SM.  Three CTAs (80 registers,
    // 36 bytes spilled) took a settled 4,096-world step from 8.05 to
    // 6.87 ms; four (64 registers) 6.95 ms.
#ifndef RBPS_FRAME_MIN_BLOCKS
#define RBPS_FRAME_MIN_BLOCKS 3
#endif
    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock, RBPS_FRAME_MIN_BLOCKS) k_phase_frame(const Engine<T, P> E, uint32_t ctr)
    {
        __shared__ BlockShared sh;
        __shared__ uint32_t sort_smem[kSmemSortWords];
        BlockTeam tm;
        each_small_world(E.small_worlds, E.n_small, E.work_counter + ctr,
                         [&](uint32_t w) { phase_frame(E, tm, w, sh, sort_smem); });
    }

    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_phase_narrow(const Engine<T, P> E, uint32_t ctr)
    {
        BlockTeam tm;
        each_small_world(E.small_worlds, E.n_small, E.work_counter + ctr, [&](uint32_t w) { phase_narrow(E, tm, w); });
    }

    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_phase_color(const Engine<T, P> E, uint32_t ctr)
    {
        __shared__ BlockShared sh;
        BlockTeam tm;
        each_small_world(E.small_worlds, E.n_small, E.work_counter + ctr,
                         [&](uint32_t w) { phase_color_integrate(E, tm, w, sh); });
    }

    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_phase_position(const Engine<T, P> E, uint32_t ctr)
    {
        BlockTeam tm;
        each_small_world(E.small_worlds, E.n_small, E.work_counter + ctr, [&](uint32_t w) { phase_position(E, tm, w); });
    }

    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_phase_velocity(const Engine<T, P> E, uint32_t ctr)
    {
        BlockTeam tm;
        each_small_world(E.small_worlds, E.n_small, E.work_counter + ctr, [&](uint32_t w) { phase_velocity(E, tm, w); });
    }

    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_phase_stats(const Engine<T, P> E, uint32_t ctr)
    {
        BlockTeam tm;
        each_small_world(E.small_worlds, E.n_small, E.work_counter + ctr, [&](uint32_t w) { phase_stats(E, tm, w); });
    }

    // One phase of one large world on the whole cooperative grid; the phases
    // are separate launches so that the GJK pass can run between the
    // narrowphase and the colouring, as it does for the small worlds.
    // Resident 256-thread CTAs per SM of the cooperative grid, as for the
    // frame: capped at 128 registers (two CTAs), collision stress went from
    // 7.45 to 6.53 ms a step and joint-heavy from 5.53 to 5.12 ms (same box);
    // three CTAs (80 registers) spilled: 6.52 and 5.69 ms.
#ifndef RBPS_BIG_MIN_BLOCKS
#define RBPS_BIG_MIN_BLOCKS 2
#endif
    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock, RBPS_BIG_MIN_BLOCKS) k_big_phase(const Engine<T, P> E, uint32_t w,
                                                                               int phase)
    {
        __shared__ BlockShared sh;
        GridTeam tm;
        switch (phase)
        {
        case kKFrame: phase_frame(E, tm, w, sh); break;
        case kKNarrow: phase_narrow(E, tm, w); break;
        case kKColor: phase_color_integrate(E, tm, w, sh); break;
        case kKPosition: phase_position(E, tm, w); break;
        case kKVelocity: phase_velocity(E, tm, w); break;
        default: phase_stats(E, tm, w); break;
        }
    }

    // Enqueues one step of every small world: 2 + 4 * substeps phase kernels
    // (work counters ctr_base .. ctr_base + 1 + 4 * substeps must be zero).
    template <class T, class P>
    cudaError_t launch_step_phases(const Engine<T, P> &e, const PhaseLaunch &pl, cudaStream_t stream)
    {
        uint32_t ctr = 0;
        k_phase_frame<T, P><<<pl.grid[kKFrame], pl.block[kKFrame], 0, stream>>>(e, ctr++);
        for (int s = 0; s < e.substeps; ++s)
        {
            if (e.gjk_list)
                cudaMemsetAsync(e.gjk_count, 0, 4, stream);
            k_phase_narrow<T, P><<<pl.grid[kKNarrow], pl.block[kKNarrow], 0, stream>>>(e, ctr++);
            launch_gjk(e, stream);
            k_phase_color<T, P><<<pl.grid[kKColor], pl.block[kKColor], 0, stream>>>(e, ctr++);
            k_phase_position<T, P><<<pl.grid[kKPosition], pl.block[kKPosition], 0, stream>>>(e, ctr++);
            k_phase_velocity<T, P><<<pl.grid[kKVelocity], pl.block[kKVelocity], 0, stream>>>(e, ctr++);
        }
        k_phase_stats<T, P><<<pl.grid[kKStats], pl.block[kKStats], 0, stream>>>(e, ctr++);
        return cudaGetLastError();
    }

    // ------------------------------------------------- batched colored pipeline
    // Colored mode over the small worlds, per step:
    //   k_phase_frame    one CTA per world: SAP update / sort / sweep, candidates
    //   k_flat_prefix    candidate prefix over the worlds
    //   k_type_count / k_type_scan / k_type_scatter
    //                    the candidates of all worlds sorted by shape pair, so a
    //                    warp of the narrowphase runs one pair routine
    // and per substep:
    //   k_flat_narrow    one thread per candidate, in shape-pair order; the
    //                    box-box class in k_flat_narrow_boxbox
    //   k_substep        one CTA per large world, one warp per other world:
    //                    greedy colouring of the contacting candidates, integrate,
    //                    position solve (colour by colour, joint errors, joint
    //                    colours), velocity update, velocity solve -- worlds
    //                    progress independently on their own team barriers
    // and last k_phase_stats.

    // Candidate prefix over the small worlds (one CTA).
    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_flat_prefix(const Engine<T, P> E)
    {
        __shared__ BlockShared sh;
        uint32_t carry = 0;
        for (uint32_t base = 0; base < E.n_small; base += blockDim.x)
        {
            const uint32_t q = base + threadIdx.x;
            uint32_t v = 0;
            if (q < E.n_small)
            {
                const WorldDev W = E.worlds[E.small_worlds[q]];
                v = world_scratch(E, W).misc[kMiscNCand];
            }
            uint32_t tot;
            const uint32_t ex = block_excl_scan(v, sh, &tot);
            if (q < E.n_small)
                E.wcoff[q] = carry + ex;
            carry += tot;
        }
        if (threadIdx.x == 0)
            E.wcoff[E.n_small] = carry;
    }

    // Shape-pair class of a candidate, 25 classes over (kind a, kind b) with
    // the kinds folded to sphere, box, capsule, plane and "other": the 16
    // pairs of the four common kinds first (ia * 4 + ib; box-box is 5), then
    // the pairs with an other kind (16-20 other first, 21-24 other second),
    // so one kernel takes [0, 16) but box-box and another [16, 25).
    __device__ __forceinline__ uint32_t kind_index(int kind)
    {
        return kind == kSphere ? 0u : kind == kBox ? 1u : kind == kCapsule ? 2u : kind == kPlane ? 3u : 4u;
    }
    constexpr uint32_t kClassBoxBox = 1u * 4u + 1u; // cand_class of a box-box pair
    constexpr uint32_t kClassCommonEnd = 16u;        // classes [0, 16): common kinds only

    __device__ __forceinline__ uint32_t pair_class(uint32_t ia, uint32_t ib)
    {
        if (ia < 4u && ib < 4u)
            return ia * 4u + ib;
        return ia == 4u ? 16u + ib : 21u + ia;
    }

    // The small world holding flat candidate f: last q with wcoff[q] <= f.
    template <class T, class P>
    __device__ __forceinline__ uint32_t world_of_flat(const Engine<T, P> &E, uint32_t f)
    {
        uint32_t lo = 0, hi = E.n_small;
        while (hi - lo > 1)
        {
            const uint32_t mid = (lo + hi) >> 1;
            if (E.wcoff[mid] <= f)
                lo = mid;
            else
                hi = mid;
        }
        return lo;
    }

    template <class T, class P>
    __device__ __forceinline__ uint32_t cand_class(const Engine<T, P> &E, const WorldDev &W, const Cand &cd)
    {
        return pair_class(kind_index(E.shape[W.coll_off + cd.ca].kind), kind_index(E.shape[W.coll_off + cd.cb].kind));
    }

    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_type_count(const Engine<T, P> E)
    {
        __shared__ uint32_t cnt[kPairClasses];
        for (uint32_t k = threadIdx.x; k < kPairClasses; k += blockDim.x)
            cnt[k] = 0;
        __syncthreads();
        const uint32_t total = E.wcoff[E.n_small];
        for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x)
        {
            const uint32_t q = world_of_flat(E, f);
            const uint32_t w = E.small_worlds[q];
            const WorldDev W = E.worlds[w];
            atomicAdd(&cnt[cand_class(E, W, E.wcand[w][f - E.wcoff[q]])], 1u);
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < kPairClasses; k += blockDim.x)
            if (cnt[k])
                atomicAdd(&E.gcol[kGcolCount + k], cnt[k]);
    }

    // Class offsets; zeroes the counts for the next step and the cursors.
    template <class T, class P>
    __global__ void k_type_scan(const Engine<T, P> E)
    {
        if (threadIdx.x != 0)
            return;
        uint32_t run = 0;
        for (uint32_t k = 0; k < kPairClasses; ++k)
        {
            const uint32_t n = E.gcol[kGcolCount + k];
            E.gcol[kGcolOff + k] = run;
            E.gcol[kGcolFill + k] = 0u;
            E.gcol[kGcolCount + k] = 0u;
            run += n;
        }
        E.gcol[kGcolOff + kPairClasses] = run;
    }

    // Each CTA takes a contiguous chunk of flat candidates, counts its
    // classes in shared memory, reserves its ranges with one global atomic
    // per class, then places its candidates.
    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_type_scatter(const Engine<T, P> E)
    {
        __shared__ uint32_t cnt[kPairClasses], base[kPairClasses];
        const uint32_t total = E.wcoff[E.n_small];
        const uint32_t chunk = (total + gridDim.x - 1) / gridDim.x;
        const uint32_t f0 = blockIdx.x * chunk;
        const uint32_t f1 = min(total, f0 + chunk);
        for (uint32_t k = threadIdx.x; k < kPairClasses; k += blockDim.x)
            cnt[k] = 0;
        __syncthreads();
        for (uint32_t f = f0 + threadIdx.x; f < f1; f += blockDim.x)
        {
            const uint32_t q = world_of_flat(E, f);
            const uint32_t w = E.small_worlds[q];
            atomicAdd(&cnt[cand_class(E, E.worlds[w], E.wcand[w][f - E.wcoff[q]])], 1u);
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < kPairClasses; k += blockDim.x)
        {
            base[k] = cnt[k] ? E.gcol[kGcolOff + k] + atomicAdd(&E.gcol[kGcolFill + k], cnt[k]) : 0u;
            cnt[k] = 0;
        }
        __syncthreads();
        for (uint32_t f = f0 + threadIdx.x; f < f1; f += blockDim.x)
        {
            const uint32_t q = world_of_flat(E, f);
            const uint32_t w = E.small_worlds[q];
            const uint32_t c = f - E.wcoff[q];
            const WorldDev W = E.worlds[w];
            const Cand cd = E.wcand[w][c];
            const uint32_t k = cand_class(E, W, cd);
            const uint32_t slot = base[k] + atomicAdd(&cnt[k], 1u);
            E.nlist[slot] = make_uint2(w, c);
            // the global collider and body indices, so the narrowphase reads
            // them with its entry instead of through the world and candidate
            // (checked here, once a step, instead of every substep)
            uint4 g = make_uint4(~0u, ~0u, ~0u, ~0u);
            if (cd.ca < W.n_coll && cd.cb < W.n_coll && cd.ba < W.n_bodies && cd.bb < W.n_bodies)
                g = make_uint4(W.coll_off + cd.ca, W.coll_off + cd.cb, W.body_off + cd.ba, W.body_off + cd.bb);
            else
                set_error_at(E.error, kErrInternal, 3, cd.ca);
            E.nglob[slot] = g;
        }
    }

    // Narrowphase of flat entry i of the class-sorted candidate list of the
    // small worlds.
    template <class T, class P, int Sel>
    __device__ __forceinline__ void narrow_flat(const Engine<T, P> &E, uint32_t i)
    {
        const uint2 e = E.nlist[i];
        const uint4 g = E.nglob[i];
        CandContacts<T, P> &out = E.wcc[e.x][e.y];
        if (g.x == ~0u) // a corrupt candidate, reported by the class sort
        {
            out.n = 0;
            return;
        }
        if (narrow_pair<T, P, Sel>(E, g.x, g.y, g.z, g.w, out) == kNeedsGjk)
        {
            uint32_t n_gjk = 0;
            queue_gjk(E, e.x, e.y, n_gjk);
            atomicAdd(world_scratch(E, E.worlds[e.x]).misc + kMiscNGjk, n_gjk);
        }
    }

    // Narrowphase of every candidate of the small worlds but the box-box
    // ones, in class order.
    // Entries [0, n) of a class-sorted range are dealt to the grid's warps
    // in chunks of E.narrow_per_warp (a multiple of 32) consecutive entries,
    // a lane taking every 32nd entry of its warp's chunk; 32 is the plain
    // grid-stride loop.  (Written out in each kernel: a helper taking the
    // kernel's Engine by reference inside a lambda made the compiler copy
    // the whole parameter block to the stack, 650 bytes a thread.)
    // Resident 256-thread narrowphase CTAs per SM, both kernels.  Unbounded,
    // k_flat_narrow launched at 162 registers (one CTA per SM) and the
    // box-box kernel at 87 (two); at three each (80 registers) the step
    // above went from 6.87 to 6.64 ms.
#ifndef RBPS_NARROW_MIN_BLOCKS
#define RBPS_NARROW_MIN_BLOCKS 3
#endif
    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock, RBPS_NARROW_MIN_BLOCKS) k_flat_narrow(const Engine<T, P> E)
    {
        // the common-kind classes but box-box: [0, off(bb)) and [off(bb + 1), off(16))
        const uint32_t total = E.gcol[kGcolOff + kClassCommonEnd];
        const uint32_t bb0 = E.gcol[kGcolOff + kClassBoxBox], bb1 = E.gcol[kGcolOff + kClassBoxBox + 1];
        const uint32_t n = total - (bb1 - bb0);
        const uint32_t per_warp = E.narrow_per_warp, lane = threadIdx.x & 31u;
        const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
        for (uint32_t base = warp * per_warp; base < n; base += n_warps * per_warp)
        {
            const uint32_t end = min(n, base + per_warp);
            for (uint32_t k = base + lane; k < end; k += 32)
                narrow_flat<T, P, kSelCommon>(E, k < bb0 ? k : k + (bb1 - bb0));
        }
    }

    // The classes with any other kind (ellipsoid, cylinder, cone, hull,
    // heightmap, mesh): [off(16), total), with every routine but box-box.
    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock, RBPS_NARROW_MIN_BLOCKS) k_flat_narrow_other(const Engine<T, P> E)
    {
        const uint32_t o0 = E.gcol[kGcolOff + kClassCommonEnd], total = E.gcol[kGcolOff + kPairClasses];
        const uint32_t n = total - o0;
        const uint32_t per_warp = E.narrow_per_warp, lane = threadIdx.x & 31u;
        const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
        for (uint32_t base = warp * per_warp; base < n; base += n_warps * per_warp)
        {
            const uint32_t end = min(n, base + per_warp);
            for (uint32_t k = base + lane; k < end; k += 32)
                narrow_flat<T, P, kSelNoBoxBox>(E, o0 + k);
        }
    }

    // The box-box class on its own: its SAT, clipping buffers and registers
    // stay out of the kernel that runs every other class.
    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock, RBPS_NARROW_MIN_BLOCKS) k_flat_narrow_boxbox(const Engine<T, P> E)
    {
        const uint32_t bb0 = E.gcol[kGcolOff + kClassBoxBox], bb1 = E.gcol[kGcolOff + kClassBoxBox + 1];
        const uint32_t n = bb1 - bb0;
        const uint32_t per_warp = E.narrow_per_warp, lane = threadIdx.x & 31u;
        const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
        for (uint32_t base = warp * per_warp; base < n; base += n_warps * per_warp)
        {
            const uint32_t end = min(n, base + per_warp);
            for (uint32_t k = base + lane; k < end; k += 32)
                narrow_flat<T, P, kSelBoxBox>(E, bb0 + k);
        }
    }

    // The rest of a substep for one world per warp: colouring, integrate
    // (Body.cpp:18-39), position solve + velocity update, velocity solve.
    // The contacting candidates of world W into S.alist, in candidate
    // order; returns their count to every thread of the team.
    // Compaction of candidate indices [0, n_cand) for which sel(c) holds into
    // out[0, count), in candidate order; returns the count to every thread.
    template <class F>
    __device__ __forceinline__ uint32_t team_compact(const WarpTeam &, uint32_t n_cand, uint32_t *out, ScanShared &,
                                                     F &&sel)
    {
        const uint32_t lane = lane_id(), lt = (1u << lane) - 1u;
        uint32_t n = 0;
        for (uint32_t base = 0; base < n_cand; base += 32)
        {
            const uint32_t c = base + lane;
            const bool take = c < n_cand && sel(c);
            const uint32_t m = __ballot_sync(0xffffffffu, take);
            if (take)
                out[n + __popc(m & lt)] = c;
            n += __popc(m);
        }
        __syncwarp();
        return n;
    }

    // A pair team's two warps exchange their counts through the CTA's scan
    // words 2h and 2h + 1 (the other half uses the other two).
    template <class F>
    __device__ __forceinline__ uint32_t team_compact(const PairTeam &tm, uint32_t n_cand, uint32_t *out,
                                                     ScanShared &sh, F &&sel)
    {
        const uint32_t lane = lane_id(), lt = (1u << lane) - 1u;
        const uint32_t w = (threadIdx.x >> 5) & 1u, slot = 2u * tm.half();
        uint32_t n = 0;
        for (uint32_t base = 0; base < n_cand; base += 64)
        {
            const uint32_t c = base + tm.rank();
            const bool take = c < n_cand && sel(c);
            const uint32_t m = __ballot_sync(0xffffffffu, take);
            if (lane == 0)
                sh.warp[slot + w] = __popc(m);
            tm.sync();
            const uint32_t below = w ? sh.warp[slot] : 0u;
            const uint32_t tot = sh.warp[slot] + sh.warp[slot + 1];
            if (take)
                out[n + below + __popc(m & lt)] = c;
            n += tot;
            tm.sync();
        }
        return n;
    }

    template <class F>
    __device__ __forceinline__ uint32_t team_compact(const BlockTeam &, uint32_t n_cand, uint32_t *out, ScanShared &sh,
                                                     F &&sel)
    {
        uint32_t n = 0;
        for (uint32_t base = 0; base < n_cand; base += blockDim.x)
        {
            const uint32_t c = base + threadIdx.x;
            const bool take = c < n_cand && sel(c);
            uint32_t tot;
            const uint32_t ex = block_excl_scan(take ? 1u : 0u, sh, &tot);
            if (take)
                out[n + ex] = c;
            n += tot;
        }
        __syncthreads();
        return n;
    }

    // The contacting candidates of the world into S.alist, in candidate
    // order, their colours reset; the others marked idle.  Returns the count;
    // adds this thread's share of the contact rows to *rows.
    template <class T, class P, class Team>
    __device__ uint32_t compact_active(const Team &tm, const Scr<T, P> &S, uint32_t n_cand, ScanShared &sh,
                                       uint32_t *rows)
    {
        return team_compact(tm, n_cand, S.alist, sh, [&](uint32_t c) {
            const int n = S.cc[c].n;
            *rows += (uint32_t)n;
            const bool act = n > 0;
            S.color[c] = act ? 0xffffffffu : kColorIdle;
            return act;
        });
    }

    // Substeps after the first of a step reuse the colouring: a candidate
    // that is still contacting keeps its colour (a regular one), and goes to
    // S.alist[0, *n_keep); the newly contacting ones (and those of the
    // overflow colour) follow in candidate order with their colour reset;
    // the rest are marked idle.  The kept candidates still share no dynamic
    // body within a colour, so first-fit colouring of the new ones against
    // the kept ones' body masks gives a valid colouring again.  Returns the
    // total count.
    template <class T, class P, class Team>
    __device__ uint32_t compact_keep_active(const Team &tm, const Scr<T, P> &S, uint32_t n_cand, ScanShared &sh,
                                            uint32_t *n_keep, uint32_t *rows)
    {
        const uint32_t kept = team_compact(tm, n_cand, S.alist, sh, [&](uint32_t c) {
            const int n = S.cc[c].n;
            *rows += (uint32_t)n;
            const bool act = n > 0;
            const uint32_t old = S.color[c];
            const bool keep = act && old < kColorSerial;
            S.color[c] = keep ? old : act ? 0xffffffffu : kColorIdle;
            return keep;
        });
        const uint32_t fresh =
            team_compact(tm, n_cand, S.alist + kept, sh, [&](uint32_t c) { return S.color[c] == 0xffffffffu; });
        *n_keep = kept;
        return kept + fresh;
    }

    // Greedy colouring of the world's contacting candidates: in candidate
    // order, each takes the lowest colour free on both of its dynamic bodies
    // (kColorSerial once a body has used all 64).  The team leader colours
    // sequentially with the per-body colour masks in `mask` (shared memory
    // when the world fits); the team then buckets the candidates by colour
    // (corder, colour offsets in misc).  The first substep of a step colours
    // every contacting candidate so; later substeps of the same step keep
    // the colours of the candidates still contacting (their masks are set
    // in parallel) and colour only the newly contacting ones first-fit
    // against them, which on resting piles leaves the leader a few
    // candidates instead of all.  Returns the number of regular colours to
    // every thread.
    // The greedy pass over one staged chunk on the team's first warp, with
    // the serial pass's result.  Candidates are taken 32 at a time; in rounds,
    // every candidate none of whose dynamic bodies belongs to an earlier
    // uncoloured candidate of its 32 takes the lowest colour free on its
    // bodies.  It sees exactly the masks the serial pass would: every earlier
    // candidate on those bodies is coloured, no later one is.  Candidates
    // coloured in one round share no dynamic body, and the earliest
    // uncoloured one is always ready, so at most 32 rounds run.  claim holds
    // a word per body of scratch (the lowest uncoloured lane on the body).
    __device__ __forceinline__ void greedy_chunk_warp(const uint32_t *stage, uint8_t *scol, uint32_t m,
                                                      unsigned long long *mask, uint32_t *cnt, uint32_t *claim)
    {
        const uint32_t lane = threadIdx.x & 31u;
        for (uint32_t k0 = 0; k0 < m; k0 += 32)
        {
            const uint32_t k = k0 + lane;
            const bool live = k < m;
            const uint32_t r = live ? stage[k] : 0u;
            const uint32_t a = r & 2047u, b = (r >> 11) & 2047u;
            const bool da = live && ((r >> 22) & 1u), db = live && ((r >> 23) & 1u);
            bool pending = live;
            while (__any_sync(0xffffffffu, pending))
            {
                if (pending)
                {
                    if (da)
                        claim[a] = ~0u;
                    if (db)
                        claim[b] = ~0u;
                }
                __syncwarp();
                if (pending)
                {
                    if (da)
                        atomicMin(&claim[a], lane);
                    if (db)
                        atomicMin(&claim[b], lane);
                }
                __syncwarp();
                if (pending && (!da || claim[a] == lane) && (!db || claim[b] == lane))
                {
                    const unsigned long long used = (da ? mask[a] : 0ull) | (db ? mask[b] : 0ull);
                    uint32_t col = kColorSerial;
                    if (used != ~0ull)
                    {
                        col = (uint32_t)(__ffsll((long long)~used) - 1);
                        const unsigned long long bit = 1ull << col;
                        if (da)
                            mask[a] |= bit;
                        if (db)
                            mask[b] |= bit;
                    }
                    scol[k] = (uint8_t)col;
                    atomicAdd(&cnt[col], 1u);
                    pending = false;
                }
                __syncwarp();
            }
        }
    }

    template <class T, class P, class Team>
    __device__ uint32_t greedy_color_world(const Engine<T, P> &E, const Team &tm, uint32_t w,
                                           unsigned long long *mask, ScanShared &sh, uint32_t *book,
                                           uint32_t *stage = nullptr, uint32_t *claim = nullptr,
                                           uint2 *slots = nullptr, uint32_t slot_cap = 0)
    {
        const WorldDev W = E.worlds[w];
        const Scr<T, P> S = world_scratch(E, W);
        uint32_t *misc = S.misc;
        // colour counts / fill cursors and offsets: the team's shared block
        // when it has one, else the world's misc words
        uint32_t *cnt = book ? book : misc + kMiscCCount;
        uint32_t *off = book ? book + 66 : misc + kMiscCOff;
        const uint32_t n_cand = misc[kMiscNCand];
        for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
            mask[b] = 0ull;
        for (uint32_t k = tm.rank(); k < 66; k += tm.size())
            cnt[k] = 0u;
        // after the first substep of a step the colouring of the same
        // candidate list is reused: kept candidates first, then the new ones
#ifndef RBPS_COLOR_REUSE
#define RBPS_COLOR_REUSE 1
#endif
        const bool reuse = RBPS_COLOR_REUSE && misc[kMiscColorValid] != 0u;
        uint32_t n_keep = 0, rows = 0;
        if (tm.leader())
            misc[kMiscNContacts] = 0u; // this substep's contact rows, summed below
        const uint32_t n_act = reuse ? compact_keep_active(tm, S, n_cand, sh, &n_keep, &rows)
                                     : compact_active(tm, S, n_cand, sh, &rows);
        if (rows) // after the compaction's closing barrier, so after the reset
            atomicAdd(misc + kMiscNContacts, rows);
        const uint8_t *type = E.B.type + W.body_off;
        for (uint32_t q = tm.rank(); q < n_keep; q += tm.size())
        {
            const uint32_t c = S.alist[q];
            const uint32_t col = S.color[c];
            const Cand cd = S.cand[c];
            const unsigned long long bit = 1ull << col;
            if (type[cd.ba] == kDynamic)
                atomicOr(&mask[cd.ba], bit);
            if (type[cd.bb] == kDynamic)
                atomicOr(&mask[cd.bb], bit);
            atomicAdd(&cnt[col], 1u);
        }
        tm.sync();
        if (stage)
        {
            // Staged: the team loads a chunk of active candidates into shared
            // memory at once, as packed (a, b, dynamic a, dynamic b) records
            // (world-local body indices < 2048), so the leader's greedy pass
            // -- the same candidates in the same order -- touches shared
            // memory only.
            uint8_t *scol = reinterpret_cast<uint8_t *>(stage + kColorStage);
            const uint32_t chunk = E.color_chunk; // <= kColorStage
            for (uint32_t q0 = n_keep; q0 < n_act; q0 += chunk)
            {
                const uint32_t m = min(chunk, n_act - q0);
                for (uint32_t k = tm.rank(); k < m; k += tm.size())
                {
                    const Cand cd = S.cand[S.alist[q0 + k]];
                    stage[k] = (cd.ba & 2047u) | ((cd.bb & 2047u) << 11) |
                               ((type[cd.ba] == kDynamic ? 1u : 0u) << 22) |
                               ((type[cd.bb] == kDynamic ? 1u : 0u) << 23);
                }
                tm.sync();
                if (claim)
                {
                    if (tm.rank() < 32)
                        greedy_chunk_warp(stage, scol, m, mask, cnt, claim);
                }
                else if (tm.leader())
                    for (uint32_t k = 0; k < m; ++k)
                    {
                        const uint32_t r = stage[k];
                        const uint32_t a = r & 2047u, b = (r >> 11) & 2047u;
                        const bool da = (r >> 22) & 1u, db = (r >> 23) & 1u;
                        const unsigned long long used = (da ? mask[a] : 0ull) | (db ? mask[b] : 0ull);
                        uint32_t col = kColorSerial;
                        if (used != ~0ull)
                        {
                            col = (uint32_t)(__ffsll((long long)~used) - 1);
                            const unsigned long long bit = 1ull << col;
                            if (da)
                                mask[a] |= bit;
                            if (db)
                                mask[b] |= bit;
                        }
                        scol[k] = (uint8_t)col;
                        cnt[col] += 1u;
                    }
                tm.sync();
                for (uint32_t k = tm.rank(); k < m; k += tm.size())
                    S.color[S.alist[q0 + k]] = scol[k];
            }
        }
        if (tm.leader())
        {
            constexpr uint32_t kAhead = 8; // candidates loaded ahead of the mask updates
            for (uint32_t q0 = n_keep; q0 < (stage ? 0u : n_act); q0 += kAhead)
            {
                uint32_t cs[kAhead];
                Cand cd[kAhead];
                bool da[kAhead], db[kAhead];
#pragma unroll
                for (uint32_t k = 0; k < kAhead; ++k)
                    if (q0 + k < n_act)
                    {
                        cs[k] = S.alist[q0 + k];
                        cd[k] = S.cand[cs[k]];
                        da[k] = type[cd[k].ba] == kDynamic;
                        db[k] = type[cd[k].bb] == kDynamic;
                    }
#pragma unroll
                for (uint32_t k = 0; k < kAhead; ++k)
                    if (q0 + k < n_act)
                    {
                        const unsigned long long used = (da[k] ? mask[cd[k].ba] : 0ull) | (db[k] ? mask[cd[k].bb] : 0ull);
                        uint32_t col = kColorSerial;
                        if (used != ~0ull)
                        {
                            col = (uint32_t)(__ffsll((long long)~used) - 1);
                            const unsigned long long bit = 1ull << col;
                            if (da[k])
                                mask[cd[k].ba] |= bit;
                            if (db[k])
                                mask[cd[k].bb] |= bit;
                        }
                        S.color[cs[k]] = col;
                        cnt[col] += 1u;
                    }
            }
            uint32_t run = 0, ncol = 0;
            for (uint32_t k = 0; k <= kColorSerial; ++k)
            {
                const uint32_t n = cnt[k];
                off[k] = run;
                cnt[k] = run; // becomes the fill cursor
                if (n && k < kColorSerial)
                    ncol = k + 1;
                run += n;
            }
            off[kColorSerial + 1] = run;
            misc[kMiscNColors] = ncol;
            if (ncol > misc[kMiscMaxColors])
                misc[kMiscMaxColors] = ncol;
            misc[kMiscColorValid] = 1u;
            if (book)
            {
                book[132] = ncol;
                book[133] = slots && n_act <= slot_cap ? 1u : 0u;
            }
        }
        tm.sync();
        // the colour-ordered slots go to shared memory when they fit
        const bool in_smem = slots && n_act <= slot_cap;
        for (uint32_t q = tm.rank(); q < n_act; q += tm.size())
        {
            const uint32_t c = S.alist[q];
            const uint32_t slot = atomicAdd(&cnt[S.color[c]], 1u);
            // a team with its world in shared memory keeps the body pair of
            // each slot beside its candidate (world-local indices < 65536), so
            // the colour-by-colour solves need not read the candidate first
            if (in_smem)
            {
                const Cand cd = S.cand[c];
                slots[slot] = make_uint2(c, cd.ba | (cd.bb << 16));
            }
            else
            {
                S.corder[slot] = c;
                if (book)
                {
                    const Cand cd = S.cand[c];
                    S.act[slot] = cd.ba | (cd.bb << 16);
                }
            }
            // the position and velocity solves read this candidate's contact
            // block colour by colour, each read behind a barrier: start it
            // on its way to L2 now, while integrate runs
            prefetch_l2_range(S.cc + c, sizeof(CandContacts<T, P>));
        }
        if (book) // the offsets also go to misc for the statistics and dumps
            for (uint32_t k = tm.rank(); k < 66; k += tm.size())
                misc[kMiscCOff + k] = off[k];
        tm.sync();
        if (!book) // the solves then take the overflow bucket by second-level colours
            color_overflow(E, tm, W, S);
        return book ? book[132] : misc[kMiscNColors];
    }

// Resident 128-thread CTAs per SM the registers must allow (128 registers a
// thread at 4).  Measured on the batched workload (4,096 worlds, settled):
// 3 CTAs (168 registers) 7.58 ms a step, 4 CTAs with the previous pose in
// shared memory (which then does not fit four) 7.89, 4 CTAs with it in
// place 7.16, 5 CTAs (96 registers, heavy spills) 7.40.
#ifndef RBPS_SUBSTEP_MIN_BLOCKS
#define RBPS_SUBSTEP_MIN_BLOCKS 4
#endif
    // The rest of a substep for every small world: colouring, integrate
    // (Body.cpp:18-39), position solve + velocity update, velocity solve.
    // The largest worlds (the first n_block_worlds of the list) get a whole
    // CTA each; the others one warp each, four per CTA.  Worlds progress
    // independently: a barrier is the team's own.
    // A team's copy of its world in shared memory: 136 words of colour
    // bookkeeping (counts / cursors, offsets, colour count), then per body
    // the colour mask, pose, previous pose and velocities, and the type;
    // `cap` bodies per array (cap a multiple of 16 keeps every array 16-byte
    // aligned).  Force, torque and the inertia tensors are read in place
    // through the batch arrays offset to the world.
// The previous pose (written once by integrate, read by the friction rows
// and the velocity update) stays in the batch arrays by default: without it
// a 512-body world's shared copy fits four 128-thread CTAs on an SM (see
// RBPS_SUBSTEP_MIN_BLOCKS).  1 keeps it in the shared copy too.
#ifndef RBPS_SMEM_PREV
#define RBPS_SMEM_PREV 0
#endif
    template <class T, class P>
    struct SmemWorld
    {
        static constexpr size_t kBook = 136 * sizeof(uint32_t);
        // colouring stage: kColorStage packed candidate records + their colours
        static constexpr size_t kStage = kColorStage * (sizeof(uint32_t) + 1);
        static constexpr bool kPrev = RBPS_SMEM_PREV != 0;
        // colour-ordered slots (candidate, packed body pair) for up to
        // kSlotsPerBody x cap contacting candidates
        static constexpr uint32_t kSlotsPerBody = 2;
        static constexpr size_t kPerBody = sizeof(unsigned long long) + (kPrev ? 2 : 1) * sizeof(V4<P>) +
                                           (kPrev ? 2 : 1) * sizeof(Q4<T>) + 2 * sizeof(V4<T>) + 1 +
                                           kSlotsPerBody * sizeof(uint2);

        __host__ __device__ static size_t bytes(uint32_t cap) { return kBook + kStage + (size_t)cap * kPerBody; }

        __device__ static Bodies<T, P> view(unsigned char *p, uint32_t cap, const Bodies<T, P> &G, uint32_t body_off,
                                            unsigned long long **mask, uint32_t **book, uint32_t **stage, uint2 **slots)
        {
            *book = reinterpret_cast<uint32_t *>(p);
            p += kBook;
            *stage = reinterpret_cast<uint32_t *>(p);
            p += kStage;
            *slots = reinterpret_cast<uint2 *>(p);
            p += (size_t)cap * kSlotsPerBody * sizeof(uint2);
            *mask = reinterpret_cast<unsigned long long *>(p);
            p += (size_t)cap * sizeof(unsigned long long);
            Bodies<T, P> V;
            V.pos = reinterpret_cast<V4<P> *>(p);
            p += (size_t)cap * sizeof(V4<P>);
            V.rot = reinterpret_cast<Q4<T> *>(p);
            p += (size_t)cap * sizeof(Q4<T>);
            if (kPrev)
            {
                V.prev_pos = reinterpret_cast<V4<P> *>(p);
                p += (size_t)cap * sizeof(V4<P>);
                V.prev_rot = reinterpret_cast<Q4<T> *>(p);
                p += (size_t)cap * sizeof(Q4<T>);
            }
            else
            {
                V.prev_pos = G.prev_pos + body_off;
                V.prev_rot = G.prev_rot + body_off;
            }
            V.lin = reinterpret_cast<V4<T> *>(p);
            p += (size_t)cap * sizeof(V4<T>);
            V.ang = reinterpret_cast<V4<T> *>(p);
            p += (size_t)cap * sizeof(V4<T>);
            V.type = p;
            V.force = G.force + body_off;
            V.torque = G.torque + body_off;
            V.inertia = G.inertia + body_off;
            V.inv_inertia = G.inv_inertia + body_off;
            return V;
        }
    };

    // The statistics of a colored step, run by the last substep when no dump
    // needs the stats phase (phase_stats, which it replaces): the state check
    // on the world's bodies as the substep leaves them (the shared copy, or
    // the batch arrays), then WorldStats from the counters the step kept
    // (the contact rows are those the colouring counted this substep).
    template <class T, class P, class Team>
    __device__ void substep_stats(const Engine<T, P> &E, const Team &tm, uint32_t w, const Bodies<T, P> &V,
                                  uint32_t boff)
    {
        const WorldDev W = E.worlds[w];
        if (E.check_state)
            for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
            {
                const V4<P> x = V.pos[boff + b];
                const Q4<T> q = V.rot[boff + b];
                const V4<T> v = V.lin[boff + b], om = V.ang[boff + b];
                const bool ok = isfinite(x.x) && isfinite(x.y) && isfinite(x.z) && isfinite(q.w) && isfinite(q.x) &&
                                isfinite(q.y) && isfinite(q.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z) &&
                                isfinite(om.x) && isfinite(om.y) && isfinite(om.z);
                if (!ok)
                    set_error_at(E.error, kErrState, 7, w);
            }
        if (tm.leader())
        {
            const uint32_t *misc = world_scratch(E, W).misc;
            WorldStats st;
            st.n_pairs = misc[kMiscNPairs];
            st.n_cand = misc[kMiscNCand];
            st.n_contacts = misc[kMiscNContacts];
            st.n_colors = misc[kMiscMaxColors];
            st.n_serial = misc[kMiscCOff + kColorSerial + 1] - misc[kMiscCOff + kColorSerial];
            st.n_gjk = misc[kMiscNGjk];
            st.pad_[0] = st.pad_[1] = 0;
            E.stats[w] = st;
        }
        tm.sync();
    }

    // The rest of a substep for one world on team tm: colouring of the
    // contacting candidates, integrate (Body.cpp:18-39), position solve +
    // velocity update, velocity solve.  With `smem` (room for `cap` bodies)
    // and a world that fits, the bodies live in shared memory for the whole
    // substep and are written back once.
    template <class T, class P, class Team>
    __device__ void substep_world(const Engine<T, P> &E, const Team &tm, uint32_t w, unsigned char *smem,
                                  uint32_t cap, ScanShared &sh)
    {
        const WorldDev W = E.worlds[w];
        const bool local = smem && W.n_bodies <= cap;
        unsigned long long *mask = nullptr;
        uint32_t *book = nullptr, *stage = nullptr;
        uint2 *slots = nullptr;
        Bodies<T, P> V = E.B;
        uint32_t boff = W.body_off;
        if (local)
        {
            V = SmemWorld<T, P>::view(smem, cap, E.B, W.body_off, &mask, &book, &stage, &slots);
            boff = 0;
        }
        else
            mask = world_scratch(E, W).bmask;
        PhaseClock clk(prof_slots(E, tm, w), false);
        // the pose copy is not loaded yet: its first words serve the
        // colouring as per-body scratch
        greedy_color_world(E, tm, w, mask, sh, book, stage, local ? reinterpret_cast<uint32_t *>(V.pos) : nullptr, slots,
                           cap * SmemWorld<T, P>::kSlotsPerBody);
        clk.mark(kPhColor);
        // integrate (Body.cpp:18-39); a world in shared memory is loaded
        // into its copy by the same pass
        for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
            if (local)
                integrate_body_into(E.B, W.body_off + b, V, b, E.h);
            else
                integrate_body(V, boff + b, E.h);
        tm.sync();
        clk.mark(kPhIntegrate);
        phase_position_on(E, tm, w, V, boff, book, slots);
        phase_velocity_on(E, tm, w, V, boff, book, slots);
        if (local)
        {
            const Bodies<T, P> &G = E.B;
            for (uint32_t b = tm.rank(); b < W.n_bodies; b += tm.size())
            {
                if (V.type[b] == kStatic)
                    continue;
                const uint32_t g = W.body_off + b;
                G.pos[g] = V.pos[b];
                G.rot[g] = V.rot[b];
                G.lin[g] = V.lin[b];
                G.ang[g] = V.ang[b];
                if (SmemWorld<T, P>::kPrev)
                {
                    G.prev_pos[g] = V.prev_pos[b];
                    G.prev_rot[g] = V.prev_rot[b];
                }
            }
            tm.sync();
        }
        if (E.stats_in_substep)
        {
            PhaseClock sclk(prof_slots(E, tm, w), false);
            substep_stats(E, tm, w, V, boff);
            sclk.mark(kPhStats);
            sclk.finish();
        }
    }

    // The largest worlds (the first n_block_worlds of the list) get a whole
    // CTA each, the next n_pair_worlds half a CTA (two warps) each, the
    // others one warp each, four per CTA.  Worlds progress independently: a
    // barrier is the team's own.  Dynamic shared memory: E.smem_cap_block
    // bodies for a CTA world, E.smem_cap_pair for each of two half-CTA
    // worlds, or E.smem_cap_warp for each of four warp worlds.
    template <class T, class P>
    __global__ void __launch_bounds__(128, RBPS_SUBSTEP_MIN_BLOCKS) k_substep(const Engine<T, P> E)
    {
        __shared__ ScanShared sh; // the colouring's compaction scans are all the teams need
        extern __shared__ __align__(16) unsigned char smem[];
        if (blockIdx.x < E.n_block_worlds)
        {
            BlockTeam tm;
            substep_world(E, tm, E.small_worlds[blockIdx.x], smem, E.smem_cap_block, sh);
            return;
        }
        const uint32_t pair_ctas = (E.n_pair_worlds + 1) / 2;
        const uint32_t b = blockIdx.x - E.n_block_worlds;
        if (b < pair_ctas)
        {
            // two mid-size worlds, one per half of the CTA, each on its own
            // named barrier (a half without a world leaves at once)
            const uint32_t k = 2 * b + (threadIdx.x >> 6);
            if (k >= E.n_pair_worlds)
                return;
            PairTeam tm;
            substep_world(E, tm, E.small_worlds[E.n_block_worlds + k],
                          smem + (threadIdx.x >> 6) * SmemWorld<T, P>::bytes(E.smem_cap_pair), E.smem_cap_pair, sh);
            return;
        }
        const uint32_t q = E.n_block_worlds + E.n_pair_worlds + (b - pair_ctas) * (blockDim.x >> 5) + warp_id();
        if (q >= E.n_small)
            return;
        WarpTeam tm;
        substep_world(E, tm, E.small_worlds[q], smem + warp_id() * SmemWorld<T, P>::bytes(E.smem_cap_warp),
                      E.smem_cap_warp, sh);
    }

    // Opens k_substep to `bytes` of dynamic shared memory.
    template <class T, class P>
    cudaError_t prepare_substep(size_t bytes)
    {
        // the attribute belongs to the kernel on the current device, shared
        // by every batch there: only ever raise it, or a batch created later
        // with smaller worlds would make an earlier one's launches fail
        cudaFuncAttributes fa;
        cudaError_t rc = cudaFuncGetAttributes(&fa, k_substep<T, P>);
        if (rc != cudaSuccess)
            return rc;
        if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes)
            return cudaSuccess;
        return cudaFuncSetAttribute(k_substep<T, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    }

    template <class T, class P>
    size_t smem_world_bytes(uint32_t cap)
    {
        return SmemWorld<T, P>::bytes(cap);
    }

    template <class T, class P>
    cudaError_t launch_step_flat(const Engine<T, P> &e, const PhaseLaunch &pl, const FlatLaunch &fl,
                                 cudaStream_t stream)
    {
        // without dumps the last substep launch also writes the statistics
        Engine<T, P> el = e;
        el.stats_in_substep = e.dump_cc || e.substeps < 1 ? 0 : 1;
        k_phase_frame<T, P><<<pl.grid[kKFrame], pl.block[kKFrame], 0, stream>>>(e, 0);
        k_flat_prefix<T, P><<<1, kMaxBlock, 0, stream>>>(e);
        k_type_count<T, P><<<fl.grid_sort, kMaxBlock, 0, stream>>>(e);
        k_type_scan<T, P><<<1, 32, 0, stream>>>(e);
        k_type_scatter<T, P><<<fl.grid_sort, kMaxBlock, 0, stream>>>(e);
        for (int s = 0; s < e.substeps; ++s)
        {
            if (e.gjk_list)
                cudaMemsetAsync(e.gjk_count, 0, 4, stream);
            if (fl.side && s < 8)
            {
                // the two narrowphase kernels touch disjoint candidates: run
                // them side by side (a fork / join the graph capture keeps)
                cudaEventRecord(fl.fork[s], stream);
                cudaStreamWaitEvent(fl.side, fl.fork[s], 0);
                k_flat_narrow_boxbox<T, P><<<fl.grid_narrow, kMaxBlock, 0, fl.side>>>(e);
                k_flat_narrow_other<T, P><<<fl.grid_narrow, kMaxBlock, 0, fl.side>>>(e);
                cudaEventRecord(fl.join[s], fl.side);
                k_flat_narrow<T, P><<<fl.grid_narrow, kMaxBlock, 0, stream>>>(e);
                cudaStreamWaitEvent(stream, fl.join[s], 0);
            }
            else
            {
                k_flat_narrow<T, P><<<fl.grid_narrow, kMaxBlock, 0, stream>>>(e);
                k_flat_narrow_boxbox<T, P><<<fl.grid_narrow, kMaxBlock, 0, stream>>>(e);
                k_flat_narrow_other<T, P><<<fl.grid_narrow, kMaxBlock, 0, stream>>>(e);
            }
            launch_gjk(e, stream);
            k_substep<T, P><<<fl.grid_solve, 128, fl.substep_smem, stream>>>(s + 1 == e.substeps ? el : e);
        }
        if (!el.stats_in_substep)
            k_phase_stats<T, P><<<pl.grid[kKStats], pl.block[kKStats], 0, stream>>>(e, 1);
        return cudaGetLastError();
    }

    // kernel 0: narrowphase, 1: substep, 2: class sort
    template <class T, class P>
    cudaError_t occupancy_flat(int kernel, int block, int *blocks_per_sm, size_t fl_smem)
    {
        if (kernel == 0)
            return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_flat_narrow<T, P>, block, 0);
        if (kernel == 2)
        {
            int a = 0, b = 0;
            cudaError_t rc = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_type_count<T, P>, block, 0);
            if (rc == cudaSuccess)
                rc = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_type_scatter<T, P>, block, 0);
            *blocks_per_sm = a < b ? a : b;
            return rc;
        }
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_substep<T, P>, block, fl_smem);
    }

    // Enqueues one step of one large world: 2 + 4 * substeps cooperative
    // phase launches, plus the GJK pass after each narrowphase when the batch
    // has one.  *launches receives the number of kernels enqueued.
    template <class T, class P>
    cudaError_t launch_step_big(const Engine<T, P> &e, uint32_t world, int grid, int block, cudaStream_t stream,
                                long *launches)
    {
        Engine<T, P> ec = e;
        int phase = 0;
        void *args[] = {(void *)&ec, (void *)&world, (void *)&phase};
        long n = 0;
        auto run = [&](int ph) {
            phase = ph;
            ++n;
            return cudaLaunchCooperativeKernel((const void *)k_big_phase<T, P>, dim3(grid), dim3(block), args, 0,
                                               stream);
        };
        cudaError_t rc = run(kKFrame);
        for (int s = 0; s < e.substeps && rc == cudaSuccess; ++s)
        {
            if (e.gjk_list && (rc = cudaMemsetAsync(e.gjk_count, 0, 4, stream)) != cudaSuccess)
                break;
            if ((rc = run(kKNarrow)) != cudaSuccess)
                break;
            if (e.gjk_list)
            {
                if ((rc = launch_gjk(e, stream)) != cudaSuccess)
                    break;
                ++n;
            }
            if ((rc = run(kKColor)) != cudaSuccess || (rc = run(kKPosition)) != cudaSuccess ||
                (rc = run(kKVelocity)) != cudaSuccess)
                break;
        }
        if (rc == cudaSuccess)
            rc = run(kKStats);
        *launches = n;
        return rc;
    }

    template <class T, class P>
    cudaError_t occupancy_phase(int kernel, int block, int *blocks_per_sm)
    {
        switch (kernel)
        {
        case kKFrame: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_phase_frame<T, P>, block, 0);
        case kKNarrow: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_phase_narrow<T, P>, block, 0);
        case kKColor: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_phase_color<T, P>, block, 0);
        case kKPosition:
            return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_phase_position<T, P>, block, 0);
        case kKVelocity:
            return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_phase_velocity<T, P>, block, 0);
        default: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_phase_stats<T, P>, block, 0);
        }
    }

    template <class T, class P>
    cudaError_t occupancy_big(int block, int *blocks_per_sm)
    {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_big_phase<T, P>, block, 0);
    }
} // namespace rbps_gpu

#define RBPS_INSTANTIATE_ENGINE(T, P)                                                                          \
    template cudaError_t rbps_gpu::launch_step_phases<T, P>(const rbps_gpu::Engine<T, P> &,                        \
                                                            const rbps_gpu::PhaseLaunch &, cudaStream_t);           \
    template cudaError_t rbps_gpu::launch_step_big<T, P>(const rbps_gpu::Engine<T, P> &, uint32_t, int, int,        \
                                                         cudaStream_t, long *);                                   \
    template cudaError_t rbps_gpu::occupancy_phase<T, P>(int, int, int *);                                         \
    template cudaError_t rbps_gpu::prepare_substep<T, P>(size_t);                                                  \
    template size_t rbps_gpu::smem_world_bytes<T, P>(uint32_t);                                                    \
    template cudaError_t rbps_gpu::launch_step_flat<T, P>(const rbps_gpu::Engine<T, P> &,                          \
                                                          const rbps_gpu::PhaseLaunch &,                            \
                                                          const rbps_gpu::FlatLaunch &, cudaStream_t);              \
    template cudaError_t rbps_gpu::occupancy_flat<T, P>(int, int, int *, size_t);                                          \
    template cudaError_t rbps_gpu::occupancy_big<T, P>(int, int *);                                               \
    template cudaError_t rbps_gpu::launch_debug_broadphase<T, P>(const rbps_gpu::Engine<T, P> &, uint32_t, int,    \
                                                                 uint32_t *, cudaStream_t);                         \
    template cudaError_t rbps_gpu::launch_io<T, P>(const rbps_gpu::Engine<T, P> &, int, double *, double *,       \
                                                   uint32_t, int, cudaStream_t);

namespace rbps_gpu
{
    // Host I/O staging: per-body forces in (3 doubles), poses out
    // (3 + 4 doubles), converted to / from the device precision.
    template <class T, class P>
    __global__ void k_forces_in(const Engine<T, P> E, const double *f, uint32_t n)
    {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            E.B.force[i] = V4<T>{T(f[3 * i]), T(f[3 * i + 1]), T(f[3 * i + 2]), T(0)};
    }

    template <class T, class P>
    __global__ void k_pose_out(const Engine<T, P> E, double *pos, double *rot, uint32_t n)
    {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        {
            const V4<P> x = E.B.pos[i];
            const Q4<T> q = E.B.rot[i];
            double o[3] = {0.0, 0.0, 0.0};
            if (E.origin)
            {
                const double *ow = E.origin + 3 * (size_t)E.body_world[i];
                o[0] = ow[0]; o[1] = ow[1]; o[2] = ow[2];
            }
            pos[3 * i] = o[0] + double(x.x);
            pos[3 * i + 1] = o[1] + double(x.y);
            pos[3 * i + 2] = o[2] + double(x.z);
            rot[4 * i] = double(q.w);
            rot[4 * i + 1] = double(q.x);
            rot[4 * i + 2] = double(q.y);
            rot[4 * i + 3] = double(q.z);
        }
    }

    template <class T, class P>
    cudaError_t launch_io(const Engine<T, P> &e, int dir, double *a, double *b, uint32_t n, int grid,
                          cudaStream_t stream)
    {
        if (dir == 0)
            k_forces_in<T, P><<<grid, 256, 0, stream>>>(e, a, n);
        else
            k_pose_out<T, P><<<grid, 256, 0, stream>>>(e, a, b, n);
        return cudaGetLastError();
    }

    // Diagnostics: only the frame's broadphase + candidate build of one
    // world on one CTA (the first phase of a step).
    template <class T, class P>
    __global__ void __launch_bounds__(kMaxBlock) k_debug_broadphase(const Engine<T, P> E, uint32_t w, uint32_t *out)
    {
        __shared__ BlockShared sh;
        BlockTeam tm;
        const WorldDev W = E.worlds[w];
        const Scr<T, P> S = world_scratch(E, W);
        const uint32_t n_pairs = broadphase(E, tm, W, S, sh);
        const uint32_t n_cand = build_candidates(E, tm, W, S, n_pairs, sh);
        if (threadIdx.x == 0)
        {
            out[0] = n_pairs;
            out[1] = n_cand;
        }
    }

    template <class T, class P>
    cudaError_t launch_debug_broadphase(const Engine<T, P> &e, uint32_t w, int block, uint32_t *out,
                                        cudaStream_t stream)
    {
        k_debug_broadphase<T, P><<<1, block, 0, stream>>>(e, w, out);
        return cudaGetLastError();
    }

} // namespace rbps_gpu
