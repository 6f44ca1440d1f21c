// engine_types.cuh - device views of one batch of worlds, shared by the host
// driver (batch.cu) and the step kernels (engine_impl.cuh).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "narrow.cuh"
#include "solver.cuh"

namespace rbps_gpu
{
    // Per-world offsets into the batch-wide arrays (all indices inside a
    // world are local: body / collider IDs follow the reference's
    // ID == slot rule).
    struct WorldDev
    {
        uint32_t body_off, n_bodies;
        uint32_t coll_off, n_coll;
        uint32_t bp_off, n_bp;       // SAP objects (non-plane colliders)
        uint32_t pc_off, n_pc;       // static plane-vs-collider candidates
        uint32_t joint_off, n_joints;
        uint32_t row_off, n_rows;
        uint32_t jc_off, n_jcolors;  // joint colour offsets: n_jcolors + 1 entries
        uint32_t pair_cap;
        uint32_t dump_slot;          // index of this world's dump slices, ~0u = none
        uint64_t scr_off;            // byte offset of the world's scratch slice
    };

    struct WorldStats
    {
        uint32_t n_pairs;      // SAP pairs (before filtering) of the last step
        uint32_t n_cand;       // narrowphase candidates
        uint32_t n_contacts;   // contact rows of the last substep
        uint32_t n_colors;     // colours used (colored mode)
        uint32_t n_serial;     // candidates in the serial overflow colour
        uint32_t n_gjk;        // candidates run through GJK/EPA, summed over the substeps
        uint32_t pad_[2];
    };

    struct FatBox
    {
        double mn[3];
        double mx[3];
    };

    // Candidate pair of the narrowphase: colliders (ca = shape A) and bodies.
    struct Cand
    {
        uint32_t ca, cb, ba, bb;
    };

    // Byte offsets of the per-executor scratch arrays.
    struct ScratchLayout
    {
        size_t ep_k2, ep_v2;     // endpoint sort ping-pong
        size_t counts;           // radix digit counts
        size_t tile_sums;        // scan partials
        size_t cnt;              // pair counts per endpoint position
        size_t pr_a, pr_b;       // raw pairs (object indices)
        size_t pk, pv, pk2, pv2; // pair sort keys / values
        size_t cflag;            // candidate filter flags
        size_t cand;             // Cand[]
        size_t cc;               // CandContacts[]
        size_t color;            // colour per candidate
        size_t bmask;            // per-body colour mask (u64)
        size_t bprio;            // per-body priority (u64)
        size_t claim;            // per-(body, colour) claims (u64), grid worlds only
        size_t yz;               // float y / z extents per SAP object (float4), grid worlds only
        size_t corder;           // candidates sorted by colour
        size_t misc;             // small counters
        size_t act, alist;       // active-candidate flags / compacted list (colored mode)
        size_t stride;           // bytes per executor
    };

    // Per-world scratch: every world owns a slice of the batch scratch buffer
    // (WorldDev::scr_off) laid out from the world's own sizes, so a world's
    // frame data (SAP pairs, candidates, contact manifolds, colours) stays
    // in place between the phase kernels of a step.  Radix-sort and scan
    // tiles are sized for the smallest team tile (kTileMin threads).
    constexpr uint32_t kTileMin = 32;

    RBPS_HD size_t scr_align(size_t x, size_t a) { return (x + a - 1) / a * a; }

    constexpr uint32_t kColorSerial = 64;  // overflow colour, solved by one thread
    constexpr uint32_t kColorStage = 256;  // candidates staged in shared memory per colouring chunk
    constexpr uint32_t kColorIdle = 65;    // candidate without contact rows this substep
    constexpr uint32_t kMaxColorRounds = 96;
    // Worlds with more bodies step on the whole cooperative grid.  They
    // colour by claims on (body, colour) slots, which colours many contacts
    // of one body per round (smaller ones use Jones-Plassmann, which needs no
    // claim table), and their SAP sweep prefilters on float y / z extents.
    constexpr uint32_t kGridWorldBodies = 4096;
    constexpr uint32_t kMiscWords = 64 + 4 * 66 + kMaxColorRounds + 8;
    // misc layout (u32 words)
    constexpr uint32_t kMiscFlags = 0;                  // [0..7] scalars
    constexpr uint32_t kMiscCCount = 8;                 // 66 colour counts
    constexpr uint32_t kMiscCOff = 8 + 66;              // 66 colour offsets (+ fill)
    constexpr uint32_t kMiscLeft = 8 + 2 * 66;          // per-round "uncoloured left"
    // second-level colours of the overflow bucket (colour kColorSerial):
    // 66 counts, then 66 offsets into corder (entry 64: still serial)
    constexpr uint32_t kMiscC2Count = kMiscLeft + kMaxColorRounds;
    constexpr uint32_t kMiscC2Off = kMiscC2Count + 66;
    // misc scalars: kMiscFlags + 1 colours of this substep, + 2 contact rows,
    // + 3 GJK candidates, + 4 unclamped SAP pairs, + 5 SAP pairs, + 6 narrowphase
    // candidates, + 7 most colours over the step's substeps
    constexpr uint32_t kMiscNColors = kMiscFlags + 1, kMiscNContacts = kMiscFlags + 2, kMiscNGjk = kMiscFlags + 3,
                       kMiscPairsRaw = kMiscFlags + 4, kMiscNPairs = kMiscFlags + 5, kMiscNCand = kMiscFlags + 6,
                       kMiscMaxColors = kMiscFlags + 7;
    // 1 while S.color holds a colouring of the current candidate list (set by
    // the colouring, cleared by the frame that rebuilds the list)
    constexpr uint32_t kMiscColorValid = kMiscC2Off + 66;
    static_assert(kMiscColorValid < kMiscWords, "misc words");

    RBPS_HD ScratchLayout make_layout(uint32_t nbp, uint32_t nb, uint32_t pair_cap, uint32_t npc, size_t cc_size)
    {
        ScratchLayout L{};
        const size_t nep = 2 * (size_t)nbp + 1;
        const size_t pc = (size_t)pair_cap + 1;
        const size_t nc = pc + npc;
        size_t nt = (nep + kTileMin - 1) / kTileMin;
        nt = nt > (pc + kTileMin - 1) / kTileMin ? nt : (pc + kTileMin - 1) / kTileMin;
        nt = nt > (nc + kTileMin - 1) / kTileMin ? nt : (nc + kTileMin - 1) / kTileMin;
        const size_t nt_max = nt + 1;
        const size_t counts = 256 * nt_max;
        const size_t ts0 = (counts + kTileMin - 1) / kTileMin;
        const size_t tsums = (ts0 > nt_max ? ts0 : nt_max) + 4;
        size_t off = 0;
        auto take = [&](size_t &field, size_t bytes) {
            off = scr_align(off, 128);
            field = off;
            off += bytes;
        };
        take(L.ep_k2, nep * 4);
        take(L.ep_v2, nep * 4);
        take(L.counts, counts * 4);
        take(L.tile_sums, tsums * 4);
        take(L.cnt, nep * 4);
        take(L.pr_a, pc * 4);
        take(L.pr_b, pc * 4);
        take(L.pk, pc * 4);
        take(L.pv, pc * 4);
        take(L.pk2, pc * 4);
        take(L.pv2, pc * 4);
        take(L.cflag, pc * 4);
        take(L.cand, nc * sizeof(Cand));
        take(L.cc, nc * cc_size);
        take(L.color, nc * 4);
        take(L.bmask, (size_t)nb * 8 + 8);
        take(L.bprio, (size_t)nb * 8 + 8);
        take(L.claim, nb > kGridWorldBodies ? (size_t)nb * 64 * 8 : 8);
        take(L.yz, nb > kGridWorldBodies ? (size_t)nbp * 16 : 16);
        take(L.corder, nc * 4);
        take(L.misc, kMiscWords * 4);
        take(L.act, nc * 4);
        take(L.alist, nc * 4);
        L.stride = scr_align(off, 256);
        return L;
    }

    // Phase-timer slots per world (Engine::prof): SM cycles summed over the
    // steps since profiling was enabled, then the CTA and the globaltimer
    // bounds (ns) of the world's last step.
    enum : uint32_t
    {
        kPhBroadphase = 0,
        kPhCandidates = 1,
        kPhNarrow = 2,
        kPhColor = 3,
        kPhIntegrate = 4,
        kPhContactPos = 5,
        kPhJointPos = 6,
        kPhVelUpdate = 7,
        kPhVelSolve = 8,
        kPhStats = 9,
        // parts of kPhBroadphase on one-CTA teams, timed by the leader
        kPhEndpointSort = 10,
        kPhSweep = 11,
        kPhPairOrder = 15,
        kProfCta = 12,
        kProfStartNs = 13,
        kProfEndNs = 14,
        kProfSlots = 16
    };

    template <class T, class P>
    struct Engine
    {
        Bodies<T, P> B;
        // colliders
        const ShapeDev *shape;
        const uint32_t *c_body;
        const V4<double> *c_lpos;
        const Q4<double> *c_lrot;
        const uint8_t *c_static;
        const V4<T> *c_mat;
        HullSetDev hulls;
        // SAP state (persistent)
        const uint32_t *bp_coll;
        FatBox *fat;
        uint32_t *ep_key;
        uint32_t *ep_id;
        uint32_t *ep_pos;
        // static plane candidates (local collider ids)
        const uint2 *plane_cand;
        // joints
        Joint<T> *joints;
        Row<T> *rows;
        const uint32_t *jorder;
        const uint32_t *jcolor_off;
        // worlds
        const WorldDev *worlds;
        WorldStats *stats;
        int *error;
        // step parameters
        double dt_frame;
        T h, inv_h;
        int substeps;
        double fat_margin, reinsert_threshold;
        int solve_mode;
        int use_vel_exp;
        int check_state; // the stats phase reports a non-finite body state (RBPS_ERR_STATE)
        // 1 on the last substep launch of a colored step without dumps: the
        // substep kernel writes the world statistics and runs the state
        // check itself, and no stats kernel follows
        int stats_in_substep;
        // launch-shape knobs of the flat coloured pipeline (autotuned; results
        // do not depend on them): narrowphase candidates a warp takes per
        // pass (a multiple of 32), and active candidates the colouring stages
        // per batch (<= kColorStage)
        uint32_t narrow_per_warp;
        uint32_t color_chunk;
        // executors
        char *scratch;            // per-world slices at WorldDev::scr_off
        uint32_t *work_counter;
        const uint32_t *small_worlds;
        uint32_t n_small;
        uint32_t n_block_worlds;  // colored batches: the first n of small_worlds step on a whole CTA
        uint32_t n_pair_worlds;   // the next n on half a CTA (two warps) each
        uint32_t smem_cap_block;  // bodies a CTA world keeps in shared memory (colored substep)
        uint32_t smem_cap_warp;   // bodies each warp world keeps in shared memory
        uint32_t smem_cap_pair;   // bodies each half-CTA world keeps in shared memory
        // parity dumps (null when disabled)
        uint32_t *dump_pairs;   // 2 * pair_cap per slot
        Cand *dump_cand;        // cand_cap per slot
        CandContacts<T, P> *dump_cc;
        uint32_t *dump_color;
        uint32_t dump_pair_cap, dump_cand_cap;
        unsigned long long *prof; // phase timers, kProfSlots per world (null = off)
        // GJK pass (batches with hull colliders): queued (world, candidate)
        // pairs of the current substep and one workspace per k_gjk thread
        uint2 *gjk_list;
        uint32_t *gjk_count;
        uint32_t gjk_cap, gjk_slots;
        // RBPS_PRECISION_FP32_POS64: per-world origin (3 doubles a world) and
        // the world of every body; body positions are stored relative to it
        const double *origin;
        const uint32_t *body_world;
        // flat colored pipeline over all small worlds (see engine_impl.cuh)
        uint32_t *wcoff;               // n_small + 1: candidate prefix over small_worlds
        uint32_t *gcol;                // global colour bookkeeping, kGcolWords
        uint2 *nlist;                  // (world, candidate) of all small worlds sorted by shape pair
        uint4 *nglob;                  // beside each entry: global colliders a, b and bodies a, b
        Cand *const *wcand;            // per world: its candidate list
        CandContacts<T, P> *const *wcc; // per world: its contact manifolds
        const uint32_t *sbodies;       // bodies of the small worlds
        uint32_t n_sbodies;
        const uint32_t *sjoints;       // joints of the small worlds grouped by joint colour
        const uint32_t *sjcoff;        // n_sjcolors + 1 offsets into sjoints
        uint32_t n_sjcolors, n_sjoints;
    };

    // gcol layout (u32 words): per shape-pair class [0, 32) counts, [32, 64)
    // fill cursors, [64, 96) offsets (entry kPairClasses = total)
    constexpr uint32_t kPairClasses = 25;
    constexpr uint32_t kGcolCount = 0, kGcolFill = 32, kGcolOff = 64, kGcolWords = 96;

    // Host entry points, instantiated per precision in engine_f64.cu /
    // engine_f32.cu.  They only enqueue work on `stream`.
    // Phase kernels of the batched step (one launch per phase).
    enum : int
    {
        kKFrame = 0,
        kKNarrow = 1,
        kKColor = 2,
        kKPosition = 3,
        kKVelocity = 4,
        kKStats = 5,
        kNumPhaseKernels = 6
    };
    struct PhaseLaunch
    {
        int grid[kNumPhaseKernels];
        int block[kNumPhaseKernels];
    };

    template <class T, class P>
    cudaError_t launch_step_phases(const Engine<T, P> &e, const PhaseLaunch &pl, cudaStream_t stream);
    // Colored mode: the frame / stats phases per world, the substeps flat
    // over all small worlds (grids: narrowphase, cooperative solves).
    struct FlatLaunch
    {
        int grid_narrow, grid_solve, block_solve;
        int grid_sort;       // the class-sort kernels: every CTA they can keep resident
        size_t substep_smem; // dynamic shared memory of k_substep
        // a second stream on which the box-box narrowphase runs beside the
        // other classes' (fork / join events), or null for one stream
        cudaStream_t side;
        cudaEvent_t fork[8], join[8]; // one pair per substep (substeps <= 8), else sequential
    };
    template <class T, class P>
    cudaError_t launch_step_flat(const Engine<T, P> &e, const PhaseLaunch &pl, const FlatLaunch &fl,
                                 cudaStream_t stream);
    template <class T, class P>
    cudaError_t occupancy_flat(int kernel, int block, int *blocks_per_sm, size_t dynamic_smem);
    // k_substep's shared-memory world copies: bytes for `cap` bodies, and
    // opening the kernel to a dynamic shared-memory size
    template <class T, class P>
    size_t smem_world_bytes(uint32_t cap);
    template <class T, class P>
    cudaError_t prepare_substep(size_t bytes);
    template <class T, class P>
    cudaError_t occupancy_phase(int kernel, int block, int *blocks_per_sm);
    template <class T, class P>
    cudaError_t launch_step_big(const Engine<T, P> &e, uint32_t world, int grid, int block, cudaStream_t stream,
                                long *launches);
    template <class T, class P>
    cudaError_t occupancy_big(int block, int *blocks_per_sm);
    template <class T, class P>
    cudaError_t launch_io(const Engine<T, P> &e, int dir, double *a, double *b, uint32_t n, int grid,
                          cudaStream_t stream);
    // Output of one device narrowphase test; the layout of rbps_manifold.
    struct CollideOut
    {
        int32_t status, n_points;
        double normal[3];
        double position[4][3];
        double depth[4];
    };
    // one warp per pair, GJK / EPA workspaces in shared memory
    template <class T, class P>
    cudaError_t launch_collide(const ShapeDev *sa, const double *ta, const ShapeDev *sb, const double *tb,
                               const HullSetDev &hulls, uint32_t n, CollideOut *out, int *err, cudaStream_t stream);
    // the GJK pass over the pairs the narrowphase queued (no-op without
    // hulls): Engine::gjk_slots CTAs, one warp per queued pair
    template <class T, class P>
    cudaError_t launch_gjk(const Engine<T, P> &e, cudaStream_t stream);
    // opens the GJK pass kernel to its shared workspaces; *ctas receives the
    // CTAs the device keeps resident at once
    template <class T, class P>
    cudaError_t prepare_gjk(int sm_count, uint32_t *ctas);
    template <class T, class P>
    cudaError_t launch_debug_broadphase(const Engine<T, P> &e, uint32_t world, int block, uint32_t *out,
                                        cudaStream_t stream);
} // namespace rbps_gpu
