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
    };

    struct WorldStats
    {
        uint32_t n_pairs;      // SAP pairs (before filtering) of the last step
        uint32_t n_cand;       // narrowphase candidates
        uint32_t n_contacts;   // contact rows of the last substep
        uint32_t n_colors;     // colours used (colored mode)
        uint32_t n_serial;     // candidates in the serial overflow colour
        uint32_t n_gjk;        // candidates that needed GJK/EPA
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
        size_t corder;           // candidates sorted by colour
        size_t misc;             // small counters
        size_t stride;           // bytes per executor
    };

    constexpr uint32_t kColorSerial = 64;  // overflow colour, solved by one thread
    constexpr uint32_t kMaxColorRounds = 96;
    constexpr uint32_t kMiscWords = 64 + 2 * 66 + kMaxColorRounds + 8;
    // misc layout (u32 words)
    constexpr uint32_t kMiscFlags = 0;                  // [0..7] scalars
    constexpr uint32_t kMiscCCount = 8;                 // 66 colour counts
    constexpr uint32_t kMiscCOff = 8 + 66;              // 66 colour offsets (+ fill)
    constexpr uint32_t kMiscLeft = 8 + 2 * 66;          // per-round "uncoloured left"

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
        // executors
        char *scratch;
        ScratchLayout lay;
        uint32_t *work_counter;
        const uint32_t *small_worlds;
        uint32_t n_small;
        // parity dumps (null when disabled)
        uint32_t *dump_pairs;   // 2 * pair_cap per slot
        Cand *dump_cand;        // cand_cap per slot
        CandContacts<T, P> *dump_cc;
        uint32_t *dump_color;
        uint32_t dump_pair_cap, dump_cand_cap;
    };

    // Host entry points, instantiated per precision in engine_f64.cu /
    // engine_f32.cu.  They only enqueue work on `stream`.
    template <class T, class P>
    cudaError_t launch_step_small(const Engine<T, P> &e, int grid, int block, cudaStream_t stream);
    template <class T, class P>
    cudaError_t launch_step_big(const Engine<T, P> &e, uint32_t world, int grid, int block, cudaStream_t stream);
    template <class T, class P>
    cudaError_t occupancy_small(int block, int *blocks_per_sm);
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
    template <class T, class P>
    cudaError_t launch_collide(const ShapeDev *sa, const double *ta, const ShapeDev *sb, const double *tb,
                               const HullSetDev &hulls, uint32_t n, CollideOut *out, cudaStream_t stream);
    template <class T, class P>
    cudaError_t launch_debug_broadphase(const Engine<T, P> &e, uint32_t world, int block, uint32_t *out,
                                        cudaStream_t stream);
} // namespace rbps_gpu
