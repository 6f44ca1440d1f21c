// batch.cu - host driver and C ABI (include/rbps_gpu.h) of the batched
// engine: scene building, upload, per-step launches and state readback.
//
// The setup surface mirrors rbps::World (include/rbps/API/World.hpp:87-213):
// create_body (BodyAPI.hpp:53-80), create_collider with the initial
// broad_phase_insert (ColliderAPI.hpp:61-91, BroadPhase.cpp:169-197),
// create_{prismatic,revolute,fixed}_joint (JointAPI.hpp:191-267).  Host-side
// arithmetic that must round like the reference (inverse inertia, initial fat
// AABBs, endpoint keys) uses the shared math headers in double.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "engine_types.cuh"
#include "rbps_gpu.h"

using namespace rbps_gpu;

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

static int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CU(...)                                                                                  \
    do                                                                                           \
    {                                                                                            \
        cudaError_t e_ = (__VA_ARGS__);                                                          \
        if (e_ != cudaSuccess)                                                                   \
            return fail(RBPS_ERR_CUDA, "%s failed: %s (%s:%d)", #__VA_ARGS__,                    \
                        cudaGetErrorString(e_), __FILE__, __LINE__);                             \
    } while (0)

extern "C" int rbps_last_error(char *buf, size_t size)
{
    if (buf && size)
    {
        std::strncpy(buf, g_last_error.c_str(), size - 1);
        buf[size - 1] = 0;
    }
    return (int)g_last_error.size();
}

extern "C" const char *rbps_version(void) { return "rbps_b200 0.1 (sm_100a)"; }

// ---------------------------------------------------------- host helpers
namespace
{
    // smat3::inverse (mat3.hpp:248-272)
    void smat3_inverse(const double *m, double *out)
    {
        const double xx = m[0], yy = m[1], zz = m[2], xy = m[3], xz = m[4], yz = m[5];
        const double det = xx * yy * zz + 2 * xy * xz * yz - xx * yz * yz - yy * xz * xz - zz * xy * xy;
        if (std::fabs(det) < kEpsilon)
        {
            for (int i = 0; i < 6; ++i)
                out[i] = 0.0;
            return;
        }
        const double inv = 1.0 / det;
        out[0] = (yy * zz - yz * yz) * inv;
        out[1] = (xx * zz - xz * xz) * inv;
        out[2] = (xx * yy - xy * xy) * inv;
        out[3] = (xz * yz - xy * zz) * inv;
        out[4] = (xy * yz - xz * yy) * inv;
        out[5] = (xy * xz - xx * yz) * inv;
    }

    uint32_t order_key_host(float f)
    {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        if ((u & 0x7fffffffu) == 0u)
            u = 0u;
        return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    }

    struct HostWorld
    {
        std::vector<rbps_body_desc> bodies;
        std::vector<double> force;  // 3 per body
        std::vector<double> torque; // 3 per body
        std::vector<rbps_collider_desc> colliders;
        std::vector<rbps_joint_desc> joints;
    };

    // A convex hull as the device needs it: vertices, local AABB, and the
    // merged-polygon and adjacency tables of convex_hull_data_create
    // (ConvexHull.hpp:149-420) for the hull-hull contact manifold.
    struct HostHull
    {
        std::vector<double> verts;
        double aabb[6];
        std::vector<uint32_t> poly_off{0}, poly_idx;
        std::vector<double> poly_n;                   // 3 per polygon
        std::vector<uint32_t> v2p_off, v2p_idx;       // polygons of each vertex
        std::vector<uint32_t> v2n_off, v2n_idx;       // polygon-edge neighbours of each vertex
        std::vector<uint32_t> p2p_off, p2p_idx;       // polygons sharing an edge with each polygon
    };

    // Restatement of convex_hull_data_create's table building
    // (ConvexHull.hpp:149-420): triangle normals; union-find over triangle
    // pairs whose normals have dot > 0.99995; per group, the boundary loop of
    // directed edges whose reverse is absent, walked from the first boundary
    // edge; the normalised sum of the group's normals; then the vertex ->
    // polygons, vertex -> neighbours and polygon -> polygons tables in the
    // same insertion order.  Groups with an empty boundary, a loop under 3
    // vertices or a zero normal sum are dropped, as there.
    void build_hull_tables(HostHull &h, const uint32_t *tris, uint32_t n_tris)
    {
        const uint32_t nv = (uint32_t)(h.verts.size() / 3);
        auto V = [&](uint32_t i) { return vec3<double>(h.verts[3 * i], h.verts[3 * i + 1], h.verts[3 * i + 2]); };
        h.poly_off.assign(1, 0);
        h.poly_idx.clear();
        h.poly_n.clear();
        h.v2p_off.clear(); h.v2p_idx.clear();
        h.v2n_off.clear(); h.v2n_idx.clear();
        h.p2p_off.clear(); h.p2p_idx.clear();
        if (!tris || n_tris == 0)
            return;
        std::vector<vec3<double>> norms(n_tris);
        for (uint32_t f = 0; f < n_tris; ++f)
        {
            const vec3<double> A = V(tris[3 * f]), B = V(tris[3 * f + 1]), C = V(tris[3 * f + 2]);
            norms[f] = normalize(cross(B - A, C - A));
        }
        std::vector<int> parent(n_tris);
        for (uint32_t i = 0; i < n_tris; ++i)
            parent[i] = (int)i;
        auto find = [&parent](int x) {
            while (parent[x] != x)
            {
                parent[x] = parent[parent[x]];
                x = parent[x];
            }
            return x;
        };
        for (uint32_t i = 0; i < n_tris; ++i)
            for (uint32_t j = i + 1; j < n_tris; ++j)
                if (dot(norms[i], norms[j]) > 0.99995)
                {
                    const int ri = find((int)i), rj = find((int)j);
                    if (ri != rj)
                        parent[ri] = rj;
                }
        std::vector<std::vector<uint32_t>> groups;
        std::vector<int> root_group(n_tris, -1);
        for (uint32_t i = 0; i < n_tris; ++i)
        {
            const int r = find((int)i);
            if (root_group[r] < 0)
            {
                root_group[r] = (int)groups.size();
                groups.emplace_back();
            }
            groups[root_group[r]].push_back(i);
        }
        for (const auto &g : groups)
        {
            std::vector<std::pair<uint32_t, uint32_t>> e, bnd;
            for (uint32_t f : g)
            {
                const uint32_t a = tris[3 * f], b = tris[3 * f + 1], c = tris[3 * f + 2];
                e.push_back({a, b});
                e.push_back({b, c});
                e.push_back({c, a});
            }
            for (size_t i = 0; i < e.size(); ++i)
            {
                bool rev = false;
                for (size_t j = 0; j < e.size(); ++j)
                    if (i != j && e[j].first == e[i].second && e[j].second == e[i].first)
                    {
                        rev = true;
                        break;
                    }
                if (!rev)
                    bnd.push_back(e[i]);
            }
            if (bnd.empty())
                continue;
            std::vector<bool> used(bnd.size(), false);
            std::vector<uint32_t> loop;
            used[0] = true;
            loop.push_back(bnd[0].first);
            uint32_t cur = bnd[0].second;
            for (size_t step = 1; step < bnd.size(); ++step)
            {
                bool found = false;
                for (size_t k = 0; k < bnd.size(); ++k)
                    if (!used[k] && bnd[k].first == cur)
                    {
                        used[k] = true;
                        loop.push_back(bnd[k].first);
                        cur = bnd[k].second;
                        found = true;
                        break;
                    }
                if (!found)
                    break;
            }
            if (loop.size() < 3)
                continue;
            vec3<double> avg(0.0, 0.0, 0.0);
            for (uint32_t f : g)
                avg = avg + norms[f];
            const double len = length(avg);
            if (len < kEpsilon)
                continue;
            avg = avg / len;
            h.poly_idx.insert(h.poly_idx.end(), loop.begin(), loop.end());
            h.poly_off.push_back((uint32_t)h.poly_idx.size());
            h.poly_n.push_back(avg.x);
            h.poly_n.push_back(avg.y);
            h.poly_n.push_back(avg.z);
        }
        const uint32_t np = (uint32_t)(h.poly_off.size() - 1);
        if (np == 0)
            return;
        std::vector<std::vector<uint32_t>> v2p(nv), v2n(nv), p2p(np);
        auto push_unique = [](std::vector<uint32_t> &v, uint32_t x) {
            if (std::find(v.begin(), v.end(), x) == v.end())
                v.push_back(x);
        };
        for (uint32_t p = 0; p < np; ++p)
        {
            const uint32_t s0 = h.poly_off[p], n = h.poly_off[p + 1] - s0;
            for (uint32_t i = 0; i < n; ++i)
            {
                const uint32_t a = h.poly_idx[s0 + i], b = h.poly_idx[s0 + (i + 1) % n];
                push_unique(v2p[a], p);
                push_unique(v2n[a], b);
                push_unique(v2n[b], a);
            }
        }
        for (uint32_t p = 0; p < np; ++p)
        {
            const uint32_t sp = h.poly_off[p], n_p = h.poly_off[p + 1] - sp;
            for (uint32_t q = 0; q < np; ++q)
            {
                if (q == p)
                    continue;
                const uint32_t sq = h.poly_off[q], n_q = h.poly_off[q + 1] - sq;
                bool shared = false;
                for (uint32_t i = 0; i < n_p && !shared; ++i)
                {
                    const uint32_t a = h.poly_idx[sp + i], b = h.poly_idx[sp + (i + 1) % n_p];
                    for (uint32_t j = 0; j < n_q; ++j)
                        if (a == h.poly_idx[sq + (j + 1) % n_q] && b == h.poly_idx[sq + j])
                        {
                            shared = true;
                            break;
                        }
                }
                if (shared)
                    p2p[p].push_back(q);
            }
        }
        auto flatten = [](const std::vector<std::vector<uint32_t>> &src, std::vector<uint32_t> &off,
                          std::vector<uint32_t> &idx) {
            off.assign(1, 0);
            idx.clear();
            for (const auto &v : src)
            {
                idx.insert(idx.end(), v.begin(), v.end());
                off.push_back((uint32_t)idx.size());
            }
        };
        flatten(v2p, h.v2p_off, h.v2p_idx);
        flatten(v2n, h.v2n_off, h.v2n_idx);
        flatten(p2p, h.p2p_off, h.p2p_idx);
    }

    struct DevBuf
    {
        void *p = nullptr;
        size_t bytes = 0;
    };

    size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
} // namespace

// Shapes the device narrowphase covers: the reference's Sphere, Box,
// Ellipsoid, Capsule, Cylinder, Cone, Plane and ConvexHull (ShapeTypes.hpp);
// Heightmap and Mesh are not on the device path.
static bool shape_supported(int s)
{
    return s == RBPS_SHAPE_SPHERE || s == RBPS_SHAPE_BOX || s == RBPS_SHAPE_ELLIPSOID || s == RBPS_SHAPE_CAPSULE ||
           s == RBPS_SHAPE_CYLINDER || s == RBPS_SHAPE_CONE || s == RBPS_SHAPE_PLANE || s == RBPS_SHAPE_HEIGHTMAP ||
           s == RBPS_SHAPE_MESH || s == RBPS_SHAPE_CONVEX_HULL;
}

// A triangle mesh as mesh_data_create builds it (Mesh.hpp).
struct HostMesh
{
    std::vector<double> verts, normals;
    std::vector<uint32_t> idx;
    MeshDesc d{};
};

// A heightmap as heightmap_data_create builds it (Heightmap.hpp).
struct HostHeightmap
{
    std::vector<float> heights;
    HmDesc d{};
};

struct rbps_batch
{
    rbps_batch_desc desc;
    std::vector<HostWorld> worlds;
    std::vector<HostHull> hulls;
    std::vector<HostHeightmap> heightmaps;
    std::vector<HostMesh> meshes;
    uint32_t team_bodies = 0; // worlds this large step on a whole CTA (set_team_split)
    uint32_t pair_bodies = 0; // worlds this large (and below team_bodies) step on half a CTA
    MeshDesc *mesh_desc = nullptr;
    double *mesh_v = nullptr, *mesh_n = nullptr;
    uint32_t *mesh_i = nullptr;
    float *hm_heights = nullptr;
    HmDesc *hm_desc = nullptr;
    bool committed = false;
    bool check_state = true; // rbps_batch_set_state_check
    uint32_t narrow_per_warp = 32;        // narrowphase candidates a warp takes per pass (autotuned)
    uint32_t color_chunk = kColorStage;   // candidates the colouring stages per batch (autotuned)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 0;
    int block = 256;

    // device allocations
    std::vector<void *> allocs;
    // typed device pointers (as raw bytes; views are built per precision)
    void *pos = nullptr, *rot = nullptr, *lin = nullptr, *ang = nullptr, *prev_pos = nullptr, *prev_rot = nullptr;
    void *force = nullptr, *torque = nullptr, *inertia = nullptr, *inv_inertia = nullptr;
    uint8_t *btype = nullptr;
    ShapeDev *shape = nullptr;
    uint32_t *c_body = nullptr;
    V4<double> *c_lpos = nullptr;
    Q4<double> *c_lrot = nullptr;
    uint8_t *c_static = nullptr;
    void *c_mat = nullptr;
    double *hull_verts = nullptr;
    uint32_t *hull_voff = nullptr;
    double *hull_aabb = nullptr;
    HullDesc *hull_desc = nullptr;
    uint32_t *hull_u32 = nullptr;
    double *hull_pn = nullptr;
    uint32_t *bp_coll = nullptr;
    FatBox *fat = nullptr;
    uint32_t *ep_key = nullptr, *ep_id = nullptr, *ep_pos = nullptr;
    uint2 *plane_cand = nullptr;
    void *joints_d = nullptr, *rows_d = nullptr;
    uint32_t *jorder = nullptr, *jcolor_off = nullptr;
    WorldDev *worlds_d = nullptr;
    WorldStats *stats_d = nullptr;
    int *error_d = nullptr;
    uint32_t *work_counter = nullptr;
    uint32_t *small_list = nullptr;
    char *scratch = nullptr; // per-world slices (WorldDev::scr_off)

    // host mirrors
    std::vector<WorldDev> wdev;
    std::vector<uint32_t> small_ids, big_ids;
    // GJK pass (hull colliders present): queued pairs and workspaces
    uint2 *gjk_list = nullptr;
    uint32_t *gjk_count = nullptr;
    uint32_t gjk_cap = 0, gjk_slots = 0;
    PhaseLaunch phase{};      // grid / block of each phase kernel
    FlatLaunch flat{};        // flat colored pipeline
    bool use_flat = false;
    uint32_t *wcoff = nullptr, *gcol = nullptr, *sbodies = nullptr, *sjoints = nullptr, *sjcoff = nullptr;
    uint2 *nlist = nullptr;
    uint4 *nglob = nullptr; // global collider / body indices beside nlist
    void **wcand = nullptr, **wcc = nullptr;
    uint32_t n_sbodies = 0, n_sjoints = 0, n_sjcolors = 0, n_block_worlds = 0;
    uint32_t smem_cap_block = 0, smem_cap_warp = 0, smem_cap_pair = 0, n_pair_worlds = 0;
    int grid_big = 0;
    uint32_t n_counters = 0;  // phase work counters per step
    uint64_t total_bodies = 0, total_dynamic = 0;
    uint32_t n_bodies_all = 0, n_coll_all = 0, n_bp_all = 0, n_joint_all = 0, n_row_all = 0;
    uint64_t steps_done = 0;
    uint64_t launches_last = 0;

    // host I/O staging (rbps_batch_step_io)
    double *io_force = nullptr, *io_pos = nullptr, *io_rot = nullptr;
    // RBPS_PRECISION_FP32_POS64: every world's bodies are stored in float
    // relative to a per-world origin held in double (3 per world), so a
    // world far from the global origin keeps float resolution near its own
    // bodies; body_world maps a body to its world (host and device copies).
    std::vector<double> origin;
    std::vector<uint32_t> body_world;
    double *origin_d = nullptr;
    uint32_t *body_world_d = nullptr;
    bool relative() const { return desc.precision == RBPS_PRECISION_FP32_POS64; }
    const double *origin_of_body(size_t g) const
    {
        static const double zero[3] = {0.0, 0.0, 0.0};
        return relative() ? origin.data() + 3 * (size_t)body_world[g] : zero;
    }
    const double *origin_of_world(uint32_t w) const
    {
        static const double zero[3] = {0.0, 0.0, 0.0};
        return relative() ? origin.data() + 3 * (size_t)w : zero;
    }

    // dumps
    bool dump = false;
    uint32_t *dump_pairs = nullptr;
    Cand *dump_cand = nullptr;
    void *dump_cc = nullptr;
    uint32_t *dump_color = nullptr;
    uint32_t dump_pair_cap = 0, dump_cand_cap = 0;
    unsigned long long *prof = nullptr; // phase timers (rbps_batch_set_profile)
    bool prof_off = true;

    size_t t_size() const { return desc.precision == RBPS_PRECISION_FP64 ? 8 : 4; }
    size_t p_size() const { return desc.precision == RBPS_PRECISION_FP64 ? 8 : 4; }

    int alloc(void **p, size_t bytes)
    {
        if (bytes == 0)
            bytes = 16;
        CU(cudaMalloc(p, bytes));
        CU(cudaMemset(*p, 0, bytes));
        allocs.push_back(*p);
        return RBPS_OK;
    }
    template <class X>
    int upload(X **p, const std::vector<X> &v)
    {
        int rc = alloc((void **)p, v.size() * sizeof(X));
        if (rc)
            return rc;
        if (!v.empty())
            CU(cudaMemcpy(*p, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice));
        return RBPS_OK;
    }
    // one step captured as a CUDA graph (replayed by rbps_batch_step)
    cudaGraphExec_t graph_exec = nullptr;
    int graph_key = -1;      // dump / profile state the graph was captured with
    bool graph_ok = true;    // false once capture was refused: launch directly
    uint64_t graph_launches = 0;

    // pipelined host I/O (rbps_batch_step_io_async): an input and an output
    // copy stream (so a step's force copy never queues behind the previous
    // step's pose copy), two device staging slots and their events
    cudaStream_t io_stream = nullptr, io_out_stream = nullptr;
    double *io_f2[2] = {nullptr, nullptr}, *io_p2[2] = {nullptr, nullptr}, *io_r2[2] = {nullptr, nullptr};
    cudaEvent_t ev_force_ready[2] = {}, ev_force_free[2] = {}, ev_pose_ready[2] = {}, ev_out_free[2] = {};
    uint32_t io_slot = 0;
    bool io_async_ready = false;
    // snapshot slots (rbps_batch_snapshot): one device buffer each, holding
    // the state arrays back to back
    std::vector<char *> snaps;

    ~rbps_batch()
    {
        if (io_stream)
            cudaStreamSynchronize(io_stream);
        if (io_out_stream)
            cudaStreamSynchronize(io_out_stream);
        if (stream)
            cudaStreamSynchronize(stream);
        for (int k = 0; k < 2; ++k)
            for (cudaEvent_t e : {ev_force_ready[k], ev_force_free[k], ev_pose_ready[k], ev_out_free[k]})
                if (e)
                    cudaEventDestroy(e);
        if (io_stream)
            cudaStreamDestroy(io_stream);
        if (io_out_stream)
            cudaStreamDestroy(io_out_stream);
        if (flat.side)
        {
            cudaStreamSynchronize(flat.side);
            for (int k = 0; k < 8; ++k)
            {
                if (flat.fork[k])
                    cudaEventDestroy(flat.fork[k]);
                if (flat.join[k])
                    cudaEventDestroy(flat.join[k]);
            }
            cudaStreamDestroy(flat.side);
        }
        if (graph_exec)
            cudaGraphExecDestroy(graph_exec);
        for (void *p : allocs)
            cudaFree(p);
        if (own_stream && stream)
            cudaStreamDestroy(stream);
    }
};

// ------------------------------------------------------------ defaults
extern "C" void rbps_batch_desc_default(rbps_batch_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->n_worlds = 1;
    d->timestep = 1.0 / 60.0;
    d->substeps = 20;
    d->precision = RBPS_PRECISION_FP64;
    d->solve_mode = RBPS_SOLVE_REFERENCE_ORDER;
    d->fat_margin = 0.1;
    d->reinsert_threshold = 0.05;
    d->use_velocity_expansion = 1;
}

extern "C" void rbps_body_desc_default(rbps_body_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->type = RBPS_BODY_DYNAMIC;
    d->mass = 1.0;
    d->inertia[0] = d->inertia[1] = d->inertia[2] = 1.0;
    d->orientation[0] = 1.0;
}

extern "C" void rbps_collider_desc_default(rbps_collider_desc *d)
{
    std::memset(d, 0, sizeof(*d));
    d->shape = RBPS_SHAPE_SPHERE;
    d->params[0] = 0.5;
    d->local_rot[0] = 1.0;
    d->restitution = 0.5;
    d->static_friction = 0.5;
    d->dynamic_friction = 0.5;
}

extern "C" void rbps_joint_desc_default(rbps_joint_desc *d, int32_t type)
{
    std::memset(d, 0, sizeof(*d));
    d->type = type;
    if (type != RBPS_JOINT_FIXED) // FixedJointParams has no axis (JointAPI.hpp:63-69)
        d->axis[0] = 1.0;
    if (type == RBPS_JOINT_REVOLUTE)
        d->limit_axis[1] = 1.0;
}

// ------------------------------------------------------------ creation
extern "C" int rbps_batch_create(const rbps_batch_desc *desc, rbps_batch **out)
{
    if (!desc || !out)
        return fail(RBPS_ERR_INVALID, "rbps_batch_create: null argument");
    if (desc->n_worlds == 0 || desc->substeps <= 0 || !(desc->timestep > 0.0))
        return fail(RBPS_ERR_INVALID, "rbps_batch_create: need n_worlds > 0, substeps > 0, timestep > 0");
    if (desc->precision < 0 || desc->precision > 2 || desc->solve_mode < 0 || desc->solve_mode > 1)
        return fail(RBPS_ERR_INVALID, "rbps_batch_create: bad precision or solve mode");
    if (desc->block_threads && (desc->block_threads % 32 || desc->block_threads > 256))
        return fail(RBPS_ERR_INVALID, "rbps_batch_create: block_threads must be a multiple of 32 and <= 256");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(RBPS_ERR_CUDA, "rbps_batch_create: no CUDA device available");
    if (desc->device < 0 || desc->device >= ndev)
        return fail(RBPS_ERR_INVALID, "rbps_batch_create: device %d out of range", desc->device);
    CU(cudaSetDevice(desc->device));
    auto b = std::make_unique<rbps_batch>();
    b->desc = *desc;
    b->worlds.resize(desc->n_worlds);
    CU(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, desc->device));
    if (desc->stream)
        b->stream = (cudaStream_t)desc->stream;
    else
    {
        CU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->own_stream = true;
    }
    b->block = desc->block_threads ? (int)desc->block_threads : 128;
    for (int k = 0; k < kNumPhaseKernels; ++k)
        b->phase.block[k] = b->block;
    // the frame kernel's duration is the largest world's SAP on one CTA:
    // twice the threads for it (8.58 -> 8.26 ms a step on 4,096 uneven worlds)
    if (!desc->block_threads)
        b->phase.block[kKFrame] = 256;
    *out = b.release();
    return RBPS_OK;
}

extern "C" int rbps_batch_destroy(rbps_batch *b)
{
    delete b;
    return RBPS_OK;
}

static int check_world(rbps_batch *b, uint32_t world, bool adding)
{
    if (!b)
        return fail(RBPS_ERR_INVALID, "null batch");
    if (world >= b->worlds.size())
        return fail(RBPS_ERR_INVALID, "world %u out of range (%zu worlds)", world, b->worlds.size());
    if (adding && b->committed)
        return fail(RBPS_ERR_INVALID, "batch already committed: no adds after rbps_batch_commit");
    return RBPS_OK;
}

extern "C" int rbps_hull_create(rbps_batch *b, const double *verts, uint32_t n_verts, const uint32_t *tris,
                                uint32_t n_tris, uint32_t *hull_id)
{
    if (!b || !verts || n_verts == 0)
        return fail(RBPS_ERR_INVALID, "rbps_hull_create: need vertices");
    if (b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_hull_create: batch already committed");
    for (uint32_t t = 0; tris && t < 3 * n_tris; ++t)
        if (tris[t] >= n_verts)
            return fail(RBPS_ERR_INVALID, "rbps_hull_create: triangle index out of range");
    HostHull h;
    h.verts.assign(verts, verts + 3 * n_verts);
    build_hull_tables(h, tris, n_tris);
    // local AABB as convex_hull_data_create computes it (ConvexHull.hpp:401-414)
    double mn[3] = {(double)1e30f, (double)1e30f, (double)1e30f};
    double mx[3] = {(double)-1e30f, (double)-1e30f, (double)-1e30f};
    for (uint32_t v = 0; v < n_verts; ++v)
        for (int k = 0; k < 3; ++k)
        {
            mn[k] = rmin(mn[k], verts[3 * v + k]);
            mx[k] = rmax(mx[k], verts[3 * v + k]);
        }
    for (int k = 0; k < 3; ++k)
    {
        h.aabb[k] = mn[k];
        h.aabb[3 + k] = mx[k];
    }
    b->hulls.push_back(std::move(h));
    if (hull_id)
        *hull_id = (uint32_t)(b->hulls.size() - 1);
    return RBPS_OK;
}

extern "C" int rbps_heightmap_create(rbps_batch *b, const float *heights, uint32_t rows, uint32_t cols,
                                     const double *scale, const double *origin, uint32_t *id)
{
    if (!b || !heights || !scale || !origin || rows < 2 || cols < 2)
        return fail(RBPS_ERR_INVALID, "rbps_heightmap_create: need heights, scale, origin and a 2 x 2 grid at least");
    if (b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_heightmap_create: batch already committed");
    HostHeightmap h;
    const size_t n = (size_t)rows * cols;
    h.heights.assign(heights, heights + n);
    h.d.rows = rows;
    h.d.cols = cols;
    for (int k = 0; k < 3; ++k)
    {
        h.d.scale[k] = scale[k];
        h.d.origin[k] = origin[k];
    }
    // heightmap_data_create: min / max over the samples in float, then
    // scaled into world heights in double
    float mn = std::numeric_limits<float>::max(), mx = std::numeric_limits<float>::lowest();
    for (size_t i = 0; i < n; ++i)
    {
        mn = std::min(mn, heights[i]);
        mx = std::max(mx, heights[i]);
    }
    h.d.min_h = (double)mn * scale[1] + origin[1];
    h.d.max_h = (double)mx * scale[1] + origin[1];
    b->heightmaps.push_back(std::move(h));
    if (id)
        *id = (uint32_t)(b->heightmaps.size() - 1);
    return RBPS_OK;
}

extern "C" int rbps_mesh_create(rbps_batch *b, const double *verts, uint32_t n_verts, const uint32_t *indices,
                                uint32_t n_faces, uint32_t *id)
{
    if (!b || !verts || !indices || n_verts == 0 || n_faces == 0)
        return fail(RBPS_ERR_INVALID, "rbps_mesh_create: need vertices and faces");
    if (b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_mesh_create: batch already committed");
    for (uint32_t t = 0; t < 3 * n_faces; ++t)
        if (indices[t] >= n_verts)
            return fail(RBPS_ERR_INVALID, "rbps_mesh_create: face index out of range");
    HostMesh m;
    m.verts.assign(verts, verts + 3 * (size_t)n_verts);
    m.idx.assign(indices, indices + 3 * (size_t)n_faces);
    auto v = [&](uint32_t k) { return vec3<double>(verts[3 * k], verts[3 * k + 1], verts[3 * k + 2]); };
    for (uint32_t f = 0; f < n_faces; ++f)
    {
        const vec3<double> A = v(indices[3 * f]), B = v(indices[3 * f + 1]), C = v(indices[3 * f + 2]);
        const vec3<double> n = normalize(cross(B - A, C - A));
        m.normals.insert(m.normals.end(), {n.x, n.y, n.z});
    }
    double mn[3] = {(double)1e30f, (double)1e30f, (double)1e30f};
    double mx[3] = {(double)-1e30f, (double)-1e30f, (double)-1e30f};
    for (uint32_t k = 0; k < n_verts; ++k)
        for (int a = 0; a < 3; ++a)
        {
            mn[a] = rmin(mn[a], verts[3 * k + a]);
            mx[a] = rmax(mx[a], verts[3 * k + a]);
        }
    for (int a = 0; a < 3; ++a)
    {
        m.d.aabb[a] = mn[a];
        m.d.aabb[3 + a] = mx[a];
    }
    m.d.nv = n_verts;
    m.d.nf = n_faces;
    b->meshes.push_back(std::move(m));
    if (id)
        *id = (uint32_t)(b->meshes.size() - 1);
    return RBPS_OK;
}

extern "C" int rbps_world_add_bodies(rbps_batch *b, uint32_t world, uint32_t n, const rbps_body_desc *d,
                                     uint32_t *first_id)
{
    int rc = check_world(b, world, true);
    if (rc)
        return rc;
    if (n && !d)
        return fail(RBPS_ERR_INVALID, "rbps_world_add_bodies: null descriptors");
    HostWorld &w = b->worlds[world];
    if (first_id)
        *first_id = (uint32_t)w.bodies.size();
    for (uint32_t i = 0; i < n; ++i)
    {
        if (d[i].type != RBPS_BODY_STATIC && !(d[i].mass > 0.0))
            return fail(RBPS_ERR_INVALID, "dynamic body needs mass > 0");
        w.bodies.push_back(d[i]);
        // create_body bakes gravity into the force (BodyAPI.hpp:61)
        w.force.push_back(0.0);
        w.force.push_back((double)(-9.8f) * d[i].mass);
        w.force.push_back(0.0);
        w.torque.insert(w.torque.end(), {0.0, 0.0, 0.0});
    }
    return RBPS_OK;
}

extern "C" int rbps_world_add_body(rbps_batch *b, uint32_t world, const rbps_body_desc *d, uint32_t *id)
{
    return rbps_world_add_bodies(b, world, 1, d, id);
}

extern "C" int rbps_world_set_body_force(rbps_batch *b, uint32_t world, uint32_t body, const double f[3],
                                         const double t[3])
{
    int rc = check_world(b, world, true);
    if (rc)
        return rc;
    HostWorld &w = b->worlds[world];
    if (body >= w.bodies.size())
        return fail(RBPS_ERR_INVALID, "body %u out of range", body);
    for (int k = 0; k < 3; ++k)
    {
        if (f)
            w.force[3 * body + k] = f[k];
        if (t)
            w.torque[3 * body + k] = t[k];
    }
    return RBPS_OK;
}

extern "C" int rbps_world_add_colliders(rbps_batch *b, uint32_t world, uint32_t n, const rbps_collider_desc *d,
                                        uint32_t *first_id)
{
    int rc = check_world(b, world, true);
    if (rc)
        return rc;
    HostWorld &w = b->worlds[world];
    if (first_id)
        *first_id = (uint32_t)w.colliders.size();
    for (uint32_t i = 0; i < n; ++i)
    {
        const rbps_collider_desc &c = d[i];
        if (c.body_id >= w.bodies.size())
            return fail(RBPS_ERR_INVALID, "collider body %u does not exist", c.body_id);
        if (!shape_supported(c.shape))
            return fail(RBPS_ERR_INVALID, "unsupported shape kind %d", c.shape);
        if (c.shape == RBPS_SHAPE_HEIGHTMAP && c.hull >= b->heightmaps.size())
            return fail(RBPS_ERR_INVALID, "collider %u: unknown heightmap %u", i, c.hull);
        if (c.shape == RBPS_SHAPE_MESH && c.hull >= b->meshes.size())
            return fail(RBPS_ERR_INVALID, "collider %u: unknown mesh %u", i, c.hull);
        if (c.shape == RBPS_SHAPE_CONVEX_HULL && c.hull >= b->hulls.size())
            return fail(RBPS_ERR_INVALID, "hull %u does not exist", c.hull);
        w.colliders.push_back(c);
    }
    return RBPS_OK;
}

extern "C" int rbps_world_add_collider(rbps_batch *b, uint32_t world, const rbps_collider_desc *d, uint32_t *id)
{
    return rbps_world_add_colliders(b, world, 1, d, id);
}

extern "C" int rbps_world_add_joint(rbps_batch *b, uint32_t world, const rbps_joint_desc *d, uint32_t *id)
{
    int rc = check_world(b, world, true);
    if (rc)
        return rc;
    HostWorld &w = b->worlds[world];
    if (!d || d->body_1 >= w.bodies.size() || d->body_2 >= w.bodies.size())
        return fail(RBPS_ERR_INVALID, "joint bodies out of range");
    if (d->type < RBPS_JOINT_PRISMATIC || d->type > RBPS_JOINT_SPHERICAL)
        return fail(RBPS_ERR_INVALID, "bad joint type %d", d->type);
    if (id)
        *id = (uint32_t)w.joints.size();
    w.joints.push_back(*d);
    return RBPS_OK;
}

// ------------------------------------------------------------ commit
namespace
{
    template <class T, class P>
    Engine<T, P> make_engine(rbps_batch *b)
    {
        Engine<T, P> e;
        std::memset(&e, 0, sizeof(e));
        e.B.pos = (V4<P> *)b->pos;
        e.B.rot = (Q4<T> *)b->rot;
        e.B.lin = (V4<T> *)b->lin;
        e.B.ang = (V4<T> *)b->ang;
        e.B.prev_pos = (V4<P> *)b->prev_pos;
        e.B.prev_rot = (Q4<T> *)b->prev_rot;
        e.B.force = (V4<T> *)b->force;
        e.B.torque = (V4<T> *)b->torque;
        e.B.inertia = (S8<T> *)b->inertia;
        e.B.inv_inertia = (S8<T> *)b->inv_inertia;
        e.B.type = b->btype;
        e.shape = b->shape;
        e.c_body = b->c_body;
        e.c_lpos = b->c_lpos;
        e.c_lrot = b->c_lrot;
        e.c_static = b->c_static;
        e.c_mat = (const V4<T> *)b->c_mat;
        e.hulls.verts = b->hull_verts;
        e.hulls.v_off = b->hull_voff;
        e.hulls.local_aabb = b->hull_aabb;
        e.hulls.desc = b->hull_desc;
        e.hulls.u32 = b->hull_u32;
        e.hulls.poly_n = b->hull_pn;
        e.hulls.hm_heights = b->hm_heights;
        e.hulls.hm_desc = b->hm_desc;
        e.hulls.mesh = b->mesh_desc;
        e.hulls.mesh_v = b->mesh_v;
        e.hulls.mesh_i = b->mesh_i;
        e.hulls.mesh_n = b->mesh_n;
        e.bp_coll = b->bp_coll;
        e.fat = b->fat;
        e.ep_key = b->ep_key;
        e.ep_id = b->ep_id;
        e.ep_pos = b->ep_pos;
        e.plane_cand = b->plane_cand;
        e.joints = (Joint<T> *)b->joints_d;
        e.rows = (Row<T> *)b->rows_d;
        e.jorder = b->jorder;
        e.jcolor_off = b->jcolor_off;
        e.worlds = b->worlds_d;
        e.stats = b->stats_d;
        e.error = b->error_d;
        const double h = b->desc.timestep / b->desc.substeps;
        e.dt_frame = b->desc.timestep;
        e.h = T(h);
        e.inv_h = T(1.0 / h);
        e.substeps = b->desc.substeps;
        e.fat_margin = b->desc.fat_margin;
        e.reinsert_threshold = b->desc.reinsert_threshold;
        e.solve_mode = b->desc.solve_mode;
        e.use_vel_exp = b->desc.use_velocity_expansion;
        e.check_state = b->check_state ? 1 : 0;
        e.stats_in_substep = 0;
        e.narrow_per_warp = b->narrow_per_warp;
        e.color_chunk = b->color_chunk;
        e.work_counter = b->work_counter;
        e.scratch = b->scratch;
        e.wcoff = b->wcoff;
        e.gcol = b->gcol;
        e.nlist = b->nlist;
        e.nglob = b->nglob;
        e.wcand = (Cand *const *)b->wcand;
        e.wcc = (CandContacts<T, P> *const *)b->wcc;
        e.sbodies = b->sbodies;
        e.n_sbodies = b->n_sbodies;
        e.sjoints = b->sjoints;
        e.sjcoff = b->sjcoff;
        e.n_sjcolors = b->n_sjcolors;
        e.n_sjoints = b->n_sjoints;
        e.small_worlds = b->small_list;
        e.n_small = (uint32_t)b->small_ids.size();
        e.n_block_worlds = b->n_block_worlds;
        e.smem_cap_block = b->smem_cap_block;
        e.smem_cap_warp = b->smem_cap_warp;
        e.n_pair_worlds = b->n_pair_worlds;
        e.smem_cap_pair = b->smem_cap_pair;
        e.dump_pairs = b->dump ? b->dump_pairs : nullptr;
        e.dump_cand = b->dump ? b->dump_cand : nullptr;
        e.dump_cc = b->dump ? (CandContacts<T, P> *)b->dump_cc : nullptr;
        e.dump_color = b->dump ? b->dump_color : nullptr;
        e.dump_pair_cap = b->dump_pair_cap;
        e.dump_cand_cap = b->dump_cand_cap;
        e.prof = b->prof_off ? nullptr : b->prof;
        e.gjk_list = b->gjk_list;
        e.gjk_count = b->gjk_count;
        e.gjk_cap = b->gjk_cap;
        e.gjk_slots = b->gjk_slots;
        e.origin = b->origin_d;
        e.body_world = b->body_world_d;
        return e;
    }

    size_t cc_size_of(int precision)
    {
        if (precision == RBPS_PRECISION_FP64)
            return sizeof(CandContacts<double, double>);
        return sizeof(CandContacts<float, float>); // FP32 and FP32_POS64
    }

    template <class T>
    void put_v4(std::vector<char> &buf, size_t idx, double x, double y, double z, double w)
    {
        T *p = (T *)(buf.data() + idx * 4 * sizeof(T));
        p[0] = T(x); p[1] = T(y); p[2] = T(z); p[3] = T(w);
    }

    constexpr uint32_t kSmallWorldBodies = kGridWorldBodies; // larger worlds step on the cooperative grid
    constexpr int kMaxBlockHost = 256; // block of the flat kernels (their __launch_bounds__)
    constexpr uint32_t kBlockTeamBodies = 256; // colored batches: worlds this large step on a whole CTA
    constexpr uint32_t kPairTeamBodies = 96;   // ... and worlds this large on half a CTA
    constexpr uint32_t kSmemBodiesMax = 1024;   // bodies a CTA world keeps in shared memory (137 KB in FP32)
} // namespace

// Worlds of `threshold` bodies or more step on a whole CTA in the substep
// kernel, worlds of `pair` bodies or more (and fewer than `threshold`) on
// half a CTA, the rest on one warp each (small_ids is sorted by body count,
// largest first); pair >= threshold leaves no half-CTA worlds.  Shared-memory
// world copies hold the largest CTA world, two half-CTA worlds or four warp
// worlds (a world beyond its cap runs on the batch arrays).
template <class T, class P>
static int set_team_split(rbps_batch *b, uint32_t threshold, uint32_t pair)
{
    pair = std::min(pair, threshold);
    const uint32_t ns = (uint32_t)b->small_ids.size();
    uint32_t nbw = 0;
    while (nbw < ns && b->wdev[b->small_ids[nbw]].n_bodies >= threshold)
        ++nbw;
    uint32_t npw = 0;
    while (nbw + npw < ns && b->wdev[b->small_ids[nbw + npw]].n_bodies >= pair)
        ++npw;
    b->n_block_worlds = nbw;
    b->n_pair_worlds = npw;
    b->flat.grid_solve = (int)(nbw + (npw + 1) / 2 + (ns - nbw - npw + 3) / 4);
    auto round16 = [](uint32_t x) { return (x + 15u) / 16u * 16u; };
    b->smem_cap_warp = round16(pair);
    b->smem_cap_pair = npw ? round16(std::min<uint32_t>(b->wdev[b->small_ids[nbw]].n_bodies, kSmemBodiesMax)) : 0;
    b->smem_cap_block = 0;
    if (nbw)
        b->smem_cap_block = round16(std::min<uint32_t>(b->wdev[b->small_ids[0]].n_bodies, kSmemBodiesMax));
    b->flat.substep_smem = std::max({4 * smem_world_bytes<T, P>(b->smem_cap_warp),
                                     2 * smem_world_bytes<T, P>(b->smem_cap_pair),
                                     smem_world_bytes<T, P>(b->smem_cap_block)});
    CU(prepare_substep<T, P>(b->flat.substep_smem));
    b->team_bodies = threshold;
    b->pair_bodies = pair;
    return RBPS_OK;
}

template <class T, class P>
static int commit_typed(rbps_batch *b)
{
    const uint32_t W = (uint32_t)b->worlds.size();
    // ---- offsets
    b->wdev.assign(W, WorldDev{});
    uint32_t nb = 0, nc = 0, nbp = 0, npc = 0, nj = 0, nr = 0, njc = 0;
    std::vector<std::vector<uint32_t>> bp_lists(W);
    std::vector<std::vector<uint2>> pc_lists(W);
    std::vector<std::vector<uint32_t>> jorders(W), joffs(W);
    for (uint32_t w = 0; w < W; ++w)
    {
        const HostWorld &hw = b->worlds[w];
        WorldDev &d = b->wdev[w];
        d.body_off = nb;
        d.n_bodies = (uint32_t)hw.bodies.size();
        d.coll_off = nc;
        d.n_coll = (uint32_t)hw.colliders.size();
        for (uint32_t c = 0; c < d.n_coll; ++c)
            if (hw.colliders[c].shape != RBPS_SHAPE_PLANE)
                bp_lists[w].push_back(c);
        d.bp_off = nbp;
        d.n_bp = (uint32_t)bp_lists[w].size();
        // plane loop of run_narrow_phase (CollisionPipeline.cpp:159-196)
        for (uint32_t pi = 0; pi < d.n_coll; ++pi)
        {
            const rbps_collider_desc &pc = hw.colliders[pi];
            if (pc.shape != RBPS_SHAPE_PLANE)
                continue;
            for (uint32_t di = 0; di < d.n_coll; ++di)
            {
                const rbps_collider_desc &dc = hw.colliders[di];
                if (di == pi || dc.shape == RBPS_SHAPE_PLANE)
                    continue;
                if (pc.is_static && dc.is_static)
                    continue;
                if (pc.body_id == dc.body_id)
                    continue;
                pc_lists[w].push_back(make_uint2(di, pi));
            }
        }
        d.pc_off = npc;
        d.n_pc = (uint32_t)pc_lists[w].size();
        d.joint_off = nj;
        d.n_joints = (uint32_t)hw.joints.size();
        d.row_off = nr;
        uint32_t rows = 0;
        for (const auto &j : hw.joints)
            rows += j.type == RBPS_JOINT_REVOLUTE ? 4 : (j.type == RBPS_JOINT_PRISMATIC ? 3 : 2); // fixed, spherical: 2
        d.n_rows = rows;
        // greedy joint colouring by shared dynamic bodies
        {
            std::vector<uint32_t> color(d.n_joints, 0);
            uint32_t ncol = 0;
            std::vector<std::vector<uint32_t>> body_cols(d.n_bodies);
            for (uint32_t j = 0; j < d.n_joints; ++j)
            {
                const auto &jd = hw.joints[j];
                std::vector<uint32_t> used;
                for (uint32_t bb : {jd.body_1, jd.body_2})
                    if (hw.bodies[bb].type != RBPS_BODY_STATIC)
                        used.insert(used.end(), body_cols[bb].begin(), body_cols[bb].end());
                uint32_t c = 0;
                while (std::find(used.begin(), used.end(), c) != used.end())
                    ++c;
                color[j] = c;
                ncol = std::max(ncol, c + 1);
                for (uint32_t bb : {jd.body_1, jd.body_2})
                    if (hw.bodies[bb].type != RBPS_BODY_STATIC)
                        body_cols[bb].push_back(c);
            }
            std::vector<uint32_t> off(ncol + 1, 0);
            for (uint32_t j = 0; j < d.n_joints; ++j)
                off[color[j] + 1]++;
            for (uint32_t c = 0; c < ncol; ++c)
                off[c + 1] += off[c];
            std::vector<uint32_t> fill(off.begin(), off.end() - 1), order(d.n_joints);
            for (uint32_t j = 0; j < d.n_joints; ++j)
                order[fill[color[j]]++] = j;
            jorders[w] = order;
            joffs[w] = off;
            d.jc_off = njc;
            d.n_jcolors = ncol;
            njc += ncol + 1;
        }
        d.pair_cap = b->desc.max_pairs_per_world ? b->desc.max_pairs_per_world
                                                 : std::max<uint32_t>(1024u, 8u * d.n_bp);
        d.dump_slot = ~0u;
        nb += d.n_bodies;
        nc += d.n_coll;
        nbp += d.n_bp;
        npc += d.n_pc;
        nj += d.n_joints;
        nr += rows;
    }
    b->n_bodies_all = nb;
    b->n_coll_all = nc;
    b->n_bp_all = nbp;
    b->n_joint_all = nj;
    b->n_row_all = nr;

    // ---- bodies
    std::vector<char> pos(nb * 4 * sizeof(P)), ppos(nb * 4 * sizeof(P));
    std::vector<char> rot(nb * 4 * sizeof(T)), lin(nb * 4 * sizeof(T)), ang(nb * 4 * sizeof(T));
    std::vector<char> frc(nb * 4 * sizeof(T)), trq(nb * 4 * sizeof(T));
    std::vector<char> inr(nb * 8 * sizeof(T)), iinr(nb * 8 * sizeof(T));
    std::vector<uint8_t> btype(nb);
    b->total_bodies = nb;
    b->total_dynamic = 0;
    b->origin.assign(3 * (size_t)W, 0.0);
    b->body_world.clear();
    if (b->relative())
    {
        // origin = centre of the box around the world's body positions
        b->body_world.resize(nb);
        for (uint32_t w = 0; w < W; ++w)
        {
            const HostWorld &hw = b->worlds[w];
            for (int k = 0; k < 3 && !hw.bodies.empty(); ++k)
            {
                double lo = hw.bodies[0].position[k], hi = lo;
                for (const auto &d : hw.bodies)
                {
                    lo = std::min(lo, d.position[k]);
                    hi = std::max(hi, d.position[k]);
                }
                b->origin[3 * (size_t)w + k] = 0.5 * (lo + hi);
            }
            for (uint32_t i = 0; i < hw.bodies.size(); ++i)
                b->body_world[b->wdev[w].body_off + i] = w;
        }
    }
    for (uint32_t w = 0; w < W; ++w)
    {
        const HostWorld &hw = b->worlds[w];
        const double *ow = b->origin_of_world(w);
        for (uint32_t i = 0; i < hw.bodies.size(); ++i)
        {
            const rbps_body_desc &d = hw.bodies[i];
            const size_t g = b->wdev[w].body_off + i;
            const bool st = d.type == RBPS_BODY_STATIC;
            const double inv_mass = st ? 0.0 : 1.0 / d.mass;
            double iinv[6] = {0, 0, 0, 0, 0, 0};
            if (!st)
                smat3_inverse(d.inertia, iinv);
            put_v4<P>(pos, g, d.position[0] - ow[0], d.position[1] - ow[1], d.position[2] - ow[2], 0);
            put_v4<P>(ppos, g, d.position[0] - ow[0], d.position[1] - ow[1], d.position[2] - ow[2], 0);
            put_v4<T>(rot, g, d.orientation[0], d.orientation[1], d.orientation[2], d.orientation[3]);
            put_v4<T>(lin, g, d.linear_velocity[0], d.linear_velocity[1], d.linear_velocity[2], inv_mass);
            put_v4<T>(ang, g, d.angular_velocity[0], d.angular_velocity[1], d.angular_velocity[2], 0);
            put_v4<T>(frc, g, hw.force[3 * i], hw.force[3 * i + 1], hw.force[3 * i + 2], 0);
            put_v4<T>(trq, g, hw.torque[3 * i], hw.torque[3 * i + 1], hw.torque[3 * i + 2], 0);
            T *I = (T *)(inr.data() + g * 8 * sizeof(T));
            T *Ii = (T *)(iinr.data() + g * 8 * sizeof(T));
            for (int k = 0; k < 6; ++k)
            {
                I[k] = T(d.inertia[k]);
                Ii[k] = T(iinv[k]);
            }
            I[6] = I[7] = Ii[6] = Ii[7] = T(0);
            btype[g] = st ? kStatic : kDynamic;
            if (!st)
                b->total_dynamic++;
        }
    }
    int rc = 0;
    auto up = [&](void **dst, const std::vector<char> &v) {
        if (rc)
            return;
        rc = b->alloc(dst, v.size());
        if (!rc && !v.empty())
            if (cudaMemcpy(*dst, v.data(), v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
                rc = fail(RBPS_ERR_CUDA, "upload failed");
    };
    up(&b->pos, pos);
    up(&b->prev_pos, ppos);
    if (b->relative())
    {
        int rc2;
        if ((rc2 = b->upload(&b->origin_d, b->origin)) || (rc2 = b->upload(&b->body_world_d, b->body_world)))
            return rc2;
    }
    up(&b->rot, rot);
    up(&b->prev_rot, rot);
    up(&b->lin, lin);
    up(&b->ang, ang);
    up(&b->force, frc);
    up(&b->torque, trq);
    up(&b->inertia, inr);
    up(&b->inv_inertia, iinr);
    if (rc)
        return rc;
    if ((rc = b->upload(&b->btype, btype)))
        return rc;

    // ---- hulls
    {
        std::vector<double> hv, ha;
        std::vector<uint32_t> hoff(1, 0);
        for (const auto &h : b->hulls)
        {
            hv.insert(hv.end(), h.verts.begin(), h.verts.end());
            hoff.push_back((uint32_t)(hv.size() / 3));
            ha.insert(ha.end(), h.aabb, h.aabb + 6);
        }
        std::vector<HullDesc> hd;
        std::vector<uint32_t> u32;
        std::vector<double> pn;
        for (const auto &h : b->hulls)
        {
            HullDesc d{};
            d.np = (uint32_t)(h.poly_off.size() - 1);
            auto put = [&u32](const std::vector<uint32_t> &v) {
                const uint32_t base = (uint32_t)u32.size();
                u32.insert(u32.end(), v.begin(), v.end());
                return base;
            };
            d.po = put(h.poly_off);
            d.pi = put(h.poly_idx);
            d.pn = (uint32_t)(pn.size() / 3);
            pn.insert(pn.end(), h.poly_n.begin(), h.poly_n.end());
            d.v2p_o = put(h.v2p_off);
            d.v2p_i = put(h.v2p_idx);
            d.v2n_o = put(h.v2n_off);
            d.v2n_i = put(h.v2n_idx);
            d.p2p_o = put(h.p2p_off);
            d.p2p_i = put(h.p2p_idx);
            hd.push_back(d);
        }
        if ((rc = b->upload(&b->hull_verts, hv)) || (rc = b->upload(&b->hull_voff, hoff)) ||
            (rc = b->upload(&b->hull_aabb, ha)) || (rc = b->upload(&b->hull_desc, hd)) ||
            (rc = b->upload(&b->hull_u32, u32)) || (rc = b->upload(&b->hull_pn, pn)))
            return rc;
    }
    // ---- heightmaps
    {
        std::vector<float> hh;
        std::vector<HmDesc> hd;
        for (const auto &h : b->heightmaps)
        {
            HmDesc d = h.d;
            d.off = (uint32_t)hh.size();
            hh.insert(hh.end(), h.heights.begin(), h.heights.end());
            hd.push_back(d);
        }
        if ((rc = b->upload(&b->hm_heights, hh)) || (rc = b->upload(&b->hm_desc, hd)))
            return rc;
    }
    // ---- triangle meshes
    {
        std::vector<double> mv, mnrm;
        std::vector<uint32_t> mi;
        std::vector<MeshDesc> md;
        for (const auto &m : b->meshes)
        {
            MeshDesc d = m.d;
            d.v0 = (uint32_t)(mv.size() / 3);
            d.f0 = (uint32_t)(mi.size() / 3);
            mv.insert(mv.end(), m.verts.begin(), m.verts.end());
            mi.insert(mi.end(), m.idx.begin(), m.idx.end());
            mnrm.insert(mnrm.end(), m.normals.begin(), m.normals.end());
            md.push_back(d);
        }
        if ((rc = b->upload(&b->mesh_desc, md)) || (rc = b->upload(&b->mesh_v, mv)) ||
            (rc = b->upload(&b->mesh_i, mi)) || (rc = b->upload(&b->mesh_n, mnrm)))
            return rc;
    }
    HullSetDev hs_host{nullptr, nullptr, nullptr};

    // ---- colliders + initial SAP state (broad_phase_insert, BroadPhase.cpp:169-197)
    std::vector<ShapeDev> shp(nc);
    std::vector<uint32_t> cbody(nc), bpc(nbp), epk(2 * (size_t)nbp), epi(2 * (size_t)nbp), epp(2 * (size_t)nbp);
    std::vector<V4<double>> clp(nc);
    std::vector<Q4<double>> clr(nc);
    std::vector<uint8_t> cst(nc);
    std::vector<char> cmat(nc * 4 * sizeof(T));
    std::vector<FatBox> fat(nbp);
    std::vector<uint2> pcs;
    pcs.reserve(npc);
    for (uint32_t w = 0; w < W; ++w)
    {
        const HostWorld &hw = b->worlds[w];
        const WorldDev &d = b->wdev[w];
        for (uint32_t c = 0; c < d.n_coll; ++c)
        {
            const rbps_collider_desc &cd = hw.colliders[c];
            const size_t g = d.coll_off + c;
            ShapeDev s{};
            s.kind = cd.shape;
            s.hull = (int)cd.hull;
            for (int k = 0; k < 4; ++k)
                s.p[k] = cd.params[k];
            shp[g] = s;
            cbody[g] = cd.body_id;
            clp[g] = V4<double>{cd.local_pos[0], cd.local_pos[1], cd.local_pos[2], 0.0};
            clr[g] = Q4<double>{cd.local_rot[0], cd.local_rot[1], cd.local_rot[2], cd.local_rot[3]};
            cst[g] = cd.is_static ? 1 : 0;
            put_v4<T>(cmat, g, cd.restitution, cd.static_friction, cd.dynamic_friction, 0);
        }
        for (uint32_t o = 0; o < d.n_bp; ++o)
        {
            const uint32_t c = bp_lists[w][o];
            const rbps_collider_desc &cd = hw.colliders[c];
            const rbps_body_desc &bd = hw.bodies[cd.body_id];
            bpc[d.bp_off + o] = c;
            tf<double> t;
            const double *ow = b->origin_of_world(w);
            const vec3<double> bp(bd.position[0] - ow[0], bd.position[1] - ow[1], bd.position[2] - ow[2]);
            const quat<double> br(bd.orientation[0], bd.orientation[1], bd.orientation[2], bd.orientation[3]);
            t.pos = bp + rotate(br, vec3<double>(cd.local_pos[0], cd.local_pos[1], cd.local_pos[2]));
            t.rot = br * quat<double>(cd.local_rot[0], cd.local_rot[1], cd.local_rot[2], cd.local_rot[3]);
            HullSetDev hs = hs_host;
            std::vector<double> la;
            if (cd.shape == RBPS_SHAPE_CONVEX_HULL)
            {
                la.assign(b->hulls[cd.hull].aabb, b->hulls[cd.hull].aabb + 6);
                hs.local_aabb = la.data();
            }
            if (cd.shape == RBPS_SHAPE_HEIGHTMAP)
                hs.hm_desc = &b->heightmaps[cd.hull].d;
            if (cd.shape == RBPS_SHAPE_MESH)
                hs.mesh = &b->meshes[cd.hull].d;
            ShapeDev s = shp[d.coll_off + c];
            s.hull = 0;
            const aabb tight = compute_aabb(s, t, hs);
            const aabb f = aabb_expand(tight, b->desc.fat_margin);
            FatBox fb;
            fb.mn[0] = f.mn.x; fb.mn[1] = f.mn.y; fb.mn[2] = f.mn.z;
            fb.mx[0] = f.mx.x; fb.mx[1] = f.mx.y; fb.mx[2] = f.mx.z;
            fat[d.bp_off + o] = fb;
            const size_t e0 = 2 * (size_t)d.bp_off;
            epk[e0 + 2 * o] = order_key_host((float)f.mn.x);
            epk[e0 + 2 * o + 1] = order_key_host((float)f.mx.x);
            epi[e0 + 2 * o] = 2 * o;
            epi[e0 + 2 * o + 1] = 2 * o + 1;
            epp[e0 + 2 * o] = 2 * o;
            epp[e0 + 2 * o + 1] = 2 * o + 1;
        }
        pcs.insert(pcs.end(), pc_lists[w].begin(), pc_lists[w].end());
    }
    if ((rc = b->upload(&b->shape, shp)) || (rc = b->upload(&b->c_body, cbody)) || (rc = b->upload(&b->c_lpos, clp)) ||
        (rc = b->upload(&b->c_lrot, clr)) || (rc = b->upload(&b->c_static, cst)) || (rc = b->upload(&b->bp_coll, bpc)) ||
        (rc = b->upload(&b->fat, fat)) || (rc = b->upload(&b->ep_key, epk)) || (rc = b->upload(&b->ep_id, epi)) ||
        (rc = b->upload(&b->ep_pos, epp)) || (rc = b->upload(&b->plane_cand, pcs)))
        return rc;
    up(&b->c_mat, cmat);
    if (rc)
        return rc;

    // ---- joints and their constraint rows (JointAPI.hpp:191-267)
    {
        std::vector<Joint<T>> js(nj);
        std::vector<Row<T>> rs(nr);
        for (uint32_t w = 0; w < W; ++w)
        {
            const HostWorld &hw = b->worlds[w];
            const WorldDev &d = b->wdev[w];
            uint32_t row = d.row_off;
            for (uint32_t j = 0; j < d.n_joints; ++j)
            {
                const rbps_joint_desc &jd = hw.joints[j];
                Joint<T> J{};
                J.r1 = V4<T>{T(jd.r_1[0]), T(jd.r_1[1]), T(jd.r_1[2]), T(0)};
                J.r2 = V4<T>{T(jd.r_2[0]), T(jd.r_2[1]), T(jd.r_2[2]), T(0)};
                J.axis = V4<T>{T(jd.axis[0]), T(jd.axis[1]), T(jd.axis[2]), T(0)};
                if (jd.type == RBPS_JOINT_REVOLUTE)
                    J.limit_axis = V4<T>{T(jd.limit_axis[0]), T(jd.limit_axis[1]), T(jd.limit_axis[2]), T(0)};
                // a spherical joint's cone is symmetric: [-upper, upper]
                const double lower = jd.type == RBPS_JOINT_SPHERICAL ? -jd.upper_limit : jd.lower_limit;
                J.lower = T(lower);
                J.upper = T(jd.upper_limit);
                J.target_pos = T(jd.target_position);
                J.target_speed = T(jd.target_speed);
                J.damping = T(jd.damping);
                // from_axis_angle of the clamped limit angle (quat.hpp:111-117)
                const double hl = lower * 0.5, hu = jd.upper_limit * 0.5;
                J.sin_lo = T(std::sin(hl));
                J.cos_lo = T(std::cos(hl));
                J.sin_hi = T(std::sin(hu));
                J.cos_hi = T(std::cos(hu));
                J.b1 = d.body_off + jd.body_1;
                J.b2 = d.body_off + jd.body_2;
                J.row0 = row;
                J.type = jd.type;
                J.act = jd.type == RBPS_JOINT_FIXED || jd.type == RBPS_JOINT_SPHERICAL ? RBPS_ACTUATION_FREE
                                                                                       : jd.actuation;
                J.limited = jd.type == RBPS_JOINT_FIXED ? 0 : jd.limited;
                int types[4];
                double comp[4] = {0, 0, 0, 0};
                int cnt;
                if (jd.type == RBPS_JOINT_REVOLUTE)
                {
                    cnt = 4;
                    types[0] = kRowRotational; types[1] = kRowPositional; types[2] = kRowRotational; types[3] = kRowRotational;
                    comp[3] = jd.compliance;
                }
                else if (jd.type == RBPS_JOINT_PRISMATIC)
                {
                    cnt = 3;
                    types[0] = kRowRotational; types[1] = kRowPositional; types[2] = kRowPositional;
                    comp[2] = jd.compliance;
                }
                else if (jd.type == RBPS_JOINT_SPHERICAL)
                {
                    cnt = 2;
                    types[0] = kRowPositional; types[1] = kRowRotational;
                    comp[0] = jd.compliance;
                }
                else
                {
                    cnt = 2;
                    types[0] = kRowRotational; types[1] = kRowPositional;
                }
                J.count = cnt;
                for (int r = 0; r < cnt; ++r)
                {
                    Row<T> R{};
                    R.dir = V4<T>{T(1.0), T(0.0), T(0.0), T(0.0)};
                    R.r1 = V4<T>{T(jd.r_1[0]), T(jd.r_1[1]), T(jd.r_1[2]), T(comp[r])};
                    R.r2 = V4<T>{T(jd.r_2[0]), T(jd.r_2[1]), T(jd.r_2[2]), T(0.0)};
                    R.b1 = J.b1;
                    R.b2 = J.b2;
                    R.type = types[r];
                    rs[row + r] = R;
                }
                row += cnt;
                js[d.joint_off + j] = J;
            }
        }
        // joint orders are world-local; colour offsets index jorder world slices
        std::vector<uint32_t> jord_g, jco_g;
        for (uint32_t w = 0, jo = 0; w < W; ++w)
        {
            const WorldDev &d = b->wdev[w];
            for (uint32_t k = 0; k < d.n_joints; ++k)
                jord_g.push_back(jorders[w][k]);
            for (uint32_t k = 0; k <= d.n_jcolors; ++k)
                jco_g.push_back(joffs[w][k] + jo);
            jo += d.n_joints;
        }
        std::vector<char> jb(js.size() * sizeof(Joint<T>)), rb(rs.size() * sizeof(Row<T>));
        if (!js.empty())
            std::memcpy(jb.data(), js.data(), jb.size());
        if (!rs.empty())
            std::memcpy(rb.data(), rs.data(), rb.size());
        up(&b->joints_d, jb);
        up(&b->rows_d, rb);
        if (rc)
            return rc;
        if ((rc = b->upload(&b->jorder, jord_g)) || (rc = b->upload(&b->jcolor_off, jco_g)))
            return rc;
    }

    // ---- executors: small worlds on persistent CTAs, large ones on the grid
    b->small_ids.clear();
    b->big_ids.clear();
    std::vector<uint32_t> order(W);
    for (uint32_t w = 0; w < W; ++w)
        order[w] = w;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t c) { return b->wdev[a].n_bodies > b->wdev[c].n_bodies; });
    uint32_t s_bp = 0, s_b = 0, s_pc = 0, s_npc = 0, g_bp = 0, g_b = 0, g_pc = 0, g_npc = 0;
    for (uint32_t w : order)
    {
        const WorldDev &d = b->wdev[w];
        if (d.n_bodies <= kSmallWorldBodies)
        {
            b->small_ids.push_back(w);
            s_bp = std::max(s_bp, d.n_bp); s_b = std::max(s_b, d.n_bodies);
            s_pc = std::max(s_pc, d.pair_cap); s_npc = std::max(s_npc, d.n_pc);
        }
        else
        {
            b->big_ids.push_back(w);
            g_bp = std::max(g_bp, d.n_bp); g_b = std::max(g_b, d.n_bodies);
            g_pc = std::max(g_pc, d.pair_cap); g_npc = std::max(g_npc, d.n_pc);
        }
    }
    const size_t ccs = cc_size_of(b->desc.precision);
    // per-world scratch slices
    size_t scr_total = 0;
    for (uint32_t w = 0; w < W; ++w)
    {
        WorldDev &d = b->wdev[w];
        d.scr_off = scr_total;
        scr_total += make_layout(d.n_bp, d.n_bodies, d.pair_cap, d.n_pc, ccs).stride;
    }
    if ((rc = b->alloc((void **)&b->scratch, std::max<size_t>(scr_total, 256))))
        return rc;
    if (!b->small_ids.empty())
    {
        for (int k = 0; k < kNumPhaseKernels; ++k)
        {
            int per_sm = 0;
            CU(occupancy_phase<T, P>(k, b->phase.block[k], &per_sm));
            if (per_sm < 1)
                return fail(RBPS_ERR_CUDA, "phase kernel %d cannot be resident with %d threads", k, b->phase.block[k]);
            b->phase.grid[k] = std::min<int>((int)b->small_ids.size(), per_sm * b->sm_count);
        }
        if ((rc = b->upload(&b->small_list, b->small_ids)))
            return rc;
    }
    if (!b->big_ids.empty())
    {
        int per_sm = 0;
        CU(occupancy_big<T, P>(b->block, &per_sm));
        if (per_sm < 1)
            return fail(RBPS_ERR_CUDA, "cooperative step kernel cannot be resident");
        b->grid_big = per_sm * b->sm_count;
    }
    b->n_counters = 2 + 4 * (uint32_t)b->desc.substeps;
    // ---- flat colored pipeline over the small worlds
    if (!b->small_ids.empty() && b->desc.solve_mode == RBPS_SOLVE_COLORED)
    {
        const uint32_t ns = (uint32_t)b->small_ids.size();
        size_t cand_cap = 0;
        std::vector<void *> wcand(W, nullptr), wcc(W, nullptr);
        std::vector<uint32_t> sbodies;
        uint32_t max_jc = 0;
        for (uint32_t w : b->small_ids)
        {
            const WorldDev &d = b->wdev[w];
            const ScratchLayout L = make_layout(d.n_bp, d.n_bodies, d.pair_cap, d.n_pc, ccs);
            wcand[w] = b->scratch + d.scr_off + L.cand;
            wcc[w] = b->scratch + d.scr_off + L.cc;
            cand_cap += (size_t)d.pair_cap + 1 + d.n_pc;
            for (uint32_t k = 0; k < d.n_bodies; ++k)
                sbodies.push_back(d.body_off + k);
            max_jc = std::max(max_jc, d.n_jcolors);
        }
        std::vector<uint32_t> sjoints, sjcoff(1, 0);
        for (uint32_t jc = 0; jc < max_jc; ++jc)
        {
            for (uint32_t w : b->small_ids)
            {
                const WorldDev &d = b->wdev[w];
                if (jc >= d.n_jcolors)
                    continue;
                for (uint32_t k = joffs[w][jc]; k < joffs[w][jc + 1]; ++k)
                    sjoints.push_back(d.joint_off + jorders[w][k]);
            }
            sjcoff.push_back((uint32_t)sjoints.size());
        }
        b->n_sbodies = (uint32_t)sbodies.size();
        b->n_sjoints = (uint32_t)sjoints.size();
        b->n_sjcolors = max_jc;
        if ((rc = b->alloc((void **)&b->wcoff, 4 * ((size_t)ns + 1))) ||
            (rc = b->alloc((void **)&b->gcol, 4 * (size_t)kGcolWords)) ||
            (rc = b->alloc((void **)&b->nlist, sizeof(uint2) * std::max<size_t>(cand_cap, 1))) ||
            (rc = b->alloc((void **)&b->nglob, sizeof(uint4) * std::max<size_t>(cand_cap, 1))) ||
            (rc = b->upload(&b->wcand, wcand)) || (rc = b->upload(&b->wcc, wcc)) ||
            (rc = b->upload(&b->sbodies, sbodies)) || (rc = b->upload(&b->sjoints, sjoints)) ||
            (rc = b->upload(&b->sjcoff, sjcoff)))
            return rc;
        CU(cudaMemset(b->gcol, 0, 4 * (size_t)kGcolWords));
        int per_sm = 0;
        CU(occupancy_flat<T, P>(0, kMaxBlockHost, &per_sm, 0));
        b->flat.grid_narrow = std::max(1, per_sm) * b->sm_count;
        // the class sort is a chain of dependent loads per candidate (a
        // binary search over the worlds): it wants every warp it can get
        CU(occupancy_flat<T, P>(2, kMaxBlockHost, &per_sm, 0));
        b->flat.grid_sort = std::max(1, per_sm) * b->sm_count;
        b->flat.block_solve = 128;
        if ((rc = set_team_split<T, P>(b, kBlockTeamBodies, kPairTeamBodies)))
            return rc;
        b->use_flat = true;
        // side stream + events for the parallel narrowphase kernels
        CU(cudaStreamCreateWithFlags(&b->flat.side, cudaStreamNonBlocking));
        for (int k = 0; k < 8; ++k)
        {
            CU(cudaEventCreateWithFlags(&b->flat.fork[k], cudaEventDisableTiming));
            CU(cudaEventCreateWithFlags(&b->flat.join[k], cudaEventDisableTiming));
        }
    }
    // ---- GJK pass: only batches with hull colliders reach it
    {
        bool any_hull = false;
        size_t cap = 0;
        for (uint32_t w = 0; w < (uint32_t)b->wdev.size(); ++w)
        {
            const WorldDev &d = b->wdev[w];
            cap += (size_t)d.pair_cap + 1 + d.n_pc;
            for (const auto &c : b->worlds[w].colliders)
                any_hull = any_hull || gjk_kind(c.shape); // pairs that go through GJK / EPA
        }
        if (any_hull && cap)
        {
            b->gjk_cap = (uint32_t)std::min<size_t>(cap, 0xffffffffu);
            // the GJK pass: one warp per queued pair, its polytope and
            // clipping buffers in shared memory; as many CTAs as stay resident
            CU(prepare_gjk<T, P>(b->sm_count, &b->gjk_slots));
            if ((rc = b->alloc((void **)&b->gjk_list, sizeof(uint2) * cap)) ||
                (rc = b->alloc((void **)&b->gjk_count, 64)))
                return rc;
        }
    }
    if ((rc = b->alloc((void **)&b->work_counter, std::max<size_t>(64, 4 * (size_t)b->n_counters))) || (rc = b->alloc((void **)&b->error_d, 64)) ||
        (rc = b->alloc((void **)&b->stats_d, sizeof(WorldStats) * W)))
        return rc;
    if ((rc = b->upload(&b->worlds_d, b->wdev)))
        return rc;
    return RBPS_OK;
}

extern "C" int rbps_batch_commit(rbps_batch *b)
{
    if (!b)
        return fail(RBPS_ERR_INVALID, "null batch");
    if (b->committed)
        return fail(RBPS_ERR_INVALID, "batch already committed");
    CU(cudaSetDevice(b->desc.device));
    int rc;
    if (b->desc.precision == RBPS_PRECISION_FP64)
        rc = commit_typed<double, double>(b);
    else
        rc = commit_typed<float, float>(b); // FP32 and FP32_POS64
    if (rc)
        return rc;
    CU(cudaDeviceSynchronize());
    b->committed = true;
    return RBPS_OK;
}

// ------------------------------------------------------------ dumps
template <class T, class P>
static int alloc_dumps(rbps_batch *b)
{
    if (b->dump_pairs)
        return RBPS_OK;
    uint32_t pc = 0, cc = 0;
    for (auto &d : b->wdev)
    {
        pc = std::max(pc, d.pair_cap);
        cc = std::max(cc, d.pair_cap + d.n_pc);
    }
    const size_t W = b->wdev.size();
    b->dump_pair_cap = pc;
    b->dump_cand_cap = cc;
    int rc;
    if ((rc = b->alloc((void **)&b->dump_pairs, W * 2 * pc * 4)) ||
        (rc = b->alloc((void **)&b->dump_cand, W * cc * sizeof(Cand))) ||
        (rc = b->alloc((void **)&b->dump_cc, W * cc * sizeof(CandContacts<T, P>))) ||
        (rc = b->alloc((void **)&b->dump_color, W * cc * 4)))
        return rc;
    for (size_t w = 0; w < W; ++w)
        b->wdev[w].dump_slot = (uint32_t)w;
    CU(cudaMemcpy(b->worlds_d, b->wdev.data(), W * sizeof(WorldDev), cudaMemcpyHostToDevice));
    // the zero fills above ran on the legacy stream; the step kernels run on
    // the batch's non-blocking stream
    CU(cudaDeviceSynchronize());
    return RBPS_OK;
}

extern "C" int rbps_batch_set_dump(rbps_batch *b, int32_t enable)
{
    if (!b || !b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_batch_set_dump: commit first");
    CU(cudaSetDevice(b->desc.device));
    CU(cudaStreamSynchronize(b->stream));
    b->dump = enable != 0;
    if (!b->dump)
        return RBPS_OK;
    if (b->desc.precision == RBPS_PRECISION_FP64)
        return alloc_dumps<double, double>(b);
    return alloc_dumps<float, float>(b);
}

// ------------------------------------------------------------ stepping
// The launches of one step on b->stream; returns the kernel count, or a
// negative status.
template <class T, class P>
static long enqueue_step(rbps_batch *b, const Engine<T, P> &e)
{
    long launches = 0;
    if (!b->small_ids.empty())
    {
        if (cudaMemsetAsync(b->work_counter, 0, 4 * (size_t)b->n_counters, b->stream) != cudaSuccess)
            return RBPS_ERR_CUDA;
        if (b->use_flat)
        {
            if (launch_step_flat<T, P>(e, b->phase, b->flat, b->stream) != cudaSuccess)
                return RBPS_ERR_CUDA;
            // frame, prefix, 3 class-sort kernels, stats (only with dumps:
            // otherwise the last substep writes them); per substep the three
            // narrowphase kernels, the GJK pass (batches with hulls) and the
            // substep
            launches += (e.dump_cc || b->desc.substeps < 1 ? 6 : 5) + (long)b->desc.substeps * (e.gjk_list ? 5 : 4);
        }
        else
        {
            if (launch_step_phases<T, P>(e, b->phase, b->stream) != cudaSuccess)
                return RBPS_ERR_CUDA;
            launches += b->n_counters + (e.gjk_list ? (long)b->desc.substeps : 0); // + the GJK passes
        }
    }
    for (uint32_t w : b->big_ids)
    {
        long k = 0;
        if (launch_step_big<T, P>(e, w, b->grid_big, b->block, b->stream, &k) != cudaSuccess)
            return RBPS_ERR_CUDA;
        launches += k;
    }
    return launches;
}

// Captures one step into b->graph_exec; on any refusal the batch falls back
// to direct launches for good.
template <class T, class P>
static void capture_step(rbps_batch *b, const Engine<T, P> &e, int key)
{
    if (b->graph_exec)
    {
        cudaGraphExecDestroy(b->graph_exec);
        b->graph_exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    {
        cudaGetLastError();
        b->graph_ok = false;
        return;
    }
    const long n = enqueue_step<T, P>(b, e);
    const cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
    cudaGraphExec_t x = nullptr;
    if (n < 0 || ec != cudaSuccess || !g || cudaGraphInstantiate(&x, g, 0) != cudaSuccess)
    {
        cudaGetLastError();
        b->graph_ok = false;
        x = nullptr;
    }
    if (g)
        cudaGraphDestroy(g);
    b->graph_exec = x;
    b->graph_key = key;
    b->graph_launches = n > 0 ? (uint64_t)n : 0;
}

template <class T, class P>
static int step_typed(rbps_batch *b, int n)
{
    Engine<T, P> e = make_engine<T, P>(b);
    const int key = (b->dump ? 1 : 0) | (e.prof ? 2 : 0) | (e.check_state ? 4 : 0);
    if (b->graph_ok && n > 0 && (!b->graph_exec || b->graph_key != key))
        capture_step<T, P>(b, e, key);
    uint64_t launches = 0;
    for (int s = 0; s < n; ++s)
    {
        if (b->graph_exec)
        {
            CU(cudaGraphLaunch(b->graph_exec, b->stream));
            launches += b->graph_launches;
        }
        else
        {
            const long k = enqueue_step<T, P>(b, e);
            if (k < 0)
                return fail(RBPS_ERR_CUDA, "step launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            launches += (uint64_t)k;
        }
    }
    b->launches_last = launches;
    return RBPS_OK;
}

extern "C" int rbps_batch_step(rbps_batch *b, int32_t n_steps)
{
    if (!b || !b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_batch_step: commit first");
    if (n_steps < 0)
        return fail(RBPS_ERR_INVALID, "rbps_batch_step: negative step count");
    CU(cudaSetDevice(b->desc.device));
    int rc;
    // the small-world view needs its scratch / layout
    if (b->desc.precision == RBPS_PRECISION_FP64)
        rc = step_typed<double, double>(b, n_steps);
    else
        rc = step_typed<float, float>(b, n_steps);
    if (!rc)
        b->steps_done += (uint64_t)n_steps;
    return rc;
}

static int check_device_error(rbps_batch *b)
{
    int err[4] = {0, 0, 0, 0};
    CU(cudaMemcpy(err, b->error_d, sizeof(err), cudaMemcpyDeviceToHost));
    if (err[0])
    {
        CU(cudaMemset(b->error_d, 0, sizeof(err)));
        CU(cudaDeviceSynchronize());
        static const char *sites[] = {"", "endpoint id out of range", "corrupt SAP pair record",
                                      "narrowphase candidate out of range", "endpoint keys not ordered after sort",
                                      "pair keys not ordered after sort", "GJK queue full",
                                      "non-finite body state"};
        const int site = (err[1] > 0 && err[1] < 8) ? err[1] : 0;
        if (err[0] == RBPS_ERR_STATE)
            return fail(err[0], "device reported error %d (non-finite body position, orientation or velocity in "
                                "world %d)", err[0], err[2]);
        return fail(err[0], "device reported error %d (%s%s%s, value %d)", err[0],
                    err[0] == RBPS_ERR_CAPACITY ? "capacity exceeded: raise max_pairs_per_world" : "step failure",
                    site ? ": " : "", sites[site], err[2]);
    }
    return RBPS_OK;
}

extern "C" int rbps_batch_set_state_check(rbps_batch *b, int32_t enable)
{
    if (!b)
        return fail(RBPS_ERR_INVALID, "rbps_batch_set_state_check: null batch");
    if (b->committed)
    {
        CU(cudaSetDevice(b->desc.device));
        CU(cudaStreamSynchronize(b->stream));
    }
    b->check_state = enable != 0;
    return RBPS_OK;
}

extern "C" int rbps_batch_synchronize(rbps_batch *b)
{
    if (!b || !b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_batch_synchronize: commit first");
    CU(cudaSetDevice(b->desc.device));
    CU(cudaStreamSynchronize(b->stream));
    if (b->io_stream)
        CU(cudaStreamSynchronize(b->io_stream));
    if (b->io_out_stream)
        CU(cudaStreamSynchronize(b->io_out_stream));
    return check_device_error(b);
}

// ------------------------------------------------------------ readback
template <class T, class P>
static int get_state_typed(rbps_batch *b, uint32_t first, uint32_t n, const rbps_state_view *v)
{
    std::vector<V4<P>> pos(n);
    std::vector<Q4<T>> rot(n);
    std::vector<V4<T>> lin(n), ang(n);
    if (v->position)
        CU(cudaMemcpy(pos.data(), (V4<P> *)b->pos + first, n * sizeof(V4<P>), cudaMemcpyDeviceToHost));
    if (v->orientation)
        CU(cudaMemcpy(rot.data(), (Q4<T> *)b->rot + first, n * sizeof(Q4<T>), cudaMemcpyDeviceToHost));
    if (v->linear_velocity)
        CU(cudaMemcpy(lin.data(), (V4<T> *)b->lin + first, n * sizeof(V4<T>), cudaMemcpyDeviceToHost));
    if (v->angular_velocity)
        CU(cudaMemcpy(ang.data(), (V4<T> *)b->ang + first, n * sizeof(V4<T>), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i)
    {
        if (v->position)
        {
            const double *o = b->origin_of_body(first + i);
            v->position[3 * i] = o[0] + double(pos[i].x);
            v->position[3 * i + 1] = o[1] + double(pos[i].y);
            v->position[3 * i + 2] = o[2] + double(pos[i].z);
        }
        if (v->orientation)
        {
            v->orientation[4 * i] = rot[i].w; v->orientation[4 * i + 1] = rot[i].x;
            v->orientation[4 * i + 2] = rot[i].y; v->orientation[4 * i + 3] = rot[i].z;
        }
        if (v->linear_velocity)
        {
            v->linear_velocity[3 * i] = lin[i].x; v->linear_velocity[3 * i + 1] = lin[i].y;
            v->linear_velocity[3 * i + 2] = lin[i].z;
        }
        if (v->angular_velocity)
        {
            v->angular_velocity[3 * i] = ang[i].x; v->angular_velocity[3 * i + 1] = ang[i].y;
            v->angular_velocity[3 * i + 2] = ang[i].z;
        }
    }
    return RBPS_OK;
}

template <class T, class P>
static int set_state_typed(rbps_batch *b, uint32_t first, uint32_t n, const rbps_state_view *v)
{
    std::vector<V4<P>> pos(n);
    std::vector<Q4<T>> rot(n);
    std::vector<V4<T>> lin(n), ang(n);
    CU(cudaMemcpy(pos.data(), (V4<P> *)b->pos + first, n * sizeof(V4<P>), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(rot.data(), (Q4<T> *)b->rot + first, n * sizeof(Q4<T>), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(lin.data(), (V4<T> *)b->lin + first, n * sizeof(V4<T>), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(ang.data(), (V4<T> *)b->ang + first, n * sizeof(V4<T>), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i)
    {
        if (v->position)
        {
            const double *o = b->origin_of_body(first + i);
            pos[i] = V4<P>{P(v->position[3 * i] - o[0]), P(v->position[3 * i + 1] - o[1]),
                           P(v->position[3 * i + 2] - o[2]), P(0)};
        }
        if (v->orientation)
            rot[i] = Q4<T>{T(v->orientation[4 * i]), T(v->orientation[4 * i + 1]), T(v->orientation[4 * i + 2]),
                           T(v->orientation[4 * i + 3])};
        if (v->linear_velocity)
            lin[i] = V4<T>{T(v->linear_velocity[3 * i]), T(v->linear_velocity[3 * i + 1]),
                           T(v->linear_velocity[3 * i + 2]), lin[i].w};
        if (v->angular_velocity)
            ang[i] = V4<T>{T(v->angular_velocity[3 * i]), T(v->angular_velocity[3 * i + 1]),
                           T(v->angular_velocity[3 * i + 2]), T(0)};
    }
    CU(cudaMemcpy((V4<P> *)b->pos + first, pos.data(), n * sizeof(V4<P>), cudaMemcpyHostToDevice));
    CU(cudaMemcpy((Q4<T> *)b->rot + first, rot.data(), n * sizeof(Q4<T>), cudaMemcpyHostToDevice));
    CU(cudaMemcpy((V4<T> *)b->lin + first, lin.data(), n * sizeof(V4<T>), cudaMemcpyHostToDevice));
    CU(cudaMemcpy((V4<T> *)b->ang + first, ang.data(), n * sizeof(V4<T>), cudaMemcpyHostToDevice));
    return RBPS_OK;
}

#define DISPATCH_PREC(b, fn, ...)                                        \
    ((b)->desc.precision == RBPS_PRECISION_FP64 ? fn<double, double>(__VA_ARGS__) : fn<float, float>(__VA_ARGS__))

static int ready(rbps_batch *b, const char *who)
{
    if (!b || !b->committed)
        return fail(RBPS_ERR_INVALID, "%s: commit first", who);
    CU(cudaSetDevice(b->desc.device));
    CU(cudaStreamSynchronize(b->stream));
    return check_device_error(b);
}

extern "C" int rbps_batch_get_state(rbps_batch *b, uint32_t world, const rbps_state_view *v)
{
    int rc = ready(b, "rbps_batch_get_state");
    if (rc)
        return rc;
    if (!v || world >= b->wdev.size())
        return fail(RBPS_ERR_INVALID, "rbps_batch_get_state: bad world or view");
    return DISPATCH_PREC(b, get_state_typed, b, b->wdev[world].body_off, b->wdev[world].n_bodies, v);
}

extern "C" int rbps_batch_set_state(rbps_batch *b, uint32_t world, const rbps_state_view *v)
{
    int rc = ready(b, "rbps_batch_set_state");
    if (rc)
        return rc;
    if (!v || world >= b->wdev.size())
        return fail(RBPS_ERR_INVALID, "rbps_batch_set_state: bad world or view");
    return DISPATCH_PREC(b, set_state_typed, b, b->wdev[world].body_off, b->wdev[world].n_bodies, v);
}

extern "C" int rbps_batch_get_state_all(rbps_batch *b, const rbps_state_view *v)
{
    int rc = ready(b, "rbps_batch_get_state_all");
    if (rc)
        return rc;
    if (!v)
        return fail(RBPS_ERR_INVALID, "null view");
    return DISPATCH_PREC(b, get_state_typed, b, 0u, b->n_bodies_all, v);
}

template <class T, class P>
static int set_forces_typed(rbps_batch *b, const double *f)
{
    std::vector<V4<T>> v(b->n_bodies_all);
    for (uint32_t i = 0; i < b->n_bodies_all; ++i)
        v[i] = V4<T>{T(f[3 * i]), T(f[3 * i + 1]), T(f[3 * i + 2]), T(0)};
    CU(cudaMemcpyAsync(b->force, v.data(), v.size() * sizeof(V4<T>), cudaMemcpyHostToDevice, b->stream));
    CU(cudaStreamSynchronize(b->stream));
    return RBPS_OK;
}

extern "C" int rbps_batch_set_forces_all(rbps_batch *b, const double *force)
{
    if (!b || !b->committed || !force)
        return fail(RBPS_ERR_INVALID, "rbps_batch_set_forces_all: commit first / null forces");
    CU(cudaSetDevice(b->desc.device));
    return DISPATCH_PREC(b, set_forces_typed, b, force);
}

extern "C" int rbps_batch_body_count(rbps_batch *b, uint32_t world, uint32_t *n)
{
    if (!b || world >= b->worlds.size() || !n)
        return fail(RBPS_ERR_INVALID, "rbps_batch_body_count: bad argument");
    *n = (uint32_t)b->worlds[world].bodies.size();
    return RBPS_OK;
}

extern "C" int rbps_batch_total_bodies(rbps_batch *b, uint64_t *n, uint64_t *nd)
{
    if (!b || !b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_batch_total_bodies: commit first");
    if (n)
        *n = b->total_bodies;
    if (nd)
        *nd = b->total_dynamic;
    return RBPS_OK;
}

static int world_stats(rbps_batch *b, uint32_t world, WorldStats *st)
{
    CU(cudaMemcpy(st, b->stats_d + world, sizeof(WorldStats), cudaMemcpyDeviceToHost));
    return RBPS_OK;
}

extern "C" int rbps_batch_get_pairs(rbps_batch *b, uint32_t world, uint32_t *pairs, uint32_t cap, uint32_t *n_out)
{
    int rc = ready(b, "rbps_batch_get_pairs");
    if (rc)
        return rc;
    if (world >= b->wdev.size())
        return fail(RBPS_ERR_INVALID, "world out of range");
    if (!b->dump)
        return fail(RBPS_ERR_INVALID, "rbps_batch_get_pairs: enable rbps_batch_set_dump before stepping");
    WorldStats st;
    if ((rc = world_stats(b, world, &st)))
        return rc;
    const uint32_t n = std::min(st.n_pairs, b->dump_pair_cap);
    if (n_out)
        *n_out = n;
    if (pairs && cap)
        CU(cudaMemcpy(pairs, b->dump_pairs + (size_t)world * 2 * b->dump_pair_cap,
                      std::min(n, cap) * 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return RBPS_OK;
}

template <class T, class P>
static int get_contacts_typed(rbps_batch *b, uint32_t world, rbps_contact *out, uint32_t cap, uint32_t *n_out)
{
    WorldStats st;
    int rc = world_stats(b, world, &st);
    if (rc)
        return rc;
    const uint32_t nc = std::min(st.n_cand, b->dump_cand_cap);
    std::vector<Cand> cand(nc);
    std::vector<CandContacts<T, P>> cc(nc);
    const size_t o = (size_t)world * b->dump_cand_cap;
    CU(cudaMemcpy(cand.data(), b->dump_cand + o, nc * sizeof(Cand), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(cc.data(), (CandContacts<T, P> *)b->dump_cc + o, nc * sizeof(CandContacts<T, P>),
                  cudaMemcpyDeviceToHost));
    uint32_t n = 0;
    for (uint32_t c = 0; c < nc; ++c)
        for (int k = 0; k < cc[c].n; ++k, ++n)
        {
            if (!out || n >= cap)
                continue;
            rbps_contact &r = out[n];
            std::memset(&r, 0, sizeof(r));
            const ContactPt<T, P> &p = cc[c].pt[k];
            r.body_a = cand[c].ba; r.body_b = cand[c].bb;
            r.collider_a = cand[c].ca; r.collider_b = cand[c].cb;
            r.normal[0] = cc[c].normal.x; r.normal[1] = cc[c].normal.y; r.normal[2] = cc[c].normal.z;
            r.r_a_local[0] = p.ra.x; r.r_a_local[1] = p.ra.y; r.r_a_local[2] = p.ra.z;
            r.r_b_local[0] = p.rb.x; r.r_b_local[1] = p.rb.y; r.r_b_local[2] = p.rb.z;
            const double *o = b->origin_of_world(world);
            r.point_on_a[0] = o[0] + p.pa.x; r.point_on_a[1] = o[1] + p.pa.y; r.point_on_a[2] = o[2] + p.pa.z;
            r.point_on_b[0] = o[0] + p.pb.x; r.point_on_b[1] = o[1] + p.pb.y; r.point_on_b[2] = o[2] + p.pb.z;
            r.penetration_depth = p.depth;
            r.normal_lambda = p.lam_n;
            r.tangent_lambda = p.lam_t;
            r.relative_velocity = p.vrel;
            r.restitution = cc[c].mat.x; r.static_friction = cc[c].mat.y; r.dynamic_friction = cc[c].mat.z;
            r.collision = p.coll;
        }
    if (n_out)
        *n_out = n;
    return RBPS_OK;
}

extern "C" int rbps_batch_get_contacts(rbps_batch *b, uint32_t world, rbps_contact *out, uint32_t cap, uint32_t *n_out)
{
    int rc = ready(b, "rbps_batch_get_contacts");
    if (rc)
        return rc;
    if (world >= b->wdev.size())
        return fail(RBPS_ERR_INVALID, "world out of range");
    if (!b->dump)
        return fail(RBPS_ERR_INVALID, "rbps_batch_get_contacts: enable rbps_batch_set_dump before stepping");
    return DISPATCH_PREC(b, get_contacts_typed, b, world, out, cap, n_out);
}

extern "C" int rbps_batch_get_colors(rbps_batch *b, uint32_t world, uint32_t *colors, uint32_t *ba, uint32_t *bb,
                                     uint32_t cap, uint32_t *n_out)
{
    int rc = ready(b, "rbps_batch_get_colors");
    if (rc)
        return rc;
    if (world >= b->wdev.size() || !b->dump)
        return fail(RBPS_ERR_INVALID, "rbps_batch_get_colors: bad world or dumps disabled");
    WorldStats st;
    if ((rc = world_stats(b, world, &st)))
        return rc;
    const uint32_t nc = std::min(st.n_cand, b->dump_cand_cap);
    if (n_out)
        *n_out = nc;
    const uint32_t n = std::min(nc, cap);
    std::vector<Cand> cand(n);
    const size_t o = (size_t)world * b->dump_cand_cap;
    if (colors && n)
        CU(cudaMemcpy(colors, b->dump_color + o, n * 4, cudaMemcpyDeviceToHost));
    if ((ba || bb) && n)
    {
        CU(cudaMemcpy(cand.data(), b->dump_cand + o, n * sizeof(Cand), cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; ++i)
        {
            if (ba)
                ba[i] = cand[i].ba;
            if (bb)
                bb[i] = cand[i].bb;
        }
    }
    return RBPS_OK;
}

extern "C" int rbps_batch_get_stats(rbps_batch *b, rbps_stats *s)
{
    int rc = ready(b, "rbps_batch_get_stats");
    if (rc)
        return rc;
    if (!s)
        return fail(RBPS_ERR_INVALID, "null stats");
    std::vector<WorldStats> st(b->wdev.size());
    CU(cudaMemcpy(st.data(), b->stats_d, st.size() * sizeof(WorldStats), cudaMemcpyDeviceToHost));
    std::memset(s, 0, sizeof(*s));
    s->steps = b->steps_done;
    for (auto &x : st)
    {
        s->pairs += x.n_pairs;
        s->candidates += x.n_cand;
        s->contacts += x.n_contacts;
        s->max_colors = std::max(s->max_colors, x.n_colors);
        s->serial_overflow += x.n_serial;
        s->gjk_pairs += x.n_gjk;
    }
    s->kernel_launches = b->launches_last;
    s->graph = b->graph_exec ? 1u : 0u;
    return RBPS_OK;
}

int rbps_internal_fail(int code, const char *msg) { return fail(code, "%s", msg); }

// Persistent SAP state of one world (BroadPhaseState::objects[].fat_aabb and
// ::endpoints, BroadPhase.hpp:88-143): fat AABBs per SAP object (6 doubles,
// object order = collider order without planes), endpoints in list order as
// (object*2 + is_max) and their float values.
extern "C" int rbps_batch_get_sap_state(rbps_batch *b, uint32_t world, double *fat, uint32_t *ep_ids,
                                        float *ep_values, uint32_t *n_objects)
{
    int rc = ready(b, "rbps_batch_get_sap_state");
    if (rc)
        return rc;
    if (world >= b->wdev.size())
        return fail(RBPS_ERR_INVALID, "world out of range");
    const WorldDev &d = b->wdev[world];
    if (n_objects)
        *n_objects = d.n_bp;
    if (fat && d.n_bp)
    {
        CU(cudaMemcpy(fat, b->fat + d.bp_off, d.n_bp * sizeof(FatBox), cudaMemcpyDeviceToHost));
        const double *o = b->origin_of_world(world);
        for (uint32_t k = 0; k < d.n_bp; ++k)
            for (int a = 0; a < 6; ++a)
                fat[6 * k + a] += o[a % 3];
    }
    if ((ep_ids || ep_values) && d.n_bp)
    {
        std::vector<uint32_t> ids(2 * d.n_bp), keys(2 * d.n_bp);
        CU(cudaMemcpy(ids.data(), b->ep_id + 2 * d.bp_off, ids.size() * 4, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(keys.data(), b->ep_key + 2 * d.bp_off, keys.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < ids.size(); ++i)
        {
            if (ep_ids)
                ep_ids[i] = ids[i];
            if (ep_values)
            {
                // invert the order-preserving key transform
                const uint32_t k = keys[i];
                const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
                float f;
                std::memcpy(&f, &u, 4);
                ep_values[i] = f;
            }
        }
    }
    return RBPS_OK;
}

// Diagnostics: runs only the broadphase + candidate build of `world` (on
// the first executor's scratch) and returns the pair / candidate counts.
template <class T, class P>
static int debug_bp_typed(rbps_batch *b, uint32_t world, uint32_t *counts)
{
    Engine<T, P> e = make_engine<T, P>(b);
    uint32_t *d = nullptr;
    CU(cudaMalloc(&d, 16));
    CU(cudaMemset(d, 0, 16));
    CU(launch_debug_broadphase<T, P>(e, world, b->block, d, b->stream));
    CU(cudaStreamSynchronize(b->stream));
    CU(cudaMemcpy(counts, d, 8, cudaMemcpyDeviceToHost));
    cudaFree(d);
    return RBPS_OK;
}

extern "C" RBPS_API int rbps_debug_broadphase(rbps_batch *b, uint32_t world, uint32_t *counts)
{
    int rc = ready(b, "rbps_debug_broadphase");
    if (rc)
        return rc;
    if (world >= b->wdev.size() || b->wdev[world].n_bodies > kSmallWorldBodies)
        return fail(RBPS_ERR_INVALID, "rbps_debug_broadphase: small worlds only");
    return DISPATCH_PREC(b, debug_bp_typed, b, world, counts);
}

// Phase timers (see rbps_batch_set_profile in rbps_gpu.h).
static_assert(kProfSlots == RBPS_PROFILE_SLOTS, "profile slot count must match the header");

extern "C" int rbps_batch_set_profile(rbps_batch *b, int32_t enable)
{
    int rc = ready(b, "rbps_batch_set_profile");
    if (rc)
        return rc;
    const size_t bytes = b->wdev.size() * kProfSlots * sizeof(unsigned long long);
    if (enable && !b->prof && (rc = b->alloc((void **)&b->prof, bytes)))
        return rc;
    if (enable)
        CU(cudaMemset(b->prof, 0, bytes));
    else
        b->prof_off = true;
    if (enable)
        b->prof_off = false;
    return RBPS_OK;
}

extern "C" int rbps_batch_get_profile(rbps_batch *b, uint64_t *out, uint32_t cap_worlds)
{
    int rc = ready(b, "rbps_batch_get_profile");
    if (rc)
        return rc;
    if (!b->prof)
        return fail(RBPS_ERR_INVALID, "rbps_batch_get_profile: profiling was never enabled");
    const size_t n = std::min<size_t>(cap_worlds, b->wdev.size());
    if (out && n)
        CU(cudaMemcpy(out, b->prof, n * kProfSlots * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    return RBPS_OK;
}

// Polygon and adjacency tables of a hull (see rbps_hull_tables in rbps_gpu.h).
extern "C" int rbps_hull_tables(const double *verts, uint32_t n_verts, const uint32_t *tris, uint32_t n_tris,
                                uint32_t cap, uint32_t *counts, uint32_t *poly_offsets, uint32_t *poly_indices,
                                double *poly_normals, uint32_t *v2p_offsets, uint32_t *v2p_indices,
                                uint32_t *v2n_offsets, uint32_t *v2n_indices, uint32_t *p2p_offsets,
                                uint32_t *p2p_indices)
{
    if (!verts || !n_verts || !counts)
        return fail(RBPS_ERR_INVALID, "rbps_hull_tables: need vertices and counts");
    for (uint32_t t = 0; tris && t < 3 * n_tris; ++t)
        if (tris[t] >= n_verts)
            return fail(RBPS_ERR_INVALID, "rbps_hull_tables: triangle index out of range");
    HostHull h;
    h.verts.assign(verts, verts + 3 * n_verts);
    build_hull_tables(h, tris, n_tris);
    const uint32_t np = (uint32_t)(h.poly_off.size() - 1);
    counts[0] = np;
    counts[1] = (uint32_t)h.poly_idx.size();
    counts[2] = (uint32_t)h.v2p_idx.size();
    counts[3] = (uint32_t)h.v2n_idx.size();
    counts[4] = (uint32_t)h.p2p_idx.size();
    const uint32_t need = std::max({np + 1, counts[1], counts[2], counts[3], counts[4], n_verts + 1});
    if (need > cap)
        return fail(RBPS_ERR_CAPACITY, "rbps_hull_tables: tables need %u entries, cap is %u", need, cap);
    auto put = [](uint32_t *dst, const std::vector<uint32_t> &v) {
        if (dst)
            std::copy(v.begin(), v.end(), dst);
    };
    put(poly_offsets, h.poly_off);
    put(poly_indices, h.poly_idx);
    if (poly_normals)
        std::copy(h.poly_n.begin(), h.poly_n.end(), poly_normals);
    put(v2p_offsets, h.v2p_off);
    put(v2p_indices, h.v2p_idx);
    put(v2n_offsets, h.v2n_off);
    put(v2n_indices, h.v2n_idx);
    put(p2p_offsets, h.p2p_off);
    put(p2p_indices, h.p2p_idx);
    return RBPS_OK;
}

// Device narrowphase of independent shape pairs (see rbps_batch_collide in
// rbps_gpu.h).
static_assert(sizeof(CollideOut) == sizeof(rbps_manifold), "CollideOut must mirror rbps_manifold");

template <class T, class P>
static int collide_typed(rbps_batch *b, uint32_t n, const std::vector<ShapeDev> &sa, const double *tf_a,
                         const std::vector<ShapeDev> &sb, const double *tf_b, rbps_manifold *out)
{
    HullSetDev hs{b->hull_verts, b->hull_voff, b->hull_aabb, b->hull_desc, b->hull_u32, b->hull_pn, b->hm_heights,
                  b->hm_desc, b->mesh_desc, b->mesh_v, b->mesh_i, b->mesh_n};
    const size_t shape_bytes = (size_t)n * sizeof(ShapeDev), tf_bytes = (size_t)n * 7 * sizeof(double);
    bool gjk = false;
    for (uint32_t i = 0; i < n && !gjk; ++i)
        gjk = (gjk_kind(sa[i].kind) || gjk_kind(sb[i].kind)) && sa[i].kind != kPlane && sb[i].kind != kPlane;
    (void)gjk; // one warp per pair, GJK workspaces in shared memory
    char *d = nullptr;
    const size_t total = 2 * shape_bytes + 2 * tf_bytes + (size_t)n * sizeof(CollideOut);
    CU(cudaMalloc(&d, total));
    ShapeDev *dsa = (ShapeDev *)d, *dsb = (ShapeDev *)(d + shape_bytes);
    double *dta = (double *)(d + 2 * shape_bytes), *dtb = (double *)(d + 2 * shape_bytes + tf_bytes);
    CollideOut *dout = (CollideOut *)(d + 2 * shape_bytes + 2 * tf_bytes);
    cudaError_t e = cudaMemcpyAsync(dsa, sa.data(), shape_bytes, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dsb, sb.data(), shape_bytes, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dta, tf_a, tf_bytes, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dtb, tf_b, tf_bytes, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = launch_collide<T, P>(dsa, dta, dsb, dtb, hs, n, dout, b->error_d, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, dout, (size_t)n * sizeof(CollideOut), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    cudaFree(d);
    if (e != cudaSuccess)
        return fail(RBPS_ERR_CUDA, "rbps_batch_collide: %s", cudaGetErrorString(e));
    return b->committed ? check_device_error(b) : RBPS_OK;
}

extern "C" int rbps_batch_collide(rbps_batch *b, uint32_t n, const rbps_collider_desc *a, const double *tf_a,
                                  const rbps_collider_desc *bd, const double *tf_b, rbps_manifold *out)
{
    if (!b)
        return fail(RBPS_ERR_INVALID, "rbps_batch_collide: null batch");
    if (n == 0)
        return RBPS_OK;
    if (!a || !bd || !tf_a || !tf_b || !out)
        return fail(RBPS_ERR_INVALID, "rbps_batch_collide: null buffer");
    std::vector<ShapeDev> sa(n), sb(n);
    bool uses_hull = false;
    for (uint32_t i = 0; i < n; ++i)
        for (int side = 0; side < 2; ++side)
        {
            const rbps_collider_desc &c = side ? bd[i] : a[i];
            if (!shape_supported(c.shape))
                return fail(RBPS_ERR_INVALID, "rbps_batch_collide: pair %u has an unknown shape %d", i, c.shape);
            if (c.shape == RBPS_SHAPE_HEIGHTMAP)
            {
                if (c.hull >= b->heightmaps.size())
                    return fail(RBPS_ERR_INVALID, "rbps_batch_collide: heightmap %u does not exist", c.hull);
                uses_hull = true;
            }
            if (c.shape == RBPS_SHAPE_MESH)
            {
                if (c.hull >= b->meshes.size())
                    return fail(RBPS_ERR_INVALID, "rbps_batch_collide: mesh %u does not exist", c.hull);
                uses_hull = true;
            }
            if (c.shape == RBPS_SHAPE_CONVEX_HULL)
            {
                if (c.hull >= b->hulls.size())
                    return fail(RBPS_ERR_INVALID, "rbps_batch_collide: hull %u does not exist", c.hull);
                uses_hull = true;
            }
            ShapeDev s{};
            s.kind = c.shape;
            s.hull = (int)c.hull;
            for (int k = 0; k < 4; ++k)
                s.p[k] = c.params[k];
            (side ? sb : sa)[i] = s;
        }
    if (uses_hull && !b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_batch_collide: commit the batch before colliding hulls");
    CU(cudaSetDevice(b->desc.device));
    return DISPATCH_PREC(b, collide_typed, b, n, sa, tf_a, sb, tf_b, out);
}

// One step with host I/O (see rbps_batch_step_io in rbps_gpu.h).
template <class T, class P>
static int step_io_typed(rbps_batch *b, const double *force_in, double *pos_out, double *rot_out)
{
    const uint32_t n = b->n_bodies_all;
    int rc;
    if (!b->io_force)
    {
        if ((rc = b->alloc((void **)&b->io_force, (size_t)n * 3 * 8)) || (rc = b->alloc((void **)&b->io_pos, (size_t)n * 3 * 8)) ||
            (rc = b->alloc((void **)&b->io_rot, (size_t)n * 4 * 8)))
            return rc;
        CU(cudaDeviceSynchronize());
    }
    Engine<T, P> e = make_engine<T, P>(b);
    const int grid = std::max(1, std::min<int>(b->sm_count * 8, (int)((n + 255) / 256)));
    if (force_in)
    {
        CU(cudaMemcpyAsync(b->io_force, force_in, (size_t)n * 3 * 8, cudaMemcpyHostToDevice, b->stream));
        CU(launch_io<T, P>(e, 0, b->io_force, nullptr, n, grid, b->stream));
    }
    if ((rc = step_typed<T, P>(b, 1)))
        return rc;
    b->steps_done += 1;
    if (pos_out || rot_out)
    {
        CU(launch_io<T, P>(e, 1, b->io_pos, b->io_rot, n, grid, b->stream));
        if (pos_out)
            CU(cudaMemcpyAsync(pos_out, b->io_pos, (size_t)n * 3 * 8, cudaMemcpyDeviceToHost, b->stream));
        if (rot_out)
            CU(cudaMemcpyAsync(rot_out, b->io_rot, (size_t)n * 4 * 8, cudaMemcpyDeviceToHost, b->stream));
    }
    CU(cudaStreamSynchronize(b->stream));
    return check_device_error(b);
}

// Pipelined variant: call k uses staging slot s = k % 2.
//   input stream:   [wait force_free[s]] H2D force -> io_f2[s], record force_ready[s]
//   compute stream: [wait force_ready[s]] forces in, record force_free[s], step,
//                   [wait out_free[s]] poses -> io_p2/io_r2[s], record pose_ready[s]
//   output stream:  [wait pose_ready[s]] D2H poses, record out_free[s]
// so the copies of call k overlap the compute of calls k - 1 and k + 1.
template <class T, class P>
static int step_io_async_typed(rbps_batch *b, const double *force_in, double *pos_out, double *rot_out)
{
    const uint32_t n = b->n_bodies_all;
    int rc;
    if (!b->io_async_ready)
    {
        CU(cudaStreamCreateWithFlags(&b->io_stream, cudaStreamNonBlocking));
        CU(cudaStreamCreateWithFlags(&b->io_out_stream, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k)
        {
            if ((rc = b->alloc((void **)&b->io_f2[k], (size_t)n * 3 * 8)) ||
                (rc = b->alloc((void **)&b->io_p2[k], (size_t)n * 3 * 8)) ||
                (rc = b->alloc((void **)&b->io_r2[k], (size_t)n * 4 * 8)))
                return rc;
            for (cudaEvent_t *e : {&b->ev_force_ready[k], &b->ev_force_free[k], &b->ev_pose_ready[k], &b->ev_out_free[k]})
                CU(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
            // every slot starts free
            CU(cudaEventRecord(b->ev_force_free[k], b->stream));
            CU(cudaEventRecord(b->ev_out_free[k], b->io_out_stream));
        }
        CU(cudaDeviceSynchronize());
        b->io_async_ready = true;
    }
    const uint32_t s = b->io_slot;
    b->io_slot ^= 1u;
    Engine<T, P> e = make_engine<T, P>(b);
    const int grid = std::max(1, std::min<int>(b->sm_count * 8, (int)((n + 255) / 256)));
    if (force_in)
    {
        CU(cudaStreamWaitEvent(b->io_stream, b->ev_force_free[s], 0));
        CU(cudaMemcpyAsync(b->io_f2[s], force_in, (size_t)n * 3 * 8, cudaMemcpyHostToDevice, b->io_stream));
        CU(cudaEventRecord(b->ev_force_ready[s], b->io_stream));
        CU(cudaStreamWaitEvent(b->stream, b->ev_force_ready[s], 0));
        CU(launch_io<T, P>(e, 0, b->io_f2[s], nullptr, n, grid, b->stream));
        CU(cudaEventRecord(b->ev_force_free[s], b->stream));
    }
    if ((rc = step_typed<T, P>(b, 1)))
        return rc;
    b->steps_done += 1;
    if (pos_out || rot_out)
    {
        CU(cudaStreamWaitEvent(b->stream, b->ev_out_free[s], 0));
        CU(launch_io<T, P>(e, 1, b->io_p2[s], b->io_r2[s], n, grid, b->stream));
        CU(cudaEventRecord(b->ev_pose_ready[s], b->stream));
        CU(cudaStreamWaitEvent(b->io_out_stream, b->ev_pose_ready[s], 0));
        if (pos_out)
            CU(cudaMemcpyAsync(pos_out, b->io_p2[s], (size_t)n * 3 * 8, cudaMemcpyDeviceToHost, b->io_out_stream));
        if (rot_out)
            CU(cudaMemcpyAsync(rot_out, b->io_r2[s], (size_t)n * 4 * 8, cudaMemcpyDeviceToHost, b->io_out_stream));
        CU(cudaEventRecord(b->ev_out_free[s], b->io_out_stream));
    }
    return RBPS_OK;
}

extern "C" int rbps_batch_step_io_async(rbps_batch *b, const double *force_in, double *position_out,
                                        double *orientation_out)
{
    if (!b || !b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_batch_step_io_async: commit first");
    CU(cudaSetDevice(b->desc.device));
    return DISPATCH_PREC(b, step_io_async_typed, b, force_in, position_out, orientation_out);
}

// ------------------------------------------------------------ snapshots
// The device arrays that carry state from one step to the next.  Everything
// else on the device is either constant after commit (shapes, inertia,
// layouts) or rebuilt every frame (candidates, contacts, colours).
template <class T, class P>
static std::vector<std::pair<void *, size_t>> state_arrays(rbps_batch *b)
{
    const size_t nb = b->n_bodies_all, nbp = b->n_bp_all;
    std::vector<std::pair<void *, size_t>> v = {
        {b->pos, nb * sizeof(V4<P>)},      {b->prev_pos, nb * sizeof(V4<P>)},
        {b->rot, nb * sizeof(Q4<T>)},      {b->prev_rot, nb * sizeof(Q4<T>)},
        {b->lin, nb * sizeof(V4<T>)},      {b->ang, nb * sizeof(V4<T>)},
        {b->force, nb * sizeof(V4<T>)},    {b->torque, nb * sizeof(V4<T>)},
        {b->fat, nbp * sizeof(FatBox)},    {b->ep_key, 2 * nbp * sizeof(uint32_t)},
        {b->ep_id, 2 * nbp * sizeof(uint32_t)}, {b->ep_pos, 2 * nbp * sizeof(uint32_t)},
        {b->joints_d, (size_t)b->n_joint_all * sizeof(Joint<T>)},
        {b->rows_d, (size_t)b->n_row_all * sizeof(Row<T>)}};
    std::vector<std::pair<void *, size_t>> out;
    for (auto &a : v)
        if (a.first && a.second)
            out.push_back(a);
    return out;
}

// dir 0: state -> slot, 1: slot -> state
template <class T, class P>
static int snapshot_copy(rbps_batch *b, char *slot, int dir)
{
    size_t off = 0;
    for (auto &a : state_arrays<T, P>(b))
    {
        void *dst = dir == 0 ? (void *)(slot + off) : a.first;
        const void *src = dir == 0 ? a.first : (const void *)(slot + off);
        CU(cudaMemcpyAsync(dst, src, a.second, cudaMemcpyDeviceToDevice, b->stream));
        off += (a.second + 255) / 256 * 256;
    }
    return RBPS_OK;
}

template <class T, class P>
static int snapshot_new(rbps_batch *b, uint32_t *slot_out)
{
    size_t bytes = 0;
    for (auto &a : state_arrays<T, P>(b))
        bytes += (a.second + 255) / 256 * 256;
    char *p = nullptr;
    int rc = b->alloc((void **)&p, std::max<size_t>(bytes, 256));
    if (rc)
        return rc;
    b->snaps.push_back(p);
    *slot_out = (uint32_t)(b->snaps.size() - 1);
    return snapshot_copy<T, P>(b, p, 0);
}

extern "C" int rbps_batch_snapshot(rbps_batch *b, uint32_t *slot_out)
{
    if (!b || !b->committed || !slot_out)
        return fail(RBPS_ERR_INVALID, "rbps_batch_snapshot: commit first, and pass slot_out");
    CU(cudaSetDevice(b->desc.device));
    return DISPATCH_PREC(b, snapshot_new, b, slot_out);
}

extern "C" int rbps_batch_snapshot_update(rbps_batch *b, uint32_t slot)
{
    if (!b || !b->committed || slot >= b->snaps.size())
        return fail(RBPS_ERR_INVALID, "rbps_batch_snapshot_update: no snapshot %u", slot);
    CU(cudaSetDevice(b->desc.device));
    return DISPATCH_PREC(b, snapshot_copy, b, b->snaps[slot], 0);
}

extern "C" int rbps_batch_restore(rbps_batch *b, uint32_t slot)
{
    if (!b || !b->committed || slot >= b->snaps.size())
        return fail(RBPS_ERR_INVALID, "rbps_batch_restore: no snapshot %u", slot);
    CU(cudaSetDevice(b->desc.device));
    return DISPATCH_PREC(b, snapshot_copy, b, b->snaps[slot], 1);
}

// ------------------------------------------------------------ autotuner
// Frame-kernel block (its grid follows from occupancy) and narrowphase grid.
template <class T, class P>
static int apply_launch(rbps_batch *b, int frame_block, int narrow_grid)
{
    if (!b->small_ids.empty())
    {
        int per_sm = 0;
        CU(occupancy_phase<T, P>(kKFrame, frame_block, &per_sm));
        if (per_sm < 1)
            return fail(RBPS_ERR_CUDA, "frame kernel cannot be resident with %d threads", frame_block);
        b->phase.block[kKFrame] = frame_block;
        b->phase.grid[kKFrame] = std::min<int>((int)b->small_ids.size(), per_sm * b->sm_count);
    }
    if (b->use_flat)
        b->flat.grid_narrow = std::max(1, narrow_grid);
    b->graph_key = -1; // recapture the step graph with the new shapes
    return RBPS_OK;
}

template <class T, class P>
static int autotune_typed(rbps_batch *b, int trials, rbps_tune_result *out)
{
    int rc;
    uint32_t slot = 0;
    if ((rc = snapshot_new<T, P>(b, &slot)))
        return rc;
    const uint64_t steps0 = b->steps_done;
    const int fb0 = b->phase.block[kKFrame], ng0 = b->flat.grid_narrow;
    std::vector<std::pair<int, int>> cand = {{fb0, ng0}};
    for (int fb : {128, 256})
        for (int f2 : {1, 2, 4}) // narrowphase grid x 1/2, 1, 2
        {
            const std::pair<int, int> c(fb, std::max(1, ng0 * f2 / 2));
            if (std::find(cand.begin(), cand.end(), c) == cand.end())
                cand.push_back(c);
        }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    double best = 1e300, first = 0.0;
    std::pair<int, int> best_c = cand[0];
    for (size_t k = 0; k < cand.size(); ++k)
    {
        if ((rc = apply_launch<T, P>(b, cand[k].first, cand[k].second)) ||
            (rc = snapshot_copy<T, P>(b, b->snaps[slot], 1)) || (rc = step_typed<T, P>(b, 1)))
            break;
        CU(cudaEventRecord(e0, b->stream));
        if ((rc = step_typed<T, P>(b, trials)))
            break;
        CU(cudaEventRecord(e1, b->stream));
        CU(cudaEventSynchronize(e1));
        float ms = 0.f;
        CU(cudaEventElapsedTime(&ms, e0, e1));
        const double per = ms / trials;
        if (k == 0)
            first = per;
        if (per < best)
        {
            best = per;
            best_c = cand[k];
        }
    }
    // then the team split of the substep kernel (CTA from / half CTA from
    // body counts), with the best shapes above
    const uint32_t tb0 = b->team_bodies, pb0 = b->pair_bodies;
    uint32_t best_t = tb0, best_p = pb0;
    uint32_t n_trials = (uint32_t)cand.size();
    if (!rc && b->use_flat)
    {
        rc = apply_launch<T, P>(b, best_c.first, best_c.second);
        const std::pair<uint32_t, uint32_t> splits[] = {{128u, 128u}, {96u, 96u}, {192u, 64u}, {256u, 64u},
                                                        {256u, 128u}, {320u, 96u}, {384u, 128u}};
        for (const auto &sp : splits)
        {
            if (rc || (sp.first == tb0 && sp.second == pb0))
                continue;
            ++n_trials;
            if ((rc = set_team_split<T, P>(b, sp.first, sp.second)) ||
                (rc = apply_launch<T, P>(b, best_c.first, best_c.second)) ||
                (rc = snapshot_copy<T, P>(b, b->snaps[slot], 1)) || (rc = step_typed<T, P>(b, 1)))
                break;
            CU(cudaEventRecord(e0, b->stream));
            if ((rc = step_typed<T, P>(b, trials)))
                break;
            CU(cudaEventRecord(e1, b->stream));
            CU(cudaEventSynchronize(e1));
            float ms = 0.f;
            CU(cudaEventElapsedTime(&ms, e0, e1));
            if (ms / trials < best)
            {
                best = ms / trials;
                best_t = sp.first;
                best_p = sp.second;
            }
        }
        if (!rc)
            rc = set_team_split<T, P>(b, best_t, best_p);
    }
    // then the narrowphase candidates per warp and the colouring batch, one
    // knob at a time with the others at their best
    const uint32_t npw0 = b->narrow_per_warp, cc0 = b->color_chunk;
    uint32_t best_npw = npw0, best_cc = cc0;
    auto time_knobs = [&](uint32_t npw, uint32_t cc, double *ms_out) -> int {
        b->narrow_per_warp = npw;
        b->color_chunk = cc;
        int r2 = apply_launch<T, P>(b, best_c.first, best_c.second);
        if (!r2)
            r2 = snapshot_copy<T, P>(b, b->snaps[slot], 1);
        if (!r2)
            r2 = step_typed<T, P>(b, 1);
        if (r2)
            return r2;
        if (cudaEventRecord(e0, b->stream) != cudaSuccess)
            return fail(RBPS_ERR_CUDA, "autotune: event record failed");
        if ((r2 = step_typed<T, P>(b, trials)))
            return r2;
        float ms = 0.f;
        if (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            return fail(RBPS_ERR_CUDA, "autotune: event timing failed");
        *ms_out = ms / trials;
        return RBPS_OK;
    };
    if (!rc && b->use_flat)
    {
        for (uint32_t npw : {64u, 128u, 256u})
        {
            double ms = 0.0;
            if (rc || npw == npw0)
                continue;
            ++n_trials;
            if ((rc = time_knobs(npw, best_cc, &ms)))
                break;
            if (ms < best)
            {
                best = ms;
                best_npw = npw;
            }
        }
        for (uint32_t cc : {64u, 128u})
        {
            double ms = 0.0;
            if (rc || cc == cc0)
                continue;
            ++n_trials;
            if ((rc = time_knobs(best_npw, cc, &ms)))
                break;
            if (ms < best)
            {
                best = ms;
                best_cc = cc;
            }
        }
    }
    b->narrow_per_warp = best_npw;
    b->color_chunk = best_cc;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc)
        return rc;
    if ((rc = apply_launch<T, P>(b, best_c.first, best_c.second)) ||
        (rc = snapshot_copy<T, P>(b, b->snaps[slot], 1)))
        return rc;
    CU(cudaStreamSynchronize(b->stream));
    b->steps_done = steps0;
    if (out)
    {
        std::memset(out, 0, sizeof(*out));
        out->frame_block = best_c.first;
        out->narrow_grid = best_c.second;
        out->ms_per_step = best;
        out->ms_per_step_default = first;
        out->trials = n_trials;
        out->team_bodies = best_t;
        out->pair_bodies = best_p;
        out->narrow_per_warp = best_npw;
        out->color_chunk = best_cc;
    }
    return check_device_error(b);
}

extern "C" int rbps_batch_autotune(rbps_batch *b, int32_t trial_steps, rbps_tune_result *out)
{
    if (!b || !b->committed || trial_steps < 1)
        return fail(RBPS_ERR_INVALID, "rbps_batch_autotune: commit first; trial_steps >= 1");
    CU(cudaSetDevice(b->desc.device));
    return DISPATCH_PREC(b, autotune_typed, b, trial_steps, out);
}

template <class T, class P>
static int set_launch_typed(rbps_batch *b, const rbps_tune_result *cfg)
{
    int rc;
    if (b->use_flat && (cfg->team_bodies || cfg->pair_bodies) &&
        (rc = set_team_split<T, P>(b, cfg->team_bodies ? cfg->team_bodies : b->team_bodies,
                                   cfg->pair_bodies ? cfg->pair_bodies : b->pair_bodies)))
        return rc;
    if (cfg->narrow_per_warp)
        b->narrow_per_warp = cfg->narrow_per_warp;
    if (cfg->color_chunk)
        b->color_chunk = cfg->color_chunk;
    return apply_launch<T, P>(b, cfg->frame_block ? cfg->frame_block : b->phase.block[kKFrame],
                              cfg->narrow_grid ? cfg->narrow_grid : b->flat.grid_narrow);
}

extern "C" int rbps_batch_set_launch(rbps_batch *b, const rbps_tune_result *cfg)
{
    if (!b || !b->committed || !cfg)
        return fail(RBPS_ERR_INVALID, "rbps_batch_set_launch: commit first; non-null configuration");
    if ((cfg->frame_block && cfg->frame_block != 128 && cfg->frame_block != 256) || cfg->narrow_grid < 0 ||
        (cfg->narrow_per_warp && (cfg->narrow_per_warp % 32 || cfg->narrow_per_warp > 4096)) ||
        (cfg->color_chunk && (cfg->color_chunk > kColorStage || cfg->color_chunk < 32)))
        return fail(RBPS_ERR_INVALID, "rbps_batch_set_launch: frame_block 128 or 256, narrow_per_warp a multiple "
                                      "of 32 up to 4096, color_chunk in [32, %u] (0 keeps a field)", kColorStage);
    CU(cudaSetDevice(b->desc.device));
    CU(cudaStreamSynchronize(b->stream));
    return DISPATCH_PREC(b, set_launch_typed, b, cfg);
}

extern "C" int rbps_batch_step_io(rbps_batch *b, const double *force_in, double *position_out, double *orientation_out)
{
    if (!b || !b->committed)
        return fail(RBPS_ERR_INVALID, "rbps_batch_step_io: commit first");
    CU(cudaSetDevice(b->desc.device));
    return DISPATCH_PREC(b, step_io_typed, b, force_in, position_out, orientation_out);
}

extern "C" int rbps_world_set_body_forces(rbps_batch *b, uint32_t world, uint32_t first, uint32_t n, const double *force)
{
    int rc = check_world(b, world, true);
    if (rc)
        return rc;
    HostWorld &w = b->worlds[world];
    if (!force || (uint64_t)first + n > w.bodies.size())
        return fail(RBPS_ERR_INVALID, "rbps_world_set_body_forces: range out of bounds");
    std::memcpy(w.force.data() + 3 * (size_t)first, force, (size_t)n * 3 * sizeof(double));
    return RBPS_OK;
}
