// vox_api.cu - host orchestration of the voxelization pipeline and the C ABI
// (pnanovdb_get_raster / pnanovdb_get_compute drop-in tables and vox_*).
//
// The reference drives raster_gaussian_3d from the host as a loop of
// 256K-prim x 8M-fragment windows with a per-window queue flush and a
// frame-lagged readback of the fragment total (raster/Raster.cpp:420-558,
// raster/GridBuild.cpp:830-942).  Here one call runs the whole chain on one
// CUDA stream with three small read-backs (candidate count, pair count, node
// counts) that size the buffers; buffers persist in the context and only
// grow, so repeated calls allocate nothing.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "pnanovdb_b200.h"
#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

using namespace vox;

namespace
{

struct DevBuf
{
    void* p = nullptr;
    size_t cap = 0;
};

struct Timers
{
    cudaEvent_t ev[8] = {};
};

} // namespace

struct vox_context_t
{
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    // host-array calls: the attribute upload runs in chunks on its own stream,
    // each chunk's k_prep launch waiting only for that chunk's copies
    struct Upload
    {
        bool active = false;
        const void* host[5] = {};     // means, quats, scales, opacities, colors
        char* dev[5] = {};
        int width[5] = { 3, 4, 3, 1, 3 }; // values per Gaussian
        size_t es = 4;                   // bytes per value
    } upload;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t up_ev[5] = {};           // [0]: the call's start on the stream, [1..4]: chunks landed
    uint32_t wait_ctl = 0; // look-back wait control (0: default limit), see vox_context_set_wait_limit
    std::string last_error;
    std::vector<DevBuf*> bufs;
    // device buffers
    DevBuf recs, footprints, frag_off, root_bits, root_prefix, root_of_rank, lower_bits, lower_prefix, lower_cell;
    DevBuf scan_status, run_status;
    DevBuf keys, ids, keys_alt, ids_alt, sort_ws;
    DevBuf vox_start, leaf_vstart, lower_lstart, lower_rank;
    DevBuf lower_origin, lower_upper_n, upper_head, upper_scan, lower_parent, upper_root_n, upper_lostart;
    DevBuf leaf_lower, leaf_lower_n, leaf_mask, leaf_origin;
    DevBuf vox_leaf, vox_n, rank_to_lower;
    // leaf-granular pipeline
    DevBuf cand_org, tile_g0, lcols, lcol_off, lc_count, lc_mask, lc_off, emit_gid, emit_flag, lflags, lpos, cand_key, cand_start, cand_mask, pair_gid;
    DevBuf s_rgba, s_dens, s_col, s_pairs, cand_cnt, cand_voff, vkeys, vslot, vpairs, pair_off, cand_vbase, cloud_pairs;
    DevBuf partials, exp_keys, exp_ids;
    // reference node order
    DevBuf nwin, win_before, cand_wkey, wkey_u, wkey_lo, wkey_leaf, wcnt, wbase, okeys, okeys_alt, ovals, ovals_alt;
    DevBuf rank_u, rank_lo, rank_leaf, leaf_popc, leaf_voff;
    DevBuf cloud_start, cloud_vs, clouds;           // batched calls: inputs, per-cloud layout
    DevBuf order; // 9 node order arrays
    DevBuf grid;
    DevBuf scal; // device scalars
    DevBuf hier_keys;
    DevBuf prim_keys_alt, prim_vals_alt; // ping-pong buffers of vox_radix_sort_key64
    DevBuf vb_work; // VoxelBVH ingestion: world-box keys, range tile counts
    DevBuf vb_keys, vb_ids_c, vb_used; // VoxelBVH ingestion: compressed sort keys (also the dual-key sort's keys)
    DevBuf dual_idx; // dual-key sort: original indices
    DevBuf vb_rec;   // VoxelBVH ingestion: per-Gaussian search records
    uint64_t* hscal = nullptr; // pinned mirror
    Epochs scan_epochs, run_epochs, sort_epochs;
    int check_sort = 0; // VOX_CHECK_SORT=1: validate key order after every sort
    int check_emit = 0; // VOX_CHECK_EMIT=1: also walk the leaves the leaf test culls; a pass there is an error
    int key64 = 0;
    int sorted_in_alt = 0;
    vox_stats_t stats{};
    Timers timers;
    SortTuning tuning;
    OnlineChoice walk_choice[4] = { OnlineChoice(2), OnlineChoice(2), OnlineChoice(2), OnlineChoice(2) }; // leaf walk: 4 or 3 CTAs per SM, per mode (window | smooth << 1)
    int walk_mode = 0;
    OnlineChoice vb_search_choice{ 2 }; // VoxelBVH level search: lane-balanced or thread per Gaussian
    int walk_variant = 0, vb_variant = 0;
    // last result
    int64_t last_P = 0;
    uint64_t last_grid_bytes = 0;
    // state the adjoint of the last differentiable call reads
    bool diff_ready = false;
    int64_t last_G = 0;
    int64_t last_V = -1; // -1: no successful call yet
    uint64_t last_value_count = 0;
    uint32_t last_flags = 0;
    float last_voxel_size = 0.f;
    NodeParams last_N{};
    LeafPassParams last_LP{};
    uint64_t last_NLC = 0, last_Q = 0;
    const float* last_cloud_vs = nullptr;
    std::vector<uint64_t> h_grid_off, h_value_base; // per cloud, last call
};

// device scalar slots (u64 each)
enum
{
    SC_F = 0,
    SC_NROOT,
    SC_NLOWER,
    SC_P,
    SC_V,
    SC_L,
    SC_LO,
    SC_U,
    SC_ERR, // int in the low half
    SC_GRID_BYTES,
    SC_NLC,  // leaf columns
    SC_Q,    // (leaf, Gaussian) pairs
    SC_NCL,  // candidate leaves
    SC_NVOX, // active voxels from the leaf masks
    SC_NWIN, // reference fragment windows (window order)
    SC_VBU,  // VoxelBVH: used key slots
    SC_BBOX, // 3 words (6 int32)
    SC_COUNT = SC_BBOX + 3,
    SC_SCRATCH = 24
};

static void set_error(vox_context_t* ctx, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx)
        ctx->last_error = buf;
    fprintf(stderr, "[pnanovdb_b200] %s\n", buf);
}

// The look-back wait control (vox_context_set_wait_limit) lives in the upper
// half of the device error word, which every call clears: re-arm it.
static void arm_wait(vox_context_t* ctx, uint64_t* sc, cudaStream_t s)
{
    if (ctx->wait_ctl)
        cudaMemcpyAsync((uint32_t*)(sc + SC_ERR) + 1, &ctx->wait_ctl, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
}

// zeroes the per-call device scalars (counts, error word) and re-arms the wait control
static void clear_scalars(vox_context_t* ctx, uint64_t* sc, cudaStream_t s)
{
    cudaMemsetAsync(sc, 0, sizeof(uint64_t) * SC_COUNT, s);
    arm_wait(ctx, sc, s);
}

static bool ensure(vox_context_t* ctx, DevBuf& b, size_t bytes)
{
    if (bytes == 0)
        bytes = 256;
    if (b.cap >= bytes)
        return true;
    if (b.p)
        cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t want = bytes + bytes / 8 + 256;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        set_error(ctx, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
        b.p = nullptr;
        return false;
    }
    b.cap = want;
    return true;
}

static int check_cuda(vox_context_t* ctx, const char* where)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        set_error(ctx, "CUDA error at %s: %s", where, cudaGetErrorString(e));
        return VOX_ERR_CUDA;
    }
    return VOX_OK;
}

static int sync_scalars(vox_context_t* ctx, const char* where)
{
    cudaMemcpyAsync(ctx->hscal, ctx->scal.p, sizeof(uint64_t) * SC_COUNT, cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
    {
        set_error(ctx, "CUDA error at %s: %s", where, cudaGetErrorString(e));
        return VOX_ERR_CUDA;
    }
    int err = (int)(ctx->hscal[SC_ERR] & 0xffffffffu);
    if (err & ERR_LOOKBACK)
    {
        set_error(ctx, "%s: a bounded device wait expired", where);
        return VOX_ERR_TIMEOUT;
    }
    if (err & ERR_RANGE)
    {
        set_error(ctx, "%s: voxel coordinates outside [-65536, 65535] (root key range of the node2 grid)", where);
        return VOX_ERR_RANGE;
    }
    if (err & ERR_FOOTPRINT)
    {
        set_error(ctx, "%s: a Gaussian's bounding box covers 2^31 or more voxels", where);
        return VOX_ERR_FOOTPRINT;
    }
    if (err & (ERR_ORDER | ERR_BOUNDS))
    {
        set_error(ctx, "%s: internal consistency check failed (%s%s)", where, (err & ERR_ORDER) ? "keys out of order " : "",
                  (err & ERR_BOUNDS) ? "index out of range" : "");
        return VOX_ERR_CUDA;
    }
    return VOX_OK;
}

static int bits_for(uint64_t n)
{
    int b = 0;
    while ((1ull << b) < n)
        b++;
    return b;
}

static float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

// ---------------------------------------------------------------------------
// the pipeline
// ---------------------------------------------------------------------------
// node_idx / addresses / value indices in the reference's window order
// (vox_order.cu): per level a sort by (creation window, parent rank, n)
static int window_order(vox_context_t* ctx, NodeParams& N, int64_t U, int64_t Lo, int64_t L, int64_t nw,
                        cudaStream_t s)
{
    const int64_t mx = std::max<int64_t>(std::max<int64_t>(U, Lo), std::max<int64_t>(L, 1));
    const int64_t W = nw > 0 ? nw : 1;
    if (!ensure(ctx, ctx->wkey_u, 8 * (size_t)(U + 1)) || !ensure(ctx, ctx->wkey_lo, 8 * (size_t)(Lo + 1)) ||
        !ensure(ctx, ctx->wkey_leaf, 8 * (size_t)(L + 1)) || !ensure(ctx, ctx->wcnt, 8 * 3 * (size_t)W) ||
        !ensure(ctx, ctx->wbase, 8 * 4 * (size_t)(W + 1)) || !ensure(ctx, ctx->okeys, 8 * (size_t)mx) ||
        !ensure(ctx, ctx->okeys_alt, 8 * (size_t)mx) || !ensure(ctx, ctx->ovals, 4 * (size_t)mx) ||
        !ensure(ctx, ctx->ovals_alt, 4 * (size_t)mx) || !ensure(ctx, ctx->rank_u, 4 * (size_t)(U + 1)) ||
        !ensure(ctx, ctx->rank_lo, 4 * (size_t)(Lo + 1)) || !ensure(ctx, ctx->rank_leaf, 4 * (size_t)(L + 1)) ||
        !ensure(ctx, ctx->leaf_popc, 8 * (size_t)(L + 1)) || !ensure(ctx, ctx->leaf_voff, 8 * (size_t)(L + 1)) ||
        !ensure(ctx, ctx->sort_ws, sort_workspace_bytes(mx, 8)) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(L + 1) * 2))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    int* d_err = (int*)(sc + SC_ERR);
    uint32_t* d_counter = (uint32_t*)(sc + SC_SCRATCH);
    uint64_t* wk_u = (uint64_t*)ctx->wkey_u.p;
    uint64_t* wk_lo = (uint64_t*)ctx->wkey_lo.p;
    uint64_t* wk_leaf = (uint64_t*)ctx->wkey_leaf.p;
    uint64_t* cnt = (uint64_t*)ctx->wcnt.p; // [3][W]
    uint64_t* base = (uint64_t*)ctx->wbase.p; // [4][W + 1]
    cudaMemsetAsync(cnt, 0, 8 * 3 * (size_t)W, s);
    launch_leaf_wkey(L, N.leaf_vstart, (const uint32_t*)ctx->vslot.p, (const uint64_t*)ctx->cand_wkey.p, wk_leaf, s);
    launch_run_min(Lo, N.lower_lstart, wk_leaf, wk_lo, s);
    launch_run_min(U, N.upper_lostart, wk_lo, wk_u, s);
    const int key_bits = 40 + bits_for((uint64_t)W + 1);
    struct Level
    {
        int64_t n;
        const uint64_t* wkey;
        const uint32_t* parent;
        const uint32_t* parent_rank;
        const uint32_t* nval;
        uint32_t nmask;
        uint32_t* rank;
    } lv[3] = { { U, wk_u, nullptr, nullptr, N.upper_root_n, 32767u, (uint32_t*)ctx->rank_u.p },
                { Lo, wk_lo, N.lower_parent, (const uint32_t*)ctx->rank_u.p, N.lower_upper_n, 32767u,
                  (uint32_t*)ctx->rank_lo.p },
                { L, wk_leaf, N.leaf_lower, (const uint32_t*)ctx->rank_lo.p, N.leaf_lower_n, 4095u,
                  (uint32_t*)ctx->rank_leaf.p } };
    for (int l = 0; l < 3; l++)
    {
        if (lv[l].n <= 0)
            continue;
        launch_level_keys(lv[l].n, lv[l].wkey, lv[l].parent, lv[l].parent_rank, lv[l].nval, lv[l].nmask,
                          (uint64_t*)ctx->okeys.p, (uint32_t*)ctx->ovals.p, cnt + (size_t)l * W, s);
        const int in_alt = sort_pairs_u64((uint64_t*)ctx->okeys.p, (uint32_t*)ctx->ovals.p, (uint64_t*)ctx->okeys_alt.p,
                                          (uint32_t*)ctx->ovals_alt.p, lv[l].n, key_bits, ctx->sort_ws.p,
                                          &ctx->sort_epochs, d_err, ctx->num_sms, s, ctx->tuning);
        const uint32_t* sv = (const uint32_t*)(in_alt ? ctx->ovals_alt.p : ctx->ovals.p);
        launch_level_rank(lv[l].n, sv, lv[l].rank, s);
        if (l == 2)
            launch_leaf_popc_sorted(L, sv, N.leaf_vstart, (uint64_t*)ctx->leaf_popc.p, s);
    }
    uint64_t* scan_status = (uint64_t*)ctx->scan_status.p;
    const size_t scan_words = ctx->scan_status.cap / sizeof(uint64_t);
    scan_exclusive_u64((const uint64_t*)ctx->leaf_popc.p, (uint64_t*)ctx->leaf_voff.p, L, 0, sc + SC_SCRATCH + 4,
                       scan_status, ctx->scan_epochs.next(scan_status, scan_words, s), d_counter, d_err, ctx->num_sms, s);
    launch_window_bases(W, cnt, cnt + W, cnt + 2 * (size_t)W, base, base + (W + 1), base + 2 * (W + 1),
                        base + 3 * (W + 1), s);
    WindowOrderParams P;
    P.U = (uint64_t)U;
    P.rank_u = lv[0].rank;
    P.rank_lo = lv[1].rank;
    P.rank_leaf = lv[2].rank;
    P.wkey_u = wk_u;
    P.wkey_lo = wk_lo;
    P.wkey_leaf = wk_leaf;
    P.base_u = base;
    P.base_lo = base + (W + 1);
    P.base_leaf = base + 2 * (W + 1);
    P.base_all = base + 3 * (W + 1);
    P.leaf_voff = (const uint64_t*)ctx->leaf_voff.p;
    P.V = (uint64_t)N.C.V;
    launch_window_place(P, N, s);
    return check_cuda(ctx, "window order");
}

// B clouds: Gaussians [h_start[b], h_start[b + 1]) with voxel size h_vs[b]
// (h_start / h_vs null: one cloud with voxel_size)
static int run_voxelize(vox_context_t* ctx, const vox_gaussians_t* gs, float voxel_size, float cull_scale,
                        uint32_t flags, int64_t B = 1, const int64_t* h_start = nullptr, const float* h_vs = nullptr)
{
    if (!ctx || !gs || gs->count < 0 || B < 1 || B > VOX_MAX_CLOUDS || (!h_vs && !(voxel_size > 0.f)))
    {
        set_error(ctx, "vox_voxelize: invalid arguments");
        return VOX_ERR_ARGS;
    }
    if (h_start)
    {
        bool ok = h_start[0] == 0 && h_start[B] == gs->count && h_vs;
        for (int64_t b = 0; ok && b < B; b++)
            ok = h_start[b] <= h_start[b + 1] && h_vs[b] > 0.f;
        if (!ok)
        {
            set_error(ctx, "vox_voxelize_batch: cloud_start must rise from 0 to the Gaussian count and every voxel size be > 0");
            return VOX_ERR_ARGS;
        }
    }
    if (gs->count > 0 && (!gs->means || !gs->quats || !gs->scales || !gs->opacities || !gs->colors))
    {
        set_error(ctx, "vox_voxelize: missing attribute array");
        return VOX_ERR_ARGS;
    }
    const bool window = (flags & VOX_FLAG_WINDOW_ORDER) != 0;
    if (window && B > 1)
    {
        set_error(ctx, "vox_voxelize_batch: the reference window node order is for one cloud per call");
        return VOX_ERR_ARGS;
    }
    ctx->diff_ready = false;
    ctx->last_V = -1;
    const bool diff = (flags & VOX_FLAG_DIFFERENTIABLE) != 0;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int64_t G = gs->count;
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    ctx->stats.gaussians = G;
    const int64_t launches0 = launch_count();
    if (!ensure(ctx, ctx->scal, sizeof(uint64_t) * SC_SCRATCH * 4))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    clear_scalars(ctx, sc, s);
    int* d_err = (int*)(sc + SC_ERR);
    uint32_t* d_counter = (uint32_t*)(sc + SC_SCRATCH);
    cudaEventRecord(ctx->timers.ev[0], s);

    // ---------------------------------------------------------------- prep
    const float cull = cull_scale > 0.f ? cull_scale : 0.05f;
    if (!ensure(ctx, ctx->recs, sizeof(GaussRec) * (size_t)(G + 1)) ||
        !ensure(ctx, ctx->footprints, sizeof(uint64_t) * (size_t)(G + 1)) ||
        !ensure(ctx, ctx->frag_off, sizeof(uint64_t) * (size_t)(G + 1)) ||
        !ensure(ctx, ctx->root_bits, sizeof(uint64_t) * 512 * B) || !ensure(ctx, ctx->root_prefix, sizeof(uint64_t) * 512 * B) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(G > 512 * B ? G : 512 * B) * 2))
        return VOX_ERR_MEMORY;
    const int64_t* d_cloud_start = nullptr;
    const float* d_cloud_vs = nullptr;
    if (h_start)
    {
        if (!ensure(ctx, ctx->cloud_start, sizeof(int64_t) * (B + 1)) || !ensure(ctx, ctx->cloud_vs, sizeof(float) * B))
            return VOX_ERR_MEMORY;
        cudaMemcpyAsync(ctx->cloud_start.p, h_start, sizeof(int64_t) * (B + 1), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(ctx->cloud_vs.p, h_vs, sizeof(float) * B, cudaMemcpyHostToDevice, s);
        d_cloud_start = (const int64_t*)ctx->cloud_start.p;
        d_cloud_vs = (const float*)ctx->cloud_vs.p;
    }
    GaussRec* recs = (GaussRec*)ctx->recs.p;
    uint64_t* footprints = (uint64_t*)ctx->footprints.p;
    uint64_t* frag_off = (uint64_t*)ctx->frag_off.p;
    uint64_t* root_bits = (uint64_t*)ctx->root_bits.p;
    uint64_t* root_prefix = (uint64_t*)ctx->root_prefix.p;
    cudaMemsetAsync(root_bits, 0, sizeof(uint64_t) * 512 * B, s);
    PrepParams P;
    P.means = gs->means;
    P.quats = gs->quats;
    P.scales = gs->scales;
    P.opac = gs->opacities;
    P.colors = gs->colors;
    P.count = G;
    P.raw = (flags & VOX_FLAG_RAW_INPUTS) ? 1 : 0;
    P.bf16 = (flags & VOX_FLAG_BF16_INPUTS) ? 1 : 0;
    P.voxel_size = voxel_size;
    P.cull_scale = cull;
    P.cloud_start = d_cloud_start;
    P.cloud_vs = d_cloud_vs;
    P.clouds = B;
    if (ctx->upload.active && G >= (1 << 20))
    {
        // four chunks: the copies of chunk c + 1 overlap the prep of chunk c
        const int NC = 4;
        cudaEventRecord(ctx->up_ev[0], s);
        cudaStreamWaitEvent(ctx->copy_stream, ctx->up_ev[0], 0);
        for (int c = 0; c < NC; c++)
        {
            const int64_t g0 = G * c / NC, g1 = G * (c + 1) / NC;
            for (int a = 0; a < 5; a++)
            {
                const size_t row = (size_t)ctx->upload.width[a] * ctx->upload.es;
                cudaMemcpyAsync(ctx->upload.dev[a] + row * g0, (const char*)ctx->upload.host[a] + row * g0,
                                row * (size_t)(g1 - g0), cudaMemcpyHostToDevice, ctx->copy_stream);
            }
            cudaEventRecord(ctx->up_ev[1 + c], ctx->copy_stream);
            cudaStreamWaitEvent(s, ctx->up_ev[1 + c], 0);
            P.g0 = g0;
            P.g1 = g1;
            launch_prep(P, recs, footprints, root_bits, d_err, s);
        }
    }
    else
    {
        if (ctx->upload.active)
            for (int a = 0; a < 5; a++)
                cudaMemcpyAsync(ctx->upload.dev[a], ctx->upload.host[a],
                                (size_t)ctx->upload.width[a] * ctx->upload.es * (size_t)G, cudaMemcpyHostToDevice, s);
        launch_prep(P, recs, footprints, root_bits, d_err, s);
    }
    ctx->upload.active = false;
    uint64_t* scan_status = (uint64_t*)ctx->scan_status.p;
    size_t scan_words = ctx->scan_status.cap / sizeof(uint64_t);
    scan_exclusive_u64(footprints, frag_off, G, 0, sc + SC_F, scan_status, ctx->scan_epochs.next(scan_status, scan_words, s),
                       d_counter, d_err, ctx->num_sms, s);
    scan_exclusive_u64(root_bits, root_prefix, 512 * B, 1, sc + SC_NROOT, scan_status,
                       ctx->scan_epochs.next(scan_status, scan_words, s), d_counter, d_err, ctx->num_sms, s);
    int rc = sync_scalars(ctx, "prep");
    if (rc)
        return rc;
    const uint64_t F = ctx->hscal[SC_F];
    const uint64_t NR = ctx->hscal[SC_NROOT];
    if (!ensure(ctx, ctx->root_of_rank, sizeof(uint32_t) * (NR + 1)))
        return VOX_ERR_MEMORY;
    launch_invert_bits(root_bits, root_prefix, 512 * B, (uint32_t*)ctx->root_of_rank.p, s);
    ctx->stats.candidates = (int64_t)F;

    // ------------------------------------------------------- lower ranks
    const int64_t lwords = (int64_t)(NR > 0 ? NR : 1) * 512;
    if (!ensure(ctx, ctx->lower_bits, sizeof(uint64_t) * lwords) ||
        !ensure(ctx, ctx->lower_prefix, sizeof(uint64_t) * lwords) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(lwords > G ? lwords : G) * 2))
        return VOX_ERR_MEMORY;
    scan_status = (uint64_t*)ctx->scan_status.p;
    scan_words = ctx->scan_status.cap / sizeof(uint64_t);
    uint64_t* lower_bits = (uint64_t*)ctx->lower_bits.p;
    uint64_t* lower_prefix = (uint64_t*)ctx->lower_prefix.p;
    cudaMemsetAsync(lower_bits, 0, sizeof(uint64_t) * lwords, s);
    launch_mark_lower(recs, G, root_bits, root_prefix, lower_bits, s);
    scan_exclusive_u64(lower_bits, lower_prefix, lwords, 1, sc + SC_NLOWER, scan_status,
                       ctx->scan_epochs.next(scan_status, scan_words, s), d_counter, d_err, ctx->num_sms, s);
    rc = sync_scalars(ctx, "lower ranks");
    if (rc)
        return rc;
    const uint64_t NL = ctx->hscal[SC_NLOWER];
    if (!ensure(ctx, ctx->lower_cell, sizeof(uint32_t) * (NL + 1)))
        return VOX_ERR_MEMORY;
    launch_invert_bits(lower_bits, lower_prefix, lwords, (uint32_t*)ctx->lower_cell.p, s);
    const int key_bits = 21 + bits_for(NL > 1 ? NL : 2);
    const int key64 = key_bits > 32 ? 1 : 0;
    ctx->key64 = key64;
    ctx->stats.key_bits = key_bits;
    cudaEventRecord(ctx->timers.ev[1], s);

    // ---------------------------------------------------------- leaf pairs
    RankTables T{ root_bits, root_prefix, lower_bits, lower_prefix };
    const size_t kb = key64 ? 8 : 4;
    const int leaf_key_bits = 12 + bits_for(NL > 1 ? NL : 2);
    if (leaf_key_bits > 32)
    {
        set_error(ctx, "voxelize: %llu touched lower-node cells (128^3 voxels) exceed the 2^20 leaf keys hold",
                  (unsigned long long)NL);
        return VOX_ERR_SIZE;
    }
    if (!ensure(ctx, ctx->lcols, 8 * (size_t)(G + 1)) || !ensure(ctx, ctx->lcol_off, 8 * (size_t)(G + 1)))
        return VOX_ERR_MEMORY;
    uint64_t* lcols = (uint64_t*)ctx->lcols.p;
    uint64_t* lcol_off = (uint64_t*)ctx->lcol_off.p;
    launch_leaf_cols(recs, G, lcols, s);
    scan_exclusive_u64(lcols, lcol_off, G, 0, sc + SC_NLC, scan_status, ctx->scan_epochs.next(scan_status, scan_words, s),
                       d_counter, d_err, ctx->num_sms, s);
    rc = sync_scalars(ctx, "leaf columns");
    if (rc)
        return rc;
    const uint64_t NLC = ctx->hscal[SC_NLC];
    if (!ensure(ctx, ctx->lc_count, 8 * (size_t)(NLC + 1)) || !ensure(ctx, ctx->lc_off, 8 * (size_t)(NLC + 1)) ||
        !ensure(ctx, ctx->lc_mask, 4 * (size_t)(NLC + 1)) || !ensure(ctx, ctx->tile_g0, 8 * (size_t)(NLC / 256 + 2)) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words((int64_t)NLC + 1) * 2))
        return VOX_ERR_MEMORY;
    scan_status = (uint64_t*)ctx->scan_status.p;
    scan_words = ctx->scan_status.cap / sizeof(uint64_t);
    LeafEmitParams LE;
    memset(&LE, 0, sizeof(LE));
    LE.recs = recs;
    LE.G = G;
    LE.lcol_off = lcol_off;
    LE.NLC = NLC;
    LE.lc_count = (uint64_t*)ctx->lc_count.p;
    LE.lc_mask = (uint32_t*)ctx->lc_mask.p;
    LE.tile_g0 = (const int64_t*)ctx->tile_g0.p;
    launch_tile_gauss(lcol_off, G, NLC, (int64_t*)ctx->tile_g0.p, s);
    LE.voxel_size = voxel_size;
    LE.cloud_vs = d_cloud_vs;
    LE.check = ctx->check_emit;
    launch_leaf_emit(LE, T, false, s);
    uint64_t* lc_off = (uint64_t*)ctx->lc_off.p;
    scan_exclusive_u64(LE.lc_count, lc_off, (int64_t)NLC, 0, sc + SC_Q, scan_status,
                       ctx->scan_epochs.next(scan_status, scan_words, s), d_counter, d_err, ctx->num_sms, s);
    rc = sync_scalars(ctx, "leaf pairs");
    if (rc)
        return rc;
    const uint64_t Q = ctx->hscal[SC_Q];
    if (Q >= 0xFFFFFFF0ull)
    {
        set_error(ctx, "voxelize: %llu (leaf, Gaussian) pairs exceed the 32-bit pair index range", (unsigned long long)Q);
        return VOX_ERR_SIZE;
    }
    if (!ensure(ctx, ctx->keys, 4 * (size_t)(Q + 1)) || !ensure(ctx, ctx->ids, 4 * (size_t)(Q + 1)) ||
        !ensure(ctx, ctx->keys_alt, 4 * (size_t)(Q + 1)) || !ensure(ctx, ctx->ids_alt, 4 * (size_t)(Q + 1)) ||
        !ensure(ctx, ctx->emit_gid, 4 * (size_t)(Q + 1)) || !ensure(ctx, ctx->pair_gid, 4 * (size_t)(Q + 1)) ||
        (ctx->check_emit && !ensure(ctx, ctx->emit_flag, (size_t)(Q + 1))) ||
        !ensure(ctx, ctx->sort_ws, sort_workspace_bytes((int64_t)Q, 4)) || !ensure(ctx, ctx->lflags, 8 * (size_t)(Q + 1)) ||
        !ensure(ctx, ctx->lpos, 8 * (size_t)(Q + 1)) || !ensure(ctx, ctx->cand_key, 4 * (size_t)(Q + 1)) ||
        !ensure(ctx, ctx->cand_org, 16 * (size_t)(Q + 1)) ||
        !ensure(ctx, ctx->cand_start, 4 * (size_t)(Q + 2)) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words((int64_t)Q + 1) * 2))
        return VOX_ERR_MEMORY;
    scan_status = (uint64_t*)ctx->scan_status.p;
    scan_words = ctx->scan_status.cap / sizeof(uint64_t);
    LE.lc_off = lc_off;
    LE.keys = (uint32_t*)ctx->keys.p;
    LE.vals = (uint32_t*)ctx->ids.p;
    LE.emit_gid = (uint32_t*)ctx->emit_gid.p;
    LE.emit_flag = ctx->check_emit ? (uint8_t*)ctx->emit_flag.p : nullptr;
    launch_leaf_emit(LE, T, true, s);
    cudaEventRecord(ctx->timers.ev[2], s);

    // ------------------------------------------ sort by leaf key, candidates
    const int in_alt = sort_pairs_u32((uint32_t*)ctx->keys.p, (uint32_t*)ctx->ids.p, (uint32_t*)ctx->keys_alt.p,
                                      (uint32_t*)ctx->ids_alt.p, (int64_t)Q, leaf_key_bits, ctx->sort_ws.p,
                                      &ctx->sort_epochs, d_err, ctx->num_sms, s, ctx->tuning);
    ctx->stats.sort_passes = (leaf_key_bits + ctx->tuning.digit_bits - 1) / ctx->tuning.digit_bits;
    ctx->stats.sort_shape = sort_shape_used((int64_t)Q, 0, ctx->tuning);
    const uint32_t* lkeys = (const uint32_t*)(in_alt ? ctx->keys_alt.p : ctx->keys.p);
    const uint32_t* lvals = (const uint32_t*)(in_alt ? ctx->ids_alt.p : ctx->ids.p);
    if (ctx->check_sort)
    {
        check_sorted(lkeys, (int64_t)Q, 0, sc + SC_SCRATCH + 2, ctx->num_sms, s);
        rc = sync_scalars(ctx, "sort");
        if (rc)
            return rc;
        uint64_t descents = 0;
        cudaMemcpy(&descents, sc + SC_SCRATCH + 2, sizeof(uint64_t), cudaMemcpyDeviceToHost);
        if (descents)
        {
            set_error(ctx, "sort: %llu keys out of order", (unsigned long long)descents);
            return VOX_ERR_CUDA;
        }
    }
    uint64_t* lflags = (uint64_t*)ctx->lflags.p;
    uint64_t* lpos = (uint64_t*)ctx->lpos.p;
    launch_leaf_heads(lkeys, (int64_t)Q, lflags, s);
    scan_exclusive_u64(lflags, lpos, (int64_t)Q, 0, sc + SC_NCL, scan_status,
                       ctx->scan_epochs.next(scan_status, scan_words, s), d_counter, d_err, ctx->num_sms, s);
    if (Q == 0)
        cudaMemsetAsync(ctx->cand_start.p, 0, 4, s);
    launch_leaf_compact(lkeys, lvals, (const uint32_t*)ctx->emit_gid.p, (int64_t)Q, lflags, lpos,
                        (const uint32_t*)ctx->lower_cell.p, (const uint32_t*)ctx->root_of_rank.p,
                        (uint32_t*)ctx->cand_key.p, (int4*)ctx->cand_org.p, (uint32_t*)ctx->cand_start.p,
                        (uint32_t*)ctx->pair_gid.p, s);
    rc = sync_scalars(ctx, "candidate leaves");
    if (rc)
        return rc;
    const int64_t NCL = (int64_t)ctx->hscal[SC_NCL];
    ctx->stats.leaf_pairs = (int64_t)Q;
    ctx->stats.candidate_leaves = NCL;
    if ((uint64_t)NCL * 512ull >= 0xFFFFFFF0ull)
    {
        set_error(ctx, "voxelize: %lld candidate leaves exceed the 2^23 the staging indices hold", (long long)NCL);
        return VOX_ERR_SIZE;
    }
    cudaEventRecord(ctx->timers.ev[3], s);

    // ------------------------------------------------------------ leaf walk
    const size_t slots = 512 * (size_t)(NCL + 1);
    if (!ensure(ctx, ctx->cand_mask, 64 * (size_t)(NCL + 1)) || !ensure(ctx, ctx->s_rgba, 4 * slots) ||
        !ensure(ctx, ctx->s_dens, 4 * slots) || !ensure(ctx, ctx->s_col, 12 * slots) || !ensure(ctx, ctx->s_pairs, 4 * slots) ||
        !ensure(ctx, ctx->cand_cnt, 8 * (size_t)(NCL + 1)) || !ensure(ctx, ctx->cand_voff, 8 * (size_t)(NCL + 1)) ||
        !ensure(ctx, ctx->cand_vbase, 8 * (size_t)(NCL + 1)) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(NCL + 1) * 2))
        return VOX_ERR_MEMORY;
    scan_status = (uint64_t*)ctx->scan_status.p;
    scan_words = ctx->scan_status.cap / sizeof(uint64_t);
    uint64_t* win_before = nullptr;
    if (window)
    {
        // windows of the reference's 256K-Gaussian batches (raster/Raster.cpp:443-444)
        const int64_t nbatch = (G + REF_PRIM_BATCH - 1) / REF_PRIM_BATCH;
        if (!ensure(ctx, ctx->nwin, 8 * (size_t)(nbatch + 1)) || !ensure(ctx, ctx->win_before, 8 * (size_t)(nbatch + 1)) ||
            !ensure(ctx, ctx->cand_wkey, 8 * (size_t)(NCL + 1)))
            return VOX_ERR_MEMORY;
        win_before = (uint64_t*)ctx->win_before.p;
        launch_batch_windows(frag_off, sc + SC_F, G, nbatch, (uint64_t*)ctx->nwin.p, s);
        scan_exclusive_u64((const uint64_t*)ctx->nwin.p, win_before, nbatch, 0, sc + SC_NWIN, scan_status,
                           ctx->scan_epochs.next(scan_status, scan_words, s), d_counter, d_err, ctx->num_sms, s);
    }
    LeafPassParams LP;
    memset(&LP, 0, sizeof(LP));
    LP.window = window ? 1 : 0;
    LP.frag_off = frag_off;
    LP.win_before = win_before;
    LP.cand_wkey = window ? (uint64_t*)ctx->cand_wkey.p : nullptr;
    LP.recs = recs;
    LP.vals = lvals;
    LP.emit_gid = (const uint32_t*)ctx->emit_gid.p;
    LP.pair_gid = (const uint32_t*)ctx->pair_gid.p;
    LP.emit_flag = ctx->check_emit ? (const uint8_t*)ctx->emit_flag.p : nullptr;
    LP.cand_key = (const uint32_t*)ctx->cand_key.p;
    LP.cand_org = (const int4*)ctx->cand_org.p;
    LP.cand_start = (const uint32_t*)ctx->cand_start.p;
    LP.NCL = NCL;
    LP.lower_cell = (const uint32_t*)ctx->lower_cell.p;
    LP.root_of_rank = (const uint32_t*)ctx->root_of_rank.p;
    LP.voxel_size = voxel_size;
    LP.cloud_vs = d_cloud_vs;
    LP.smooth = diff ? 1 : 0;
    LP.cand_mask = (uint64_t*)ctx->cand_mask.p;
    LP.s_rgba = (uint32_t*)ctx->s_rgba.p;
    LP.s_dens = (float*)ctx->s_dens.p;
    LP.s_col = (float*)ctx->s_col.p;
    LP.s_pairs = (uint32_t*)ctx->s_pairs.p;
    LP.total_pairs = sc + SC_P;
    LP.err = d_err;
    LP.cand_vbase = (const uint64_t*)ctx->cand_vbase.p;
    LP.cand_voff = (const uint64_t*)ctx->cand_voff.p;
    LP.key64 = key64;
    ctx->walk_mode = (LP.window ? 1 : 0) | (LP.smooth ? 2 : 0); // the modes differ in cost per pair
    ctx->walk_variant = ctx->walk_choice[ctx->walk_mode].pick((int64_t)Q);
    ctx->stats.walk_ctas_per_sm = launch_leaf_pass(LP, d_counter, ctx->num_sms, s, ctx->walk_variant);
    cudaEventRecord(ctx->timers.ev[4], s);
    launch_leaf_popc(LP.cand_mask, NCL, (uint64_t*)ctx->cand_cnt.p, s);
    scan_exclusive_u64((const uint64_t*)ctx->cand_cnt.p, (uint64_t*)ctx->cand_voff.p, NCL, 0, sc + SC_NVOX, scan_status,
                       ctx->scan_epochs.next(scan_status, scan_words, s), d_counter, d_err, ctx->num_sms, s);
    rc = sync_scalars(ctx, "leaf walk");
    if (rc)
        return rc;
    const int64_t VX = (int64_t)ctx->hscal[SC_NVOX];
    const int64_t P_pairs = (int64_t)ctx->hscal[SC_P];
    ctx->stats.pairs = P_pairs;
    ctx->last_P = P_pairs;
    if (!ensure(ctx, ctx->vkeys, kb * (size_t)(VX + 1)) || !ensure(ctx, ctx->vslot, 4 * (size_t)(VX + 1)))
        return VOX_ERR_MEMORY;
    launch_voxel_keys(LP.cand_mask, LP.cand_key, LP.cand_voff, NCL, ctx->vkeys.p, key64, (uint32_t*)ctx->vslot.p, s);
    const void* skeys = ctx->vkeys.p;

    // ------------------------------------------- runs over the voxel keys
    const int64_t rtiles = runs_tile_count(VX);
    if (!ensure(ctx, ctx->vox_start, 4 * (size_t)(VX + 2)) || !ensure(ctx, ctx->leaf_vstart, 4 * (size_t)(VX + 2)) ||
        !ensure(ctx, ctx->lower_lstart, 4 * (size_t)(NL + 2)) || !ensure(ctx, ctx->lower_rank, 4 * (size_t)(NL + 2)) ||
        !ensure(ctx, ctx->run_status, sizeof(uint64_t) * 3 * (size_t)(rtiles + 1)) ||
        !ensure(ctx, ctx->vox_leaf, 4 * (size_t)(VX + 2)) || !ensure(ctx, ctx->vox_n, 2 * (size_t)(VX + 2)))
        return VOX_ERR_MEMORY;
    RunParams Rp;
    Rp.P = VX;
    Rp.vox_start = (uint32_t*)ctx->vox_start.p;
    Rp.vox_leaf = (uint32_t*)ctx->vox_leaf.p;
    Rp.vox_n = (uint16_t*)ctx->vox_n.p;
    Rp.leaf_vstart = (uint32_t*)ctx->leaf_vstart.p;
    Rp.lower_lstart = (uint32_t*)ctx->lower_lstart.p;
    Rp.lower_rank = (uint32_t*)ctx->lower_rank.p;
    Rp.counts = sc + SC_V;
    Rp.status = (uint64_t*)ctx->run_status.p;
    Rp.epoch = ctx->run_epochs.next(Rp.status, ctx->run_status.cap / sizeof(uint64_t), s);
    Rp.counter = d_counter;
    Rp.err = d_err;
    Rp.lower_cap = NL + 2;
    if (VX == 0)
    {
        cudaMemsetAsync(Rp.vox_start, 0, 4, s);
        cudaMemsetAsync(Rp.leaf_vstart, 0, 4, s);
        cudaMemsetAsync(Rp.lower_lstart, 0, 4, s);
    }
    launch_runs(Rp, skeys, key64, s);
    rc = sync_scalars(ctx, "runs");
    if (rc)
        return rc;
    const int64_t V = (int64_t)ctx->hscal[SC_V], L = (int64_t)ctx->hscal[SC_L], Lo = (int64_t)ctx->hscal[SC_LO];

    // ---------------------------------------------------------- node tables
    if (!ensure(ctx, ctx->lower_origin, 12 * (size_t)(Lo + 1)) || !ensure(ctx, ctx->lower_upper_n, 4 * (size_t)(Lo + 1)) ||
        !ensure(ctx, ctx->upper_head, 8 * (size_t)(Lo + 1)) || !ensure(ctx, ctx->upper_scan, 8 * (size_t)(Lo + 1)) ||
        !ensure(ctx, ctx->lower_parent, 4 * (size_t)(Lo + 1)) || !ensure(ctx, ctx->upper_root_n, 4 * (size_t)(Lo + 1)) ||
        !ensure(ctx, ctx->upper_lostart, 4 * (size_t)(Lo + 2)) || !ensure(ctx, ctx->leaf_lower, 4 * (size_t)(L + 1)) ||
        !ensure(ctx, ctx->leaf_lower_n, 4 * (size_t)(L + 1)) || !ensure(ctx, ctx->leaf_mask, 64 * (size_t)(L + 1)) ||
        !ensure(ctx, ctx->leaf_origin, 12 * (size_t)(L + 1)) || !ensure(ctx, ctx->rank_to_lower, 4 * (size_t)(NL + 1)) ||
        !ensure(ctx, ctx->order, 8 * 3 * (size_t)((Lo + 1) * 2 + (L + 1))) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(Lo + 1) * 2))
        return VOX_ERR_MEMORY;
    // per-cloud tables: 3 x (B + 1) u32 starts, L u32 leaf clouds, 9 x (B + 1) u64 layout words, 6 B i32 bbox
    const size_t cl_u32 = 3 * (size_t)(B + 1), cl_u64 = 9 * (size_t)(B + 1);
    const size_t cl_bytes = 8 * cl_u64 + 4 * (cl_u32 + (size_t)L + 6 * (size_t)B) + 64;
    if (!ensure(ctx, ctx->clouds, cl_bytes))
        return VOX_ERR_MEMORY;
    scan_status = (uint64_t*)ctx->scan_status.p;
    scan_words = ctx->scan_status.cap / sizeof(uint64_t);
    NodeParams N;
    N.Lo = Lo;
    N.L = L;
    N.lower_rank = (const uint32_t*)ctx->lower_rank.p;
    N.lower_cell = (const uint32_t*)ctx->lower_cell.p;
    N.root_of_rank = (const uint32_t*)ctx->root_of_rank.p;
    N.lower_lstart = (const uint32_t*)ctx->lower_lstart.p;
    N.leaf_vstart = (const uint32_t*)ctx->leaf_vstart.p;
    N.vox_start = (const uint32_t*)ctx->vox_start.p;
    N.lower_origin = (int32_t*)ctx->lower_origin.p;
    N.lower_upper_n = (uint32_t*)ctx->lower_upper_n.p;
    N.rank_to_lower = (uint32_t*)ctx->rank_to_lower.p;
    N.upper_head = (uint64_t*)ctx->upper_head.p;
    N.upper_scan = (uint64_t*)ctx->upper_scan.p;
    N.lower_parent = (uint32_t*)ctx->lower_parent.p;
    N.upper_root_n = (uint32_t*)ctx->upper_root_n.p;
    N.upper_lostart = (uint32_t*)ctx->upper_lostart.p;
    N.upper_count = sc + SC_U;
    N.leaf_lower = (uint32_t*)ctx->leaf_lower.p;
    N.leaf_lower_n = (uint32_t*)ctx->leaf_lower_n.p;
    N.leaf_mask = (uint64_t*)ctx->leaf_mask.p;
    N.leaf_origin = (int32_t*)ctx->leaf_origin.p;
    uint64_t* ord = (uint64_t*)ctx->order.p;
    N.upper_idx = ord;
    N.upper_addr = ord + (Lo + 1);
    N.upper_vidx = ord + 2 * (Lo + 1);
    N.lower_idx = ord + 3 * (Lo + 1);
    N.lower_addr = ord + 4 * (Lo + 1);
    N.lower_vidx = ord + 5 * (Lo + 1);
    N.leaf_idx = ord + 6 * (Lo + 1);
    N.leaf_addr = ord + 6 * (Lo + 1) + (L + 1);
    N.leaf_vidx = ord + 6 * (Lo + 1) + 2 * (L + 1);
    {
        CloudParams& C = N.C;
        uint64_t* w64 = (uint64_t*)ctx->clouds.p;
        C.B = B;
        C.vstart = w64;
        C.grid_off = w64 + (B + 1);
        C.value_base = w64 + 2 * (B + 1);
        C.node2_bytes = w64 + 3 * (B + 1);
        C.bbox_off = w64 + 4 * (B + 1);
        C.rgba_off = w64 + 5 * (B + 1);
        C.dens_off = w64 + 6 * (B + 1);
        C.col_off = w64 + 7 * (B + 1);
        uint32_t* w32 = (uint32_t*)(w64 + cl_u64);
        C.upper_start = w32;
        C.lower_start = w32 + (B + 1);
        C.leaf_start = w32 + 2 * (B + 1);
        C.leaf_cloud = w32 + cl_u32;
        C.bbox = (int32_t*)(w32 + cl_u32 + L);
        C.cloud_vs = d_cloud_vs;
        C.voxel_size = voxel_size;
        C.cloud_start = d_cloud_start;
        C.frag_off = frag_off;
        C.F_total = sc + SC_F;
        C.G = G;
        C.P = P_pairs;
        C.V = V;
        C.node_order = (flags & VOX_FLAG_WINDOW_ORDER) ? 1u : 0u;
        cudaMemsetAsync(C.upper_start, 0, 4 * cl_u32, s); // clouds without nodes start at 0
    }
    launch_lower_info(N, s);
    scan_exclusive_u64(N.upper_head, N.upper_scan, Lo, 0, sc + SC_SCRATCH + 1, scan_status,
                       ctx->scan_epochs.next(scan_status, scan_words, s), d_counter, d_err, ctx->num_sms, s);
    launch_upper_info(N, s);
    launch_leaf_tables(N, skeys, key64, s);
    launch_cloud_layout(N, s);
    cudaMemcpyAsync(sc + SC_GRID_BYTES, N.C.grid_off + B, sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
    rc = sync_scalars(ctx, "node tables");
    if (rc)
        return rc;
    const uint64_t U = Lo > 0 ? ctx->hscal[SC_U] : 0;
    const uint64_t grid_bytes = ctx->hscal[SC_GRID_BYTES];
    if (window)
    {
        rc = window_order(ctx, N, (int64_t)U, Lo, L, (int64_t)ctx->hscal[SC_NWIN], s);
        if (rc)
            return rc;
    }
    else
        launch_canonical_order(N, U, s);

    // --------------------------------------------------------- grid buffer
    // every cloud's grid: header, node2 region, bbox, RGBA8, density, colour
    if (!ensure(ctx, ctx->grid, grid_bytes))
        return VOX_ERR_MEMORY;
    uint8_t* grid = (uint8_t*)ctx->grid.p;
    launch_zero_gaps(N, grid, grid_bytes, s);
    launch_leaf_masks(N, LP.cand_mask, (const uint32_t*)ctx->vslot.p, s);
    uint64_t* cloud_pairs = nullptr;
    if (B > 1)
    {
        if (!ensure(ctx, ctx->cloud_pairs, 8 * (size_t)(B + 1)))
            return VOX_ERR_MEMORY;
        cloud_pairs = (uint64_t*)ctx->cloud_pairs.p;
        cudaMemsetAsync(cloud_pairs, 0, 8 * (size_t)B, s);
    }
    ValueParams VA;
    VA.V = V;
    VA.vslot = (const uint32_t*)ctx->vslot.p;
    VA.s_rgba = LP.s_rgba;
    VA.s_dens = LP.s_dens;
    VA.s_col = LP.s_col;
    VA.s_pairs = LP.s_pairs;
    VA.cloud_pairs = cloud_pairs;
    VA.cand_vbase = (uint64_t*)ctx->cand_vbase.p;
    VA.vox_leaf = (const uint32_t*)ctx->vox_leaf.p;
    VA.vox_n = (const uint16_t*)ctx->vox_n.p;
    VA.out = grid;
    launch_values(VA, N, s);
    N.C.cloud_pairs = cloud_pairs;
    N.C.P = P_pairs;
    cudaEventRecord(ctx->timers.ev[5], s);
    launch_leaf_bbox(N, s);
    launch_write_nodes(N, U, grid, s);
    launch_write_headers(N, grid, s);
    ctx->h_grid_off.resize((size_t)B + 1);
    ctx->h_value_base.resize((size_t)B + 1);
    cudaMemcpyAsync(ctx->h_grid_off.data(), N.C.grid_off, sizeof(uint64_t) * (B + 1), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ctx->h_value_base.data(), N.C.value_base, sizeof(uint64_t) * (B + 1), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(ctx->timers.ev[6], s);
    rc = sync_scalars(ctx, "accumulate");
    if (rc)
        return rc;
    rc = check_cuda(ctx, "accumulate");
    if (rc)
        return rc;
    const uint64_t value_count = ctx->h_value_base[(size_t)B];

    ctx->last_grid_bytes = grid_bytes;
    vox_stats_t& st = ctx->stats;
    st.voxels = V;
    st.uppers = (int64_t)U;
    st.lowers = Lo;
    st.leaves = L;
    st.value_count = (int64_t)value_count;
    st.grid_bytes = (int64_t)grid_bytes;
    st.ms_prep = elapsed(ctx->timers.ev[0], ctx->timers.ev[1]);
    st.ms_emit = elapsed(ctx->timers.ev[1], ctx->timers.ev[2]);       // (leaf, Gaussian) pairs
    st.ms_sort = elapsed(ctx->timers.ev[2], ctx->timers.ev[3]);       // sort + candidate leaves
    st.ms_accumulate = elapsed(ctx->timers.ev[3], ctx->timers.ev[4]); // leaf walk: test, RGBA8, float sums
    ctx->walk_choice[ctx->walk_mode].report((int64_t)Q, ctx->walk_variant, st.ms_accumulate);
    st.ms_build = elapsed(ctx->timers.ev[4], ctx->timers.ev[6]);      // topology, values, node2
    st.ms_total = elapsed(ctx->timers.ev[0], ctx->timers.ev[6]);
    st.kernel_launches = launch_count() - launches0;
    ctx->last_G = G;
    ctx->last_V = V;
    ctx->last_value_count = value_count;
    ctx->last_flags = flags;
    ctx->last_voxel_size = voxel_size;
    ctx->last_cloud_vs = d_cloud_vs;
    ctx->last_N = N;
    LP.pair_off = nullptr; // built on demand by vox_copy_pairs
    ctx->last_LP = LP;
    ctx->last_NLC = NLC;
    ctx->last_Q = Q;
    ctx->diff_ready = diff;
    return VOX_OK;
}

static int run_backward(vox_context_t* ctx, const vox_gaussians_t* gs, const float* grad_density,
                        const float* grad_color, float* d_means, float* d_quats, float* d_scales, float* d_opacities,
                        float* d_colors)
{
    if (!ctx || !gs)
    {
        set_error(ctx, "vox_backward: invalid arguments");
        return VOX_ERR_ARGS;
    }
    if (!ctx->diff_ready)
    {
        set_error(ctx, "vox_backward: the context's last call was not a successful VOX_FLAG_DIFFERENTIABLE voxelization");
        return VOX_ERR_ARGS;
    }
    if (gs->count != ctx->last_G)
    {
        set_error(ctx, "vox_backward: %lld Gaussians, the forward had %lld", (long long)gs->count, (long long)ctx->last_G);
        return VOX_ERR_ARGS;
    }
    const int64_t G = gs->count;
    if (G > 0 && (!gs->means || !gs->quats || !gs->scales || !gs->opacities || !gs->colors))
    {
        set_error(ctx, "vox_backward: missing attribute array");
        return VOX_ERR_ARGS;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int64_t launches0 = launch_count();
    const uint64_t Q = ctx->last_Q;
    if (!ensure(ctx, ctx->partials, sizeof(float) * BWD_NACC * (size_t)(Q + 1)))
        return VOX_ERR_MEMORY;
    cudaEventRecord(ctx->timers.ev[0], s);
    cudaMemsetAsync((uint64_t*)ctx->scal.p + SC_ERR, 0, sizeof(uint64_t), s);
    arm_wait(ctx, (uint64_t*)ctx->scal.p, s);
    float* partials = (float*)ctx->partials.p;
    if (grad_density || grad_color)
    {
        LeafPassParams LP = ctx->last_LP;
        LP.grad_density = grad_density;
        LP.grad_color = grad_color;
        LP.partials = partials;
        launch_leaf_backward(LP, (uint32_t*)((uint64_t*)ctx->scal.p + SC_SCRATCH), ctx->num_sms, s);
    }
    else
        cudaMemsetAsync(partials, 0, sizeof(float) * BWD_NACC * (size_t)Q, s);
    BwdFinalParams F;
    memset(&F, 0, sizeof(F));
    F.partials = partials;
    F.lcol_off = (const uint64_t*)ctx->lcol_off.p;
    F.lc_off = (const uint64_t*)ctx->lc_off.p;
    F.NLC = ctx->last_NLC;
    F.Q = Q;
    F.G = G;
    F.means = gs->means;
    F.quats = gs->quats;
    F.scales = gs->scales;
    F.opacities = gs->opacities;
    F.colors = gs->colors;
    F.raw = (ctx->last_flags & VOX_FLAG_RAW_INPUTS) ? 1 : 0;
    F.bf16 = (ctx->last_flags & VOX_FLAG_BF16_INPUTS) ? 1 : 0;
    F.voxel_size = ctx->last_voxel_size;
    F.cloud_vs = ctx->last_cloud_vs;
    F.recs = (const GaussRec*)ctx->recs.p;
    F.d_means = d_means;
    F.d_quats = d_quats;
    F.d_scales = d_scales;
    F.d_opacities = d_opacities;
    F.d_colors = d_colors;
    launch_bwd_finalize(F, s);
    cudaEventRecord(ctx->timers.ev[1], s);
    int rc = sync_scalars(ctx, "backward");
    if (rc)
        return rc;
    rc = check_cuda(ctx, "backward");
    if (rc)
        return rc;
    ctx->stats.ms_backward = elapsed(ctx->timers.ev[0], ctx->timers.ev[1]);
    ctx->stats.kernel_launches = launch_count() - launches0;
    return VOX_OK;
}

// coordinates of the active voxels by value index (clouds back to back)
__global__ void k_voxel_coords(int64_t V, const uint32_t* vox_leaf, const uint16_t* vox_n, const int32_t* leaf_origin,
                               const uint32_t* leaf_vstart, const uint64_t* leaf_vidx, const uint32_t* leaf_cloud,
                               const uint64_t* value_base, int32_t* out)
{
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V)
        return;
    const uint32_t l = vox_leaf[v], n = vox_n[v];
    const uint64_t slot = value_base[leaf_cloud[l]] + leaf_vidx[l] + (uint64_t)(v - leaf_vstart[l]);
    out[3 * slot + 0] = leaf_origin[3 * l + 0] + (int32_t)(n >> 6);
    out[3 * slot + 1] = leaf_origin[3 * l + 1] + (int32_t)((n >> 3) & 7);
    out[3 * slot + 2] = leaf_origin[3 * l + 2] + (int32_t)(n & 7);
}

// hierarchical key of a compact key: rank -> cell -> (root_n, upper_n)
__global__ void k_export_keys(const void* keys, int key64, const uint32_t* lower_cell, const uint32_t* root_of_rank,
                              int64_t n, uint64_t* out)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    uint64_t k = key64 ? ((const uint64_t*)keys)[i] : (uint64_t)((const uint32_t*)keys)[i];
    uint32_t cell = lower_cell[k >> 21];
    uint64_t rn = root_of_rank[cell >> 15];
    out[i] = (rn << 36) | ((uint64_t)(cell & 32767u) << 21) | (k & ((1ull << 21) - 1ull));
}

// ---------------------------------------------------------------------------
// vox_* C ABI
// ---------------------------------------------------------------------------
extern "C" {

vox_context_t* vox_context_create(int device)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0)
    {
        cudaGetLastError();
        set_error(nullptr, "vox_context_create: no CUDA device");
        return nullptr;
    }
    if (device < 0 || device >= count)
        device = 0;
    vox_context_t* ctx = new vox_context_t();
    ctx->device = device;
    cudaSetDevice(device);
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost((void**)&ctx->hscal, sizeof(uint64_t) * SC_SCRATCH * 8) != cudaSuccess)
    {
        set_error(nullptr, "vox_context_create: stream / pinned allocation failed");
        delete ctx;
        return nullptr;
    }
    for (auto& e : ctx->timers.ev)
        cudaEventCreate(&e);
    cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
    for (auto& e : ctx->up_ev)
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    const char* chk = getenv("VOX_CHECK_SORT");
    ctx->check_sort = (chk && chk[0] == '1') ? 1 : 0;
    const char* chk_emit = getenv("VOX_CHECK_EMIT");
    ctx->check_emit = (chk_emit && chk_emit[0] == '1') ? 1 : 0;
    // VOX_SORT_SHAPE=c fixes the sort's tuner candidate (0-4: onesweep tile
    // shapes, 5-9: the same shapes as three-kernel passes), for tests and timing
    const char* shp = getenv("VOX_SORT_SHAPE");
    if (shp && shp[0] >= '0' && shp[0] <= '9' && shp[1] == 0)
        ctx->tuning.shape = shp[0] - '0';
    return ctx;
}

void vox_context_destroy(vox_context_t* ctx)
{
    if (!ctx)
        return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    DevBuf* all[] = { &ctx->recs, &ctx->footprints, &ctx->frag_off, &ctx->root_bits, &ctx->root_prefix,
                      &ctx->root_of_rank, &ctx->lower_bits, &ctx->lower_prefix, &ctx->lower_cell, &ctx->scan_status,
                      &ctx->run_status, &ctx->keys, &ctx->ids, &ctx->keys_alt, &ctx->ids_alt,
                      &ctx->sort_ws, &ctx->vox_start, &ctx->leaf_vstart, &ctx->lower_lstart, &ctx->lower_rank,
                      &ctx->lower_origin, &ctx->lower_upper_n, &ctx->upper_head, &ctx->upper_scan,
                      &ctx->lower_parent, &ctx->upper_root_n, &ctx->upper_lostart, &ctx->leaf_lower,
                      &ctx->leaf_lower_n, &ctx->leaf_mask, &ctx->leaf_origin, &ctx->order, &ctx->grid, &ctx->scal,
                      &ctx->vox_leaf, &ctx->vox_n, &ctx->rank_to_lower,
                      &ctx->hier_keys, &ctx->prim_keys_alt, &ctx->prim_vals_alt, &ctx->vb_work, &ctx->vb_keys, &ctx->vb_ids_c, &ctx->vb_used, &ctx->dual_idx, &ctx->vb_rec, &ctx->cloud_start,
                      &ctx->cloud_vs, &ctx->clouds, &ctx->lcols, &ctx->lcol_off, &ctx->lc_count, &ctx->lc_mask, &ctx->lc_off,
                      &ctx->cand_org, &ctx->tile_g0, &ctx->emit_gid, &ctx->emit_flag, &ctx->lflags, &ctx->lpos, &ctx->cand_key, &ctx->cand_start,
                      &ctx->cand_mask, &ctx->pair_gid, &ctx->s_rgba, &ctx->s_dens, &ctx->s_col, &ctx->s_pairs, &ctx->cand_cnt,
                      &ctx->cand_voff, &ctx->vkeys, &ctx->vslot, &ctx->vpairs, &ctx->pair_off, &ctx->cand_vbase, &ctx->cloud_pairs,
                      &ctx->partials, &ctx->exp_keys, &ctx->exp_ids, &ctx->nwin, &ctx->win_before,
                      &ctx->cand_wkey, &ctx->wkey_u, &ctx->wkey_lo, &ctx->wkey_leaf, &ctx->wcnt, &ctx->wbase,
                      &ctx->okeys, &ctx->okeys_alt, &ctx->ovals, &ctx->ovals_alt, &ctx->rank_u, &ctx->rank_lo,
                      &ctx->rank_leaf, &ctx->leaf_popc, &ctx->leaf_voff };
    for (DevBuf* b : all)
        if (b->p)
            cudaFree(b->p);
    for (auto& e : ctx->timers.ev)
        if (e)
            cudaEventDestroy(e);
    for (auto& e : ctx->up_ev)
        if (e)
            cudaEventDestroy(e);
    if (ctx->copy_stream)
    {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->hscal)
        cudaFreeHost(ctx->hscal);
    if (ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
}

void* vox_context_stream(vox_context_t* ctx)
{
    return ctx ? (void*)ctx->stream : nullptr;
}

int vox_context_set_wait_limit(vox_context_t* ctx, uint32_t max_polls, int withhold_publication)
{
    if (!ctx)
        return VOX_ERR_ARGS;
    if (max_polls == VOX_WAIT_DEFAULT && !withhold_publication)
    {
        ctx->wait_ctl = 0;
        return VOX_OK;
    }
    const uint32_t lim = max_polls > 0x7ffffffeu ? 0x7ffffffeu : max_polls;
    ctx->wait_ctl = (lim + 1u) | (withhold_publication ? 0x80000000u : 0u);
    return VOX_OK;
}

const char* vox_last_error(vox_context_t* ctx)
{
    return ctx ? ctx->last_error.c_str() : "no context";
}

int vox_voxelize_batch(vox_context_t* ctx, const vox_gaussians_t* gaussians, int64_t clouds, const int64_t* cloud_start,
                       const float* voxel_sizes, float cull_scale, uint32_t flags, void** grids,
                       uint64_t* grid_offsets, uint64_t* value_offsets)
{
    if (!cloud_start || !voxel_sizes)
    {
        set_error(ctx, "vox_voxelize_batch: cloud_start and voxel_sizes are required");
        return VOX_ERR_ARGS;
    }
    int rc = run_voxelize(ctx, gaussians, voxel_sizes[0], cull_scale, flags, clouds, cloud_start, voxel_sizes);
    if (rc)
        return rc;
    if (grids)
        *grids = ctx->grid.p;
    if (grid_offsets)
        memcpy(grid_offsets, ctx->h_grid_off.data(), sizeof(uint64_t) * (size_t)(clouds + 1));
    if (value_offsets)
        memcpy(value_offsets, ctx->h_value_base.data(), sizeof(uint64_t) * (size_t)(clouds + 1));
    return VOX_OK;
}

int vox_backward(vox_context_t* ctx, const vox_gaussians_t* gaussians, const float* grad_density, const float* grad_color,
                 float* grad_means, float* grad_quats, float* grad_scales, float* grad_opacities, float* grad_colors)
{
    return run_backward(ctx, gaussians, grad_density, grad_color, grad_means, grad_quats, grad_scales, grad_opacities,
                        grad_colors);
}

int vox_voxelize(vox_context_t* ctx, const vox_gaussians_t* gaussians, float voxel_size, float cull_scale,
                 uint32_t flags, void** grid, uint64_t* grid_bytes)
{
    int rc = run_voxelize(ctx, gaussians, voxel_size, cull_scale, flags);
    if (rc)
        return rc;
    if (grid)
        *grid = ctx->grid.p;
    if (grid_bytes)
        *grid_bytes = ctx->last_grid_bytes;
    return VOX_OK;
}

int vox_voxelize_host(vox_context_t* ctx, const vox_gaussians_t* gaussians, float voxel_size, float cull_scale,
                      uint32_t flags, void* out, uint64_t out_capacity, uint64_t* grid_bytes)
{
    if (!ctx || !gaussians)
        return VOX_ERR_ARGS;
    cudaSetDevice(ctx->device);
    const int64_t n = gaussians->count;
    DevBuf& in = ctx->hier_keys; // reused as the attribute upload area between calls
    const size_t es = (flags & VOX_FLAG_BF16_INPUTS) ? 2 : 4; // bytes per attribute value
    const size_t per = 16 * sizeof(float);
    if (!ensure(ctx, in, per * (size_t)(n + 1)))
        return VOX_ERR_MEMORY;
    float* d = (float*)in.p;
    vox_gaussians_t dg;
    dg.count = n;
    // the arrays back to back, in their own element size
    char* db = (char*)d;
    dg.means = (const float*)db;
    dg.quats = (const float*)(db + 3 * n * es);
    dg.scales = (const float*)(db + 7 * n * es);
    dg.opacities = (const float*)(db + 10 * n * es);
    dg.colors = (const float*)(db + 11 * n * es);
    // the copies are issued by run_voxelize's prep step (chunked, overlapping k_prep)
    const void* hs[5] = { gaussians->means, gaussians->quats, gaussians->scales, gaussians->opacities, gaussians->colors };
    const void* ds[5] = { dg.means, dg.quats, dg.scales, dg.opacities, dg.colors };
    for (int a = 0; a < 5; a++)
    {
        ctx->upload.host[a] = hs[a];
        ctx->upload.dev[a] = (char*)ds[a];
    }
    ctx->upload.es = es;
    ctx->upload.active = n > 0;
    int rc = run_voxelize(ctx, &dg, voxel_size, cull_scale, flags);
    ctx->upload.active = false;
    if (rc)
        return rc;
    if (grid_bytes)
        *grid_bytes = ctx->last_grid_bytes;
    if (!out)
        return VOX_OK;
    if (out_capacity < ctx->last_grid_bytes)
    {
        set_error(ctx, "vox_voxelize_host: output capacity %llu < grid size %llu", (unsigned long long)out_capacity,
                  (unsigned long long)ctx->last_grid_bytes);
        return VOX_ERR_SIZE;
    }
    cudaMemcpyAsync(out, ctx->grid.p, ctx->last_grid_bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return check_cuda(ctx, "vox_voxelize_host copy");
    return VOX_OK;
}

int vox_copy_grid(vox_context_t* ctx, void* out, uint64_t capacity)
{
    if (!ctx || !out)
        return VOX_ERR_ARGS;
    if (capacity < ctx->last_grid_bytes)
        return VOX_ERR_SIZE;
    cudaSetDevice(ctx->device);
    // host or device destination (unified addressing)
    cudaMemcpyAsync(out, ctx->grid.p, ctx->last_grid_bytes, cudaMemcpyDefault, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return check_cuda(ctx, "vox_copy_grid");
    return VOX_OK;
}

int vox_copy_grid_rgba8(vox_context_t* ctx, void* out, uint64_t capacity, uint64_t* bytes)
{
    if (!ctx || !bytes)
        return VOX_ERR_ARGS;
    if (ctx->last_V < 0 || ctx->h_grid_off.size() != 2)
    {
        set_error(ctx, "vox_copy_grid_rgba8: no single-cloud grid");
        return VOX_ERR_ARGS;
    }
    cudaSetDevice(ctx->device);
    vox_grid_header_t h;
    cudaMemcpyAsync(&h, ctx->grid.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return check_cuda(ctx, "vox_copy_grid_rgba8");
    const uint64_t n = h.rgba8_offset + 4 * h.value_count;
    *bytes = n;
    if (!out)
        return VOX_OK;
    if (capacity < n)
        return VOX_ERR_SIZE;
    h.grid_bytes = n;
    h.density_offset = 0;
    h.color_offset = 0;
    cudaMemcpyAsync(out, &h, sizeof(h), cudaMemcpyDefault, ctx->stream);
    cudaMemcpyAsync((uint8_t*)out + sizeof(h), (const uint8_t*)ctx->grid.p + sizeof(h), n - sizeof(h), cudaMemcpyDefault,
                    ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return check_cuda(ctx, "vox_copy_grid_rgba8");
    return VOX_OK;
}

int vox_voxel_coords(vox_context_t* ctx, int32_t* d_ijk, int64_t capacity)
{
    if (!ctx || (!d_ijk && capacity > 0))
        return VOX_ERR_ARGS;
    if (ctx->last_V < 0)
    {
        set_error(ctx, "vox_voxel_coords: no grid");
        return VOX_ERR_ARGS;
    }
    const int64_t V = ctx->last_V;
    if (capacity < (int64_t)ctx->last_value_count)
        return VOX_ERR_SIZE;
    if (V == 0)
        return VOX_OK;
    cudaSetDevice(ctx->device);
    const NodeParams& N = ctx->last_N;
    { k_voxel_coords<<<(unsigned)((V + 255) / 256), 256, 0, ctx->stream>>>(V, (const uint32_t*)ctx->vox_leaf.p, (const uint16_t*)ctx->vox_n.p, N.leaf_origin, N.leaf_vstart, N.leaf_vidx, N.C.leaf_cloud, N.C.value_base, d_ijk); count_launch(); }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return check_cuda(ctx, "vox_voxel_coords");
    return VOX_OK;
}

int vox_copy_pairs(vox_context_t* ctx, uint64_t* keys, uint32_t* ids, int64_t capacity)
{
    if (!ctx)
        return VOX_ERR_ARGS;
    if (ctx->last_V < 0)
    {
        set_error(ctx, "vox_copy_pairs: no grid");
        return VOX_ERR_ARGS;
    }
    const int64_t P = ctx->last_P;
    if (capacity < P)
        return VOX_ERR_SIZE;
    if (P == 0)
        return VOX_OK;
    cudaSetDevice(ctx->device);
    const size_t kb = ctx->key64 ? 8 : 4;
    if (!ensure(ctx, ctx->exp_keys, kb * (size_t)P) || !ensure(ctx, ctx->exp_ids, 4 * (size_t)P))
        return VOX_ERR_MEMORY;
    // pairs before each voxel: the staged per-voxel counts in run order, scanned
    const int64_t V = ctx->last_V;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    if (!ensure(ctx, ctx->vpairs, 8 * (size_t)(V + 1)) || !ensure(ctx, ctx->pair_off, 8 * (size_t)(V + 1)) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(V + 1) * 2))
        return VOX_ERR_MEMORY;
    uint64_t* scan_status = (uint64_t*)ctx->scan_status.p;
    const size_t scan_words = ctx->scan_status.cap / sizeof(uint64_t);
    launch_voxel_pairs(V, (const uint32_t*)ctx->vslot.p, (const uint32_t*)ctx->s_pairs.p, (uint64_t*)ctx->vpairs.p,
                       ctx->stream);
    scan_exclusive_u64((const uint64_t*)ctx->vpairs.p, (uint64_t*)ctx->pair_off.p, V, 0, sc + SC_SCRATCH + 3,
                       scan_status, ctx->scan_epochs.next(scan_status, scan_words, ctx->stream),
                       (uint32_t*)(sc + SC_SCRATCH), (int*)(sc + SC_ERR), ctx->num_sms, ctx->stream);
    // replay the leaf walk, writing every passing pair at its voxel's pair offset
    LeafPassParams LP = ctx->last_LP;
    LP.pair_off = (const uint64_t*)ctx->pair_off.p;
    LP.out_keys = ctx->exp_keys.p;
    LP.out_ids = (uint32_t*)ctx->exp_ids.p;
    launch_leaf_export(LP, (uint32_t*)((uint64_t*)ctx->scal.p + SC_SCRATCH), ctx->num_sms, ctx->stream);
    DevBuf tmp;
    if (!ensure(ctx, tmp, 8 * (size_t)P))
        return VOX_ERR_MEMORY;
    k_export_keys<<<(unsigned)((P + 255) / 256), 256, 0, ctx->stream>>>(
        ctx->exp_keys.p, ctx->key64, (const uint32_t*)ctx->lower_cell.p, (const uint32_t*)ctx->root_of_rank.p, P,
        (uint64_t*)tmp.p);
    count_launch();
    if (keys)
        cudaMemcpyAsync(keys, tmp.p, 8 * (size_t)P, cudaMemcpyDeviceToHost, ctx->stream);
    if (ids)
        cudaMemcpyAsync(ids, ctx->exp_ids.p, 4 * (size_t)P, cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    cudaFree(tmp.p);
    if (e != cudaSuccess)
        return check_cuda(ctx, "vox_copy_pairs");
    return VOX_OK;
}

void vox_get_stats(vox_context_t* ctx, vox_stats_t* out)
{
    if (ctx && out)
        *out = ctx->stats;
}

int vox_global_scan_u64(vox_context_t* ctx, const uint64_t* d_in, uint64_t* d_out, int64_t n, int inclusive,
                        uint64_t* d_total)
{
    if (!ctx || n < 0 || (n > 0 && (!d_in || !d_out)) || !d_total)
        return VOX_ERR_ARGS;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (!ensure(ctx, ctx->scal, sizeof(uint64_t) * SC_SCRATCH * 4) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(n > 512 ? n : 512) * 2))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    clear_scalars(ctx, sc, s);
    uint64_t* status = (uint64_t*)ctx->scan_status.p;
    scan_exclusive_u64(d_in, d_out, n, inclusive ? 2 : 0, d_total, status,
                       ctx->scan_epochs.next(status, ctx->scan_status.cap / sizeof(uint64_t), s),
                       (uint32_t*)(sc + SC_SCRATCH), (int*)(sc + SC_ERR), ctx->num_sms, s);
    return sync_scalars(ctx, "vox_global_scan_u64");
}

int vox_global_scan_u32(vox_context_t* ctx, const uint32_t* d_in, uint32_t* d_out, int64_t n, int inclusive,
                        uint32_t* d_total)
{
    if (!ctx || n < 0 || (n > 0 && (!d_in || !d_out)))
        return VOX_ERR_ARGS;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (!ensure(ctx, ctx->scal, sizeof(uint64_t) * SC_SCRATCH * 4) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(n > 512 ? n : 512) * 2))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    clear_scalars(ctx, sc, s);
    uint64_t* status = (uint64_t*)ctx->scan_status.p;
    scan_u32(d_in, d_out, n, inclusive ? 1 : 0, 0, sc + SC_F, status,
             ctx->scan_epochs.next(status, ctx->scan_status.cap / sizeof(uint64_t), s), (uint32_t*)(sc + SC_SCRATCH),
             (int*)(sc + SC_ERR), s);
    if (d_total)
        cudaMemcpyAsync(d_total, sc + SC_F, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s); // low half: mod 2^32
    return sync_scalars(ctx, "vox_global_scan_u32");
}

int vox_global_scan_max_u32(vox_context_t* ctx, const uint32_t* d_in, uint32_t* d_out, int64_t n)
{
    if (!ctx || n < 0 || (n > 0 && (!d_in || !d_out)))
        return VOX_ERR_ARGS;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (!ensure(ctx, ctx->scal, sizeof(uint64_t) * SC_SCRATCH * 4) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(n > 512 ? n : 512) * 2))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    clear_scalars(ctx, sc, s);
    uint64_t* status = (uint64_t*)ctx->scan_status.p;
    scan_u32(d_in, d_out, n, 1, 1, sc + SC_F, status,
             ctx->scan_epochs.next(status, ctx->scan_status.cap / sizeof(uint64_t), s), (uint32_t*)(sc + SC_SCRATCH),
             (int*)(sc + SC_ERR), s);
    return sync_scalars(ctx, "vox_global_scan_max_u32");
}

int vox_radix_sort_u32(vox_context_t* ctx, uint32_t* d_keys, uint32_t* d_vals, int64_t n, uint32_t key_bit_count)
{
    if (!ctx || n < 0 || (n > 0 && (!d_keys || !d_vals)) || key_bit_count > 32)
        return VOX_ERR_ARGS;
    if (n <= 1 || key_bit_count == 0)
        return VOX_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (!ensure(ctx, ctx->scal, sizeof(uint64_t) * SC_SCRATCH * 4) ||
        !ensure(ctx, ctx->prim_keys_alt, 4 * (size_t)n) || !ensure(ctx, ctx->prim_vals_alt, 4 * (size_t)n) ||
        !ensure(ctx, ctx->sort_ws, sort_workspace_bytes(n, 4)))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    clear_scalars(ctx, sc, s);
    int in_alt = sort_pairs_u32(d_keys, d_vals, (uint32_t*)ctx->prim_keys_alt.p, (uint32_t*)ctx->prim_vals_alt.p, n,
                                (int)key_bit_count, ctx->sort_ws.p, &ctx->sort_epochs, (int*)(sc + SC_ERR),
                                ctx->num_sms, s, ctx->tuning);
    if (in_alt)
    {
        cudaMemcpyAsync(d_keys, ctx->prim_keys_alt.p, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d_vals, ctx->prim_vals_alt.p, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s);
    }
    return sync_scalars(ctx, "vox_radix_sort_u32");
}

int vox_radix_sort_dual_key(vox_context_t* ctx, uint32_t* d_keys_low, uint32_t* d_keys_high, uint32_t* d_vals,
                            int64_t n, uint32_t key_low_bit_count, uint32_t key_high_bit_count)
{
    if (!ctx || n < 0 || (n > 0 && (!d_keys_low || !d_keys_high || !d_vals)) || key_low_bit_count > 32 ||
        key_high_bit_count > 32 || n > 0xffffffffll)
        return VOX_ERR_ARGS;
    const int bits = (int)(key_low_bit_count + key_high_bit_count);
    if (n <= 1 || bits == 0)
        return VOX_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (!ensure(ctx, ctx->scal, sizeof(uint64_t) * SC_SCRATCH * 4) || !ensure(ctx, ctx->vb_keys, 8 * (size_t)n) ||
        !ensure(ctx, ctx->prim_keys_alt, 8 * (size_t)n) || !ensure(ctx, ctx->prim_vals_alt, 4 * (size_t)n) ||
        !ensure(ctx, ctx->dual_idx, 4 * (size_t)n) || !ensure(ctx, ctx->sort_ws, sort_workspace_bytes(n, 8)))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    int* err = (int*)(sc + SC_ERR);
    clear_scalars(ctx, sc, s);
    // one stable sort by (high, low): the order of the reference's sort by
    // the low key then, stably, by the high key (ParallelPrimitives.cpp:527-683)
    uint64_t* key = (uint64_t*)ctx->vb_keys.p;
    uint32_t* idx = (uint32_t*)ctx->dual_idx.p;
    dual_combine(d_keys_low, d_keys_high, n, (int)key_low_bit_count, (int)key_high_bit_count, key, idx, ctx->num_sms, s);
    const int in_alt = sort_pairs_u64(key, idx, (uint64_t*)ctx->prim_keys_alt.p, (uint32_t*)ctx->prim_vals_alt.p, n,
                                      bits, ctx->sort_ws.p, &ctx->sort_epochs, err, ctx->num_sms, s, ctx->tuning);
    const uint32_t* sidx = in_alt ? (const uint32_t*)ctx->prim_vals_alt.p : idx;
    // copies of the inputs in buffers the sorted indices do not live in
    uint32_t* low_c = (uint32_t*)ctx->vb_keys.p;
    uint32_t* high_c = low_c + n;
    uint32_t* val_c = (uint32_t*)ctx->prim_keys_alt.p;
    cudaMemcpyAsync(low_c, d_keys_low, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(high_c, d_keys_high, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(val_c, d_vals, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s);
    dual_gather(sidx, n, low_c, high_c, val_c, d_keys_low, d_keys_high, d_vals, err, ctx->num_sms, s);
    return sync_scalars(ctx, "vox_radix_sort_dual_key");
}

int vox_radix_sort_key64(vox_context_t* ctx, uint64_t* d_keys, uint32_t* d_vals, int64_t n, uint32_t key_bit_count)
{
    if (!ctx || n < 0 || (n > 0 && (!d_keys || !d_vals)) || key_bit_count > 64)
        return VOX_ERR_ARGS;
    if (n <= 1 || key_bit_count == 0)
        return VOX_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (!ensure(ctx, ctx->scal, sizeof(uint64_t) * SC_SCRATCH * 4) ||
        !ensure(ctx, ctx->prim_keys_alt, 8 * (size_t)n) || !ensure(ctx, ctx->prim_vals_alt, 4 * (size_t)n) ||
        !ensure(ctx, ctx->sort_ws, sort_workspace_bytes(n, 8)))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    clear_scalars(ctx, sc, s);
    SortTuning& t = ctx->tuning;
    int in_alt = sort_pairs_u64(d_keys, d_vals, (uint64_t*)ctx->prim_keys_alt.p, (uint32_t*)ctx->prim_vals_alt.p, n,
                                (int)key_bit_count, ctx->sort_ws.p, &ctx->sort_epochs, (int*)(sc + SC_ERR),
                                ctx->num_sms, s, t);
    if (in_alt)
    {
        cudaMemcpyAsync(d_keys, ctx->prim_keys_alt.p, 8 * (size_t)n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d_vals, ctx->prim_vals_alt.p, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s);
    }
    return sync_scalars(ctx, "vox_radix_sort_key64");
}

int vox_voxelbvh_transform_inverse(const float* m, float* inv)
{
    if (!m || !inv)
        return VOX_ERR_ARGS;
    double a[4][8];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++)
        {
            if (!std::isfinite(m[4 * r + c]))
                return VOX_ERR_ARGS;
            a[r][c] = (double)m[4 * r + c];
            a[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    double scale = 0.0;
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++)
            scale = std::fmax(scale, std::fabs(a[r][c]));
    if (scale == 0.0)
        return VOX_ERR_ARGS;
    for (int col = 0; col < 4; col++)
    {
        int piv = col;
        for (int r = col + 1; r < 4; r++)
            if (std::fabs(a[r][col]) > std::fabs(a[piv][col]))
                piv = r;
        if (std::fabs(a[piv][col]) <= 1e-12 * scale)
            return VOX_ERR_ARGS;
        if (piv != col)
            for (int c = 0; c < 8; c++)
                std::swap(a[piv][c], a[col][c]);
        const double d = a[col][col];
        for (int c = 0; c < 8; c++)
            a[col][c] /= d;
        for (int r = 0; r < 4; r++)
        {
            if (r == col)
                continue;
            const double f = a[r][col];
            if (f != 0.0)
                for (int c = 0; c < 8; c++)
                    a[r][c] -= f * a[col][c];
        }
    }
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++)
            inv[4 * r + c] = (float)a[r][4 + c];
    return VOX_OK;
}

static int bit_length(int64_t v)
{
    int b = 0;
    while (v > 0)
    {
        b++;
        v >>= 1;
    }
    return b;
}

int vox_voxelbvh_ijkl_from_gaussians(vox_context_t* ctx, const float* d_means, const float* d_opacities,
                                     const float* d_quats, const float* d_scales, int64_t count, uint32_t resolution,
                                     const float* transform, uint64_t* d_ijkl, uint32_t* d_prim_id, uint32_t* d_range,
                                     float* d_world_bbox, int64_t* range_count)
{
    // resolution 1..4096: validate_resolution (raster/VoxelBVH.cpp:30-33)
    if (!ctx || count < 0 || count > (1ll << 29) - 1 || resolution < 1u || resolution > 4096u || !d_world_bbox)
        return VOX_ERR_ARGS;
    if (count > 0 && (!d_means || !d_opacities || !d_quats || !d_scales || !d_ijkl || !d_prim_id || !d_range ||
                      ((uintptr_t)d_ijkl & 15u) || ((uintptr_t)d_prim_id & 15u)))
        return VOX_ERR_ARGS;
    VoxelBvhParams P{};
    P.means = d_means;
    P.opac = d_opacities;
    P.quats = d_quats;
    P.scales = d_scales;
    P.n = count;
    P.resolution = resolution;
    if (transform)
    {
        if (vox_voxelbvh_transform_inverse(transform, P.ti) != VOX_OK)
        {
            set_error(ctx, "vox_voxelbvh_ijkl_from_gaussians: transform is singular or not finite");
            return VOX_ERR_ARGS;
        }
        for (int i = 0; i < 16; i++)
            P.t[i] = transform[i];
        P.has_xform = 1;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int64_t launches0 = launch_count();
    const int64_t N = 8 * count;
    const int64_t tiles = vb_range_tiles(N);
    if (!ensure(ctx, ctx->scal, sizeof(uint64_t) * SC_SCRATCH * 4) ||
        !ensure(ctx, ctx->vb_work, 256 + sizeof(uint64_t) * (size_t)(2 * tiles + 2)) ||
        !ensure(ctx, ctx->scan_status, sizeof(uint64_t) * scan_status_words(tiles > 512 ? tiles : 512) * 2))
        return VOX_ERR_MEMORY;
    if (N > 1 && (!ensure(ctx, ctx->vb_keys, 8 * (size_t)N) || !ensure(ctx, ctx->prim_keys_alt, 8 * (size_t)N) ||
                  !ensure(ctx, ctx->prim_vals_alt, 4 * (size_t)N) || !ensure(ctx, ctx->sort_ws, sort_workspace_bytes(N, 8))))
        return VOX_ERR_MEMORY;
    uint64_t* sc = (uint64_t*)ctx->scal.p;
    int* err = (int*)(sc + SC_ERR);
    clear_scalars(ctx, sc, s);
    P.box_keys = (uint32_t*)ctx->vb_work.p;
    P.cell_minmax = (int*)(sc + SC_BBOX);
    P.world_bbox = d_world_bbox;
    P.keys = d_ijkl;
    P.ids = d_prim_id;
    P.err = err;
    uint64_t* tile_cnt = (uint64_t*)((char*)ctx->vb_work.p + 256);
    uint64_t* tile_off = tile_cnt + tiles;
    uint64_t* d_total = tile_off + tiles;
    cudaEventRecord(ctx->timers.ev[0], s);
    launch_vb_init(P.box_keys, P.cell_minmax, s);
    launch_vb_box(P, ctx->num_sms, s);
    // the level search variant: the tuner's choice, or VOX_VB_SEARCH=thread / lane
    const char* search = getenv("VOX_VB_SEARCH");
    ctx->vb_variant = search && search[0] == 't' ? 1 : search && search[0] == 'l' ? 0 : ctx->vb_search_choice.pick(count);
    ctx->stats.vb_search = ctx->vb_variant;
    if (ctx->vb_variant == 1)
        launch_vb_ijkl(P, s);
    else
    {
        if (!ensure(ctx, ctx->vb_rec, sizeof(float) * 24 * (size_t)(count > 0 ? count : 1)))
            return VOX_ERR_MEMORY;
        P.rec = (float*)ctx->vb_rec.p;
        launch_vb_search(P, ctx->num_sms, s);
    }
    cudaEventRecord(ctx->timers.ev[1], s);
    int rc = check_cuda(ctx, "vox_voxelbvh_ijkl_from_gaussians");
    if (rc == VOX_OK)
        rc = sync_scalars(ctx, "vox_voxelbvh_ijkl_from_gaussians");
    if (rc == VOX_ERR_RANGE)
        set_error(ctx, "vox_voxelbvh_ijkl_from_gaussians: a Gaussian's box is not finite or maps outside "
                       "[-65536, 65536] voxels (a zero-size world box)");
    if (rc != VOX_OK)
        return rc;

    // Sort key: the emitted cells' coordinate range sizes a compressed key
    // (4 level bits + the bits of i, j, k) in the same order as the 64-bit
    // key, which the radix sort then covers in fewer passes; with a cell
    // outside [0, 2^16) the 64-bit keys themselves are sorted (64 key bits,
    // radix_sort_key64 of VoxelBVH.cpp:1374-1378).  Only unused slots: already
    // in order.
    const int* mm = (const int*)(ctx->hscal + SC_BBOX);
    VbRangeParams R{};
    R.range = d_range;
    R.keys_out = d_ijkl;
    R.ids_out = d_prim_id;
    int key32 = 0, sort_bits = 0;
    int64_t n_sorted = N; // the slots the sort and the range kernels cover (the used ones when compacted)
    const void* sorted_keys = d_ijkl;
    const bool any_cell = mm[3] >= mm[0];
    // VOX_VB_SORT64=1 sorts the 64-bit keys even when they compress (testing)
    const char* force64 = getenv("VOX_VB_SORT64");
    const bool compress = any_cell && mm[0] >= 0 && mm[1] >= 0 && mm[2] >= 0 && mm[3] < 65536 && mm[4] < 65536 &&
                          mm[5] < 65536 && !(force64 && force64[0] == '1');
    cudaEventRecord(ctx->timers.ev[2], s);
    if (N > 1 && any_cell)
    {
        uint64_t* alt_k = (uint64_t*)ctx->prim_keys_alt.p;
        uint32_t* alt_v = (uint32_t*)ctx->prim_vals_alt.p;
        int in_alt = 0;
        if (compress)
        {
            for (int a = 0; a < 3; a++)
                R.bits[a] = bit_length(mm[3 + a]);
            sort_bits = 4 + R.bits[0] + R.bits[1] + R.bits[2];
            key32 = sort_bits <= 32;
            R.sentinel = sort_bits >= 64 ? ~0ull : (1ull << sort_bits) - 1;
            R.expand = 1;
            // only the used slots are sorted: per-Gaussian counts, their scan (the total U
            // read back to size the sort), then the compressed keys and ids compacted
            if (!ensure(ctx, ctx->vb_ids_c, 4 * (size_t)N) || !ensure(ctx, ctx->vb_used, 8 * (size_t)(count + 1)))
                return VOX_ERR_MEMORY;
            uint32_t* used = (uint32_t*)ctx->vb_used.p;
            uint32_t* uoff = used + count + 1;
            uint32_t* ids_c = (uint32_t*)ctx->vb_ids_c.p;
            launch_vb_used(d_prim_id, count, used, s);
            uint64_t* status = (uint64_t*)ctx->scan_status.p;
            scan_u32(used, uoff, count, 0, 0, sc + SC_VBU, status,
                     ctx->scan_epochs.next(status, ctx->scan_status.cap / sizeof(uint64_t), s),
                     (uint32_t*)(sc + SC_SCRATCH), err, s);
            rc = sync_scalars(ctx, "vox_voxelbvh_ijkl_from_gaussians");
            if (rc != VOX_OK)
                return rc;
            n_sorted = (int64_t)ctx->hscal[SC_VBU];
            launch_vb_compress_used(d_ijkl, d_prim_id, count, used, uoff, R, ctx->vb_keys.p, ids_c, key32, ctx->num_sms,
                                    s);
            if (key32)
                in_alt = sort_pairs_u32((uint32_t*)ctx->vb_keys.p, ids_c, (uint32_t*)alt_k, alt_v, n_sorted, sort_bits,
                                        ctx->sort_ws.p, &ctx->sort_epochs, err, ctx->num_sms, s, ctx->tuning);
            else
                in_alt = sort_pairs_u64((uint64_t*)ctx->vb_keys.p, ids_c, alt_k, alt_v, n_sorted, sort_bits,
                                        ctx->sort_ws.p, &ctx->sort_epochs, err, ctx->num_sms, s, ctx->tuning);
            sorted_keys = in_alt ? (const void*)alt_k : (const void*)ctx->vb_keys.p;
            R.ids_src = in_alt ? alt_v : ids_c;
        }
        else
        {
            sort_bits = 64;
            in_alt = sort_pairs_u64(d_ijkl, d_prim_id, alt_k, alt_v, N, 64, ctx->sort_ws.p, &ctx->sort_epochs, err,
                                    ctx->num_sms, s, ctx->tuning);
            if (in_alt)
                cudaMemcpyAsync(d_ijkl, alt_k, 8 * (size_t)N, cudaMemcpyDeviceToDevice, s);
        }
        if (in_alt && !compress)
            R.ids_src = alt_v;
    }
    cudaEventRecord(ctx->timers.ev[3], s);
    if (n_sorted > 0)
    {
        const int64_t rtiles = vb_range_tiles(n_sorted);
        launch_vb_range_count(sorted_keys, key32, n_sorted, tile_cnt, s);
        uint64_t* status = (uint64_t*)ctx->scan_status.p;
        scan_exclusive_u64(tile_cnt, tile_off, rtiles, 0, d_total, status,
                           ctx->scan_epochs.next(status, ctx->scan_status.cap / sizeof(uint64_t), s),
                           (uint32_t*)(sc + SC_SCRATCH), err, ctx->num_sms, s);
        launch_vb_range_scatter(sorted_keys, key32, n_sorted, tile_off, d_total, R, s);
        if (n_sorted < N) // compacted: the unused run [U, N) is the last range
            launch_vb_tail(n_sorted, N, d_total, sc + SC_F, R, ctx->num_sms, s);
        else
            cudaMemcpyAsync(sc + SC_F, d_total, sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
    }
    cudaEventRecord(ctx->timers.ev[4], s);
    rc = check_cuda(ctx, "vox_voxelbvh_ijkl_from_gaussians");
    if (rc != VOX_OK)
        return rc;
    rc = sync_scalars(ctx, "vox_voxelbvh_ijkl_from_gaussians");
    if (rc != VOX_OK)
        return rc;
    if (range_count)
        *range_count = (int64_t)ctx->hscal[SC_F];
    auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    };
    vox_stats_t& st = ctx->stats;
    st.ms_vb_keys = elapsed(ctx->timers.ev[0], ctx->timers.ev[1]);
    if (!search)
        ctx->vb_search_choice.report(count, ctx->vb_variant, st.ms_vb_keys);
    st.ms_vb_sort = elapsed(ctx->timers.ev[2], ctx->timers.ev[3]);
    st.ms_vb_ranges = elapsed(ctx->timers.ev[3], ctx->timers.ev[4]);
    st.vb_sort_bits = sort_bits;
    st.vb_launches = launch_count() - launches0;
    return VOX_OK;
}

} // extern "C"
