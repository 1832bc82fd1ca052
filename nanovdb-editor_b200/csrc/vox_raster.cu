// vox_raster.cu - per-Gaussian records, rank tables, run detection and the
// node2 tree of the Gaussian -> node2 voxelization.
//
// Reference path (raster/Raster.cpp:420-558): two passes of fragment windows,
// each re-running gaussian_prim / fanout / gaussian_frag_{alloc,color} and an
// incremental 4-level tree build with atomics.  Here:
//   k_prep        one record per Gaussian (bbox, inverse rotation, alpha
//                 constants), footprint, touched root tiles
//   k_mark_lower  touched lower-node cells (128^3 voxels) per Gaussian bbox
//   [vox_leaf.cu] (leaf, Gaussian) pairs, sort, one CTA per candidate leaf:
//                 value masks, RGBA8, float sums; active voxel keys
//   k_runs        unique-key runs of the sorted voxel keys -> voxels, leaves,
//                 lower nodes
//   k_lower_info / k_upper_info / k_leaf_info / k_cloud_*   node tables and
//                 per-cloud layout
//   k_write_*     node2 nodes, per-cloud headers, written exactly
#include <cstdio>
#include <cuda_runtime.h>

#include "pnanovdb_b200.h"
#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

// ------------------------------------------------------------------ prep ----
__global__ void __launch_bounds__(256) k_prep(PrepParams P, GaussRec* recs, uint64_t* footprints,
                                              unsigned long long* root_bits, int* err)
{
    const int64_t g = P.g0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (P.g1 < 0 ? P.count : P.g1))
        return;
    GaussRec R;
    int32_t bmax[3];
    uint32_t cloud = 0;
    if (P.cloud_start)
    {
        // last cloud whose start is <= g
        int64_t lo = 0, hi = P.clouds;
        while (lo < hi)
        {
            int64_t mid = (lo + hi) >> 1;
            if (P.cloud_start[mid] <= g)
                lo = mid + 1;
            else
                hi = mid;
        }
        cloud = (uint32_t)(lo - 1);
    }
    const float vs = P.cloud_vs ? P.cloud_vs[cloud] : P.voxel_size;
    uint64_t fp = make_record(P, g, vs, R, bmax);
    R.q5.w = (int32_t)cloud;
    if (fp)
    {
        int e = 0;
        for (int a = 0; a < 3; a++)
        {
            int32_t lo = (&R.q4.x)[a];
            if (lo < -65536 || bmax[a] > 65535)
                e |= ERR_RANGE;
        }
        if (fp >= (1ull << 31))
            e |= ERR_FOOTPRINT;
        if (e)
        {
            atomicOr(err, e);
            fp = 0;
            R.q4.w = 0;
        }
    }
    recs[g] = R;
    footprints[g] = fp;
    if (fp)
    {
        // root tiles (4096^3 voxels) spanned by the bbox
        for (int32_t x = R.q4.x >> 12; x <= (bmax[0] >> 12); x++)
            for (int32_t y = R.q4.y >> 12; y <= (bmax[1] >> 12); y++)
                for (int32_t z = R.q4.z >> 12; z <= (bmax[2] >> 12); z++)
                {
                    const uint64_t rn = root_index(cloud, x << 12, y << 12, z << 12);
                    atomicOr(&root_bits[rn >> 6], 1ull << (rn & 63));
                }
    }
}

__global__ void __launch_bounds__(256) k_mark_lower(const GaussRec* recs, int64_t G, const uint64_t* root_bits,
                                                    const uint64_t* root_prefix, unsigned long long* lower_bits)
{
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G)
        return;
    GaussRec R = recs[g];
    if (!R.q4.w)
        return;
    int32_t mn[3] = { R.q4.x, R.q4.y, R.q4.z };
    int32_t mx[3] = { R.q4.x + R.q5.x - 1, R.q4.y + R.q5.y - 1, R.q4.z + R.q5.z - 1 };
    for (int32_t x = mn[0] >> 7; x <= (mx[0] >> 7); x++)
        for (int32_t y = mn[1] >> 7; y <= (mx[1] >> 7); y++)
            for (int32_t z = mn[2] >> 7; z <= (mx[2] >> 7); z++)
            {
                int32_t cx = x << 7, cy = y << 7, cz = z << 7;
                uint64_t rr = bit_rank(root_bits, root_prefix, root_index(rec_cloud(R), cx, cy, cz));
                uint64_t cell = rr * 32768ull + upper_n_of(cx, cy, cz);
                atomicOr(&lower_bits[cell >> 6], 1ull << (cell & 63));
            }
}

// inverse tables: rank -> root_n, rank -> cell
__global__ void k_invert_bits(const uint64_t* bits, const uint64_t* prefix, int64_t words, uint32_t* out)
{
    int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words)
        return;
    uint64_t b = bits[w];
    uint64_t r = prefix[w];
    while (b)
    {
        int bit = __ffsll((long long)b) - 1;
        out[r++] = (uint32_t)(w * 64 + bit);
        b &= b - 1;
    }
}

// ------------------------------------------------------------------ runs ----
// Unique-key run detection over the sorted keys.  Warp-contiguous loads
// (element = warp chunk + item * 32 + lane), heads found against the
// previous key (shuffle across lanes, carried across items), counted with
// ballots, three exclusive counts (voxels, leaves, lower nodes) across the
// tile and across tiles with a decoupled look-back.
constexpr int RUN_BLOCK = 256;
constexpr int RUN_ITEMS = 16;
constexpr int RUN_WARPS = RUN_BLOCK / 32;
constexpr int RUN_TILE = RUN_BLOCK * RUN_ITEMS;

template <class K>
__global__ void __launch_bounds__(RUN_BLOCK) k_runs(RunParams Rp, const K* __restrict__ keys)
{
    __shared__ uint32_t s_wtot[3][RUN_WARPS];
    __shared__ uint64_t s_ex[3];
    __shared__ uint32_t s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0)
        s_tile = atomicAdd(Rp.counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const int64_t P = Rp.P;
    const int64_t wbase = (int64_t)tile * RUN_TILE + (int64_t)warp * (32 * RUN_ITEMS);
    K k[RUN_ITEMS];
    uint32_t bv[RUN_ITEMS], bl[RUN_ITEMS], blo[RUN_ITEMS];
    K carry = (wbase > 0 && wbase - 1 < P) ? keys[wbase - 1] : (K)0;
    uint32_t tv = 0, tl = 0, tlo = 0;
#pragma unroll
    for (int i = 0; i < RUN_ITEMS; i++)
    {
        const int64_t idx = wbase + i * 32 + lane;
        const bool valid = idx < P;
        k[i] = valid ? keys[idx] : (K)0;
        K prev = __shfl_up_sync(0xffffffffu, k[i], 1);
        if (lane == 0)
            prev = carry;
        carry = __shfl_sync(0xffffffffu, k[i], 31);
        const bool first = idx == 0;
        const bool hv = valid && (first || k[i] != prev);
        const bool hl = valid && (first || (k[i] >> 9) != (prev >> 9));
        const bool hlo = valid && (first || (k[i] >> 21) != (prev >> 21));
        bv[i] = __ballot_sync(0xffffffffu, hv);
        bl[i] = __ballot_sync(0xffffffffu, hl);
        blo[i] = __ballot_sync(0xffffffffu, hlo);
        tv += __popc(bv[i]);
        tl += __popc(bl[i]);
        tlo += __popc(blo[i]);
    }
    if (lane == 0)
    {
        s_wtot[0][warp] = tv;
        s_wtot[1][warp] = tl;
        s_wtot[2][warp] = tlo;
    }
    __syncthreads();
    if (threadIdx.x < 3)
    {
        uint64_t agg = 0;
        for (int w = 0; w < RUN_WARPS; w++)
            agg += s_wtot[threadIdx.x][w];
        s_ex[threadIdx.x] = lookback_exclusive(Rp.status + threadIdx.x, tile, agg, Rp.epoch, Rp.err, 3);
    }
    __syncthreads();
    uint64_t v = s_ex[0], l = s_ex[1], lo = s_ex[2];
    for (int w = 0; w < warp; w++)
    {
        v += s_wtot[0][w];
        l += s_wtot[1][w];
        lo += s_wtot[2][w];
    }
    const uint32_t le = (lane == 31) ? 0xffffffffu : ((1u << (lane + 1)) - 1u);
#pragma unroll
    for (int i = 0; i < RUN_ITEMS; i++)
    {
        const int64_t idx = wbase + i * 32 + lane;
        // inclusive counts at this element: heads up to and including it
        const uint64_t vi = v + __popc(bv[i] & le), li = l + __popc(bl[i] & le), loi = lo + __popc(blo[i] & le);
        if ((blo[i] >> lane) & 1u)
        {
            // distinct lower ranks never exceed the touched-cell count; more
            // heads mean the keys are not sorted: report, never write past it
            if (loi < Rp.lower_cap)
            {
                Rp.lower_lstart[loi - 1] = (uint32_t)(li - 1);
                Rp.lower_rank[loi - 1] = (uint32_t)((uint64_t)k[i] >> 21);
            }
            else
                atomicOr(Rp.err, ERR_ORDER);
        }
        if ((bl[i] >> lane) & 1u)
            Rp.leaf_vstart[li - 1] = (uint32_t)(vi - 1);
        if ((bv[i] >> lane) & 1u)
        {
            Rp.vox_start[vi - 1] = (uint32_t)idx;
            Rp.vox_leaf[vi - 1] = (uint32_t)(li - 1);
            Rp.vox_n[vi - 1] = (uint16_t)((uint32_t)k[i] & 511u);
        }
        if (idx == P - 1)
        {
            Rp.vox_start[vi] = (uint32_t)P;
            Rp.leaf_vstart[li] = (uint32_t)vi;
            if (loi < Rp.lower_cap)
                Rp.lower_lstart[loi] = (uint32_t)li;
            Rp.counts[0] = vi;
            Rp.counts[1] = li;
            Rp.counts[2] = loi;
        }
        v += __popc(bv[i]);
        l += __popc(bl[i]);
        lo += __popc(blo[i]);
    }
}

// ------------------------------------------------------------- node tables ----

// per lower node: origin, parent upper; per upper: root_n, lower range
__global__ void k_lower_info(NodeParams N)
{
    int64_t lo = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lo >= N.Lo)
        return;
    uint32_t cell = N.lower_cell[N.lower_rank[lo]];
    uint32_t rr = cell >> 15, un = cell & 32767u;
    uint32_t rn = N.root_of_rank[rr];
    int32_t o[3];
    root_tile_origin(rn, o);
    o[0] += (int32_t)((un >> 10) & 31) * 128;
    o[1] += (int32_t)((un >> 5) & 31) * 128;
    o[2] += (int32_t)(un & 31) * 128;
    N.lower_origin[3 * lo + 0] = o[0];
    N.lower_origin[3 * lo + 1] = o[1];
    N.lower_origin[3 * lo + 2] = o[2];
    N.lower_upper_n[lo] = un;
    N.rank_to_lower[N.lower_rank[lo]] = (uint32_t)lo;
    bool head = lo == 0 || (N.lower_cell[N.lower_rank[lo - 1]] >> 15) != rr;
    N.upper_head[lo] = head ? 1ull : 0ull;
}

__global__ void k_upper_info(NodeParams N)
{
    int64_t lo = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lo >= N.Lo)
        return;
    const bool head = N.upper_head[lo] != 0ull;
    const uint64_t u = N.upper_scan[lo] + (head ? 1ull : 0ull) - 1ull; // heads in [0, lo] minus one
    if (head)
    {
        uint32_t cell = N.lower_cell[N.lower_rank[lo]];
        N.upper_root_n[u] = N.root_of_rank[cell >> 15];
        N.upper_lostart[u] = (uint32_t)lo;
    }
    N.lower_parent[lo] = (uint32_t)u;
    if (lo == N.Lo - 1)
    {
        N.upper_lostart[u + 1] = (uint32_t)N.Lo;
        *N.upper_count = u + 1;
    }
}

// ---------------------------------------------------------------- clouds ----
__device__ __forceinline__ uint32_t upper_cloud(const NodeParams& N, uint64_t u)
{
    return N.upper_root_n[u] >> 15;
}
__device__ __forceinline__ uint32_t lower_cloud(const NodeParams& N, uint64_t lo)
{
    return N.upper_root_n[N.lower_parent[lo]] >> 15;
}

// fills start[b] for clouds (prev, cur] with i; the last element closes the table
__device__ __forceinline__ void fill_starts(uint32_t* start, int64_t i, int64_t n, int64_t prev, int64_t cur, int64_t B)
{
    for (int64_t b = prev + 1; b <= cur; b++)
        start[b] = (uint32_t)i;
    if (i == n - 1)
        for (int64_t b = cur + 1; b <= B; b++)
            start[b] = (uint32_t)n;
}

// first upper / lower / leaf of every cloud (nodes are ordered by cloud first);
// the upper count is read on the device
__global__ void k_cloud_starts(NodeParams N)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t U = (int64_t)*N.upper_count, B = N.C.B;
    if (t < U)
        fill_starts(N.C.upper_start, t, U, t ? (int64_t)upper_cloud(N, t - 1) : -1, upper_cloud(N, t), B);
    if (t < N.Lo)
        fill_starts(N.C.lower_start, t, N.Lo, t ? (int64_t)lower_cloud(N, t - 1) : -1, lower_cloud(N, t), B);
    if (t < N.L)
    {
        const uint32_t c = lower_cloud(N, N.leaf_lower[t]);
        N.C.leaf_cloud[t] = c;
        fill_starts(N.C.leaf_start, t, N.L, t ? (int64_t)lower_cloud(N, N.leaf_lower[t - 1]) : -1, c, B);
    }
}

__device__ __forceinline__ uint64_t al256(uint64_t x)
{
    return (x + 255) / 256 * 256;
}

// one CTA: per-cloud node counts -> grid layout, grid offsets and value bases
// (exclusive scans over the clouds, 1024 at a time)
__global__ void __launch_bounds__(1024) k_cloud_layout(NodeParams N)
{
    __shared__ uint64_t s_warp[33];
    __shared__ uint64_t s_carry[2];
    const CloudParams& C = N.C;
    if (threadIdx.x == 0)
        s_carry[0] = s_carry[1] = 0;
    __syncthreads();
    for (int64_t c0 = 0; c0 < C.B; c0 += blockDim.x)
    {
        const int64_t b = c0 + threadIdx.x;
        uint64_t size = 0, vc = 0;
        uint64_t node2 = 0, o_bbox = 0, o_rgba = 0, o_dens = 0, o_col = 0;
        if (b < C.B)
        {
            const uint64_t U = C.upper_start[b + 1] - C.upper_start[b];
            const uint64_t Lo = C.lower_start[b + 1] - C.lower_start[b];
            const uint64_t L = C.leaf_start[b + 1] - C.leaf_start[b];
            const uint64_t v0 = C.leaf_start[b] < (uint64_t)N.L ? N.leaf_vstart[C.leaf_start[b]] : (uint64_t)C.V;
            C.vstart[b] = v0;
            if (b == C.B - 1)
                C.vstart[C.B] = (uint64_t)C.V;
            const uint64_t v1 = C.leaf_start[b + 1] < (uint64_t)N.L ? N.leaf_vstart[C.leaf_start[b + 1]] : (uint64_t)C.V;
            vc = 2 + (v1 - v0);
            node2 = n2_node_bytes(0) + U * n2_node_bytes(1) + Lo * n2_node_bytes(2) + L * n2_node_bytes(3);
            o_bbox = al256(VOX_GRID_HEADER_BYTES + node2);
            o_rgba = al256(o_bbox + 32);
            o_dens = al256(o_rgba + 4 * vc);
            o_col = al256(o_dens + 4 * vc);
            size = al256(o_col + 12 * vc);
            for (int a = 0; a < 6; a++)
                C.bbox[6 * b + a] = a < 3 ? 0x7FFFFFFF : (int32_t)0x80000000;
        }
        uint64_t tot_size, tot_vc;
        const uint64_t ex_size = block_excl_scan_u64(size, s_warp, tot_size);
        const uint64_t ex_vc = block_excl_scan_u64(vc, s_warp, tot_vc);
        if (b < C.B)
        {
            const uint64_t g = s_carry[0] + ex_size;
            C.grid_off[b] = g;
            C.value_base[b] = s_carry[1] + ex_vc;
            C.node2_bytes[b] = node2;
            C.bbox_off[b] = g + o_bbox;
            C.rgba_off[b] = g + o_rgba;
            C.dens_off[b] = g + o_dens;
            C.col_off[b] = g + o_col;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            s_carry[0] += tot_size;
            s_carry[1] += tot_vc;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        C.grid_off[C.B] = s_carry[0];
        C.value_base[C.B] = s_carry[1];
    }
}

// canonical (single fragment window) node order inside every cloud's grid:
// uppers, lowers, leaves, each in hierarchical key order; node addresses
// (absolute in the output buffer) follow node_idx order
__global__ void k_canonical_order(NodeParams N, uint64_t U)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t root_sz = n2_node_bytes(0), up_sz = n2_node_bytes(1), lo_sz = n2_node_bytes(2),
                   lf_sz = n2_node_bytes(3);
    const CloudParams& C = N.C;
    if (t < (int64_t)U)
    {
        const uint32_t b = upper_cloud(N, t);
        const uint64_t local = (uint64_t)t - C.upper_start[b];
        N.upper_idx[t] = 1 + local;
        N.upper_addr[t] = C.grid_off[b] + VOX_GRID_HEADER_BYTES + root_sz + local * up_sz;
        N.upper_vidx[t] = 2;
    }
    if (t < N.Lo)
    {
        const uint32_t b = lower_cloud(N, t);
        const uint64_t Ub = C.upper_start[b + 1] - C.upper_start[b];
        const uint64_t local = (uint64_t)t - C.lower_start[b];
        N.lower_idx[t] = 1 + Ub + local;
        N.lower_addr[t] = C.grid_off[b] + VOX_GRID_HEADER_BYTES + root_sz + Ub * up_sz + local * lo_sz;
        N.lower_vidx[t] = 2;
    }
    if (t < N.L)
    {
        const uint32_t b = C.leaf_cloud[t];
        const uint64_t Ub = C.upper_start[b + 1] - C.upper_start[b];
        const uint64_t Lob = C.lower_start[b + 1] - C.lower_start[b];
        const uint64_t local = (uint64_t)t - C.leaf_start[b];
        N.leaf_idx[t] = 1 + Ub + Lob + local;
        N.leaf_addr[t] = C.grid_off[b] + VOX_GRID_HEADER_BYTES + root_sz + Ub * up_sz + Lob * lo_sz + local * lf_sz;
        N.leaf_vidx[t] = 2 + ((uint64_t)N.leaf_vstart[t] - C.vstart[b]);
    }
}

// per cloud: the grid header (vox_grid_header_t) and the bbox blind data
__global__ void k_write_headers(NodeParams N, uint8_t* out)
{
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const CloudParams& C = N.C;
    if (b >= C.B)
        return;
    const uint64_t g = C.grid_off[b];
    vox_grid_header_t h;
    memset(&h, 0, sizeof(h));
    const uint64_t vc = 2 + (C.vstart[b + 1] - C.vstart[b]);
    h.magic = VOX_GRID_MAGIC;
    h.version = 1;
    h.header_bytes = VOX_GRID_HEADER_BYTES;
    h.grid_bytes = C.grid_off[b + 1] - g;
    h.node2_offset = VOX_GRID_HEADER_BYTES;
    h.node2_bytes = C.node2_bytes[b];
    h.upper_count = C.upper_start[b + 1] - C.upper_start[b];
    h.lower_count = C.lower_start[b + 1] - C.lower_start[b];
    h.leaf_count = C.leaf_start[b + 1] - C.leaf_start[b];
    h.node_order = C.node_order;
    h.value_count = vc;
    h.bbox_offset = C.bbox_off[b] - g;
    h.rgba8_offset = C.rgba_off[b] - g;
    h.density_offset = C.dens_off[b] - g;
    h.color_offset = C.col_off[b] - g;
    h.voxel_size = C.cloud_vs ? C.cloud_vs[b] : C.voxel_size;
    if (vc > 2)
        for (int a = 0; a < 6; a++)
            h.bbox[a] = C.bbox[6 * b + a];
    h.pair_count = C.cloud_pairs ? C.cloud_pairs[b] : (uint64_t)C.P;
    const int64_t g0 = C.cloud_start ? C.cloud_start[b] : 0, g1 = C.cloud_start ? C.cloud_start[b + 1] : C.G;
    const uint64_t f0 = g0 < C.G ? C.frag_off[g0] : *C.F_total, f1 = g1 < C.G ? C.frag_off[g1] : *C.F_total;
    h.candidate_count = f1 - f0;
    const uint32_t* src = (const uint32_t*)&h;
    uint32_t* dst = (uint32_t*)(out + g);
    for (int w = 0; w < (int)(sizeof(h) / 4); w++)
        dst[w] = src[w];
    int32_t* bb = (int32_t*)(out + C.bbox_off[b]);
    for (int a = 0; a < 6; a++)
        bb[a] = h.bbox[a];
}

// per leaf: lower_n in its parent and origin
template <class K>
__global__ void __launch_bounds__(256) k_leaf_info(NodeParams N, const K* __restrict__ keys)
{
    int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= N.L)
        return;
    const K key0 = keys[N.vox_start[N.leaf_vstart[l]]];
    const uint32_t ln = (uint32_t)((uint64_t)key0 >> 9) & 4095u;
    const uint32_t lo = N.leaf_lower[l];
    N.leaf_lower_n[l] = ln;
    N.leaf_origin[3 * l + 0] = N.lower_origin[3 * lo + 0] + (int32_t)((ln >> 8) & 15) * 8;
    N.leaf_origin[3 * l + 1] = N.lower_origin[3 * lo + 1] + (int32_t)((ln >> 4) & 15) * 8;
    N.leaf_origin[3 * l + 2] = N.lower_origin[3 * lo + 2] + (int32_t)(ln & 15) * 8;
}

// bbox of the active voxels from the leaf masks (grid_build_compute_bbox.slang)
__global__ void __launch_bounds__(256) k_leaf_bbox(NodeParams N)
{
    __shared__ int32_t s_bb[6];
    if (threadIdx.x < 6)
        s_bb[threadIdx.x] = threadIdx.x < 3 ? 0x7FFFFFFF : (int32_t)0x80000000;
    __syncthreads();
    const int64_t l0 = (int64_t)blockIdx.x * blockDim.x;
    const int64_t lz = min((int64_t)N.L, l0 + (int64_t)blockDim.x) - 1;
    // leaves of one cloud reduce in shared memory; a CTA spanning clouds goes to global per leaf
    const uint32_t cb = N.C.leaf_cloud[l0];
    const bool one_cloud = N.C.leaf_cloud[lz] == cb;
    int64_t l = l0 + threadIdx.x;
    if (l < N.L)
    {
        int32_t mn[3] = { 8, 8, 8 }, mx[3] = { -1, -1, -1 };
        for (int w = 0; w < 8; w++)
        {
            uint64_t m = N.leaf_mask[8 * l + w];
            while (m)
            {
                int n = w * 64 + __ffsll((long long)m) - 1;
                m &= m - 1;
                int32_t c[3] = { n >> 6, (n >> 3) & 7, n & 7 };
                for (int a = 0; a < 3; a++)
                {
                    mn[a] = min(mn[a], c[a]);
                    mx[a] = max(mx[a], c[a]);
                }
            }
        }
        int32_t* bb = one_cloud ? s_bb : N.C.bbox + 6 * (uint64_t)N.C.leaf_cloud[l];
        for (int a = 0; a < 3; a++)
        {
            atomicMin(&bb[a], N.leaf_origin[3 * l + a] + mn[a]);
            atomicMax(&bb[3 + a], N.leaf_origin[3 * l + a] + mx[a]);
        }
    }
    __syncthreads();
    if (one_cloud)
    {
        if (threadIdx.x < 3)
            atomicMin(&N.C.bbox[6 * (uint64_t)cb + threadIdx.x], s_bb[threadIdx.x]);
        else if (threadIdx.x < 6)
            atomicMax(&N.C.bbox[6 * (uint64_t)cb + threadIdx.x], s_bb[threadIdx.x]);
    }
}

// leaf -> lower index (leaves of lower lo are [lower_lstart[lo], lower_lstart[lo+1]))
__global__ void k_leaf_lower(NodeParams N)
{
    int64_t lo = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lo >= N.Lo)
        return;
    for (uint32_t l = N.lower_lstart[lo]; l < N.lower_lstart[lo + 1]; l++)
        N.leaf_lower[l] = (uint32_t)lo;
}

// ------------------------------------------------------------ node2 write ----
// prefix words of a mask (grid_build_count_new.slang:49-88): field (w & 3) of
// word (w >> 2) = popcount(mask[0 .. w-1]); field 0 of word 0 = total.
// One CTA, mask of nw words in shared memory.
__device__ void write_prefix_block(uint64_t* dst, const uint64_t* s_mask, uint32_t nw, uint32_t* s_scan)
{
    // exclusive scan of popcounts into s_scan[0..nw], serial per 32-word chunk
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x)
        s_scan[w] = __popcll(s_mask[w]);
    __syncthreads();
    if (threadIdx.x == 0)
    {
        uint32_t run = 0;
        for (uint32_t w = 0; w < nw; w++)
        {
            uint32_t c = s_scan[w];
            s_scan[w] = run;
            run += c;
        }
        s_scan[nw] = run;
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < nw / 4; q += blockDim.x)
    {
        uint64_t word = 0;
        for (uint32_t f = 0; f < 4; f++)
        {
            uint32_t w = 4 * q + f;
            uint32_t v = (w == 0) ? s_scan[nw] : s_scan[w];
            word |= ((uint64_t)(v & 0xFFFFu)) << (16 * f);
        }
        dst[q] = word;
    }
    __syncthreads();
}

// one CTA per cloud: the root of that cloud's grid
__global__ void __launch_bounds__(1024) k_write_root(NodeParams N, uint8_t* out)
{
    __shared__ uint64_t s_mask[512];
    __shared__ uint32_t s_scan[513];
    const uint64_t b = blockIdx.x;
    const uint64_t root_addr = N.C.grid_off[b] + VOX_GRID_HEADER_BYTES;
    uint64_t* W = (uint64_t*)(out + root_addr);
    const uint32_t u0 = N.C.upper_start[b];
    const uint64_t U = N.C.upper_start[b + 1] - u0;
    for (int i = threadIdx.x; i < 512; i += blockDim.x)
        s_mask[i] = 0;
    __syncthreads();
    for (uint64_t u = threadIdx.x; u < U; u += blockDim.x)
    {
        uint32_t rn = N.upper_root_n[u0 + u] & 32767u;
        atomicOr((unsigned long long*)&s_mask[rn >> 6], 1ull << (rn & 63));
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        W[N2_OFF_NODE_IDX] = 0;
        W[N2_OFF_VALUE_IDX] = 2;
    }
    for (int i = threadIdx.x; i < 512; i += blockDim.x)
    {
        W[n2_off_child_mask(0) + i] = s_mask[i];
        W[N2_OFF_KEY_MASK_ROOT + i] = s_mask[i];
    }
    write_prefix_block(W + n2_off_child_prefix(0), s_mask, 512, s_scan);
    write_prefix_block(W + N2_OFF_KEY_PREFIX_ROOT, s_mask, 512, s_scan);
    uint64_t* ch = W + n2_off_children(0);
    for (uint32_t e = threadIdx.x; e < 65536u; e += blockDim.x)
    {
        uint64_t val = N2_END_KEY;
        if (e < U)
            val = N.upper_addr[u0 + e] - root_addr;
        else if (e < 2 * U)
        {
            uint32_t rn = N.upper_root_n[u0 + e - U] & 32767u;
            int32_t x = (int32_t)(((rn >> 10) & 31) << 12), y = (int32_t)(((rn >> 5) & 31) << 12),
                    z = (int32_t)((rn & 31) << 12);
            x = x >= 65536 ? x - 131072 : x;
            y = y >= 65536 ? y - 131072 : y;
            z = z >= 65536 ? z - 131072 : z;
            val = (uint64_t)((uint32_t)z >> 12) | ((uint64_t)((uint32_t)y >> 12) << 21) |
                  ((uint64_t)((uint32_t)x >> 12) << 42);
        }
        ch[e] = val;
    }
}

__global__ void __launch_bounds__(512) k_write_upper(NodeParams N, uint8_t* node2)
{
    __shared__ uint64_t s_mask[512];
    __shared__ uint32_t s_scan[513];
    const uint64_t u = blockIdx.x;
    uint64_t* W = (uint64_t*)(node2 + N.upper_addr[u]);
    for (int i = threadIdx.x; i < 512; i += blockDim.x)
        s_mask[i] = 0;
    __syncthreads();
    const uint32_t lo0 = N.upper_lostart[u], lo1 = N.upper_lostart[u + 1];
    for (uint32_t lo = lo0 + threadIdx.x; lo < lo1; lo += blockDim.x)
    {
        uint32_t un = N.lower_upper_n[lo];
        atomicOr((unsigned long long*)&s_mask[un >> 6], 1ull << (un & 63));
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        W[N2_OFF_NODE_IDX] = N.upper_idx[u];
        W[N2_OFF_VALUE_IDX] = N.upper_vidx[u];
    }
    for (int i = threadIdx.x; i < 512; i += blockDim.x)
        W[n2_off_child_mask(1) + i] = s_mask[i];
    write_prefix_block(W + n2_off_child_prefix(1), s_mask, 512, s_scan);
    uint64_t* ch = W + n2_off_children(1);
    for (uint32_t lo = lo0 + threadIdx.x; lo < lo1; lo += blockDim.x)
        ch[lo - lo0] = N.lower_addr[lo] - N.upper_addr[u];
}

__global__ void __launch_bounds__(256) k_write_lower(NodeParams N, uint8_t* node2)
{
    __shared__ uint64_t s_mask[64];
    __shared__ uint32_t s_scan[65];
    const uint64_t lo = blockIdx.x;
    uint64_t* W = (uint64_t*)(node2 + N.lower_addr[lo]);
    for (int i = threadIdx.x; i < 64; i += blockDim.x)
        s_mask[i] = 0;
    __syncthreads();
    const uint32_t l0 = N.lower_lstart[lo], l1 = N.lower_lstart[lo + 1];
    for (uint32_t l = l0 + threadIdx.x; l < l1; l += blockDim.x)
    {
        uint32_t ln = N.leaf_lower_n[l];
        atomicOr((unsigned long long*)&s_mask[ln >> 6], 1ull << (ln & 63));
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        W[N2_OFF_NODE_IDX] = N.lower_idx[lo];
        W[N2_OFF_VALUE_IDX] = N.lower_vidx[lo];
    }
    for (int i = threadIdx.x; i < 64; i += blockDim.x)
        W[n2_off_child_mask(2) + i] = s_mask[i];
    write_prefix_block(W + n2_off_child_prefix(2), s_mask, 64, s_scan);
    uint64_t* ch = W + n2_off_children(2);
    for (uint32_t l = l0 + threadIdx.x; l < l1; l += blockDim.x)
        ch[l - l0] = N.leaf_addr[l] - N.lower_addr[lo];
}

// one leaf per 16 lanes, one 64-bit word per lane (128 B per leaf)
__global__ void __launch_bounds__(256) k_write_leaf(NodeParams N, uint8_t* node2)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t l = t >> 4;
    int w = (int)(t & 15);
    if (l >= N.L)
        return;
    const uint64_t* m = N.leaf_mask + 8 * l;
    uint64_t val = 0;
    if (w == 0)
        val = N.leaf_idx[l];
    else if (w == 1)
        val = N.leaf_vidx[l];
    else if (w == 6 || w == 7)
    {
        // prefix fields for mask words 4(w-6) .. 4(w-6)+3
        uint32_t c[9];
        c[0] = 0;
        for (int q = 0; q < 8; q++)
            c[q + 1] = c[q] + __popcll(m[q]);
        for (int f = 0; f < 4; f++)
        {
            int mw = 4 * (w - 6) + f;
            uint32_t v = mw == 0 ? c[8] : c[mw];
            val |= ((uint64_t)(v & 0xFFFFu)) << (16 * f);
        }
    }
    else if (w >= 8)
        val = m[w - 8];
    ((uint64_t*)(node2 + N.leaf_addr[l]))[w] = val;
}

// =================================================================== launch
void launch_prep(const PrepParams& P, GaussRec* recs, uint64_t* footprints, uint64_t* root_bits, int* err,
                 cudaStream_t s)
{
    const int64_t n = (P.g1 < 0 ? P.count : P.g1) - P.g0;
    if (n <= 0)
        return;
    { k_prep<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, recs, footprints, (unsigned long long*)root_bits, err); count_launch(); }
}

void launch_mark_lower(const GaussRec* recs, int64_t G, const uint64_t* root_bits, const uint64_t* root_prefix,
                       uint64_t* lower_bits, cudaStream_t s)
{
    if (G <= 0)
        return;
    { k_mark_lower<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(recs, G, root_bits, root_prefix,
                                                           (unsigned long long*)lower_bits); count_launch(); }
}

void launch_invert_bits(const uint64_t* bits, const uint64_t* prefix, int64_t words, uint32_t* out, cudaStream_t s)
{
    if (words <= 0)
        return;
    { k_invert_bits<<<(unsigned)((words + 255) / 256), 256, 0, s>>>(bits, prefix, words, out); count_launch(); }
}


void launch_runs(const RunParams& Rp, const void* keys, int key64, cudaStream_t s)
{
    if (Rp.P <= 0)
        return;
    cudaMemsetAsync(Rp.counter, 0, sizeof(uint32_t), s);
    int64_t tiles = (Rp.P + RUN_TILE - 1) / RUN_TILE;
    if (key64)
        { k_runs<uint64_t><<<(unsigned)tiles, RUN_BLOCK, 0, s>>>(Rp, (const uint64_t*)keys); count_launch(); }
    else
        { k_runs<uint32_t><<<(unsigned)tiles, RUN_BLOCK, 0, s>>>(Rp, (const uint32_t*)keys); count_launch(); }
}
int64_t runs_tile_count(int64_t P)
{
    return (P + RUN_TILE - 1) / RUN_TILE;
}

void launch_lower_info(const NodeParams& N, cudaStream_t s)
{
    if (N.Lo <= 0)
        return;
    { k_lower_info<<<(unsigned)((N.Lo + 255) / 256), 256, 0, s>>>(N); count_launch(); }
}
void launch_upper_info(const NodeParams& N, cudaStream_t s)
{
    if (N.Lo <= 0)
        return;
    { k_upper_info<<<(unsigned)((N.Lo + 255) / 256), 256, 0, s>>>(N); count_launch(); }
}
void launch_leaf_tables(const NodeParams& N, const void* keys, int key64, cudaStream_t s)
{
    if (N.L <= 0)
        return;
    { k_leaf_lower<<<(unsigned)((N.Lo + 255) / 256), 256, 0, s>>>(N); count_launch(); }
    unsigned blocks = (unsigned)((N.L + 255) / 256);
    if (key64)
        { k_leaf_info<uint64_t><<<blocks, 256, 0, s>>>(N, (const uint64_t*)keys); count_launch(); }
    else
        { k_leaf_info<uint32_t><<<blocks, 256, 0, s>>>(N, (const uint32_t*)keys); count_launch(); }
}
void launch_leaf_bbox(const NodeParams& N, cudaStream_t s)
{
    if (N.L <= 0)
        return;
    { k_leaf_bbox<<<(unsigned)((N.L + 255) / 256), 256, 0, s>>>(N); count_launch(); }
}
void launch_canonical_order(const NodeParams& N, uint64_t U, cudaStream_t s)
{
    int64_t m = N.L;
    if ((int64_t)U > m)
        m = (int64_t)U;
    if (N.Lo > m)
        m = N.Lo;
    if (m <= 0)
        return;
    { k_canonical_order<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(N, U); count_launch(); }
}
void launch_write_nodes(const NodeParams& N, uint64_t U, uint8_t* out, cudaStream_t s)
{
    { k_write_root<<<(unsigned)N.C.B, 1024, 0, s>>>(N, out); count_launch(); }
    if (U)
        { k_write_upper<<<(unsigned)U, 512, 0, s>>>(N, out); count_launch(); }
    if (N.Lo)
        { k_write_lower<<<(unsigned)N.Lo, 256, 0, s>>>(N, out); count_launch(); }
    if (N.L)
        { k_write_leaf<<<(unsigned)((N.L * 16 + 255) / 256), 256, 0, s>>>(N, out); count_launch(); }
}
void launch_cloud_layout(const NodeParams& N, cudaStream_t s)
{
    // U <= Lo, so Lo + L threads cover every level
    const int64_t n = N.Lo > N.L ? N.Lo : N.L;
    if (n > 0)
        { k_cloud_starts<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(N); count_launch(); }
    { k_cloud_layout<<<1, 1024, 0, s>>>(N); count_launch(); }
}
// Zero every byte of each cloud's grid that the node / value writers leave
// alone: header, node2 region, bbox, the two background values of each value
// array and the alignment gaps (the values 2 .. vc - 1 are all written).
__device__ __forceinline__ void zero_range(uint8_t* out, uint64_t a, uint64_t b, uint64_t i, uint64_t n)
{
    // a, b multiples of 4
    const uint64_t a16 = (a + 15) & ~15ull, b16 = b & ~15ull;
    if (a16 >= b16)
    {
        for (uint64_t o = a + 4 * i; o < b; o += 4 * n)
            *reinterpret_cast<uint32_t*>(out + o) = 0u;
        return;
    }
    for (uint64_t o = a + 4 * i; o < a16; o += 4 * n)
        *reinterpret_cast<uint32_t*>(out + o) = 0u;
    for (uint64_t o = a16 + 16 * i; o < b16; o += 16 * n)
        *reinterpret_cast<uint4*>(out + o) = make_uint4(0u, 0u, 0u, 0u);
    for (uint64_t o = b16 + 4 * i; o < b; o += 4 * n)
        *reinterpret_cast<uint32_t*>(out + o) = 0u;
}

__global__ void k_zero_gaps(NodeParams N, uint8_t* out)
{
    const CloudParams& C = N.C;
    const int64_t b = blockIdx.y;
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, n = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t vc = 2 + (C.vstart[b + 1] - C.vstart[b]);
    zero_range(out, C.grid_off[b], C.rgba_off[b] + 8, i, n);
    zero_range(out, C.rgba_off[b] + 4 * vc, C.dens_off[b] + 8, i, n);
    zero_range(out, C.dens_off[b] + 4 * vc, C.col_off[b] + 24, i, n);
    zero_range(out, C.col_off[b] + 12 * vc, C.grid_off[b + 1], i, n);
}

void launch_zero_gaps(const NodeParams& N, uint8_t* out, uint64_t grid_bytes, cudaStream_t s)
{
    if (N.C.B <= 0)
        return;
    uint64_t bx = grid_bytes / (uint64_t)N.C.B / (1ull << 19);
    bx = bx < 1 ? 1 : (bx > 1024 ? 1024 : bx);
    { k_zero_gaps<<<dim3((unsigned)bx, (unsigned)N.C.B), 256, 0, s>>>(N, out); count_launch(); }
}

void launch_write_headers(const NodeParams& N, uint8_t* out, cudaStream_t s)
{
    { k_write_headers<<<(unsigned)((N.C.B + 127) / 128), 128, 0, s>>>(N, out); count_launch(); }
}
} // namespace vox
