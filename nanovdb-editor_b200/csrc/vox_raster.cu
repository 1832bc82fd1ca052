// vox_raster.cu - emit -> (sort) -> build -> accumulate kernels of the
// Gaussian -> node2 voxelization.
//
// Reference path (raster/Raster.cpp:420-558): two passes of fragment windows,
// each re-running gaussian_prim / fanout / gaussian_frag_{alloc,color} and an
// incremental 4-level tree build with atomics.  Here instead:
//   k_prep        one record per Gaussian (bbox, inverse rotation, alpha
//                 constants), footprint, touched root tiles
//   k_mark_lower  touched lower-node cells (128^3 voxels) per Gaussian bbox
//   k_emit        load-balanced fragment test over all candidate fragments,
//                 passing pairs compacted in (Gaussian, fragment) order with a
//                 decoupled look-back, written as (compact voxel key, id)
//   [sort]        onesweep radix sort by key (stable: ids stay ascending)
//   k_runs        unique-key runs -> voxels, leaves, lower nodes
//   k_leaf_masks / k_node_* / k_write_*  node2 tables written exactly
//   k_accumulate  per voxel, pairs in (key, id) order: RGBA8 max + float sums
#include <cstdio>
#include <cuda_runtime.h>

#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

// ------------------------------------------------------------------ prep ----
__global__ void __launch_bounds__(256) k_prep(PrepParams P, GaussRec* recs, uint64_t* footprints,
                                              unsigned long long* root_bits, int* err)
{
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P.count)
        return;
    GaussRec R;
    int32_t bmax[3];
    uint64_t fp = make_record(P, g, R, bmax);
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
                    uint32_t rn = root_n_of(x << 12, y << 12, z << 12);
                    atomicOr(&root_bits[rn >> 6], 1ull << (rn & 63));
                }
    }
}

__device__ __forceinline__ uint64_t bit_rank(const uint64_t* bits, const uint64_t* prefix, uint64_t idx)
{
    uint64_t w = bits[idx >> 6];
    return prefix[idx >> 6] + (uint64_t)__popcll(w & ((1ull << (idx & 63)) - 1ull));
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
                uint64_t rr = bit_rank(root_bits, root_prefix, root_n_of(cx, cy, cz));
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

// ------------------------------------------------------------------ emit ----
constexpr int EMIT_BLOCK = 256;
constexpr int EMIT_CPT = 16;
constexpr int EMIT_TILE = EMIT_BLOCK * EMIT_CPT;

__device__ __forceinline__ int64_t upper_bound_u64(const uint64_t* a, int64_t lo, int64_t hi, uint64_t v)
{
    while (lo < hi)
    {
        int64_t mid = (lo + hi) >> 1;
        if (a[mid] <= v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

template <class K>
__device__ __forceinline__ K compact_key(const RankTables& T, int32_t x, int32_t y, int32_t z)
{
    uint64_t rr = bit_rank(T.root_bits, T.root_prefix, root_n_of(x, y, z));
    uint64_t cell = rr * 32768ull + upper_n_of(x, y, z);
    uint64_t lr = bit_rank(T.lower_bits, T.lower_prefix, cell);
    return (K)((lr << 21) | ((uint64_t)lower_n_of(x, y, z) << 9) | (uint64_t)leaf_n_of(x, y, z));
}

template <class K>
struct EmitSmem
{
    K stage_k[EMIT_TILE];
    uint32_t stage_i[EMIT_TILE];
    K out_k[EMIT_TILE];
    uint32_t out_i[EMIT_TILE];
    uint64_t s_warp[33];
    uint64_t gofs;
    int64_t g_lo, g_hi;
    uint32_t tile;
};

template <class K>
__global__ void __launch_bounds__(EMIT_BLOCK) k_emit(EmitParams E, RankTables T, K* __restrict__ out_k,
                                                       uint32_t* __restrict__ out_i)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    EmitSmem<K>& S = *reinterpret_cast<EmitSmem<K>*>(smem_raw);
    const uint64_t F = E.F;
    const int64_t ntiles = (int64_t)((F + EMIT_TILE - 1) / EMIT_TILE);
    while (true)
    {
        if (threadIdx.x == 0)
        {
            uint32_t t = atomicAdd(E.counter, 1u);
            S.tile = t;
            if ((int64_t)t < ntiles)
            {
                uint64_t c0 = (uint64_t)t * EMIT_TILE;
                uint64_t c1 = min(c0 + EMIT_TILE, F) - 1;
                S.g_lo = upper_bound_u64(E.frag_off, 0, E.G, c0) - 1;
                S.g_hi = upper_bound_u64(E.frag_off, S.g_lo, E.G, c1);
            }
        }
        __syncthreads();
        const int64_t tile = S.tile;
        if (tile >= ntiles)
            break;
        const uint64_t cbeg = (uint64_t)tile * EMIT_TILE + (uint64_t)threadIdx.x * EMIT_CPT;
        const uint64_t cend = min(cbeg + EMIT_CPT, F);
        uint32_t cnt = 0;
        if (cbeg < cend)
        {
            int64_t g = upper_bound_u64(E.frag_off, S.g_lo, S.g_hi, cbeg) - 1;
            uint64_t c = cbeg;
            while (c < cend)
            {
                // Gaussian g owns [frag_off[g], frag_off[g] + footprint)
                if (g >= E.G)
                {
                    atomicOr(E.err, ERR_BOUNDS);
                    break;
                }
                const GaussRec R = E.recs[g];
                const uint64_t gbeg = E.frag_off[g];
                const uint64_t gend = gbeg + (uint64_t)R.q5.x * (uint64_t)R.q5.y * (uint64_t)R.q5.z;
                if (!R.q4.w || c >= gend)
                {
                    g++;
                    continue;
                }
                const RInv M = rinv_of(R);
                const uint32_t ry = (uint32_t)R.q5.y, rz = (uint32_t)R.q5.z;
                uint32_t r = (uint32_t)(c - gbeg);
                // fragment decode, x slowest / z fastest (gaussian_frag_alloc.slang:55-58)
                int32_t i = (int32_t)(r / (rz * ry)), j = (int32_t)((r / rz) % ry), k = (int32_t)(r % rz);
                const uint64_t stop = min(cend, gend);
                for (; c < stop; c++)
                {
                    int32_t x = R.q4.x + i, y = R.q4.y + j, z = R.q4.z + k;
                    Aabb b = voxel_local_aabb(R, M, E.voxel_size, x, y, z);
                    if (aabb_hits_unit_sphere(b))
                    {
                        S.stage_k[threadIdx.x * EMIT_CPT + cnt] = compact_key<K>(T, x, y, z);
                        S.stage_i[threadIdx.x * EMIT_CPT + cnt] = (uint32_t)g;
                        cnt++;
                    }
                    if (++k == (int32_t)rz)
                    {
                        k = 0;
                        if (++j == (int32_t)ry)
                        {
                            j = 0;
                            ++i;
                        }
                    }
                }
            }
        }
        uint64_t tile_total;
        uint64_t texcl = block_excl_scan_u64(cnt, S.s_warp, tile_total);
        if (threadIdx.x == 0)
            S.gofs = lookback_exclusive(E.status, (uint64_t)tile, tile_total, E.epoch, E.err);
        for (uint32_t m = 0; m < cnt; m++)
        {
            S.out_k[texcl + m] = S.stage_k[threadIdx.x * EMIT_CPT + m];
            S.out_i[texcl + m] = S.stage_i[threadIdx.x * EMIT_CPT + m];
        }
        __syncthreads();
        const uint64_t gofs = S.gofs;
        for (uint32_t m = threadIdx.x; m < (uint32_t)tile_total; m += EMIT_BLOCK)
        {
            uint64_t dst = gofs + m;
            if (dst < E.cap)
            {
                out_k[dst] = S.out_k[m];
                out_i[dst] = S.out_i[m];
            }
        }
        if (threadIdx.x == 0 && tile == ntiles - 1)
        {
            *E.total = gofs + tile_total;
            if (gofs + tile_total > E.cap)
                atomicOr(E.err, ERR_CAPACITY);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ runs ----
constexpr int RUN_BLOCK = 256;
constexpr int RUN_ITEMS = 8;
constexpr int RUN_TILE = RUN_BLOCK * RUN_ITEMS;

template <class K>
__global__ void __launch_bounds__(RUN_BLOCK) k_runs(RunParams Rp, const K* __restrict__ keys)
{
    __shared__ uint64_t s_warp[33];
    __shared__ uint64_t s_ex[3];
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0)
        s_tile = atomicAdd(Rp.counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const int64_t P = Rp.P;
    const int64_t base = (int64_t)tile * RUN_TILE + (int64_t)threadIdx.x * RUN_ITEMS;
    K prev = (base > 0 && base - 1 < P) ? keys[base - 1] : (K)0;
    uint32_t fl[RUN_ITEMS];
    uint64_t cv = 0, cl = 0, clo = 0;
#pragma unroll
    for (int t = 0; t < RUN_ITEMS; t++)
    {
        int64_t idx = base + t;
        uint32_t f = 0;
        if (idx < P)
        {
            K k = keys[idx];
            bool first = idx == 0;
            bool hv = first || k != prev;
            bool hl = first || (k >> 9) != (prev >> 9);
            bool hlo = first || (k >> 21) != (prev >> 21);
            f = (hv ? 1u : 0u) | (hl ? 2u : 0u) | (hlo ? 4u : 0u);
            prev = k;
        }
        fl[t] = f;
        cv += f & 1u;
        cl += (f >> 1) & 1u;
        clo += (f >> 2) & 1u;
    }
    uint64_t tv, tl, tlo;
    uint64_t ev = block_excl_scan_u64(cv, s_warp, tv);
    uint64_t el = block_excl_scan_u64(cl, s_warp, tl);
    uint64_t elo = block_excl_scan_u64(clo, s_warp, tlo);
    if (threadIdx.x < 3)
    {
        uint64_t agg = threadIdx.x == 0 ? tv : (threadIdx.x == 1 ? tl : tlo);
        s_ex[threadIdx.x] = lookback_exclusive(Rp.status + threadIdx.x, tile, agg, Rp.epoch, Rp.err, 3);
    }
    __syncthreads();
    uint64_t v = s_ex[0] + ev, l = s_ex[1] + el, lo = s_ex[2] + elo;
#pragma unroll
    for (int t = 0; t < RUN_ITEMS; t++)
    {
        int64_t idx = base + t;
        if (idx >= P)
            break;
        uint32_t f = fl[t];
        if (f & 4u)
        {
            // distinct lower ranks never exceed the touched-cell count; more
            // heads mean the keys are not sorted: report, never write past it
            if (lo + 1 < Rp.lower_cap)
            {
                Rp.lower_lstart[lo] = (uint32_t)l;
                Rp.lower_rank[lo] = (uint32_t)((uint64_t)keys[idx] >> 21);
            }
            else
                atomicOr(Rp.err, ERR_ORDER);
            lo++;
        }
        if (f & 2u)
        {
            Rp.leaf_vstart[l] = (uint32_t)v;
            l++;
        }
        if (f & 1u)
        {
            Rp.vox_start[v] = (uint32_t)idx;
            v++;
        }
        if (idx == P - 1)
        {
            Rp.vox_start[v] = (uint32_t)P;
            Rp.leaf_vstart[l] = (uint32_t)v;
            if (lo < Rp.lower_cap)
                Rp.lower_lstart[lo] = (uint32_t)l;
            Rp.counts[0] = v;
            Rp.counts[1] = l;
            Rp.counts[2] = lo;
        }
    }
}

// ------------------------------------------------------------- node tables ----
__device__ __forceinline__ void root_tile_origin(uint32_t rn, int32_t o[3])
{
    int32_t x = (int32_t)((rn >> 10) & 31), y = (int32_t)((rn >> 5) & 31), z = (int32_t)(rn & 31);
    o[0] = (x >= 16 ? x - 32 : x) * 4096;
    o[1] = (y >= 16 ? y - 32 : y) * 4096;
    o[2] = (z >= 16 ? z - 32 : z) * 4096;
}

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

// canonical (single fragment window) node order: uppers, lowers, leaves, each
// in hierarchical key order; node addresses follow node_idx order
__global__ void k_canonical_order(NodeParams N, uint64_t U)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t root_sz = n2_node_bytes(0), up_sz = n2_node_bytes(1), lo_sz = n2_node_bytes(2),
                   lf_sz = n2_node_bytes(3);
    if (t < (int64_t)U)
    {
        N.upper_idx[t] = 1 + t;
        N.upper_addr[t] = root_sz + (uint64_t)t * up_sz;
        N.upper_vidx[t] = 2;
    }
    if (t < N.Lo)
    {
        N.lower_idx[t] = 1 + U + t;
        N.lower_addr[t] = root_sz + U * up_sz + (uint64_t)t * lo_sz;
        N.lower_vidx[t] = 2;
    }
    if (t < N.L)
    {
        N.leaf_idx[t] = 1 + U + N.Lo + t;
        N.leaf_addr[t] = root_sz + U * up_sz + (uint64_t)N.Lo * lo_sz + (uint64_t)t * lf_sz;
        N.leaf_vidx[t] = 2 + (uint64_t)N.leaf_vstart[t];
    }
}

// leaf value masks (+ bbox of active voxels, grid_build_compute_bbox.slang)
template <class K>
__global__ void __launch_bounds__(256) k_leaf_masks(NodeParams N, const K* __restrict__ keys)
{
    const int lane = threadIdx.x & 31;
    int64_t l = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (l >= N.L)
        return;
    uint32_t v0 = N.leaf_vstart[l], v1 = N.leaf_vstart[l + 1];
    uint64_t m[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
    int32_t mn[3] = { 8, 8, 8 }, mx[3] = { -1, -1, -1 };
    K key0 = keys[N.vox_start[v0]];
    for (uint32_t v = v0 + lane; v < v1; v += 32)
    {
        uint32_t n = (uint32_t)keys[N.vox_start[v]] & 511u;
        m[n >> 6] |= 1ull << (n & 63);
        int32_t c[3] = { (int32_t)(n >> 6), (int32_t)((n >> 3) & 7), (int32_t)(n & 7) };
        for (int a = 0; a < 3; a++)
        {
            mn[a] = min(mn[a], c[a]);
            mx[a] = max(mx[a], c[a]);
        }
    }
#pragma unroll
    for (int w = 0; w < 8; w++)
        for (int o = 16; o > 0; o >>= 1)
            m[w] |= __shfl_xor_sync(0xffffffffu, m[w], o);
    for (int a = 0; a < 3; a++)
        for (int o = 16; o > 0; o >>= 1)
        {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    if (lane < 8)
        N.leaf_mask[8 * l + lane] = m[lane];
    if (lane == 0)
    {
        // leaf origin from its lower node and lower_n
        uint32_t ln = (uint32_t)((uint64_t)key0 >> 9) & 4095u;
        uint32_t lo = N.leaf_lower[l];
        int32_t o[3] = { N.lower_origin[3 * lo + 0] + (int32_t)((ln >> 8) & 15) * 8,
                         N.lower_origin[3 * lo + 1] + (int32_t)((ln >> 4) & 15) * 8,
                         N.lower_origin[3 * lo + 2] + (int32_t)(ln & 15) * 8 };
        N.leaf_origin[3 * l + 0] = o[0];
        N.leaf_origin[3 * l + 1] = o[1];
        N.leaf_origin[3 * l + 2] = o[2];
        for (int a = 0; a < 3; a++)
        {
            atomicMin(&N.bbox[a], o[a] + mn[a]);
            atomicMax(&N.bbox[3 + a], o[a] + mx[a]);
        }
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

__global__ void __launch_bounds__(1024) k_write_root(NodeParams N, uint64_t U, uint8_t* node2)
{
    __shared__ uint64_t s_mask[512];
    __shared__ uint32_t s_scan[513];
    uint64_t* W = (uint64_t*)node2;
    for (int i = threadIdx.x; i < 512; i += blockDim.x)
        s_mask[i] = 0;
    __syncthreads();
    for (uint64_t u = threadIdx.x; u < U; u += blockDim.x)
    {
        uint32_t rn = N.upper_root_n[u];
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
            val = N.upper_addr[e];
        else if (e < 2 * U)
        {
            uint32_t rn = N.upper_root_n[e - U];
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

__global__ void k_leaf_lower_n(NodeParams N, const void* keys_v, int key64)
{
    int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= N.L)
        return;
    uint64_t key = key64 ? ((const uint64_t*)keys_v)[N.vox_start[N.leaf_vstart[l]]]
                         : (uint64_t)((const uint32_t*)keys_v)[N.vox_start[N.leaf_vstart[l]]];
    N.leaf_lower_n[l] = (uint32_t)(key >> 9) & 4095u;
}

// ------------------------------------------------------------- accumulate ----
// one warp per leaf, one lane per voxel; each lane walks its voxel's pairs in
// (key, id) order so the float sums have a fixed sequential order
template <class K>
__global__ void __launch_bounds__(256) k_accumulate(AccumParams A, NodeParams N, const uint32_t* __restrict__ ids)
{
    const int lane = threadIdx.x & 31;
    int64_t l = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (l >= N.L)
        return;
    const uint32_t v0 = N.leaf_vstart[l], v1 = N.leaf_vstart[l + 1];
    const int32_t ox = N.leaf_origin[3 * l + 0], oy = N.leaf_origin[3 * l + 1], oz = N.leaf_origin[3 * l + 2];
    const uint64_t vbase = N.leaf_vidx[l];
    const K* keys = (const K*)A.keys;
    for (uint32_t v = v0 + lane; v < v1; v += 32)
    {
        const uint32_t p0 = N.vox_start[v], p1 = N.vox_start[v + 1];
        const uint32_t n = (uint32_t)keys[p0] & 511u;
        const int32_t x = ox + (int32_t)(n >> 6), y = oy + (int32_t)((n >> 3) & 7), z = oz + (int32_t)(n & 7);
        uint32_t rgba = 0;
        float dsum = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
        for (uint32_t p = p0; p < p1; p++)
        {
            const GaussRec R = A.recs[ids[p]];
            const RInv M = rinv_of(R);
            Aabb b = voxel_local_aabb(R, M, A.voxel_size, x, y, z);
            float a = pair_alpha(R, b);
            uint32_t c = pack_rgba8(R, a);
            rgba = c > rgba ? c : rgba;
            dsum = VOX_FADD(dsum, a);
            c0 = VOX_FADD(c0, VOX_FMUL(a, R.q7.x));
            c1 = VOX_FADD(c1, VOX_FMUL(a, R.q7.y));
            c2 = VOX_FADD(c2, VOX_FMUL(a, R.q7.z));
        }
        const uint64_t vi = vbase + (v - v0);
        A.rgba8[vi] = rgba;
        A.density[vi] = dsum;
        A.color[3 * vi + 0] = dsum > 0.f ? VOX_FDIV(c0, dsum) : 0.f;
        A.color[3 * vi + 1] = dsum > 0.f ? VOX_FDIV(c1, dsum) : 0.f;
        A.color[3 * vi + 2] = dsum > 0.f ? VOX_FDIV(c2, dsum) : 0.f;
    }
}

// =================================================================== launch
void launch_prep(const PrepParams& P, GaussRec* recs, uint64_t* footprints, uint64_t* root_bits, int* err,
                 cudaStream_t s)
{
    if (P.count <= 0)
        return;
    { k_prep<<<(unsigned)((P.count + 255) / 256), 256, 0, s>>>(P, recs, footprints, (unsigned long long*)root_bits, err); count_launch(); }
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

template <class K>
static void launch_emit_t(const EmitParams& E, const RankTables& T, K* out_k, uint32_t* out_i, int num_sms,
                          cudaStream_t s)
{
    if (E.F == 0)
    {
        cudaMemsetAsync(E.total, 0, sizeof(uint64_t), s);
        return;
    }
    const size_t smem = sizeof(EmitSmem<K>);
    cudaFuncSetAttribute(k_emit<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_emit<K>, EMIT_BLOCK, smem);
    if (per_sm < 1)
        per_sm = 1;
    int64_t tiles = (int64_t)((E.F + EMIT_TILE - 1) / EMIT_TILE);
    int64_t grid = (int64_t)num_sms * per_sm;
    if (grid > tiles)
        grid = tiles;
    cudaMemsetAsync(E.counter, 0, sizeof(uint32_t), s);
    { k_emit<K><<<(unsigned)grid, EMIT_BLOCK, smem, s>>>(E, T, out_k, out_i); count_launch(); }
}
void launch_emit_u32(const EmitParams& E, const RankTables& T, uint32_t* out_k, uint32_t* out_i, int num_sms,
                     cudaStream_t s)
{
    launch_emit_t<uint32_t>(E, T, out_k, out_i, num_sms, s);
}
void launch_emit_u64(const EmitParams& E, const RankTables& T, uint64_t* out_k, uint32_t* out_i, int num_sms,
                     cudaStream_t s)
{
    launch_emit_t<uint64_t>(E, T, out_k, out_i, num_sms, s);
}
int64_t emit_tile_count(uint64_t F)
{
    return (int64_t)((F + EMIT_TILE - 1) / EMIT_TILE);
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
    { k_leaf_lower_n<<<(unsigned)((N.L + 255) / 256), 256, 0, s>>>(N, keys, key64); count_launch(); }
    unsigned blocks = (unsigned)((N.L * 32 + 255) / 256);
    if (key64)
        { k_leaf_masks<uint64_t><<<blocks, 256, 0, s>>>(N, (const uint64_t*)keys); count_launch(); }
    else
        { k_leaf_masks<uint32_t><<<blocks, 256, 0, s>>>(N, (const uint32_t*)keys); count_launch(); }
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
void launch_write_nodes(const NodeParams& N, uint64_t U, uint8_t* node2, cudaStream_t s)
{
    { k_write_root<<<1, 1024, 0, s>>>(N, U, node2); count_launch(); }
    if (U)
        { k_write_upper<<<(unsigned)U, 512, 0, s>>>(N, node2); count_launch(); }
    if (N.Lo)
        { k_write_lower<<<(unsigned)N.Lo, 256, 0, s>>>(N, node2); count_launch(); }
    if (N.L)
        { k_write_leaf<<<(unsigned)((N.L * 16 + 255) / 256), 256, 0, s>>>(N, node2); count_launch(); }
}
void launch_accumulate(const AccumParams& A, const NodeParams& N, const uint32_t* ids, int key64, cudaStream_t s)
{
    if (N.L <= 0)
        return;
    unsigned blocks = (unsigned)((N.L * 32 + 255) / 256);
    if (key64)
        { k_accumulate<uint64_t><<<blocks, 256, 0, s>>>(A, N, ids); count_launch(); }
    else
        { k_accumulate<uint32_t><<<blocks, 256, 0, s>>>(A, N, ids); count_launch(); }
}

} // namespace vox
