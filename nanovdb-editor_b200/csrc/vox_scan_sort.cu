// vox_scan_sort.cu - single-pass scans and the onesweep LSD radix sort that
// replace the reference's ParallelPrimitives (raster/ParallelPrimitives.cpp:
// global_scan* at :151-310, radix_sort_key64 at :685-869).
//
// Both use decoupled look-back: CTAs take tiles in order from an atomic
// counter, publish their tile aggregate, then walk back over predecessors'
// published (aggregate | inclusive) words.  All waits are bounded
// (LB_SPIN_LIMIT); a timeout sets the device error word and the call fails.
#include <atomic>
#include <cstdio>
#include <cuda_runtime.h>

#include "vox_device.cuh"
#include "vox_internal.h"

namespace vox
{

static std::atomic<int64_t> g_launches{ 0 };
int64_t launch_count()
{
    return g_launches.load(std::memory_order_relaxed);
}
void count_launch()
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

// ===================================================================== scan
constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

// status words of a scan of n elements: four per tile for the u64 scan (its
// full 64-bit look-back), one per tile for the u32 scans
size_t scan_status_words(int64_t n)
{
    return 4 * ((size_t)((n + SCAN_TILE - 1) / SCAN_TILE) + 1);
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_excl(const uint64_t* in, uint64_t* out, int64_t n, int mode,
                                                            uint64_t* total, uint64_t* status, uint32_t epoch,
                                                            uint32_t* counter, int* err)
{
    __shared__ uint64_t s_warp[33];
    __shared__ uint64_t s_excl;
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0)
        s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const int64_t base = (int64_t)tile * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    uint64_t v[SCAN_ITEMS];
    uint64_t sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        int64_t idx = base + i;
        uint64_t x = idx < n ? in[idx] : 0ull;
        if (mode & 1)
            x = (uint64_t)__popcll(x);
        v[i] = x;
        sum += x;
    }
    uint64_t block_total;
    uint64_t texcl = block_excl_scan_u64(sum, s_warp, block_total);
    if (threadIdx.x == 0)
        s_excl = lookback_exclusive_wide(status, tile, block_total, epoch, err);
    __syncthreads();
    uint64_t run = s_excl + texcl;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        int64_t idx = base + i;
        if (idx < n)
        {
            out[idx] = (mode & 2) ? run + v[i] : run;
            run += v[i];
            if (idx == n - 1)
                *total = run;
        }
    }
}

void scan_exclusive_u64(const uint64_t* in, uint64_t* out, int64_t n, int mode, uint64_t* total, uint64_t* status,
                        uint32_t epoch, uint32_t* counter, int* err, int num_sms, cudaStream_t s)
{
    (void)num_sms;
    if (n <= 0)
    {
        cudaMemsetAsync(total, 0, sizeof(uint64_t), s);
        return;
    }
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    { k_scan_excl<<<(unsigned)tiles, SCAN_BLOCK, 0, s>>>(in, out, n, mode, total, status, epoch, counter, err); count_launch(); }
}

// u32 scans: the reference's global_scan (sum, wrapping mod 2^32) and
// global_scan_max (running maximum), inclusive or exclusive; sums are carried
// in 64 bits (the look-back keeps them mod 2^55, a multiple of 2^32)
template <bool MAX>
__device__ __forceinline__ uint64_t scan_op(uint64_t a, uint64_t b)
{
    return MAX ? (a > b ? a : b) : a + b;
}

template <bool MAX>
__device__ __forceinline__ uint64_t block_excl_scan_op(uint64_t v, uint64_t* s_warp, uint64_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const uint64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o)
            incl = scan_op<MAX>(incl, t);
    }
    if (lane == 31)
        s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0)
    {
        const uint64_t w = lane < nwarps ? s_warp[lane] : 0;
        uint64_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const uint64_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o)
                wi = scan_op<MAX>(wi, t);
        }
        const uint64_t prev = __shfl_up_sync(0xffffffffu, wi, 1);
        if (lane < nwarps)
            s_warp[lane] = lane == 0 ? 0 : prev; // exclusive over warps
        if (lane == nwarps - 1)
            s_warp[32] = wi;
    }
    __syncthreads();
    total = s_warp[32];
    // exclusive within the warp: the inclusive value of the lane before
    const uint64_t before = __shfl_up_sync(0xffffffffu, incl, 1);
    const uint64_t r = scan_op<MAX>(s_warp[warp], lane == 0 ? 0 : before);
    __syncthreads();
    return r;
}

template <bool MAX>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, int inclusive,
                                                           uint64_t* total, uint64_t* status, uint32_t epoch,
                                                           uint32_t* counter, int* err)
{
    __shared__ uint64_t s_warp[33];
    __shared__ uint64_t s_excl;
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0)
        s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const int64_t base = (int64_t)tile * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint64_t agg = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        const int64_t idx = base + i;
        v[i] = idx < n ? in[idx] : 0u;
        agg = scan_op<MAX>(agg, (uint64_t)v[i]);
    }
    uint64_t block_total;
    const uint64_t texcl = block_excl_scan_op<MAX>(agg, s_warp, block_total);
    if (threadIdx.x == 0)
        s_excl = lookback_exclusive(status, tile, block_total, epoch, err, 1, MAX);
    __syncthreads();
    uint64_t run = scan_op<MAX>(s_excl, texcl);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        const int64_t idx = base + i;
        if (idx < n)
        {
            const uint64_t next = scan_op<MAX>(run, (uint64_t)v[i]);
            out[idx] = (uint32_t)(inclusive ? next : run);
            run = next;
            if (idx == n - 1)
                *total = run;
        }
    }
}

void scan_u32(const uint32_t* in, uint32_t* out, int64_t n, int inclusive, int max_op, uint64_t* total,
              uint64_t* status, uint32_t epoch, uint32_t* counter, int* err, cudaStream_t s)
{
    if (n <= 0)
    {
        cudaMemsetAsync(total, 0, sizeof(uint64_t), s);
        return;
    }
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    const int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (max_op)
        k_scan_u32<true><<<(unsigned)tiles, SCAN_BLOCK, 0, s>>>(in, out, n, inclusive, total, status, epoch, counter, err);
    else
        k_scan_u32<false><<<(unsigned)tiles, SCAN_BLOCK, 0, s>>>(in, out, n, inclusive, total, status, epoch, counter, err);
    count_launch();
}

// dual-key sort helpers: (high, low) -> one 64-bit key + original index, and
// the gather of the three arrays by the sorted indices
__global__ void k_dual_combine(const uint32_t* low, const uint32_t* high, int64_t n, int low_bits, int high_bits,
                               uint64_t* key, uint32_t* idx)
{
    const uint64_t ml = low_bits >= 32 ? 0xffffffffull : ((1ull << low_bits) - 1);
    const uint64_t mh = high_bits >= 32 ? 0xffffffffull : ((1ull << high_bits) - 1);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        key[i] = (((uint64_t)high[i] & mh) << low_bits) | ((uint64_t)low[i] & ml);
        idx[i] = (uint32_t)i;
    }
}

__global__ void k_dual_gather(const uint32_t* sidx, int64_t n, const uint32_t* low_c, const uint32_t* high_c,
                              const uint32_t* val_c, uint32_t* low, uint32_t* high, uint32_t* val, int* err)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        const uint32_t j = sidx[i];
        if ((int64_t)j >= n)
        {
            atomicOr(err, ERR_BOUNDS);
            continue;
        }
        low[i] = low_c[j];
        high[i] = high_c[j];
        val[i] = val_c[j];
    }
}

void dual_combine(const uint32_t* low, const uint32_t* high, int64_t n, int low_bits, int high_bits, uint64_t* key,
                  uint32_t* idx, int num_sms, cudaStream_t s)
{
    if (n <= 0)
        return;
    int64_t grid = (n + 255) / 256;
    if (grid > (int64_t)num_sms * 16)
        grid = (int64_t)num_sms * 16;
    k_dual_combine<<<(unsigned)grid, 256, 0, s>>>(low, high, n, low_bits, high_bits, key, idx);
    count_launch();
}

void dual_gather(const uint32_t* sidx, int64_t n, const uint32_t* low_c, const uint32_t* high_c, const uint32_t* val_c,
                 uint32_t* low, uint32_t* high, uint32_t* val, int* err, int num_sms, cudaStream_t s)
{
    if (n <= 0)
        return;
    int64_t grid = (n + 255) / 256;
    if (grid > (int64_t)num_sms * 16)
        grid = (int64_t)num_sms * 16;
    k_dual_gather<<<(unsigned)grid, 256, 0, s>>>(sidx, n, low_c, high_c, val_c, low, high, val, err);
    count_launch();
}

// ===================================================================== sort
// Tile: block threads x items keys (SORT_SHAPES).  One up-front pass computes the
// digit histograms of every pass (global counts are permutation-invariant);
// each scatter pass then finds, per digit, the count in earlier tiles with a
// decoupled look-back over 64-bit epoch-tagged words (55-bit counts).
constexpr int SORT_MAX_PASSES = 8;
struct SortShapeInfo
{
    int block, items, tile;
};
constexpr int SORT_NSHAPES = 5;
constexpr SortShapeInfo SORT_SHAPES[SORT_NSHAPES] = { { 512, 16, 8192 }, { 256, 16, 4096 }, { 256, 12, 3072 },
                                                      { 256, 8, 2048 }, { 512, 8, 4096 } };
constexpr int SORT_TILE_MIN = 2048; // status words are sized for the smallest tile

struct SortWs
{
    uint32_t* hist;      // [passes][256]
    uint64_t* base;      // [passes][256]
    uint32_t* counters;  // [passes]
    uint64_t* status;    // [tiles][256]
    uint32_t* tile_hist; // [256][tiles]: per-tile digit counts, then their global offsets (three-kernel passes)
    int64_t tiles;
};

static size_t align256(size_t x)
{
    return (x + 255) / 256 * 256;
}

static SortWs carve(void* ws, int64_t n)
{
    SortWs w;
    w.tiles = (n + SORT_TILE_MIN - 1) / SORT_TILE_MIN;
    char* p = (char*)ws;
    w.hist = (uint32_t*)p;
    p += align256(sizeof(uint32_t) * SORT_MAX_PASSES * 256);
    w.base = (uint64_t*)p;
    p += align256(sizeof(uint64_t) * SORT_MAX_PASSES * 256);
    w.counters = (uint32_t*)p;
    p += align256(sizeof(uint32_t) * (SORT_MAX_PASSES + 1));
    w.status = (uint64_t*)p;
    p += align256(sizeof(uint64_t) * (w.tiles + 1) * 256);
    w.tile_hist = (uint32_t*)p;
    return w;
}

size_t sort_workspace_bytes(int64_t n, int key_bytes)
{
    (void)key_bytes;
    int64_t tiles = (n + SORT_TILE_MIN - 1) / SORT_TILE_MIN;
    return align256(sizeof(uint32_t) * SORT_MAX_PASSES * 256) + align256(sizeof(uint64_t) * SORT_MAX_PASSES * 256) +
           align256(sizeof(uint32_t) * (SORT_MAX_PASSES + 1)) + align256(sizeof(uint64_t) * (tiles + 1) * 256) +
           align256(sizeof(uint32_t) * (tiles + 1) * 256);
}

size_t sort_status_words(int64_t n)
{
    return (size_t)((n + SORT_TILE_MIN - 1) / SORT_TILE_MIN + 1) * 256;
}

template <class K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift, uint32_t mask)
{
    return (uint32_t)(k >> shift) & mask;
}

// up-front histogram of every pass's digit (per-CTA shared counters, then
// one global atomic per bin); counts fit 32 bits for n < 2^32
// digit width of pass p: `bits`, the last pass only the key bits left, so
// bits at and above key_bits never take part in the order
__host__ __device__ __forceinline__ int pass_bits(int p, int bits, int key_bits)
{
    const int left = key_bits - p * bits;
    return left < bits ? left : bits;
}

template <class K>
__global__ void __launch_bounds__(512) k_sort_hist(const K* keys, int64_t n, int passes, int bits, int key_bits,
                                                            uint32_t* hist)
{
    __shared__ uint32_t s_h[SORT_MAX_PASSES * 256];
    for (int i = threadIdx.x; i < SORT_MAX_PASSES * 256; i += blockDim.x)
        s_h[i] = 0;
    __syncthreads();
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x)
    {
        K k = keys[idx];
        for (int p = 0; p < passes; p++)
            atomicAdd(&s_h[p * 256 + digit_of(k, p * bits, (1u << pass_bits(p, bits, key_bits)) - 1u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        if (s_h[i])
            atomicAdd(&hist[i], s_h[i]);
}

// base[pass][d] = sum_{d' < d} hist[pass][d']
__global__ void k_sort_bases(const uint32_t* hist, uint64_t* base, int passes)
{
    __shared__ uint64_t s_warp[33];
    const int d = threadIdx.x; // 256 threads
    for (int p = 0; p < passes; p++)
    {
        uint64_t all;
        base[p * 256 + d] = block_excl_scan_u64((uint64_t)hist[p * 256 + d], s_warp, all);
    }
}

// onesweep tile shapes: threads x keys per thread (x minimum resident CTAs,
// which caps registers); the tuner times one pass of each and keeps the
// fastest per key width and size class
template <class K, int BLOCK, int ITEMS>
struct SortSmem
{
    K keys[BLOCK * ITEMS];
    uint32_t vals[BLOCK * ITEMS];
    uint32_t warp_hist[BLOCK / 32][256];
    uint32_t digit_excl[256];
    uint64_t gbase[256];
    uint64_t s_warp[33];
    uint32_t tile;
};

// LB: the tile's digit offsets from a decoupled look-back over the tiles before
// it (tiles claimed in order by an atomic ticket); otherwise from offsets, the
// digit-major exclusive scan of every tile's digit counts (tile = block index)
template <class K, int BLOCK, int ITEMS, int MINB, bool LB = true>
__global__ void __launch_bounds__(BLOCK, MINB) k_onesweep(const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                                          K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                          int64_t n, int shift, int bits, const uint64_t* base,
                                                          uint64_t* status, uint32_t epoch, uint32_t* counter, int* err,
                                                          const uint32_t* offsets = nullptr, int64_t ntiles = 0)
{
    constexpr int TILE = BLOCK * ITEMS;
    constexpr int WARPS = BLOCK / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<K, BLOCK, ITEMS>& S = *reinterpret_cast<SortSmem<K, BLOCK, ITEMS>*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t mask = (1u << bits) - 1u;
    const int radix = 1 << bits;

    if (threadIdx.x == 0)
        S.tile = LB ? atomicAdd(counter, 1u) : blockIdx.x;
    for (int i = lane; i < 256; i += 32)
        S.warp_hist[warp][i] = 0;
    __syncthreads();
    const int64_t tile = S.tile;
    const int64_t tile_base = tile * TILE;
    const int tile_count = (int)min((int64_t)TILE, n - tile_base);

    // load: warp-contiguous chunks, item-major within a warp (stable order = (item, lane))
    K k[ITEMS];
    uint32_t v[ITEMS];
    uint32_t rank[ITEMS];
    const int64_t wbase = tile_base + (int64_t)warp * (32 * ITEMS);
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
    {
        int64_t idx = wbase + i * 32 + lane;
        if (idx < n)
        {
            k[i] = keys_in[idx];
            v[i] = vals_in[idx];
        }
    }
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
    {
        int64_t idx = wbase + i * 32 + lane;
        bool valid = idx < n;
        uint32_t d = valid ? digit_of(k[i], shift, mask) : 0xFFFFu;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = __popc(peers & lt);
        uint32_t leader = __ffs(peers) - 1;
        // the group's leader reserves its slots; the others take its old count
        uint32_t prev = 0u;
        if (valid && (uint32_t)lane == leader)
            prev = atomicAdd(&S.warp_hist[warp][d], (uint32_t)__popc(peers));
        prev = __shfl_sync(0xffffffffu, prev, (int)leader);
        rank[i] = prev + before;
    }
    __syncthreads();

    // per digit: exclusive over warps, tile total, exclusive over digits
    uint64_t total = 0;
    if (threadIdx.x < 256)
    {
        uint32_t run = 0;
        for (int w = 0; w < WARPS; w++)
        {
            uint32_t c = S.warp_hist[w][threadIdx.x];
            S.warp_hist[w][threadIdx.x] = run;
            run += c;
        }
        total = run;
    }
    uint64_t all;
    uint64_t dexcl = block_excl_scan_u64(threadIdx.x < 256 ? total : 0ull, S.s_warp, all);
    if (threadIdx.x < 256)
    {
        S.digit_excl[threadIdx.x] = (uint32_t)dexcl;
        const int d = threadIdx.x;
        if (d < radix)
        {
            // count of digit d in all earlier tiles.  Walked before the shared-memory
            // scatter: the inclusive prefix this tile publishes is what shortens its
            // successors' walks (publishing it after the scatter measured slower)
            if constexpr (LB)
            {
                uint64_t excl = lookback_exclusive(status + d, (uint64_t)tile, total, epoch, err, 256);
                S.gbase[d] = base[d] + excl - dexcl;
            }
            else
                S.gbase[d] = (uint64_t)offsets[(int64_t)d * ntiles + tile] - dexcl;
        }
    }
    __syncthreads();

    // scatter into shared memory in digit order
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
    {
        int64_t idx = wbase + i * 32 + lane;
        if (idx < n)
        {
            uint32_t d = digit_of(k[i], shift, mask);
            uint32_t pos = S.digit_excl[d] + S.warp_hist[warp][d] + rank[i];
            if (pos < (uint32_t)TILE)
            {
                S.keys[pos] = k[i];
                S.vals[pos] = v[i];
            }
            else
                atomicOr(err, ERR_BOUNDS);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tile_count; i += BLOCK)
    {
        K kk = S.keys[i];
        uint32_t d = digit_of(kk, shift, mask);
        uint64_t dst = S.gbase[d] + (uint64_t)i;
        if (dst < (uint64_t)n)
        {
            keys_out[dst] = kk;
            vals_out[dst] = S.vals[i];
        }
        else
            atomicOr(err, ERR_BOUNDS);
    }
}

// one onesweep pass with shape `shape` (SORT_SHAPES)
template <class K>
static void onesweep_pass(int shape, const K* src_k, const uint32_t* src_v, K* dst_k, uint32_t* dst_v, int64_t n,
                          int shift, int bits, const uint64_t* base, uint64_t* status, uint32_t epoch,
                          uint32_t* counter, int* err, cudaStream_t s)
{
    const int64_t tiles = (n + SORT_SHAPES[shape].tile - 1) / SORT_SHAPES[shape].tile;
#define VOX_ONESWEEP(B, I, M)                                                                                      \
    {                                                                                                              \
        const size_t smem = sizeof(SortSmem<K, B, I>);                                                             \
        cudaFuncSetAttribute(k_onesweep<K, B, I, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);      \
        k_onesweep<K, B, I, M><<<(unsigned)tiles, B, smem, s>>>(src_k, src_v, dst_k, dst_v, n, shift, bits, base, \
                                                                 status, epoch, counter, err);                     \
        count_launch();                                                                                            \
    }
    switch (shape)
    {
    case 0: VOX_ONESWEEP(512, 16, 1) break;
    case 1: VOX_ONESWEEP(256, 16, 2) break;
    case 2: VOX_ONESWEEP(256, 12, 3) break;
    case 3: VOX_ONESWEEP(256, 8, 4) break;
    default: VOX_ONESWEEP(512, 8, 2) break;
    }
#undef VOX_ONESWEEP
}

// Three-kernel pass (no look-back chain): per-tile digit counts, then per digit
// an exclusive scan over the tiles plus the digit's global base, then the
// onesweep tile ranking and scatter with those offsets.  The same stable result
// as the onesweep pass; it reads the keys once more but no tile waits on
// another, which wins where the look-back chain's latency bounds the pass.
template <class K, int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK) k_tile_hist(const K* __restrict__ keys, int64_t n, int shift, int bits,
                                                     uint32_t* __restrict__ tile_hist, int64_t ntiles)
{
    __shared__ uint32_t h[BLOCK / 32][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t mask = (1u << bits) - 1u;
    for (int i = lane; i < 256; i += 32)
        h[warp][i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * (BLOCK * ITEMS);
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
    {
        const int64_t idx = base + (int64_t)i * BLOCK + threadIdx.x;
        if (idx < n)
            atomicAdd(&h[warp][digit_of(keys[idx], shift, mask)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d <= (int)mask; d += BLOCK)
    {
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < BLOCK / 32; w++)
            c += h[w][d];
        tile_hist[(int64_t)d * ntiles + blockIdx.x] = c;
    }
}

// one block per digit: the row of tile counts -> base[d] + exclusive prefix, in place
__global__ void __launch_bounds__(256) k_tile_offsets(uint32_t* tile_hist, int64_t ntiles, const uint64_t* base)
{
    __shared__ uint64_t s_warp[33];
    uint32_t* row = tile_hist + (int64_t)blockIdx.x * ntiles;
    uint64_t running = base[blockIdx.x];
    for (int64_t c0 = 0; c0 < ntiles; c0 += 256 * 4)
    {
        const int64_t t0 = c0 + (int64_t)threadIdx.x * 4;
        uint32_t v[4];
        uint64_t sum = 0;
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            v[q] = t0 + q < ntiles ? row[t0 + q] : 0u;
            sum += v[q];
        }
        uint64_t all;
        uint64_t ex = running + block_excl_scan_u64(sum, s_warp, all);
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (t0 + q < ntiles)
            {
                row[t0 + q] = (uint32_t)ex;
                ex += v[q];
            }
        running += all;
    }
}

template <class K>
static void three_kernel_pass(int shape, const K* src_k, const uint32_t* src_v, K* dst_k, uint32_t* dst_v, int64_t n,
                              int shift, int bits, const uint64_t* base, uint32_t* tile_hist, int* err, cudaStream_t s)
{
    const int64_t tiles = (n + SORT_SHAPES[shape].tile - 1) / SORT_SHAPES[shape].tile;
#define VOX_THREEK(B, I, M)                                                                                        \
    {                                                                                                              \
        k_tile_hist<K, B, I><<<(unsigned)tiles, B, 0, s>>>(src_k, n, shift, bits, tile_hist, tiles);               \
        count_launch();                                                                                            \
        k_tile_offsets<<<1u << bits, 256, 0, s>>>(tile_hist, tiles, base);                                         \
        count_launch();                                                                                            \
        const size_t smem = sizeof(SortSmem<K, B, I>);                                                             \
        cudaFuncSetAttribute(k_onesweep<K, B, I, M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        k_onesweep<K, B, I, M, false><<<(unsigned)tiles, B, smem, s>>>(src_k, src_v, dst_k, dst_v, n, shift, bits,   \
                                                                        base, nullptr, 0u, nullptr, err, tile_hist, \
                                                                        tiles);                                    \
        count_launch();                                                                                            \
    }
    switch (shape)
    {
    case 0: VOX_THREEK(512, 16, 1) break;
    case 1: VOX_THREEK(256, 16, 2) break;
    case 2: VOX_THREEK(256, 12, 3) break;
    case 3: VOX_THREEK(256, 8, 4) break;
    default: VOX_THREEK(512, 8, 2) break;
    }
#undef VOX_THREEK
}

// candidate c of the tuner: tile shape c % SORT_NSHAPES, onesweep (c < SORT_NSHAPES) or three kernels
constexpr int SORT_NCAND = 2 * SORT_NSHAPES;

template <class K>
static void sort_pass(int cand, const K* src_k, const uint32_t* src_v, K* dst_k, uint32_t* dst_v, int64_t n, int shift,
                      int bits, const uint64_t* base, const SortWs& w, Epochs* epochs, size_t words, uint32_t* counter,
                      int* err, cudaStream_t s)
{
    // the three-kernel offsets are 32-bit: n < 2^32 (every caller's limit; onesweep otherwise)
    if (cand < SORT_NSHAPES || n >= (1ll << 32))
    {
        cand %= SORT_NSHAPES;
        const uint32_t epoch = epochs->next(w.status, words, s);
        onesweep_pass<K>(cand, src_k, src_v, dst_k, dst_v, n, shift, bits, base, w.status, epoch, counter, err, s);
    }
    else
        three_kernel_pass<K>(cand - SORT_NSHAPES, src_k, src_v, dst_k, dst_v, n, shift, bits, base, w.tile_hist, err, s);
}

static int size_class(int64_t n)
{
    int c = 0;
    while (c < 39 && (1ll << (c + 1)) <= n)
        c++;
    return c;
}

template <class K>
static int sort_pairs_impl(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, int64_t n, int key_bits,
                           void* workspace, Epochs* epochs, int* err, int num_sms, cudaStream_t s, SortTuning& tune)
{
    if (n <= 1 || key_bits <= 0)
        return 0;
    const int bits = tune.digit_bits < 1 ? 8 : (tune.digit_bits > 8 ? 8 : tune.digit_bits);
    int passes = (key_bits + bits - 1) / bits;
    if (passes > SORT_MAX_PASSES)
        passes = SORT_MAX_PASSES;
    SortWs w = carve(workspace, n);
    cudaMemsetAsync(w.hist, 0, sizeof(uint32_t) * SORT_MAX_PASSES * 256, s);
    cudaMemsetAsync(w.counters, 0, sizeof(uint32_t) * (SORT_MAX_PASSES + 1), s);
    int64_t hist_grid = (int64_t)num_sms * 4;
    int64_t need = (n + 511) / 512;
    if (hist_grid > need)
        hist_grid = need;
    { k_sort_hist<K><<<(unsigned)hist_grid, 512, 0, s>>>(keys, n, passes, bits, key_bits, w.hist); count_launch(); }
    { k_sort_bases<<<1, 256, 0, s>>>(w.hist, w.base, passes); count_launch(); }
    const size_t words = sort_status_words(n);
    const int kw = sizeof(K) == 8 ? 1 : 0, sc = size_class(n);
    int shape = tune.shape >= 0 && tune.shape < SORT_NCAND ? tune.shape : tune.best[kw][sc];
    if (shape < 0)
    {
        // tuner: time pass 0 of every candidate on this data (the output is rewritten below)
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float best_ms = 1e30f;
        shape = 0;
        for (int t = 0; t < SORT_NCAND; t++)
        {
            cudaMemsetAsync(w.counters + SORT_MAX_PASSES, 0, sizeof(uint32_t), s);
            cudaEventRecord(e0, s);
            sort_pass<K>(t, keys, vals, keys_alt, vals_alt, n, 0, pass_bits(0, bits, key_bits), w.base, w, epochs, words,
                         w.counters + SORT_MAX_PASSES, err, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best_ms)
            {
                best_ms = ms;
                shape = t;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        tune.best[kw][sc] = shape;
    }
    K* src_k = keys;
    uint32_t* src_v = vals;
    K* dst_k = keys_alt;
    uint32_t* dst_v = vals_alt;
    for (int p = 0; p < passes; p++)
    {
        sort_pass<K>(shape, src_k, src_v, dst_k, dst_v, n, p * bits, pass_bits(p, bits, key_bits), w.base + p * 256, w,
                     epochs, words, w.counters + p, err, s);
        K* tk = src_k;
        src_k = dst_k;
        dst_k = tk;
        uint32_t* tv = src_v;
        src_v = dst_v;
        dst_v = tv;
    }
    return (passes & 1) ? 1 : 0;
}

int sort_shape_used(int64_t n, int key64, const SortTuning& tune)
{
    if (tune.shape >= 0 && tune.shape < SORT_NCAND)
        return tune.shape;
    return n > 1 ? tune.best[key64 ? 1 : 0][size_class(n)] : -1;
}

int sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, int64_t n, int key_bits,
                   void* workspace, Epochs* epochs, int* err, int num_sms, cudaStream_t s, SortTuning& tune)
{
    return sort_pairs_impl<uint32_t>(keys, vals, keys_alt, vals_alt, n, key_bits, workspace, epochs, err, num_sms, s,
                                     tune);
}
int sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, int64_t n, int key_bits,
                   void* workspace, Epochs* epochs, int* err, int num_sms, cudaStream_t s, SortTuning& tune)
{
    return sort_pairs_impl<uint64_t>(keys, vals, keys_alt, vals_alt, n, key_bits, workspace, epochs, err, num_sms, s,
                                     tune);
}

} // namespace vox

namespace vox
{
// counts adjacent pairs with keys[i] < keys[i - 1] (a read-only validation pass)
template <class K>
__global__ void k_check_sorted(const K* keys, int64_t n, unsigned long long* descents)
{
    unsigned long long local = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < n; i += (int64_t)gridDim.x * blockDim.x)
        local += keys[i] < keys[i - 1] ? 1ull : 0ull;
    for (int o = 16; o > 0; o >>= 1)
        local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local)
        atomicAdd(descents, local);
}

void check_sorted(const void* keys, int64_t n, int key64, uint64_t* descents, int num_sms, cudaStream_t s)
{
    cudaMemsetAsync(descents, 0, sizeof(uint64_t), s);
    if (n <= 1)
        return;
    if (key64)
    {
        k_check_sorted<uint64_t><<<num_sms * 4, 256, 0, s>>>((const uint64_t*)keys, n, (unsigned long long*)descents);
        count_launch();
    }
    else
    {
        k_check_sorted<uint32_t><<<num_sms * 4, 256, 0, s>>>((const uint32_t*)keys, n, (unsigned long long*)descents);
        count_launch();
    }
}
} // namespace vox
