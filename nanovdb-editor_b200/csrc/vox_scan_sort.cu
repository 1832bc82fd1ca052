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

size_t scan_status_words(int64_t n)
{
    return (size_t)((n + SCAN_TILE - 1) / SCAN_TILE) + 1;
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
        if (mode == 1)
            x = (uint64_t)__popcll(x);
        v[i] = x;
        sum += x;
    }
    uint64_t block_total;
    uint64_t texcl = block_excl_scan_u64(sum, s_warp, block_total);
    if (threadIdx.x == 0)
        s_excl = lookback_exclusive(status, tile, block_total, epoch, err);
    __syncthreads();
    uint64_t run = s_excl + texcl;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        int64_t idx = base + i;
        if (idx < n)
        {
            out[idx] = run;
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

// ===================================================================== sort
// Tile: SORT_BLOCK threads x SORT_ITEMS keys.  Keys are processed in
// portions of at most 2^29 keys so that 32-bit look-back words (2 flag bits,
// 30-bit count) never overflow; each portion's digit bases come from the
// up-front histogram pass.
constexpr int SORT_BLOCK = 512;
constexpr int SORT_WARPS = SORT_BLOCK / 32;
constexpr int SORT_ITEMS = 16;
constexpr int SORT_TILE = SORT_BLOCK * SORT_ITEMS;
constexpr int SORT_TILES_PER_PORTION = 1 << 16;
constexpr int64_t SORT_PORTION = (int64_t)SORT_TILE * SORT_TILES_PER_PORTION; // 2^29
constexpr int SORT_MAX_PASSES = 8;
constexpr uint32_t ST_AGG = 1u << 30;
constexpr uint32_t ST_INCL = 2u << 30;
constexpr uint32_t ST_VAL = (1u << 30) - 1u;

struct SortWs
{
    uint32_t* hist;      // [portions][passes][256]
    uint64_t* base;      // [portions][passes][256]
    uint32_t* status;    // [tiles][256]
    uint32_t* counters;  // [passes]
    int64_t tiles, portions;
};

static size_t align256(size_t x)
{
    return (x + 255) / 256 * 256;
}

static SortWs carve(void* ws, int64_t n)
{
    SortWs w;
    w.tiles = (n + SORT_TILE - 1) / SORT_TILE;
    w.portions = (n + SORT_PORTION - 1) / SORT_PORTION;
    if (w.portions < 1)
        w.portions = 1;
    char* p = (char*)ws;
    w.hist = (uint32_t*)p;
    p += align256(sizeof(uint32_t) * w.portions * SORT_MAX_PASSES * 256);
    w.base = (uint64_t*)p;
    p += align256(sizeof(uint64_t) * w.portions * SORT_MAX_PASSES * 256);
    w.counters = (uint32_t*)p;
    p += align256(sizeof(uint32_t) * SORT_MAX_PASSES);
    w.status = (uint32_t*)p;
    return w;
}

size_t sort_workspace_bytes(int64_t n, int key_bytes)
{
    (void)key_bytes;
    int64_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
    int64_t portions = (n + SORT_PORTION - 1) / SORT_PORTION;
    if (portions < 1)
        portions = 1;
    return align256(sizeof(uint32_t) * portions * SORT_MAX_PASSES * 256) +
           align256(sizeof(uint64_t) * portions * SORT_MAX_PASSES * 256) + align256(sizeof(uint32_t) * SORT_MAX_PASSES) +
           align256(sizeof(uint32_t) * (tiles + 1) * 256);
}

template <class K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift, uint32_t mask)
{
    return (uint32_t)(k >> shift) & mask;
}

// up-front histogram of every pass's digit, per portion
template <class K>
__global__ void __launch_bounds__(SORT_BLOCK) k_sort_hist(const K* keys, int64_t n, int passes, int bits,
                                                            uint32_t* hist)
{
    __shared__ uint32_t s_h[SORT_MAX_PASSES * 256];
    const uint32_t mask = (1u << bits) - 1u;
    for (int i = threadIdx.x; i < SORT_MAX_PASSES * 256; i += blockDim.x)
        s_h[i] = 0;
    __syncthreads();
    int64_t cur_portion = -1;
    const int64_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x)
    {
        int64_t portion = t / SORT_TILES_PER_PORTION;
        if (portion != cur_portion)
        {
            __syncthreads();
            if (cur_portion >= 0)
            {
                for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
                {
                    if (s_h[i])
                        atomicAdd(&hist[cur_portion * SORT_MAX_PASSES * 256 + i], s_h[i]);
                    s_h[i] = 0;
                }
            }
            cur_portion = portion;
            __syncthreads();
        }
        int64_t b = t * SORT_TILE;
        for (int i = threadIdx.x; i < SORT_TILE; i += blockDim.x)
        {
            int64_t idx = b + i;
            if (idx < n)
            {
                K k = keys[idx];
                for (int p = 0; p < passes; p++)
                    atomicAdd(&s_h[p * 256 + digit_of(k, p * bits, mask)], 1u);
            }
        }
    }
    __syncthreads();
    if (cur_portion >= 0)
        for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
            if (s_h[i])
                atomicAdd(&hist[cur_portion * SORT_MAX_PASSES * 256 + i], s_h[i]);
}

// base[portion][pass][d] = sum_{d' < d} total[pass][d'] + sum_{p' < portion} hist[p'][pass][d]
__global__ void k_sort_bases(const uint32_t* hist, uint64_t* base, int64_t portions, int passes)
{
    __shared__ uint64_t s_warp[33];
    const int d = threadIdx.x; // 256 threads
    for (int p = 0; p < passes; p++)
    {
        uint64_t tot = 0;
        for (int64_t q = 0; q < portions; q++)
            tot += hist[q * SORT_MAX_PASSES * 256 + p * 256 + d];
        uint64_t all;
        uint64_t excl = block_excl_scan_u64(tot, s_warp, all);
        uint64_t run = excl;
        for (int64_t q = 0; q < portions; q++)
        {
            base[q * SORT_MAX_PASSES * 256 + p * 256 + d] = run;
            run += hist[q * SORT_MAX_PASSES * 256 + p * 256 + d];
        }
    }
}

__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <class K>
struct SortSmem
{
    K keys[SORT_TILE];
    uint32_t vals[SORT_TILE];
    uint32_t warp_hist[SORT_WARPS][256];
    uint32_t digit_excl[256];
    uint64_t gbase[256];
    uint64_t s_warp[33];
    uint32_t tile;
};

template <class K>
__global__ void __launch_bounds__(SORT_BLOCK) k_onesweep(const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                                           K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                           int64_t n, int shift, int bits, const uint64_t* base,
                                                           int pass, uint32_t* status, uint32_t* counter, int* err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<K>& S = *reinterpret_cast<SortSmem<K>*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t mask = (1u << bits) - 1u;
    const int radix = 1 << bits;

    if (threadIdx.x == 0)
        S.tile = atomicAdd(counter, 1u);
    for (int i = lane; i < 256; i += 32)
        S.warp_hist[warp][i] = 0;
    __syncthreads();
    const int64_t tile = S.tile;
    const int64_t tile_base = tile * SORT_TILE;
    const int64_t portion = tile / SORT_TILES_PER_PORTION;
    const int64_t ptile = tile % SORT_TILES_PER_PORTION;
    const int tile_count = (int)min((int64_t)SORT_TILE, n - tile_base);

    // load: warp-contiguous chunks, item-major within a warp (stable order = (item, lane))
    K k[SORT_ITEMS];
    uint32_t v[SORT_ITEMS];
    uint32_t rank[SORT_ITEMS];
    const int64_t wbase = tile_base + (int64_t)warp * (32 * SORT_ITEMS);
#pragma unroll
    for (int i = 0; i < SORT_ITEMS; i++)
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
    for (int i = 0; i < SORT_ITEMS; i++)
    {
        int64_t idx = wbase + i * 32 + lane;
        bool valid = idx < n;
        uint32_t d = valid ? digit_of(k[i], shift, mask) : 0xFFFFu;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = __popc(peers & lt);
        uint32_t leader = __ffs(peers) - 1;
        uint32_t prev = valid ? S.warp_hist[warp][d] : 0u;
        __syncwarp();
        if (valid && (uint32_t)lane == leader)
            S.warp_hist[warp][d] = prev + __popc(peers);
        __syncwarp();
        rank[i] = prev + before;
    }
    __syncthreads();

    // per digit: exclusive over warps, tile total, exclusive over digits
    uint64_t total = 0;
    if (threadIdx.x < 256)
    {
        uint32_t run = 0;
        for (int w = 0; w < SORT_WARPS; w++)
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
        uint64_t excl = 0;
        if (d < radix)
        {
            uint32_t* st = status + (size_t)tile * 256 + d;
            if (ptile == 0)
            {
                st_release_u32(st, ST_INCL | ((uint32_t)total & ST_VAL));
            }
            else
            {
                st_release_u32(st, ST_AGG | ((uint32_t)total & ST_VAL));
                int64_t p = tile - 1;
                const int64_t pfirst = portion * SORT_TILES_PER_PORTION;
                uint32_t spins = 0;
                while (p >= pfirst)
                {
                    uint32_t sv = ld_acquire_u32(status + (size_t)p * 256 + d);
                    uint32_t flag = sv & ~ST_VAL;
                    if (flag == 0)
                    {
                        if (++spins > LB_SPIN_LIMIT)
                        {
                            atomicExch(err, ERR_LOOKBACK);
                            break;
                        }
                        __nanosleep(20);
                        continue;
                    }
                    excl += sv & ST_VAL;
                    if (flag == ST_INCL)
                        break;
                    p--;
                }
                st_release_u32(st, ST_INCL | ((uint32_t)(excl + total) & ST_VAL));
            }
            S.gbase[d] = base[portion * SORT_MAX_PASSES * 256 + pass * 256 + d] + excl - dexcl;
        }
    }
    __syncthreads();

    // scatter into shared memory in digit order
#pragma unroll
    for (int i = 0; i < SORT_ITEMS; i++)
    {
        int64_t idx = wbase + i * 32 + lane;
        if (idx < n)
        {
            uint32_t d = digit_of(k[i], shift, mask);
            uint32_t pos = S.digit_excl[d] + S.warp_hist[warp][d] + rank[i];
            S.keys[pos] = k[i];
            S.vals[pos] = v[i];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tile_count; i += SORT_BLOCK)
    {
        K kk = S.keys[i];
        uint32_t d = digit_of(kk, shift, mask);
        uint64_t dst = S.gbase[d] + (uint64_t)i;
        keys_out[dst] = kk;
        vals_out[dst] = S.vals[i];
    }
}

template <class K>
static int sort_pairs_impl(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, int64_t n, int key_bits,
                           void* workspace, int* err, int num_sms, cudaStream_t s, const SortTuning& tune)
{
    if (n <= 1 || key_bits <= 0)
        return 0;
    const int bits = tune.digit_bits < 1 ? 8 : (tune.digit_bits > 8 ? 8 : tune.digit_bits);
    int passes = (key_bits + bits - 1) / bits;
    if (passes > SORT_MAX_PASSES)
        passes = SORT_MAX_PASSES;
    SortWs w = carve(workspace, n);
    cudaMemsetAsync(w.hist, 0, sizeof(uint32_t) * w.portions * SORT_MAX_PASSES * 256, s);
    cudaMemsetAsync(w.counters, 0, sizeof(uint32_t) * SORT_MAX_PASSES, s);
    int hist_grid = num_sms * 2;
    if ((int64_t)hist_grid > w.tiles)
        hist_grid = (int)w.tiles;
    { k_sort_hist<K><<<hist_grid, SORT_BLOCK, 0, s>>>(keys, n, passes, bits, w.hist); count_launch(); }
    { k_sort_bases<<<1, 256, 0, s>>>(w.hist, w.base, w.portions, passes); count_launch(); }
    const size_t smem = sizeof(SortSmem<K>);
    cudaFuncSetAttribute(k_onesweep<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    K* src_k = keys;
    uint32_t* src_v = vals;
    K* dst_k = keys_alt;
    uint32_t* dst_v = vals_alt;
    for (int p = 0; p < passes; p++)
    {
        cudaMemsetAsync(w.status, 0, sizeof(uint32_t) * (size_t)w.tiles * 256, s);
        { k_onesweep<K><<<(unsigned)w.tiles, SORT_BLOCK, smem, s>>>(src_k, src_v, dst_k, dst_v, n, p * bits, bits,
                                                                   w.base, p, w.status, w.counters + p, err); count_launch(); }
        K* tk = src_k;
        src_k = dst_k;
        dst_k = tk;
        uint32_t* tv = src_v;
        src_v = dst_v;
        dst_v = tv;
    }
    return (passes & 1) ? 1 : 0;
}

int sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, int64_t n, int key_bits,
                   void* workspace, int* err, int num_sms, cudaStream_t s, const SortTuning& tune)
{
    return sort_pairs_impl<uint32_t>(keys, vals, keys_alt, vals_alt, n, key_bits, workspace, err, num_sms, s, tune);
}
int sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, int64_t n, int key_bits,
                   void* workspace, int* err, int num_sms, cudaStream_t s, const SortTuning& tune)
{
    return sort_pairs_impl<uint64_t>(keys, vals, keys_alt, vals_alt, n, key_bits, workspace, err, num_sms, s, tune);
}

} // namespace vox
