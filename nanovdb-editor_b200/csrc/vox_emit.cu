// vox_emit.cu - fragment test and (voxel key, Gaussian id) emission.
//
// Replaces the reference's per-window fan-out + gaussian_frag_alloc
// (raster/GridBuild.cpp:830-942, raster/shaders/gaussian_frag_alloc.slang).
// The candidate voxels of a Gaussian are the columns (i, j) of its bbox, each
// a run of k.  Work is tiled over the column index space (one column per
// thread) so every phase is uniform across a warp:
//   A  each thread bounds its column's k-range (column_interval, a
//      conservative bound that never drops a passing voxel);
//   B  a block scan flattens the bounded candidates; rounds of one candidate
//      per thread run the reference test; passing pairs are compacted in
//      (Gaussian, i, j, k) order with ballots into a shared-memory stage;
//   C  the tile's pair count is published with a decoupled look-back and the
//      stage is written out.  Tiles whose bounded candidates exceed the stage
//      count first and test again while writing.
#include <cstdio>
#include <cuda_runtime.h>

#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

constexpr int EMIT_BLOCK = 256;
constexpr int EMIT_WARPS = EMIT_BLOCK / 32;
constexpr int EMIT_STAGE = 8192;

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
__device__ __forceinline__ K compact_key(const RankTables& T, uint32_t cloud, int32_t x, int32_t y, int32_t z)
{
    uint64_t rr = bit_rank(T.root_bits, T.root_prefix, root_index(cloud, x, y, z));
    uint64_t cell = rr * 32768ull + upper_n_of(x, y, z);
    uint64_t lr = bit_rank(T.lower_bits, T.lower_prefix, cell);
    return (K)((lr << 21) | ((uint64_t)lower_n_of(x, y, z) << 9) | (uint64_t)leaf_n_of(x, y, z));
}

template <class K>
struct EmitSmem
{
    K stage_k[EMIT_STAGE];
    uint32_t stage_i[EMIT_STAGE];
    uint32_t col_g[EMIT_BLOCK];
    int32_t col_i[EMIT_BLOCK], col_j[EMIT_BLOCK], col_klo[EMIT_BLOCK];
    int32_t col_blo[EMIT_BLOCK], col_bhi[EMIT_BLOCK]; // bound, for CHECK
    uint32_t col_pre[EMIT_BLOCK + 1];
    uint32_t warp_cnt[EMIT_WARPS];
    uint64_t s_warp[33];
    uint64_t gofs;
    int64_t g_lo, g_hi;
    uint32_t tile;
};

// candidate e of the tile -> column (last column whose prefix is <= e)
__device__ __forceinline__ int find_column(const uint32_t* pre, uint32_t e)
{
    int lo = 0, hi = EMIT_BLOCK;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (pre[mid] <= e)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo - 1;
}

// runs the reference test on candidate e; returns pass and the pair
template <class K, bool CHECK>
__device__ __forceinline__ bool test_candidate(const EmitParams& E, const RankTables& T, EmitSmem<K>& S, uint32_t e,
                                               K& key, uint32_t& gid)
{
    const int col = find_column(S.col_pre, e);
    const int32_t k = S.col_klo[col] + (int32_t)(e - S.col_pre[col]);
    const int32_t i = S.col_i[col], j = S.col_j[col];
    gid = S.col_g[col];
    const GaussRec R = E.recs[gid];
    const RInv M = rinv_of(R);
    const bool pass = aabb_hits_unit_sphere(voxel_local_aabb(R, M, rec_vs(R, E.voxel_size, E.cloud_vs), i, j, k));
    if (CHECK && pass && (k < S.col_blo[col] || k > S.col_bhi[col]))
        atomicOr(E.err, ERR_BOUNDS); // the column bound would have dropped a passing voxel
    if (pass)
        key = compact_key<K>(T, rec_cloud(R), i, j, k);
    return pass;
}

// CHECK = true tests every voxel of every column and flags ERR_BOUNDS if one
// outside the column bound passes (validation runs, VOX_CHECK_EMIT=1)
template <class K, bool CHECK>
__global__ void __launch_bounds__(EMIT_BLOCK) k_emit(EmitParams E, RankTables T, K* __restrict__ out_k,
                                                       uint32_t* __restrict__ out_i)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    EmitSmem<K>& S = *reinterpret_cast<EmitSmem<K>*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint64_t NC = E.NC;
    const int64_t ntiles = (int64_t)((NC + EMIT_BLOCK - 1) / EMIT_BLOCK);
    while (true)
    {
        if (threadIdx.x == 0)
        {
            uint32_t t = atomicAdd(E.counter, 1u);
            S.tile = t;
            if ((int64_t)t < ntiles)
            {
                uint64_t c0 = (uint64_t)t * EMIT_BLOCK;
                uint64_t c1 = min(c0 + EMIT_BLOCK, NC) - 1;
                S.g_lo = upper_bound_u64(E.col_off, 0, E.G, c0) - 1;
                S.g_hi = upper_bound_u64(E.col_off, S.g_lo, E.G, c1);
            }
        }
        __syncthreads();
        const int64_t tile = S.tile;
        if (tile >= ntiles)
            break;

        // ---- A: bound one column per thread
        const uint64_t c = (uint64_t)tile * EMIT_BLOCK + threadIdx.x;
        uint32_t m = 0;
        if (c < NC)
        {
            const int64_t g = upper_bound_u64(E.col_off, S.g_lo, S.g_hi, c) - 1;
            const GaussRec R = E.recs[g];
            const RInv M = rinv_of(R);
            const uint32_t lc = (uint32_t)(c - E.col_off[g]);
            const int32_t i = R.q4.x + (int32_t)(lc / (uint32_t)R.q5.y);
            const int32_t j = R.q4.y + (int32_t)(lc % (uint32_t)R.q5.y);
            int32_t klo, khi;
            column_interval(R, M, rec_vs(R, E.voxel_size, E.cloud_vs), i, j, klo, khi);
            S.col_g[threadIdx.x] = (uint32_t)g;
            S.col_i[threadIdx.x] = i;
            S.col_j[threadIdx.x] = j;
            if (CHECK)
            {
                S.col_blo[threadIdx.x] = klo;
                S.col_bhi[threadIdx.x] = khi;
                klo = R.q4.z;
                khi = R.q4.z + R.q5.z - 1;
            }
            S.col_klo[threadIdx.x] = klo;
            m = klo <= khi ? (uint32_t)(khi - klo + 1) : 0u;
        }
        uint64_t mtot;
        const uint64_t mex = block_excl_scan_u64(m, S.s_warp, mtot);
        S.col_pre[threadIdx.x] = (uint32_t)mex;
        if (threadIdx.x == 0)
            S.col_pre[EMIT_BLOCK] = (uint32_t)mtot;
        __syncthreads();
        const uint32_t Mt = (uint32_t)mtot;

        // ---- B + C
        uint32_t npass = 0;
        if (Mt <= EMIT_STAGE)
        {
            for (uint32_t base = 0; base < Mt; base += EMIT_BLOCK)
            {
                const uint32_t e = base + threadIdx.x;
                K key = 0;
                uint32_t gid = 0;
                const bool pass = e < Mt && test_candidate<K, CHECK>(E, T, S, e, key, gid);
                const uint32_t bal = __ballot_sync(0xffffffffu, pass);
                if (lane == 0)
                    S.warp_cnt[warp] = __popc(bal);
                __syncthreads();
                uint32_t wpre = 0, rtot = 0;
                for (int w = 0; w < EMIT_WARPS; w++)
                {
                    const uint32_t x = S.warp_cnt[w];
                    wpre += w < warp ? x : 0u;
                    rtot += x;
                }
                if (pass)
                {
                    const uint32_t pos = npass + wpre + __popc(bal & lt);
                    S.stage_k[pos] = key;
                    S.stage_i[pos] = gid;
                }
                npass += rtot;
                __syncthreads();
            }
            if (threadIdx.x == 0)
                S.gofs = lookback_exclusive(E.status, (uint64_t)tile, npass, E.epoch, E.err);
            __syncthreads();
            const uint64_t gofs = S.gofs;
            for (uint32_t q = threadIdx.x; q < npass; q += EMIT_BLOCK)
            {
                const uint64_t dst = gofs + q;
                if (dst < E.cap)
                {
                    out_k[dst] = S.stage_k[q];
                    out_i[dst] = S.stage_i[q];
                }
            }
        }
        else
        {
            // more bounded candidates than the stage holds: count, publish, test again and write
            for (uint32_t base = 0; base < Mt; base += EMIT_BLOCK)
            {
                const uint32_t e = base + threadIdx.x;
                K key = 0;
                uint32_t gid = 0;
                const bool pass = e < Mt && test_candidate<K, false>(E, T, S, e, key, gid);
                npass += __popc(__ballot_sync(0xffffffffu, pass)); // per warp
            }
            if (lane == 0)
                S.warp_cnt[warp] = npass;
            __syncthreads();
            uint32_t tot = 0;
            for (int w = 0; w < EMIT_WARPS; w++)
                tot += S.warp_cnt[w];
            if (threadIdx.x == 0)
                S.gofs = lookback_exclusive(E.status, (uint64_t)tile, tot, E.epoch, E.err);
            __syncthreads();
            uint64_t run = S.gofs;
            npass = tot;
            for (uint32_t base = 0; base < Mt; base += EMIT_BLOCK)
            {
                const uint32_t e = base + threadIdx.x;
                K key = 0;
                uint32_t gid = 0;
                const bool pass = e < Mt && test_candidate<K, CHECK>(E, T, S, e, key, gid);
                const uint32_t bal = __ballot_sync(0xffffffffu, pass);
                if (lane == 0)
                    S.warp_cnt[warp] = __popc(bal);
                __syncthreads();
                uint32_t wpre = 0, rtot = 0;
                for (int w = 0; w < EMIT_WARPS; w++)
                {
                    const uint32_t x = S.warp_cnt[w];
                    wpre += w < warp ? x : 0u;
                    rtot += x;
                }
                if (pass)
                {
                    const uint64_t dst = run + wpre + __popc(bal & lt);
                    if (dst < E.cap)
                    {
                        out_k[dst] = key;
                        out_i[dst] = gid;
                    }
                }
                run += rtot;
                __syncthreads();
            }
        }
        if (threadIdx.x == 0 && tile == ntiles - 1)
        {
            const uint64_t total = S.gofs + npass;
            *E.total = total;
            if (total > E.cap)
                atomicOr(E.err, ERR_CAPACITY);
        }
        __syncthreads();
    }
}

template <class K>
static void launch_emit_t(const EmitParams& E, const RankTables& T, K* out_k, uint32_t* out_i, int num_sms,
                          cudaStream_t s)
{
    if (E.NC == 0)
    {
        cudaMemsetAsync(E.total, 0, sizeof(uint64_t), s);
        return;
    }
    const size_t smem = sizeof(EmitSmem<K>);
    auto kern = E.check ? k_emit<K, true> : k_emit<K, false>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, EMIT_BLOCK, smem);
    if (per_sm < 1)
        per_sm = 1;
    int64_t tiles = (int64_t)((E.NC + EMIT_BLOCK - 1) / EMIT_BLOCK);
    int64_t grid = (int64_t)num_sms * per_sm;
    if (grid > tiles)
        grid = tiles;
    cudaMemsetAsync(E.counter, 0, sizeof(uint32_t), s);
    { kern<<<(unsigned)grid, EMIT_BLOCK, smem, s>>>(E, T, out_k, out_i); count_launch(); }
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
int64_t emit_tile_count(uint64_t NC)
{
    return (int64_t)((NC + EMIT_BLOCK - 1) / EMIT_BLOCK);
}

} // namespace vox
