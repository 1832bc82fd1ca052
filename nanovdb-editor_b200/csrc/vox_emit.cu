// vox_emit.cu - fragment test and (voxel key, Gaussian id) emission.
//
// Replaces the reference's per-window fan-out + gaussian_frag_alloc
// (raster/GridBuild.cpp:830-942, raster/shaders/gaussian_frag_alloc.slang).
// The candidate voxels of a Gaussian are the columns (i, j) of its bbox, each
// a run of k.  Work is tiled over the column index space (one column per
// thread) so every phase is uniform across a warp:
//   A  each thread bounds its column's k-range (column_interval, a
//      conservative bound that never drops a passing voxel) and stages the
//      column's share of the reference test in shared memory: by the
//      monotone-corner identity the local AABB of voxel (i, j, k) is
//      fl(fl(S_xy + z_term) * inv_ls) * inv_s per axis, where S_xy (the
//      rounded sum of the x and y corner products) depends on the column only;
//   B  a block scan flattens the bounded candidates; a byte map sends each
//      candidate to its column; every warp tests a contiguous slice of the
//      candidates and compacts the passing pairs into its own stage slice with
//      ballots, in (Gaussian, i, j, k) order;
//   C  the tile's pair count is published with a decoupled look-back and the
//      warps copy their slices out.  Tiles with more bounded candidates than
//      the stage holds count first, publish, and test again while writing.
#include <cstdio>
#include <cuda_runtime.h>

#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

constexpr int EMIT_BLOCK = 256;
constexpr int EMIT_WARPS = EMIT_BLOCK / 32;
constexpr int EMIT_STAGE = 4096;
constexpr uint32_t EMIT_FAST_MAX = EMIT_STAGE - EMIT_BLOCK; // per-warp slices rounded to 32 stay inside

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
struct EmitSmem
{
    K stage_k[EMIT_STAGE];
    uint32_t stage_i[EMIT_STAGE];
    uint8_t cand_col[EMIT_STAGE]; // candidate -> column (fast path)
    // per column: the column's share of the reference test
    float sxy_lo[3][EMIT_BLOCK], sxy_hi[3][EMIT_BLOCK];
    float mz[3][EMIT_BLOCK];    // rinv[r][2]
    float inv_s[3][EMIT_BLOCK]; // 1 / s_r
    float inv_ls[EMIT_BLOCK], posz[EMIT_BLOCK], vs[EMIT_BLOCK];
    uint32_t col_g[EMIT_BLOCK], col_cloud[EMIT_BLOCK];
    int32_t col_i[EMIT_BLOCK], col_j[EMIT_BLOCK], col_klo[EMIT_BLOCK];
    int32_t col_kb[EMIT_BLOCK];  // 128-voxel block of col_klo
    uint32_t col_lr[EMIT_BLOCK]; // lower rank of (i, j, col_klo)
    int32_t col_blo[EMIT_BLOCK], col_bhi[EMIT_BLOCK]; // bound, for CHECK
    uint32_t col_pre[EMIT_BLOCK + 1];
    uint32_t warp_cnt[EMIT_WARPS], warp_pre[EMIT_WARPS];
    uint64_t s_warp[33];
    uint64_t gofs;
    int64_t g_lo, g_hi;
    uint32_t tile, tile_total;
};

__device__ __forceinline__ uint32_t lower_rank_of(const RankTables& T, uint32_t cloud, int32_t x, int32_t y, int32_t z)
{
    const uint64_t rr = bit_rank(T.root_bits, T.root_prefix, root_index(cloud, x, y, z));
    const uint64_t cell = rr * 32768ull + upper_n_of(x, y, z);
    return (uint32_t)bit_rank(T.lower_bits, T.lower_prefix, cell);
}

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

// the reference test (gaussian_frag_alloc.slang:84-162) of voxel k of column c,
// bit-identical to voxel_local_aabb + aabb_hits_unit_sphere
template <class K>
__device__ __forceinline__ bool column_test(const EmitSmem<K>& S, int c, int32_t k)
{
    const float vsf = S.vs[c], pos = S.posz[c];
    const float v0 = (float)k;
    const float v1 = VOX_FADD(v0, 1.f);
    const float c0 = VOX_FSUB(VOX_FMUL(v0, vsf), pos);
    const float c1 = VOX_FSUB(VOX_FMUL(v1, vsf), pos);
    const float il = S.inv_ls[c];
    float d2 = 1.f;
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        float zn, zx;
        minmax_prod(c0, c1, S.mz[r][c], zn, zx);
        const float lo = VOX_FMUL(VOX_FMUL(VOX_FADD(S.sxy_lo[r][c], zn), il), S.inv_s[r][c]);
        const float hi = VOX_FMUL(VOX_FMUL(VOX_FADD(S.sxy_hi[r][c], zx), il), S.inv_s[r][c]);
        if (0.f < lo)
            d2 = VOX_FSUB(d2, VOX_FMUL(lo, lo));
        else if (0.f > hi)
            d2 = VOX_FSUB(d2, VOX_FMUL(hi, hi));
    }
    return d2 > 0.f;
}

// runs the test on candidate e of column c; returns pass and the pair
template <class K, bool CHECK>
__device__ __forceinline__ bool test_candidate(const RankTables& T, const EmitSmem<K>& S, int c, uint32_t e, K& key,
                                               uint32_t& gid, int* err)
{
    const int32_t k = S.col_klo[c] + (int32_t)(e - S.col_pre[c]);
    const bool pass = column_test<K>(S, c, k);
    if (CHECK && pass && (k < S.col_blo[c] || k > S.col_bhi[c]))
        atomicOr(err, ERR_BOUNDS); // the column bound would have dropped a passing voxel
    if (pass)
    {
        const int32_t i = S.col_i[c], j = S.col_j[c];
        gid = S.col_g[c];
        const uint32_t lr = (k >> 7) == S.col_kb[c] ? S.col_lr[c] : lower_rank_of(T, S.col_cloud[c], i, j, k);
        key = (K)(((uint64_t)lr << 21) | ((uint64_t)lower_n_of(i, j, k) << 9) | (uint64_t)leaf_n_of(i, j, k));
    }
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

        // ---- A: bound and stage one column per thread
        const int c = threadIdx.x;
        const uint64_t cg = (uint64_t)tile * EMIT_BLOCK + c;
        uint32_t m = 0;
        if (cg < NC)
        {
            const int64_t g = upper_bound_u64(E.col_off, S.g_lo, S.g_hi, cg) - 1;
            const GaussRec R = E.recs[g];
            const RInv M = rinv_of(R);
            const float vsf = rec_vs(R, E.voxel_size, E.cloud_vs);
            const uint32_t lc = (uint32_t)(cg - E.col_off[g]);
            const int32_t i = R.q4.x + (int32_t)(lc / (uint32_t)R.q5.y);
            const int32_t j = R.q4.y + (int32_t)(lc % (uint32_t)R.q5.y);
            int32_t klo, khi;
            column_interval(R, M, vsf, i, j, klo, khi);
            float cx0, cx1, cy0, cy1;
            axis_corners(vsf, R.q0.x, i, cx0, cx1);
            axis_corners(vsf, R.q0.y, j, cy0, cy1);
            const float is[3] = { R.q3.y, R.q3.z, R.q3.w };
#pragma unroll
            for (int r = 0; r < 3; r++)
            {
                float xn, xx, yn, yx;
                minmax_prod(cx0, cx1, M.m[r][0], xn, xx);
                minmax_prod(cy0, cy1, M.m[r][1], yn, yx);
                S.sxy_lo[r][c] = VOX_FADD(xn, yn);
                S.sxy_hi[r][c] = VOX_FADD(xx, yx);
                S.mz[r][c] = M.m[r][2];
                S.inv_s[r][c] = is[r];
            }
            S.inv_ls[c] = R.q0.w;
            S.posz[c] = R.q0.z;
            S.vs[c] = vsf;
            S.col_g[c] = (uint32_t)g;
            S.col_cloud[c] = rec_cloud(R);
            S.col_i[c] = i;
            S.col_j[c] = j;
            if (CHECK)
            {
                S.col_blo[c] = klo;
                S.col_bhi[c] = khi;
                klo = R.q4.z;
                khi = R.q4.z + R.q5.z - 1;
            }
            S.col_klo[c] = klo;
            m = klo <= khi ? (uint32_t)(khi - klo + 1) : 0u;
            S.col_kb[c] = klo >> 7;
            S.col_lr[c] = m ? lower_rank_of(T, rec_cloud(R), i, j, klo) : 0u;
        }
        uint64_t mtot;
        const uint64_t mex = block_excl_scan_u64(m, S.s_warp, mtot);
        S.col_pre[c] = (uint32_t)mex;
        if (c == 0)
            S.col_pre[EMIT_BLOCK] = (uint32_t)mtot;
        const uint32_t Mt = (uint32_t)mtot;
        if (Mt <= EMIT_FAST_MAX)
            for (uint32_t q = 0; q < m; q++)
                S.cand_col[mex + q] = (uint8_t)c;
        __syncthreads();

        // ---- B + C
        uint32_t npass = 0;
        if (Mt <= EMIT_FAST_MAX)
        {
            // warp w tests candidates [e0, e0 + chunk) into stage slice [e0, ...)
            const uint32_t chunk = (Mt + EMIT_BLOCK - 1) / EMIT_BLOCK * 32;
            const uint32_t e0 = warp * chunk, e1 = min(Mt, e0 + chunk);
            uint32_t wcount = 0;
            for (uint32_t base = e0; base < e1; base += 32)
            {
                const uint32_t e = base + lane;
                K key = 0;
                uint32_t gid = 0;
                const bool pass = e < e1 && test_candidate<K, CHECK>(T, S, S.cand_col[e], e, key, gid, E.err);
                const uint32_t bal = __ballot_sync(0xffffffffu, pass);
                if (pass)
                {
                    const uint32_t pos = e0 + wcount + __popc(bal & lt);
                    S.stage_k[pos] = key;
                    S.stage_i[pos] = gid;
                }
                wcount += __popc(bal);
            }
            if (lane == 0)
                S.warp_cnt[warp] = wcount;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                uint32_t run = 0;
                for (int w = 0; w < EMIT_WARPS; w++)
                {
                    S.warp_pre[w] = run;
                    run += S.warp_cnt[w];
                }
                S.tile_total = run;
                S.gofs = lookback_exclusive(E.status, (uint64_t)tile, run, E.epoch, E.err);
            }
            __syncthreads();
            npass = S.tile_total;
            const uint64_t gofs = S.gofs + S.warp_pre[warp];
            const uint32_t cnt = S.warp_cnt[warp];
            for (uint32_t q = lane; q < cnt; q += 32)
            {
                const uint64_t dst = gofs + q;
                if (dst < E.cap)
                {
                    out_k[dst] = S.stage_k[e0 + q];
                    out_i[dst] = S.stage_i[e0 + q];
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
                const bool pass =
                    e < Mt && test_candidate<K, false>(T, S, find_column(S.col_pre, e), e, key, gid, E.err);
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
                const bool pass =
                    e < Mt && test_candidate<K, CHECK>(T, S, find_column(S.col_pre, e), e, key, gid, E.err);
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
