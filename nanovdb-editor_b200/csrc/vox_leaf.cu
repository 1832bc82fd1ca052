// vox_leaf.cu - leaf-granular voxelization: (leaf, Gaussian) pairs, one CTA
// per candidate leaf.
//
// The reference tests every (voxel, Gaussian) fragment of a Gaussian's bbox in
// 8M-fragment windows and inserts passing voxels into its tree with atomics
// (raster/Raster.cpp:420-558, gaussian_frag_alloc.slang, grid_build_*.slang,
// gaussian_frag_color.slang).  Here the unit of sorting is the leaf (8^3
// voxels, the node2 leaf of PNanoVDBExt.h:72-81):
//   k_leaf_cols / k_leaf_emit   per Gaussian, the leaf cells of its bbox whose
//       box may reach its 0.01-opacity ellipsoid (a conservative test in
//       double), written as (leaf key, emission index) in Gaussian-major
//       order; a stable sort by leaf key keeps each leaf's Gaussians in
//       ascending id;
//   k_leaf_heads / k_leaf_compact   runs of equal leaf keys -> candidate leaves;
//   k_leaf_pass   one CTA per candidate leaf, one thread per voxel (two per
//       thread): the CTA walks the leaf's Gaussians in ascending id and every
//       thread runs the reference test (gaussian_frag_alloc.slang:84-162) on
//       its voxels, keeps the RGBA8 maximum (gaussian_frag_color.slang:239-246)
//       and sums the float channels in (voxel key, Gaussian id) order; the
//       leaf's value mask comes from ballots;
//   k_leaf_popc / k_voxel_keys   active voxels as sorted compact keys, which
//       the run / node-table / node2-writer stage turns into the tree;
//   k_values      staged values to their value index.
// The adjoint (k_leaf_backward) and the sorted pair list (k_leaf_export)
// replay the same walk.
#include <cstdio>
#include <cuda_runtime.h>

#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

constexpr int LP_THREADS = 256; // two voxels per thread: leaf_n = t and t + 256
constexpr int LP_CHUNK = 32;    // Gaussian records staged in shared memory per round

__device__ __forceinline__ int64_t upper_bound_u64_l(const uint64_t* a, int64_t lo, int64_t hi, uint64_t v)
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

// ------------------------------------------------------------ emission ----
__global__ void k_leaf_cols(const GaussRec* recs, int64_t G, uint64_t* lcols)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G)
        return;
    const GaussRec R = recs[g];
    if (!R.q4.w)
    {
        lcols[g] = 0;
        return;
    }
    const int32_t lx0 = R.q4.x >> 3, lx1 = (R.q4.x + R.q5.x - 1) >> 3;
    const int32_t ly0 = R.q4.y >> 3, ly1 = (R.q4.y + R.q5.y - 1) >> 3;
    lcols[g] = (uint64_t)(lx1 - lx0 + 1) * (uint64_t)(ly1 - ly0 + 1);
}

// May a voxel of the leaf at origin o pass the reference test?  The local AABB
// of the leaf box (monotone-corner identity, in double) contains every voxel's
// local AABB; the float test's rounding is bounded by delta = 1e-5 (1 + B), B
// bounding the magnitudes it sums (a worst-case error bound of the float test
// is below 1.1e-6 B).
__device__ __forceinline__ bool leaf_may_hit(const GaussRec& R, const RInv& M, float vsf, int32_t ox, int32_t oy,
                                             int32_t oz)
{
    const double vs = vsf;
    const int32_t o[3] = { ox, oy, oz };
    const double mu[3] = { R.q0.x, R.q0.y, R.q0.z };
    const double inv_s[3] = { R.q3.y, R.q3.z, R.q3.w };
    double lo[3], hi[3], E[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const double w0 = (double)o[a] * vs, w1 = (double)(o[a] + 8) * vs;
        lo[a] = w0 - mu[a];
        hi[a] = w1 - mu[a];
        E[a] = fmax(fabs(w0), fabs(w1)) + fabs(mu[a]) + vs;
    }
    double sum = 0.0, B = 0.0;
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        const double sc = (double)R.q0.w * inv_s[r];
        double mn = 0.0, mx = 0.0, mag = 0.0;
#pragma unroll
        for (int a = 0; a < 3; a++)
        {
            const double m = (double)M.m[r][a];
            const double p0 = lo[a] * m, p1 = hi[a] * m;
            mn += fmin(p0, p1);
            mx += fmax(p0, p1);
            mag += fabs(m) * E[a];
        }
        mn *= sc;
        mx *= sc;
        const double d = mn > 0.0 ? mn : (mx < 0.0 ? -mx : 0.0);
        sum += d * d;
        B = fmax(B, mag * sc);
    }
    const double bound = 1.0 + 1e-5 * (1.0 + B);
    return sum < bound * bound;
}

__device__ __forceinline__ uint32_t leaf_key_of(const GaussRec& R, int32_t x, int32_t y, int32_t z,
                                                const uint64_t* root_bits, const uint64_t* root_prefix,
                                                const uint64_t* lower_bits, const uint64_t* lower_prefix)
{
    const uint64_t rr = bit_rank(root_bits, root_prefix, root_index(rec_cloud(R), x, y, z));
    const uint64_t cell = rr * 32768ull + upper_n_of(x, y, z);
    const uint64_t lr = bit_rank(lower_bits, lower_prefix, cell);
    return (uint32_t)((lr << 12) | lower_n_of(x, y, z));
}

// one thread per leaf column (lx, ly) of a Gaussian's bbox, looping over lz
// the Gaussian of each 256-column tile's first column
__global__ void k_tile_gauss(const uint64_t* lcol_off, int64_t G, uint64_t NLC, int64_t* tile_g0)
{
    const uint64_t tile = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tile * 256 < NLC)
        tile_g0[tile] = upper_bound_u64_l(lcol_off, 0, G, tile * 256) - 1;
}

// Blocks walk 256-column tiles; a tile's Gaussians [g0, g1] (g1 = the next
// tile's first) have their column offsets copied to shared memory, where each
// thread finds its column's Gaussian.
template <bool WRITE>
__global__ void __launch_bounds__(256) k_leaf_emit(LeafEmitParams P, RankTables T)
{
    __shared__ uint64_t s_off[257];
    const uint64_t ntiles = (P.NLC + 255) / 256;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int64_t g0 = P.tile_g0[tile];
        const int64_t g1 = tile + 1 < ntiles ? P.tile_g0[tile + 1] : P.G - 1;
        const int64_t n = g1 - g0 + 1;
        if (n <= 256 && (int64_t)threadIdx.x < n)
            s_off[threadIdx.x] = P.lcol_off[g0 + threadIdx.x];
        __syncthreads();
        const uint64_t t = tile * 256 + threadIdx.x;
        if (t < P.NLC)
        {
        int64_t g;
        if (n <= 256)
        {
            int64_t lo = 0, hi = n; // upper bound of t in s_off[0, n)
            while (lo < hi)
            {
                const int64_t mid = (lo + hi) >> 1;
                if (s_off[mid] <= t)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            g = g0 + lo - 1;
        }
        else
            g = upper_bound_u64_l(P.lcol_off, g0, g1 + 1, t) - 1;
        const GaussRec R = P.recs[g];
        const RInv M = rinv_of(R);
        const float vsf = rec_vs(R, P.voxel_size, P.cloud_vs);
        const int32_t lx0 = R.q4.x >> 3, ly0 = R.q4.y >> 3, ly1 = (R.q4.y + R.q5.y - 1) >> 3;
        const int32_t lz0 = R.q4.z >> 3, lz1 = (R.q4.z + R.q5.z - 1) >> 3;
        const uint32_t Ly = (uint32_t)(ly1 - ly0 + 1);
        const uint32_t local = (uint32_t)(t - P.lcol_off[g]);
        const int32_t ox = (lx0 + (int32_t)(local / Ly)) * 8, oy = (ly0 + (int32_t)(local % Ly)) * 8;
        uint64_t e = WRITE ? P.lc_off[t] : 0;
        uint64_t npairs = 0;
        // the write pass reuses the count pass's test results (first 32 leaves)
        const uint32_t known = WRITE ? P.lc_mask[t] : 0u;
        uint32_t mask = 0;
        for (int32_t lz = lz0; lz <= lz1; lz++)
        {
            const int32_t oz = lz * 8;
            const int32_t i = lz - lz0;
            const bool hit = (WRITE && i < 32) ? ((known >> i) & 1u) != 0u : leaf_may_hit(R, M, vsf, ox, oy, oz);
            if (!WRITE && hit && i < 32)
                mask |= 1u << i;
            if (hit || P.check)
            {
                if (WRITE)
                {
                    P.keys[e] = leaf_key_of(R, ox, oy, oz, T.root_bits, T.root_prefix, T.lower_bits, T.lower_prefix);
                    P.vals[e] = (uint32_t)e;
                    P.emit_gid[e] = (uint32_t)g;
                    if (P.check)
                        P.emit_flag[e] = hit ? 0 : 1;
                    e++;
                }
                npairs++;
            }
        }
        if (!WRITE)
        {
            P.lc_count[t] = npairs;
            P.lc_mask[t] = mask;
        }
        }
        __syncthreads();
    }
}

__global__ void k_leaf_heads(const uint32_t* keys, int64_t Q, uint64_t* flags)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Q)
        flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1ull : 0ull;
}

// origin of the leaf with compact key lower_rank << 12 | lower_n
__device__ __forceinline__ void leaf_origin_of_key(uint32_t key, const uint32_t* lower_cell,
                                                   const uint32_t* root_of_rank, int32_t o[3])
{
    const uint32_t lr = key >> 12, ln = key & 4095u;
    const uint32_t cell = lower_cell[lr];
    const uint32_t un = cell & 32767u;
    root_tile_origin(root_of_rank[cell >> 15] & 32767u, o);
    o[0] += (int32_t)((un >> 10) & 31) * 128 + (int32_t)((ln >> 8) & 15) * 8;
    o[1] += (int32_t)((un >> 5) & 31) * 128 + (int32_t)((ln >> 4) & 15) * 8;
    o[2] += (int32_t)(un & 31) * 128 + (int32_t)(ln & 15) * 8;
}

// candidate leaves (key, origin, first pair) from the run heads; each sorted pair's Gaussian id
__global__ void k_leaf_compact(const uint32_t* keys, const uint32_t* vals, const uint32_t* emit_gid, int64_t Q,
                               const uint64_t* flags, const uint64_t* pos, const uint32_t* lower_cell,
                               const uint32_t* root_of_rank, uint32_t* cand_key, int4* cand_org,
                               uint32_t* cand_start, uint32_t* pair_gid)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Q)
        return;
    pair_gid[i] = emit_gid[vals[i]];
    if (flags[i])
    {
        int32_t o[3];
        leaf_origin_of_key(keys[i], lower_cell, root_of_rank, o);
        cand_org[pos[i]] = make_int4(o[0], o[1], o[2], 0);
        cand_key[pos[i]] = keys[i];
        cand_start[pos[i]] = (uint32_t)i;
    }
    if (i == Q - 1)
        cand_start[pos[i] + flags[i]] = (uint32_t)Q;
}

// ------------------------------------------------------------ leaf walk ----
struct LeafSmem
{
    GaussRec rec[LP_CHUNK];
    uint32_t gid[LP_CHUNK];
    uint32_t eidx[LP_CHUNK];
    uint8_t flag[LP_CHUNK];
    uint64_t mask[8];
    float red[LP_THREADS / 32][BWD_NACC];
    uint32_t pairs;
    uint32_t cand;
};

__device__ __forceinline__ void cand_origin(const LeafPassParams& P, uint32_t key, int32_t o[3])
{
    leaf_origin_of_key(key, P.lower_cell, P.root_of_rank, o);
}

__device__ __forceinline__ bool in_bbox(const GaussRec& R, int32_t x, int32_t y, int32_t z)
{
    return (uint32_t)(x - R.q4.x) < (uint32_t)R.q5.x && (uint32_t)(y - R.q4.y) < (uint32_t)R.q5.y &&
           (uint32_t)(z - R.q4.z) < (uint32_t)R.q5.z;
}

// stage Gaussians [q0, q0 + cnt) of the sorted pair list
__device__ __forceinline__ void stage_chunk(const LeafPassParams& P, LeafSmem& S, uint32_t q0, uint32_t cnt)
{
    const int t = threadIdx.x;
    if (t < (int)cnt * 8)
    {
        const uint32_t j = (uint32_t)t >> 3, w = (uint32_t)t & 7u;
        const uint32_t e = P.vals[q0 + j];
        const uint32_t g = P.emit_gid[e];
        reinterpret_cast<float4*>(&S.rec[j])[w] = reinterpret_cast<const float4*>(&P.recs[g])[w];
        if (w == 0)
        {
            S.gid[j] = g;
            S.eidx[j] = e;
            S.flag[j] = P.emit_flag ? P.emit_flag[e] : 0;
        }
    }
}

// ------------------------------------------------------ forward leaf walk
// A CTA walks a stream of candidate leaves in chunks of LQ_CHUNK Gaussians
// (a leaf's Gaussians in ascending id).  Per chunk:
//   test   the part of each Gaussian's bbox inside the leaf, one (Gaussian,
//          column) per thread: the column's x / y share once, then its z run,
//          each z's corner products shared with the next; passing (Gaussian,
//          voxel) pairs go to a shared queue;
//   alpha  one queued pair per thread: the reference's RGBA8 alpha and the
//          float channels' stable alpha, accumulated per voxel with shared
//          atomics - RGBA8 maximum, pair count, 64-bit fixed-point density /
//          colour sums (exact, so independent of order);
//   flush  once a leaf's last alpha is done: its staged values, value mask
//          and pair count.
// One barrier per chunk: phase i runs the flush of the leaf that ended with
// chunk i - 2, the alpha of chunk i - 1, the test of chunk i, and the staging
// of chunk i + 1 (lanes of the last warp copy its records with cp.async and
// place its boxes).  Chunk data is triple-buffered, queues double-buffered,
// the per-voxel accumulators double-buffered by leaf parity.
constexpr int LQ_CHUNK = 12;
constexpr int LQ_STAGE_T0 = LP_THREADS - 32; // lanes 0..LQ_CHUNK-1 of the last warp stage the next chunk

// A record slot padded to 144 B: the same field of a chunk's 8 records falls in
// 8 different shared-memory banks (a 128 B stride puts them all in one).
struct RecSlot
{
    GaussRec r;
    float4 pad;
};

struct LeafChunk
{
    RecSlot rec[LQ_CHUNK];                               // first member: 16-byte aligned for cp.async
    int32_t bx0[LQ_CHUNK], by0[LQ_CHUNK], bz0[LQ_CHUNK]; // box origin, leaf-relative
    uint32_t bny[LQ_CHUNK], bnz[LQ_CHUNK];               // box extents in y and z
    uint32_t bdiv_y[LQ_CHUNK];                           // 65536 / ny, rounded up (exact division below 64)
    uint32_t bcol[LQ_CHUNK];                             // box columns, nx * ny (0: empty box)
    uint32_t rgb24[LQ_CHUNK];                            // the colour bytes of the packed RGBA8 value
    float vs[LQ_CHUNK];
    // leaf_pair_consts of each (leaf, Gaussian), by row
    float lo0[3][LQ_CHUNK], wid[3][LQ_CHUNK]; // the float channels' AABB of the leaf's voxel (0, 0, 0)
    float stp[3][3][LQ_CHUNK];                 // [r][a]: the scaled voxel steps ([r][2]: the z step of the test)
    float dab[3][LQ_CHUNK];                    // reference / float-channel AABB difference bound
    float lo_t[LQ_CHUNK], hi_t[LQ_CHUNK];      // the linear z classification's thresholds
    uint32_t anchor[LQ_CHUNK];                 // the float channels' anchor voxel (packed)
    uint32_t cstart[16];    // first column of box j (boxes past the chunk's count: empty); [LQ_CHUNK]: all
    uint8_t flag[LQ_CHUNK];
    uint64_t wf0[LQ_CHUNK], wbase[LQ_CHUNK]; // reference windows: fragment offset in its batch, windows before
};

struct LeafAcc
{
    unsigned long long dens[512];   // fixed-point sums
    unsigned long long col[3][512];
    uint32_t cnt[512];              // passing pairs
    uint32_t rgba[512];             // packed RGBA8 maximum
    unsigned long long wmin;        // creation window (reference node order)
};

struct LeafQSmem
{
    LeafChunk ch[3];
    LeafAcc acc[1];
    uint16_t queue[2][LQ_CHUNK * 512];
    uint16_t defer[LP_THREADS / 32][64]; // per warp: queued pairs whose RGBA8 byte the bound left open
    uint32_t dcount[LP_THREADS / 32];     // per warp: the open pairs left at the end of its alpha
    uint32_t dfin;                        // warps done with this phase's alpha
    uint32_t qn[3];
    int32_t nxt_o[2][3]; // the next chunk (by phase parity): leaf origin and sorted pair range
    uint32_t nxt_q0[2], nxt_p1[2];
    uint32_t cand_next[2];
    uint32_t cand;
    unsigned long long pairs;
};

// The reference test on the boxes of a chunk, one box column per thread, its
// passing (Gaussian, voxel) pairs appended to queue (entry j << 9 | leaf_n).
// Bit-identical to voxel_local_aabb + aabb_hits_unit_sphere per voxel: the z
// corner c1 of voxel z is c0 of voxel z + 1 (integer-valued floats), and "lo >
// 0: subtract lo^2, else hi < 0: subtract hi^2" selects the pre-scale bound
// with the same sign (inv_ls, inv_s > 0; an underflow to zero subtracts zero).
// Every thread of the CTA calls it (warp-synchronous queue slots).  PER_WARP:
// warp w appends to its own region queue[w * 512, ...) at warp-local
// positions and stores its count in qcount[w] - a deterministic order (a warp
// tests at most 2 x 32 columns of 8 voxels).  Otherwise one shared queue, a
// shared atomic per warp and round.
//
// APPROX (a LeafChunk, carrying the leaf_pair_consts of each Gaussian): each
// voxel of the column is first classified from the float channels' local AABB
// (stable_leaf_aabb: per column the x / y terms once, then one fma per row
// and voxel), and only voxels near the sphere run the reference test.  Per
// row that AABB is within delta_r = dab_r of the reference's
// (leaf_pair_consts), so the selected values (max(lo, min(hi, 0)),
// 1-Lipschitz in both bounds) differ by at most delta_r and the vectors of the
// three by eta <= Delta = sum delta_r in norm.  The reference passes a voxel
// when its fl-evaluated 1 - S > 0: surely if S < 1 - 2^-22 (three subtractions
// and squares of values below 1) and surely not if S > 1 + 2^-20.  With D the
// fma-summed squares of the float values (relative error <= 3 2^-24) and
// Delta <= 1/16, (sqrt(D) + eta)^2 < 1 - 2^-22 holds when D < lo_t = 1 -
// (2 Delta + 2^-19), and (sqrt(D) - eta)^2 > 1 + 2^-20 when D > hi_t = 1 +
// (2 Delta + Delta^2 + 2^-18) (the slack covers the roundings of the
// thresholds themselves).  Voxels with D in [lo_t, hi_t] (or NaN), and every
// voxel of a (leaf, Gaussian) with Delta > 1/16 (lo_t = -1, hi_t = inf), take
// the reference test.  In CHECK mode every voxel also takes it and a
// difference sets ERR_BOUNDS.
template <bool CHECK, bool PER_WARP = false, bool APPROX = false, class Chunk>
__device__ __forceinline__ void leaf_test_chunk(const LeafPassParams& P, const Chunk& C, uint32_t cnt,
                                                const int32_t o[3], uint16_t* queue, uint32_t* qcount, int t, int lane,
                                                uint32_t rot = 0)
{
    uint32_t wbase = 0; // PER_WARP: entries this warp has written
    if (PER_WARP)
        queue += (t >> 5) * (LQ_CHUNK * 64);
    uint32_t start[LQ_CHUNK + 1];
    uint32_t T;
    if constexpr (APPROX)
        T = C.cstart[LQ_CHUNK]; // the staged prefix (no registers held across the rounds)
    else
    {
        start[0] = 0;
#pragma unroll
        for (int j = 0; j < LQ_CHUNK; j++)
            start[j + 1] = start[j] + (j < (int)cnt ? C.bcol[j] : 0u);
        T = start[LQ_CHUNK];
    }
    // rounds of 32 columns dealt to the warps in turn, starting at warp rot (mod 8):
    // the forward continues the deal where the alpha's rounds of 32 pairs stopped,
    // so the warps' loads in a phase differ by at most one round
    const uint32_t first = (uint32_t)(((t >> 5) - (int)(rot & 7u)) & 7);
    for (uint32_t tu = first; tu * 32u < T; tu += LP_THREADS / 32)
    {
        const uint32_t e = tu * 32u + (uint32_t)lane;
        uint32_t zmask = 0, ebase = 0;
        if (e < T)
        {
            // j: the last box whose first column is <= e (empty boxes skipped); sj its first column
            int j = 0;
            uint32_t sj = 0;
            if constexpr (APPROX)
            {
#pragma unroll
                for (int s = 8; s; s >>= 1)
                    if (j + s < LQ_CHUNK && C.cstart[j + s] <= e)
                        j += s;
                sj = C.cstart[j];
            }
            else
            {
#pragma unroll
                for (int q = 1; q < LQ_CHUNK; q++) // without a dynamically indexed (local memory) array
                {
                    const bool ge = e >= start[q];
                    j += ge ? 1 : 0;
                    sj = ge ? start[q] : sj;
                }
            }
            const uint32_t local = e - sj;
            const uint32_t dx = (local * C.bdiv_y[j]) >> 16;
            const uint32_t dy = local - dx * C.bny[j];
            const int32_t rx = C.bx0[j] + (int32_t)dx, ry = C.by0[j] + (int32_t)dy, rz0 = C.bz0[j];
            const GaussRec& R = C.rec[j].r;
            const float vsf = C.vs[j];
            const uint32_t nz = C.bnz[j];
            if constexpr (APPROX)
            {
                // the float channels' AABB of the run's voxels (stable_leaf_aabb: the
                // column's x / y terms once, then one fma per row and voxel), within
                // delta_r of the reference's for every voxel of the leaf
                const uint32_t anc = C.anchor[j];
                const float tx = (float)(rx - (int32_t)(anc & 255u)), ty = (float)(ry - (int32_t)((anc >> 8) & 255u)),
                            tz0 = (float)(rz0 - (int32_t)(anc >> 16));
                float base[3], wid[3], st[3];
#pragma unroll
                for (int r = 0; r < 3; r++)
                {
                    base[r] = VOX_FFMA(ty, C.stp[r][1][j], VOX_FFMA(tx, C.stp[r][0][j], C.lo0[r][j]));
                    wid[r] = C.wid[r][j];
                    st[r] = C.stp[r][2][j];
                }
                const float lo_t = C.lo_t[j], hi_t = C.hi_t[j];
                uint32_t unc = 0;
                {
                    float kf = tz0;
#pragma unroll 1 // measured: unrolling by 2, 4 or 8 is slower
                    for (uint32_t k = 0; k < nz; k++, kf += 1.f)
                    {
                        float D = 0.f;
#pragma unroll
                        for (int r = 0; r < 3; r++)
                        {
                            const float a = VOX_FFMA(kf, st[r], base[r]), b = VOX_FADD(a, wid[r]);
                            const float xs = fmaxf(a, fminf(b, 0.f));
                            D = __fmaf_rn(xs, xs, D);
                        }
                        zmask |= (D < lo_t ? 1u : 0u) << k;
                        unc |= (D > hi_t ? 0u : 1u) << k; // not surely failing (NaN included)
                    }
                    unc &= ~zmask; // neither surely passing nor surely failing
                }
                // the reference test of one voxel, from the record (nothing of the column kept live)
                auto exact_voxel = [&](uint32_t k) -> uint32_t {
                    const Aabb b = voxel_local_aabb(R, rinv_of(R), vsf, o[0] + rx, o[1] + ry, o[2] + rz0 + (int32_t)k);
                    return aabb_hits_unit_sphere(b) ? 1u << k : 0u;
                };
                for (uint32_t m = unc; m; m &= m - 1u)
                    zmask |= exact_voxel((uint32_t)(__ffs(m) - 1));
                if (CHECK)
                {
                    uint32_t ex = 0;
                    for (uint32_t k = 0; k < nz; k++)
                        ex |= exact_voxel(k);
                    if (ex != zmask)
                        atomicOr(P.err, ERR_BOUNDS); // a linear classification differs from the reference test
                }
            }
            else
            {
                const RInv M = rinv_of(R);
                const float il = R.q0.w, pz = R.q0.z;
                const float is[3] = { R.q3.y, R.q3.z, R.q3.w };
                float cx0, cx1, cy0, cy1;
                axis_corners(vsf, R.q0.x, o[0] + rx, cx0, cx1);
                axis_corners(vsf, R.q0.y, o[1] + ry, cy0, cy1);
                float slo[3], shi[3], pa[3];
                float v = (float)(o[2] + rz0);
                float cz = VOX_FSUB(VOX_FMUL(v, vsf), pz);
#pragma unroll
                for (int r = 0; r < 3; r++)
                {
                    float xn, xx, yn, yx;
                    minmax_prod(cx0, cx1, M.m[r][0], xn, xx);
                    minmax_prod(cy0, cy1, M.m[r][1], yn, yx);
                    slo[r] = VOX_FADD(xn, yn);
                    shi[r] = VOX_FADD(xx, yx);
                    pa[r] = VOX_FMUL(cz, M.m[r][2]);
                }
                // the reference test along the z run
#pragma unroll 2
                for (uint32_t k = 0; k < nz; k++)
                {
                    v = VOX_FADD(v, 1.f);
                    cz = VOX_FSUB(VOX_FMUL(v, vsf), pz);
                    float d2 = 1.f;
#pragma unroll
                    for (int r = 0; r < 3; r++)
                    {
                        // the corner offsets grow with z: per row the smaller product is the
                        // lower corner's when the matrix entry is >= 0 (fl(c m) is monotone
                        // in c; a tie differs at most in the sign of a zero, which is squared)
                        const float pb = VOX_FMUL(cz, M.m[r][2]);
                        const bool up = M.m[r][2] >= 0.f;
                        const float zn = up ? pa[r] : pb, zx = up ? pb : pa[r];
                        pa[r] = pb;
                        const float xl = VOX_FADD(slo[r], zn), xh = VOX_FADD(shi[r], zx);
                        // xl <= xh: the bound of the row's interval nearest to zero, or zero
                        const float xs = VOX_FADD(fmaxf(xl, 0.f), fminf(xh, 0.f));
                        const float sv = VOX_FMUL(VOX_FMUL(xs, il), is[r]);
                        d2 = VOX_FSUB(d2, VOX_FMUL(sv, sv));
                    }
                    zmask |= (d2 > 0.f ? 1u : 0u) << k;
                }
            }
            ebase = ((uint32_t)j << 9) | (uint32_t)((rx << 6) | (ry << 3) | rz0);
            if (CHECK && zmask && C.flag[j])
                atomicOr(P.err, ERR_BOUNDS); // the leaf test would have dropped a passing voxel
        }
        // queue slots: warp inclusive scan of the pass counts, one shared atomic per warp
        const uint32_t np = (uint32_t)__popc(zmask);
        uint32_t incl = np;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off)
                incl += y;
        }
        uint32_t qb = 0;
        if (PER_WARP)
        {
            qb = wbase + incl - np;
            wbase += __shfl_sync(0xffffffffu, incl, 31);
        }
        else
        {
            if (lane == 31 && incl)
                qb = atomicAdd(qcount, incl);
            qb = __shfl_sync(0xffffffffu, qb, 31) + incl - np;
        }
        for (uint32_t m = zmask; m; m &= m - 1)
            queue[qb++] = (uint16_t)(ebase + (uint32_t)(__ffs(m) - 1));
    }
    if (PER_WARP && lane == 0)
        qcount[t >> 5] = wbase;
}

// the part of a Gaussian's bbox inside the leaf at o
template <class Chunk>
__device__ __forceinline__ void leaf_box_fields(Chunk& C, int j, const GaussRec& R, const int32_t o[3])
{
    const int32_t x0 = max(R.q4.x, o[0]) - o[0], x1 = min(R.q4.x + R.q5.x - 1, o[0] + 7) - o[0];
    const int32_t y0 = max(R.q4.y, o[1]) - o[1], y1 = min(R.q4.y + R.q5.y - 1, o[1] + 7) - o[1];
    const int32_t z0 = max(R.q4.z, o[2]) - o[2], z1 = min(R.q4.z + R.q5.z - 1, o[2] + 7) - o[2];
    const bool empty = x1 < x0 || y1 < y0 || z1 < z0;
    const uint32_t ny = empty ? 1u : (uint32_t)(y1 - y0 + 1), nz = empty ? 1u : (uint32_t)(z1 - z0 + 1);
    C.bx0[j] = x0;
    C.by0[j] = y0;
    C.bz0[j] = z0;
    C.bny[j] = ny;
    C.bnz[j] = nz;
    C.bdiv_y[j] = (65536u + ny - 1u) / ny;
    C.bcol[j] = empty ? 0u : (uint32_t)(x1 - x0 + 1) * ny;
}

// all stagers (lanes 0 .. LQ_CHUNK - 1 of the last warp), once the boxes of the
// chunk's cnt Gaussians are placed: the chunk's column prefix
__device__ __forceinline__ void leaf_stage_prefix(LeafChunk& C, int js, uint32_t cnt)
{
    uint32_t b = js < (int)cnt ? C.bcol[js] : 0u;
#pragma unroll
    for (int off = 1; off < LQ_CHUNK; off <<= 1)
    {
        const uint32_t y = __shfl_up_sync((1u << LQ_CHUNK) - 1u, b, off);
        if (js >= off)
            b += y;
    }
    C.cstart[js + 1] = b;
    if (js == 0)
        C.cstart[0] = 0;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// the record of sorted leaf pair q into shared memory (asynchronous); returns its Gaussian id
__device__ __forceinline__ uint32_t leaf_stage_issue(const LeafPassParams& P, GaussRec* dst, uint32_t q)
{
    const uint32_t g = P.pair_gid[q];
    const float4* src = reinterpret_cast<const float4*>(&P.recs[g]);
#pragma unroll
    for (int w = 0; w < 8; w++)
        cp_async16(reinterpret_cast<float4*>(dst) + w, src + w);
    return g;
}

// once the record landed: the part of the Gaussian's bbox inside the leaf at o
template <bool CHECK, bool WINDOW>
__device__ __forceinline__ void leaf_stage_box(const LeafPassParams& P, LeafChunk& C, int j, uint32_t q, uint32_t g,
                                               const int32_t o[3])
{
    const GaussRec& R = C.rec[j].r;
    leaf_box_fields(C, j, R, o);
    C.rgb24[j] = rgba8_byte(R.q7.x) | (rgba8_byte(R.q7.y) << 8) | (rgba8_byte(R.q7.z) << 16);
    C.vs[j] = rec_vs(R, P.voxel_size, P.cloud_vs);
    const LeafPairConst K = leaf_pair_consts(R, C.vs[j], o);
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        C.lo0[r][j] = K.lo0[r];
        C.wid[r][j] = K.W[r];
        C.dab[r][j] = K.dab[r];
#pragma unroll
        for (int a = 0; a < 3; a++)
            C.stp[r][a][j] = K.A[r][a];
    }
    C.lo_t[j] = K.lo_t;
    C.hi_t[j] = K.hi_t;
    C.anchor[j] = K.r0;
    C.flag[j] = CHECK ? P.emit_flag[P.vals[q]] : 0;
    if (WINDOW)
    {
        const int64_t batch = (int64_t)g / REF_PRIM_BATCH;
        C.wf0[j] = P.frag_off[g] - P.frag_off[batch * REF_PRIM_BATCH];
        C.wbase[j] = P.win_before[batch];
    }
}

template <bool CHECK, bool WINDOW, int MINB = 4>
__global__ void __launch_bounds__(LP_THREADS, MINB) k_leaf_pass(LeafPassParams P, uint32_t* counter)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LeafQSmem& S = *reinterpret_cast<LeafQSmem*>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int js = t - LQ_STAGE_T0; // staging slot (0 .. LQ_CHUNK - 1 on the stagers)
    const bool stager = js >= 0 && js < LQ_CHUNK;
    if (t == 0)
    {
        S.cand = atomicAdd(counter, 1u);
        S.cand_next[0] = atomicAdd(counter, 1u);
        S.pairs = 0;
        S.qn[0] = S.qn[1] = S.qn[2] = 0;
        S.dfin = 0;
        S.acc[0].wmin = ~0ull;
    }
#pragma unroll
    for (int b = 0; b < 1; b++)
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const int n = t + 256 * h;
            S.acc[b].dens[n] = 0;
            S.acc[b].col[0][n] = S.acc[b].col[1][n] = S.acc[b].col[2][n] = 0;
            S.acc[b].cnt[n] = 0;
            S.acc[b].rgba[n] = 0;
        }
    __syncthreads();
    // the chunk being tested (t*), the chunk whose alpha runs (a*), the leaf being flushed (f*)
    int64_t tc = S.cand;
    if (tc >= P.NCL)
        return;
    int64_t cn = S.cand_next[0];
    int32_t to[3];
    {
        const int4 o4 = P.cand_org[tc];
        to[0] = o4.x;
        to[1] = o4.y;
        to[2] = o4.z;
    }
    // stagers: the next leaf's origin and pair range, loaded as soon as the leaf
    // is known and used at the current leaf's end; lane 0 claims the leaf after
    // it just as early, so no leaf end waits on global memory
    int4 pre_org = make_int4(0, 0, 0, 0);
    uint32_t pre_q0 = 0, pre_p1 = 0, cn2 = 0;
    bool cn_fresh = true;
    uint32_t tq0 = P.cand_start[tc], tp1 = P.cand_start[tc + 1];
    if (stager)
    {
        const uint32_t c0 = min((uint32_t)LQ_CHUNK, tp1 - tq0);
        if (js < (int)c0)
        {
            const uint32_t g = leaf_stage_issue(P, &S.ch[0].rec[js].r, tq0 + (uint32_t)js);
            cp_async_wait_all();
            leaf_stage_box<CHECK, WINDOW>(P, S.ch[0], js, tq0 + (uint32_t)js, g, to);
        }
        leaf_stage_prefix(S.ch[0], js, c0);
    }
    __syncthreads();
    bool t_valid = true, a_valid = false, f_valid = false, a_leaf_end = false;
    int tpar = 0, apar = 0, fpar = 0;
    int64_t ac = 0, fc = 0;
    int32_t ao[3] = { 0, 0, 0 };
    uint32_t i = 0; // phase
    while (t_valid || a_valid || f_valid)
    {
        const int tb = (int)(i % 3u), ab = (int)((i + 2u) % 3u), nb = (int)((i + 1u) % 3u);
        const bool t_leaf_end = t_valid && tq0 + LQ_CHUNK >= tp1;
        const int64_t nc = t_leaf_end ? cn : tc;
        const bool n_valid = t_valid && nc < P.NCL;
        if (stager && cn_fresh)
        {
            if (cn < P.NCL)
            {
                pre_org = P.cand_org[cn];
                pre_q0 = P.cand_start[cn];
                pre_p1 = P.cand_start[cn + 1];
                if (js == 0)
                    cn2 = atomicAdd(counter, 1u);
            }
        }
        cn_fresh = false;
        // ---- stagers: the next chunk's pair range, its record copies
        uint32_t nq0 = 0, np1 = 0, ncnt = 0, ng = 0;
        if (stager && n_valid)
        {
            nq0 = t_leaf_end ? pre_q0 : tq0 + LQ_CHUNK;
            np1 = t_leaf_end ? pre_p1 : tp1;
            ncnt = min((uint32_t)LQ_CHUNK, np1 - nq0);
            if (js < (int)ncnt)
                ng = leaf_stage_issue(P, &S.ch[nb].rec[js].r, nq0 + (uint32_t)js);
        }
        // ---- flush of the leaf whose last alpha ran in the previous phase
        if (f_valid)
        {
            LeafAcc& A = S.acc[0];
            uint32_t cnt[2];
#pragma unroll
            for (int h = 0; h < 2; h++)
            {
                const uint32_t n = (uint32_t)(t + 256 * h);
                cnt[h] = A.cnt[n];
                if (cnt[h])
                {
                    const uint64_t slot = (uint64_t)fc * 512u + n;
                    const float ds = fx_to_float(A.dens[n]);
                    float col[3];
#pragma unroll
                    for (int k = 0; k < 3; k++)
                    {
                        col[k] = fx_to_float(A.col[k][n]);
                        if (!P.smooth)
                            col[k] = ds > 0.f ? VOX_FDIV(col[k], ds) : 0.f;
                    }
                    P.s_rgba[slot] = A.rgba[n];
                    P.s_dens[slot] = ds;
                    P.s_col[3 * slot + 0] = col[0];
                    P.s_col[3 * slot + 1] = col[1];
                    P.s_col[3 * slot + 2] = col[2];
                    P.s_pairs[slot] = cnt[h];
                    A.dens[n] = 0;
                    A.col[0][n] = A.col[1][n] = A.col[2][n] = 0;
                    A.cnt[n] = 0;
                    A.rgba[n] = 0;
                }
            }
            // value mask: voxel t of warp w is bit lane of 32-bit word w (w + 8 for voxel t + 256)
            const uint32_t ba = __ballot_sync(0xffffffffu, cnt[0] > 0), bb = __ballot_sync(0xffffffffu, cnt[1] > 0);
            unsigned long long wp = cnt[0] + cnt[1];
#pragma unroll
            for (int off = 16; off; off >>= 1)
                wp += __shfl_xor_sync(0xffffffffu, wp, off);
            if (lane == 0)
            {
                uint32_t* m32 = reinterpret_cast<uint32_t*>(P.cand_mask + 8 * (uint64_t)fc);
                m32[warp] = ba;
                m32[8 + warp] = bb;
                if (wp)
                    atomicAdd(&S.pairs, wp);
            }
            if (WINDOW && t == 0)
            {
                P.cand_wkey[fc] = A.wmin;
                A.wmin = ~0ull;
            }
            __syncthreads(); // the next leaf's alpha reuses the accumulators
        }
        const uint32_t a_rounds = a_valid ? (S.qn[ab] + 31u) / 32u : 0u; // the alpha's rounds of 32 pairs
        // ---- alpha of the previous chunk, one queued pair per thread.  A pair
        // whose RGBA8 byte the bound leaves open (a few percent) is deferred to
        // its warp's list and the reference's byte is evaluated 32 pairs at a
        // time, so the rare branch costs one converged pass per 32 pairs.
        if (a_valid)
        {
            const LeafChunk& C = S.ch[ab];
            LeafAcc& A = S.acc[0];
            const uint16_t* queue = S.queue[(i + 1u) & 1u];
            const uint32_t qn = S.qn[ab];
            uint16_t* dq = S.defer[warp];
            uint32_t dn = 0; // this warp's deferred pairs (warp-uniform)
            auto ref_byte = [&](uint32_t q) {
                const uint32_t j = q >> 9, n = q & 511u;
                const GaussRec& R = C.rec[j].r;
                const uint32_t a8 = ref_alpha_byte(R, C.vs[j], ao[0] + (int32_t)(n >> 6),
                                                   ao[1] + (int32_t)((n >> 3) & 7u), ao[2] + (int32_t)(n & 7u));
                atomicMax(&A.rgba[n], (a8 << 24) | C.rgb24[j]);
            };
            for (uint32_t e0 = (uint32_t)(t & ~31); e0 < qn; e0 += LP_THREADS) // warp-uniform trip count
            {
                const uint32_t e = e0 + (uint32_t)lane;
                bool defer = false;
                uint32_t q = 0;
                if (e < qn)
                {
                    q = queue[e];
                    const uint32_t j = q >> 9, n = q & 511u;
                    const GaussRec& R = C.rec[j].r;
                    const float vsf = C.vs[j];
                    const int32_t x = ao[0] + (int32_t)(n >> 6), yy = ao[1] + (int32_t)((n >> 3) & 7),
                                  zz = ao[2] + (int32_t)(n & 7);
                    float a;
                    uint32_t a8;
                    if (P.smooth)
                    {
                        SmoothTerms st;
                        a = smooth_kernel(R, rinv_of(R), vsf, x, yy, zz, st);
                        a8 = ref_alpha_byte(R, vsf, x, yy, zz);
                    }
                    else
                    {
                        float lo0[3], wid[3], stp[3][3];
#pragma unroll
                        for (int r = 0; r < 3; r++)
                        {
                            lo0[r] = C.lo0[r][j];
                            wid[r] = C.wid[r][j];
#pragma unroll
                            for (int a = 0; a < 3; a++)
                                stp[r][a] = C.stp[r][a][j];
                        }
                        const AlphaF af = pair_alpha_f_ex(R, stable_leaf_aabb(lo0, wid, stp, C.anchor[j], (int32_t)(n >> 6),
                                                                              (int32_t)((n >> 3) & 7u), (int32_t)(n & 7u)));
                        a = af.a1;
                        bool decided;
                        const float dab[3] = { C.dab[0][j], C.dab[1][j], C.dab[2][j] };
                        a8 = alpha_byte_bound(R, af, dab, decided);
                        defer = !decided;
                        if (CHECK && decided && a8 != ref_alpha_byte(R, vsf, x, yy, zz))
                            atomicOr(P.err, ERR_BOUNDS); // the margin failed to cover the reference's byte
                    }
                    atomicAdd(&A.cnt[n], 1u);
                    if (!defer)
                        atomicMax(&A.rgba[n], (a8 << 24) | C.rgb24[j]);
                    atomicAdd(&A.dens[n], fx_of_unit(a));
                    atomicAdd(&A.col[0][n], fx_of(VOX_FMUL(a, R.q7.x)));
                    atomicAdd(&A.col[1][n], fx_of(VOX_FMUL(a, R.q7.y)));
                    atomicAdd(&A.col[2][n], fx_of(VOX_FMUL(a, R.q7.z)));
                    if (WINDOW)
                    {
                        // the reference's window of this fragment: x-major index in the bbox
                        // (gaussian_frag_alloc.slang:55-58) after the Gaussian's batch offset
                        const uint64_t r = (uint64_t)(x - R.q4.x) * (uint64_t)R.q5.y * (uint64_t)R.q5.z +
                                           (uint64_t)(yy - R.q4.y) * (uint64_t)R.q5.z + (uint64_t)(zz - R.q4.z);
                        atomicMin(&A.wmin, (unsigned long long)(C.wbase[j] + (C.wf0[j] + r) / REF_WINDOW));
                    }
                }
                const uint32_t bal = __ballot_sync(0xffffffffu, defer);
                if (bal)
                {
                    if (defer)
                        dq[dn + (uint32_t)__popc(bal & ((1u << lane) - 1u))] = (uint16_t)q;
                    dn += (uint32_t)__popc(bal);
                    if (dn >= 32u) // dn <= 63: a batch of 32, the rest moved to the front
                    {
                        __syncwarp();
                        ref_byte(dq[lane]);
                        const uint32_t rest = dn - 32u;
                        const uint16_t mv = (uint32_t)lane < rest ? dq[32 + lane] : (uint16_t)0;
                        __syncwarp();
                        if ((uint32_t)lane < rest)
                            dq[lane] = mv;
                        __syncwarp();
                        dn = rest;
                    }
                }
            }
            // the open pairs left in every warp's list (fewer than 32 each): the last
            // warp to finish this phase's alpha evaluates all of them, 32 at a time
            // (the chunk's records stay in place until the next phase's staging)
            uint32_t fin = 0;
            if (lane == 0)
            {
                S.dcount[warp] = dn;
                __threadfence_block();
                fin = atomicAdd(&S.dfin, 1u);
            }
            fin = __shfl_sync(0xffffffffu, fin, 0);
            if (fin == LP_THREADS / 32 - 1)
            {
                __threadfence_block();
                const uint32_t c = (uint32_t)lane < LP_THREADS / 32 ? *(volatile uint32_t*)&S.dcount[lane] : 0u;
                uint32_t incl = c;
#pragma unroll
                for (int off = 1; off < LP_THREADS / 32; off <<= 1)
                {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
                    if (lane >= off)
                        incl += y;
                }
                const uint32_t total = __shfl_sync(0xffffffffu, incl, LP_THREADS / 32 - 1);
                for (uint32_t b = 0; b < total; b += 32)
                {
                    const uint32_t item = b + (uint32_t)lane;
                    // the warp list holding item: the first w whose inclusive count exceeds it
                    uint32_t w = 0, before = 0;
#pragma unroll
                    for (int v = 0; v < LP_THREADS / 32; v++)
                    {
                        const uint32_t iv = __shfl_sync(0xffffffffu, incl, v);
                        const bool past = item >= iv;
                        w += past ? 1u : 0u;
                        before = past ? iv : before;
                    }
                    if (item < total)
                        ref_byte(*(volatile uint16_t*)&S.defer[w][item - before]);
                }
                if (lane == 0)
                    S.dfin = 0;
            }
        }
        // ---- test of this chunk
        if (t_valid)
            leaf_test_chunk<CHECK, false, true>(P, S.ch[tb], min((uint32_t)LQ_CHUNK, tp1 - tq0), to, S.queue[i & 1u],
                                                &S.qn[tb], t, lane, a_rounds);
        // the counter the test of phase i + 1 fills: last read by the alpha of phase i - 1
        if (t == 0)
            S.qn[nb] = 0;
        // ---- stagers: the next chunk's boxes (their own copies have landed)
        if (stager && n_valid)
        {
            int32_t no[3] = { to[0], to[1], to[2] };
            if (t_leaf_end)
            {
                no[0] = pre_org.x;
                no[1] = pre_org.y;
                no[2] = pre_org.z;
            }
            if (js < (int)ncnt)
            {
                cp_async_wait_all();
                leaf_stage_box<CHECK, WINDOW>(P, S.ch[nb], js, nq0 + (uint32_t)js, ng, no);
            }
            leaf_stage_prefix(S.ch[nb], js, ncnt);
            if (js == 0)
            {
                const int pp = (int)(i & 1u);
                S.nxt_o[pp][0] = no[0];
                S.nxt_o[pp][1] = no[1];
                S.nxt_o[pp][2] = no[2];
                S.nxt_q0[pp] = nq0;
                S.nxt_p1[pp] = np1;
                if (t_leaf_end)
                    S.cand_next[pp] = cn2;
            }
        }
        __syncthreads();
        // ---- advance: flush <- alpha (at a leaf end), alpha <- test, test <- next
        f_valid = a_valid && a_leaf_end;
        fc = ac;
        fpar = apar;
        a_valid = t_valid;
        a_leaf_end = t_leaf_end;
        ac = tc;
        apar = tpar;
        ao[0] = to[0];
        ao[1] = to[1];
        ao[2] = to[2];
        if (n_valid)
        {
            const int pp = (int)(i & 1u);
            if (t_leaf_end)
            {
                cn = S.cand_next[pp];
                cn_fresh = true;
                tpar ^= 1;
            }
            tc = nc;
            tq0 = S.nxt_q0[pp];
            tp1 = S.nxt_p1[pp];
            to[0] = S.nxt_o[pp][0];
            to[1] = S.nxt_o[pp][1];
            to[2] = S.nxt_o[pp][2];
        }
        t_valid = n_valid;
        i++;
    }
    if (t == 0 && S.pairs)
        atomicAdd((unsigned long long*)P.total_pairs, S.pairs);
}

__device__ __forceinline__ uint32_t mask_rank(const uint64_t* m, uint32_t n)
{
    uint32_t r = 0;
    for (uint32_t w = 0; w < (n >> 6); w++)
        r += __popcll(m[w]);
    return r + __popcll(m[n >> 6] & ((1ull << (n & 63)) - 1ull));
}

// adjoint: per (leaf, Gaussian) pair, the sum of its voxel pairs' terms,
// stored by the leaf pair's emission index.  The forward walk's pipeline: phase
// p flushes the sums of chunk p - 2, runs the adjoint terms of chunk p - 1's
// queued pairs, tests chunk p's columns (the same test) and stages chunk p + 1.
// The queue has one region per warp at warp-local positions, so its order is
// fixed; a pair's terms are summed per Gaussian across each warp (shuffles)
// into that warp's slots, and the flush adds the warps' slots in warp order:
// deterministic, no atomics.
struct LeafBChunk
{
    RecSlot rec[LQ_CHUNK]; // first member: 16-byte aligned for cp.async
    int32_t bx0[LQ_CHUNK], by0[LQ_CHUNK], bz0[LQ_CHUNK];
    uint32_t bny[LQ_CHUNK], bnz[LQ_CHUNK], bdiv_y[LQ_CHUNK], bcol[LQ_CHUNK];
    float vs[LQ_CHUNK];
    uint8_t flag[LQ_CHUNK];
    uint32_t eidx[LQ_CHUNK]; // emission index of each leaf pair
    uint64_t mask[8];        // the leaf's value mask
    uint64_t vbase;          // value index of the leaf's first voxel
};

struct LeafGradSum
{
    float part[LP_THREADS / 32][LQ_CHUNK][BWD_NACC]; // per warp: a fixed set of rounds, summed in order
    uint32_t eidx[LQ_CHUNK];
    uint32_t cnt;
};

// a warp tests at most ceil(LQ_CHUNK * 64 / LP_THREADS) rounds of 32 columns of
// up to 8 voxels; its queue region (LQ_CHUNK * 64 entries) must hold them all
static_assert(((LQ_CHUNK * 64 + LP_THREADS - 1) / LP_THREADS) * 32 * 8 <= LQ_CHUNK * 64,
              "per-warp queue regions too small for this chunk size");

struct LeafBSmem
{
    LeafBChunk ch[3];
    LeafGradSum gs[2];
    uint16_t queue[2][LQ_CHUNK * 512]; // per warp regions of LQ_CHUNK * 64 entries
    uint32_t wqn[2][LP_THREADS / 32];   // entries per warp region
    int32_t nxt_o[2][3];
    uint32_t nxt_q0[2], nxt_p1[2];
    uint32_t cand_next[2];
    uint32_t cand;
};

// stager js of the chunk at sorted pair q0 of candidate c (origin o): the leaf's
// mask word js, and for js < cnt its record's box once the copy has landed
__device__ __forceinline__ void leaf_bstage(const LeafPassParams& P, LeafBChunk& C, int js, uint32_t cnt, uint32_t q0,
                                            int64_t c, const int32_t o[3])
{
    if (js < 8)
        C.mask[js] = P.cand_mask[8 * (uint64_t)c + js];
    if (js == 0)
        C.vbase = P.cand_vbase[c];
    if (js < (int)cnt)
    {
        cp_async_wait_all();
        leaf_box_fields(C, js, C.rec[js].r, o);
        C.vs[js] = rec_vs(C.rec[js].r, P.voxel_size, P.cloud_vs);
        C.flag[js] = 0;
        C.eidx[js] = P.vals[q0 + (uint32_t)js];
    }
}

__global__ void __launch_bounds__(LP_THREADS, 3) k_leaf_backward(LeafPassParams P, uint32_t* counter)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LeafBSmem& S = *reinterpret_cast<LeafBSmem*>(smem_raw);
    const int t = threadIdx.x, lane = t & 31;
    const int js = t - LQ_STAGE_T0;
    const bool stager = js >= 0 && js < LQ_CHUNK;
    if (t == 0)
    {
        S.cand = atomicAdd(counter, 1u);
        S.cand_next[0] = atomicAdd(counter, 1u);
    }
    for (int i = t; i < (LP_THREADS / 32) * LQ_CHUNK * BWD_NACC; i += LP_THREADS)
    {
        (&S.gs[0].part[0][0][0])[i] = 0.f;
        (&S.gs[1].part[0][0][0])[i] = 0.f;
    }
    __syncthreads();
    int64_t tc = S.cand;
    if (tc >= P.NCL)
        return;
    int64_t cn = S.cand_next[0];
    int32_t to[3];
    cand_origin(P, P.cand_key[tc], to);
    uint32_t tq0 = P.cand_start[tc], tp1 = P.cand_start[tc + 1];
    if (stager)
    {
        const uint32_t cnt = min((uint32_t)LQ_CHUNK, tp1 - tq0);
        if (js < (int)cnt)
            leaf_stage_issue(P, &S.ch[0].rec[js].r, tq0 + (uint32_t)js);
        leaf_bstage(P, S.ch[0], js, cnt, tq0, tc, to);
    }
    __syncthreads();
    bool t_valid = true, a_valid = false, f_valid = false;
    uint32_t acnt = 0;
    int32_t ao[3] = { 0, 0, 0 };
    uint32_t p = 0;
    while (t_valid || a_valid || f_valid)
    {
        const int tb = (int)(p % 3u), ab = (int)((p + 2u) % 3u), nb = (int)((p + 1u) % 3u);
        const bool t_end = t_valid && tq0 + LQ_CHUNK >= tp1;
        const int64_t nc = t_end ? cn : tc;
        const bool n_valid = t_valid && nc < P.NCL;
        uint32_t nq0 = 0, np1 = 0, ncnt = 0;
        if (stager && n_valid)
        {
            nq0 = t_end ? P.cand_start[nc] : tq0 + LQ_CHUNK;
            np1 = t_end ? P.cand_start[nc + 1] : tp1;
            ncnt = min((uint32_t)LQ_CHUNK, np1 - nq0);
            if (js < (int)ncnt)
                leaf_stage_issue(P, &S.ch[nb].rec[js].r, nq0 + (uint32_t)js);
        }
        // ---- flush: chunk p - 2's sums to its leaf pairs' partials
        if (f_valid)
        {
            LeafGradSum& Gs = S.gs[p & 1u];
            const uint32_t n = Gs.cnt * BWD_NACC;
            for (uint32_t i = (uint32_t)t; i < n; i += LP_THREADS)
            {
                const uint32_t j = i / BWD_NACC, k = i - j * BWD_NACC;
                float v = 0.f;
                for (int w = 0; w < LP_THREADS / 32; w++)
                {
                    v += Gs.part[w][j][k];
                    Gs.part[w][j][k] = 0.f;
                }
                P.partials[(uint64_t)Gs.eidx[j] * BWD_NACC + k] = v;
            }
        }
        // ---- adjoint terms of chunk p - 1's queued pairs
        if (a_valid)
        {
            const LeafBChunk& C = S.ch[ab];
            LeafGradSum& Gs = S.gs[(p + 1u) & 1u];
            if (t < LQ_CHUNK)
                Gs.eidx[t] = C.eidx[t];
            if (t == 0)
                Gs.cnt = acnt;
            const uint16_t* queue = S.queue[(p + 1u) & 1u];
            const uint32_t* wqn = S.wqn[(p + 1u) & 1u];
            uint32_t wstart[LP_THREADS / 32 + 1];
            wstart[0] = 0;
#pragma unroll
            for (int w = 0; w < LP_THREADS / 32; w++)
                wstart[w + 1] = wstart[w] + wqn[w];
            const uint32_t qn = wstart[LP_THREADS / 32];
            const int warp = t >> 5;
            for (uint32_t b0 = 0; b0 < qn; b0 += LP_THREADS)
            {
                const uint32_t e = b0 + (uint32_t)t;
                int j = -1;
                float cc[BWD_NACC];
#pragma unroll
                for (int k = 0; k < BWD_NACC; k++)
                    cc[k] = 0.f;
                if (e < qn)
                {
                    // entry e of the concatenated warp regions
                    uint32_t wr = 0, ws = 0;
#pragma unroll
                    for (int w = 1; w < LP_THREADS / 32; w++)
                    {
                        const bool ge = e >= wstart[w];
                        wr = ge ? (uint32_t)w : wr;
                        ws = ge ? wstart[w] : ws;
                    }
                    const uint32_t q = queue[wr * (LQ_CHUNK * 64) + (e - ws)];
                    j = (int)(q >> 9);
                    const uint32_t n = q & 511u;
                    const GaussRec& R = C.rec[j].r;
                    const RInv M = rinv_of(R);
                    const float vsf = C.vs[j];
                    const int32_t x = ao[0] + (int32_t)(n >> 6), yy = ao[1] + (int32_t)((n >> 3) & 7), zz = ao[2] + (int32_t)(n & 7);
                    SmoothTerms st;
                    const float Kw = smooth_kernel(R, M, vsf, x, yy, zz, st);
                    if (st.e > SMOOTH_TAU)
                    {
                        const uint64_t vi = C.vbase + mask_rank(C.mask, n);
                        const float gd = P.grad_density ? P.grad_density[vi] : 0.f;
                        float gc[3] = { 0.f, 0.f, 0.f };
                        if (P.grad_color)
                            for (int k = 0; k < 3; k++)
                                gc[k] = P.grad_color[3 * vi + k];
                        const float GK = gd + gc[0] * R.q7.x + gc[1] * R.q7.y + gc[2] * R.q7.z;
                        cc[0] = GK * st.E;
#pragma unroll
                        for (int r = 0; r < 3; r++)
                        {
                            const float dzr = -GK * st.e * st.z[r];
                            const float du = dzr * (r == 0 ? R.q3.y : (r == 1 ? R.q3.z : R.q3.w));
                            cc[1 + r] = du;
                            cc[4 + r] = dzr * st.z[r];
#pragma unroll
                            for (int a = 0; a < 3; a++)
                                cc[7 + 3 * r + a] = du * st.d[a];
                        }
                        cc[16] = Kw * gc[0];
                        cc[17] = Kw * gc[1];
                        cc[18] = Kw * gc[2];
                    }
                }
                // per Gaussian present in this warp: its terms summed across the warp
                // (fixed shuffle tree) into this warp's slots
                uint32_t todo = __ballot_sync(0xffffffffu, j >= 0);
                while (todo)
                {
                    const int jx = __shfl_sync(0xffffffffu, j, __ffs(todo) - 1);
                    const bool mine = j == jx;
#pragma unroll
                    for (int k = 0; k < BWD_NACC; k++)
                    {
                        float v = mine ? cc[k] : 0.f;
#pragma unroll
                        for (int off = 16; off; off >>= 1)
                            v += __shfl_xor_sync(0xffffffffu, v, off);
                        if (lane == 0)
                            Gs.part[warp][jx][k] += v;
                    }
                    todo &= ~__ballot_sync(0xffffffffu, mine);
                }
            }
        }
        // ---- test of chunk p
        if (t_valid)
            leaf_test_chunk<false, true>(P, S.ch[tb], min((uint32_t)LQ_CHUNK, tp1 - tq0), to, S.queue[p & 1u],
                                         S.wqn[p & 1u], t, lane);
        // ---- stagers: chunk p + 1's mask words and boxes
        if (stager && n_valid)
        {
            int32_t no[3] = { to[0], to[1], to[2] };
            if (t_end)
                cand_origin(P, P.cand_key[nc], no);
            leaf_bstage(P, S.ch[nb], js, ncnt, nq0, nc, no);
            if (js == 0)
            {
                const int pp = (int)(p & 1u);
                S.nxt_o[pp][0] = no[0];
                S.nxt_o[pp][1] = no[1];
                S.nxt_o[pp][2] = no[2];
                S.nxt_q0[pp] = nq0;
                S.nxt_p1[pp] = np1;
                if (t_end)
                    S.cand_next[pp] = atomicAdd(counter, 1u);
            }
        }
        __syncthreads();
        f_valid = a_valid;
        a_valid = t_valid;
        acnt = t_valid ? min((uint32_t)LQ_CHUNK, tp1 - tq0) : 0u;
        ao[0] = to[0];
        ao[1] = to[1];
        ao[2] = to[2];
        if (n_valid)
        {
            const int pp = (int)(p & 1u);
            if (t_end)
                cn = S.cand_next[pp];
            tc = nc;
            tq0 = S.nxt_q0[pp];
            tp1 = S.nxt_p1[pp];
            to[0] = S.nxt_o[pp][0];
            to[1] = S.nxt_o[pp][1];
            to[2] = S.nxt_o[pp][2];
        }
        t_valid = n_valid;
        p++;
    }
}

// the sorted (voxel key, Gaussian id) pair list: per voxel, its Gaussians in
// ascending id, at the voxel's pair offset
__global__ void __launch_bounds__(LP_THREADS) k_leaf_export(LeafPassParams P, uint32_t* counter)
{
    __shared__ LeafSmem S;
    const int t = threadIdx.x;
    while (true)
    {
        if (t == 0)
            S.cand = atomicAdd(counter, 1u);
        __syncthreads();
        const int64_t c = S.cand;
        if (c >= P.NCL)
            break;
        if (t < 8)
            S.mask[t] = P.cand_mask[8 * (uint64_t)c + t];
        const uint32_t key = P.cand_key[c];
        int32_t o[3];
        cand_origin(P, key, o);
        __syncthreads();
        const int32_t xa = o[0] + (t >> 6), y = o[1] + ((t >> 3) & 7), z = o[2] + (t & 7), xb = xa + 4;
        uint64_t dst[2] = { 0, 0 };
        bool act[2];
#pragma unroll
        for (int h = 0; h < 2; h++)
        {
            const uint32_t n = (uint32_t)(t + 256 * h);
            act[h] = (S.mask[n >> 6] >> (n & 63)) & 1ull;
            if (act[h])
                dst[h] = P.pair_off[P.cand_voff[c] + mask_rank(S.mask, n)];
        }
        const uint32_t p0 = P.cand_start[c], p1 = P.cand_start[c + 1];
        for (uint32_t q0 = p0; q0 < p1; q0 += LP_CHUNK)
        {
            const uint32_t cnt = min((uint32_t)LP_CHUNK, p1 - q0);
            stage_chunk(P, S, q0, cnt);
            __syncthreads();
            for (uint32_t j = 0; j < cnt; j++)
            {
                const GaussRec& R = S.rec[j];
                const RInv M = rinv_of(R);
                const float vsf = rec_vs(R, P.voxel_size, P.cloud_vs);
#pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const int32_t x = h ? xb : xa;
                    if (!act[h] || !in_bbox(R, x, y, z))
                        continue;
                    if (!aabb_hits_unit_sphere(voxel_local_aabb(R, M, vsf, x, y, z)))
                        continue;
                    const uint64_t k = ((uint64_t)key << 9) | (uint32_t)(t + 256 * h);
                    if (P.key64)
                        ((uint64_t*)P.out_keys)[dst[h]] = k;
                    else
                        ((uint32_t*)P.out_keys)[dst[h]] = (uint32_t)k;
                    P.out_ids[dst[h]] = S.gid[j];
                    dst[h]++;
                }
            }
            __syncthreads();
        }
    }
}

__global__ void k_leaf_popc(const uint64_t* cand_mask, int64_t NCL, uint64_t* counts)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= NCL)
        return;
    uint64_t n = 0;
    for (int w = 0; w < 8; w++)
        n += (uint64_t)__popcll(cand_mask[8 * c + w]);
    counts[c] = n;
}

// one warp per candidate leaf, 32 voxels per round: each active voxel's rank is
// the popcount of the mask bits below it, so the writes are contiguous
template <class K>
__global__ void k_voxel_keys(const uint64_t* cand_mask, const uint32_t* cand_key, const uint64_t* cand_voff,
                             int64_t NCL, K* vkeys, uint32_t* vslot)
{
    const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= NCL)
        return;
    const uint32_t* m32 = reinterpret_cast<const uint32_t*>(cand_mask + 8 * c);
    const uint32_t mine = m32[lane & 15];
    uint64_t base = cand_voff[c];
    const uint64_t lk = (uint64_t)cand_key[c] << 9;
    const uint32_t lt = (1u << lane) - 1u;
    for (int r = 0; r < 16; r++)
    {
        const uint32_t bits = __shfl_sync(0xffffffffu, mine, r);
        if ((bits >> lane) & 1u)
        {
            const uint64_t at = base + (uint64_t)__popc(bits & lt);
            const uint32_t n = (uint32_t)(32 * r + lane);
            vkeys[at] = (K)(lk | n);
            vslot[at] = (uint32_t)(c * 512 + n);
        }
        base += (uint64_t)__popc(bits);
    }
}

// staged values -> value index of every active voxel; leaf masks
__global__ void k_values(ValueParams A, NodeParams N)
{
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= A.V)
        return;
    const uint32_t slot = A.vslot[v];
    const uint32_t l = A.vox_leaf[v];
    const uint32_t n = A.vox_n[v];
    const uint64_t vi = N.leaf_vidx[l] + (uint64_t)(v - N.leaf_vstart[l]);
    const uint32_t b = N.C.leaf_cloud[l];
    ((uint32_t*)(A.out + N.C.rgba_off[b]))[vi] = A.s_rgba[slot];
    ((float*)(A.out + N.C.dens_off[b]))[vi] = A.s_dens[slot];
    float* col = (float*)(A.out + N.C.col_off[b]);
    col[3 * vi + 0] = A.s_col[3 * (uint64_t)slot + 0];
    col[3 * vi + 1] = A.s_col[3 * (uint64_t)slot + 1];
    col[3 * vi + 2] = A.s_col[3 * (uint64_t)slot + 2];
    if ((uint64_t)v == N.leaf_vstart[l])
        A.cand_vbase[slot >> 9] = N.C.value_base[b] + N.leaf_vidx[l];
    (void)n;
    if (A.cloud_pairs)
    {
        // pairs per cloud: a warp whose voxels share a cloud adds once
        uint64_t pc = A.s_pairs[slot];
        const uint32_t peers = __match_any_sync(__activemask(), b);
        for (int off = 16; off; off >>= 1)
        {
            const uint64_t o = __shfl_down_sync(__activemask(), pc, off);
            pc += ((threadIdx.x & 31) + off < 32 && ((peers >> ((threadIdx.x & 31) + off)) & 1u)) ? o : 0ull;
        }
        if ((threadIdx.x & 31) == __ffs(peers) - 1)
            atomicAdd((unsigned long long*)&A.cloud_pairs[b], (unsigned long long)pc);
    }
}

// every leaf's value mask is its candidate leaf's mask
__global__ void k_leaf_masks(int64_t L, const uint32_t* leaf_vstart, const uint32_t* vslot, const uint64_t* cand_mask,
                             uint64_t* leaf_mask)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L * 8)
        return;
    const int64_t l = t >> 3;
    const uint32_t c = vslot[leaf_vstart[l]] >> 9;
    leaf_mask[t] = cand_mask[8 * (uint64_t)c + (t & 7)];
}

// pairs per voxel (run order) from the staged counts
__global__ void k_voxel_pairs(int64_t V, const uint32_t* vslot, const uint32_t* s_pairs, uint64_t* vpairs)
{
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < V)
        vpairs[v] = s_pairs[vslot[v]];
}

// ---------------------------------------------------------------- launch ----
void launch_leaf_cols(const GaussRec* recs, int64_t G, uint64_t* lcols, cudaStream_t s)
{
    if (G <= 0)
        return;
    { k_leaf_cols<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(recs, G, lcols); count_launch(); }
}

void launch_tile_gauss(const uint64_t* lcol_off, int64_t G, uint64_t NLC, int64_t* tile_g0, cudaStream_t s)
{
    if (NLC == 0)
        return;
    const uint64_t ntiles = (NLC + 255) / 256;
    { k_tile_gauss<<<(unsigned)((ntiles + 255) / 256), 256, 0, s>>>(lcol_off, G, NLC, tile_g0); count_launch(); }
}

void launch_leaf_emit(const LeafEmitParams& P, const RankTables& T, bool write, cudaStream_t s)
{
    if (P.NLC == 0)
        return;
    uint64_t blocks = (P.NLC + 255) / 256;
    if (blocks > 148ull * 64)
        blocks = 148ull * 64;
    if (write)
        { k_leaf_emit<true><<<(unsigned)blocks, 256, 0, s>>>(P, T); count_launch(); }
    else
        { k_leaf_emit<false><<<(unsigned)blocks, 256, 0, s>>>(P, T); count_launch(); }
}

void launch_leaf_heads(const uint32_t* keys, int64_t Q, uint64_t* flags, cudaStream_t s)
{
    if (Q <= 0)
        return;
    { k_leaf_heads<<<(unsigned)((Q + 255) / 256), 256, 0, s>>>(keys, Q, flags); count_launch(); }
}

void launch_leaf_compact(const uint32_t* keys, const uint32_t* vals, const uint32_t* emit_gid, int64_t Q,
                         const uint64_t* flags, const uint64_t* pos, const uint32_t* lower_cell,
                         const uint32_t* root_of_rank, uint32_t* cand_key, int4* cand_org, uint32_t* cand_start,
                         uint32_t* pair_gid, cudaStream_t s)
{
    if (Q <= 0)
        return;
    { k_leaf_compact<<<(unsigned)((Q + 255) / 256), 256, 0, s>>>(keys, vals, emit_gid, Q, flags, pos, lower_cell, root_of_rank, cand_key, cand_org, cand_start, pair_gid); count_launch(); }
}

static unsigned walk_grid(int64_t NCL, int num_sms)
{
    int64_t g = (int64_t)num_sms * 8;
    return (unsigned)(g < NCL ? g : (NCL > 0 ? NCL : 1));
}

int launch_leaf_pass(const LeafPassParams& P, uint32_t* counter, int num_sms, cudaStream_t s, int variant)
{
    if (P.NCL <= 0)
        return 0;
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    const size_t smem = sizeof(LeafQSmem);
    auto kern = P.emit_flag ? (P.window ? k_leaf_pass<true, true> : k_leaf_pass<true, false>)
                : variant == 1 ? (P.window ? k_leaf_pass<false, true, 3> : k_leaf_pass<false, false, 3>)
                               : (P.window ? k_leaf_pass<false, true> : k_leaf_pass<false, false>);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, LP_THREADS, smem);
    int64_t grid = (int64_t)num_sms * (per_sm > 0 ? per_sm : 1);
    if (grid > P.NCL)
        grid = P.NCL;
    { kern<<<(unsigned)grid, LP_THREADS, smem, s>>>(P, counter); count_launch(); }
    return per_sm;
}

void launch_leaf_backward(const LeafPassParams& P, uint32_t* counter, int num_sms, cudaStream_t s)
{
    if (P.NCL <= 0)
        return;
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    const size_t smem = sizeof(LeafBSmem);
    cudaFuncSetAttribute(k_leaf_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_leaf_backward, LP_THREADS, smem);
    int64_t grid = (int64_t)num_sms * (per_sm > 0 ? per_sm : 1);
    if (grid > P.NCL)
        grid = P.NCL;
    { k_leaf_backward<<<(unsigned)grid, LP_THREADS, smem, s>>>(P, counter); count_launch(); }
}

void launch_leaf_export(const LeafPassParams& P, uint32_t* counter, int num_sms, cudaStream_t s)
{
    if (P.NCL <= 0)
        return;
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    { k_leaf_export<<<walk_grid(P.NCL, num_sms), LP_THREADS, 0, s>>>(P, counter); count_launch(); }
}

void launch_leaf_popc(const uint64_t* cand_mask, int64_t NCL, uint64_t* counts, cudaStream_t s)
{
    if (NCL <= 0)
        return;
    { k_leaf_popc<<<(unsigned)((NCL + 255) / 256), 256, 0, s>>>(cand_mask, NCL, counts); count_launch(); }
}

void launch_voxel_keys(const uint64_t* cand_mask, const uint32_t* cand_key, const uint64_t* cand_voff, int64_t NCL,
                       void* vkeys, int key64, uint32_t* vslot, cudaStream_t s)
{
    if (NCL <= 0)
        return;
    const unsigned blocks = (unsigned)((NCL * 32 + 255) / 256);
    if (key64)
        { k_voxel_keys<uint64_t><<<blocks, 256, 0, s>>>(cand_mask, cand_key, cand_voff, NCL, (uint64_t*)vkeys, vslot); count_launch(); }
    else
        { k_voxel_keys<uint32_t><<<blocks, 256, 0, s>>>(cand_mask, cand_key, cand_voff, NCL, (uint32_t*)vkeys, vslot); count_launch(); }
}

void launch_values(const ValueParams& A, const NodeParams& N, cudaStream_t s)
{
    if (A.V <= 0)
        return;
    { k_values<<<(unsigned)((A.V + 255) / 256), 256, 0, s>>>(A, N); count_launch(); }
}

void launch_leaf_masks(const NodeParams& N, const uint64_t* cand_mask, const uint32_t* vslot, cudaStream_t s)
{
    if (N.L <= 0)
        return;
    { k_leaf_masks<<<(unsigned)((N.L * 8 + 255) / 256), 256, 0, s>>>(N.L, N.leaf_vstart, vslot, cand_mask, N.leaf_mask); count_launch(); }
}

void launch_voxel_pairs(int64_t V, const uint32_t* vslot, const uint32_t* s_pairs, uint64_t* vpairs, cudaStream_t s)
{
    if (V <= 0)
        return;
    { k_voxel_pairs<<<(unsigned)((V + 255) / 256), 256, 0, s>>>(V, vslot, s_pairs, vpairs); count_launch(); }
}

} // namespace vox
