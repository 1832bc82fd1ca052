// vox_voxelbvh.cu - VoxelBVH Gaussian ingestion: per Gaussian, the finest
// power-of-two cell level at which at most 8 cells overlap its 0.01-opacity
// ellipsoid, those cells as 64-bit keys i << 48 | j << 32 | k << 16 | level,
// and after the key sort the [start, end) range of every distinct key
// (raster/VoxelBVH.cpp:1225-1435, ijkl_from_gaussians).
//
// Kernels, all on the caller's stream:
//   k_vb_init           world-box accumulator = (+inf, -inf)
//   k_vb_box            per-Gaussian transformed 8-corner box, warp-reduced,
//                       one atomicMin / atomicMax per warp on order-preserving
//                       integer keys (deterministic; -0 orders below +0)
//                       (voxelbvh_gaussians_bbox_reduce1/2.slang)
//   k_vb_setup          a 96-byte search record per Gaussian (mean,
//                       rotation, 1 / (local_scale scale), cell box, status)
//   k_vb_search         the level search from 11 down, stopping once more
//                       than 8 cells overlap, lane-balanced: a persistent loop
//                       in which every lane tests one cell per iteration and
//                       takes its next Gaussian when its search ends; 8 keys
//                       and 8 ids per Gaussian in 16-byte stores
//                       (voxelbvh_gaussians_to_ijkl.slang:25-250)
//   k_vb_ijkl           the same search, one thread per Gaussian with the
//                       per-axis reuse below (VOX_VB_SEARCH=thread)
//   k_vb_used,          the used slots (a prefix of each Gaussian's 8) counted and
//   k_vb_compress_used  scanned, their keys compressed to 4 + bits(i) + bits(j) +
//                       bits(k) bits (32-bit when they fit), sized by the
//                       emitted cells' range the search reduces: the same
//                       order in fewer radix passes, and compacted (the
//                       unused slots, all-ones key and id, are the sorted tail)
//   (sort)              stable LSD sort of the used compressed keys (of all
//                       64-bit keys when a cell lies outside [0, 2^15))
//   k_vb_range_count    starts per 2048-key tile
//   (scan)              exclusive scan of the tile counts
//   k_vb_range_scatter  headers [2r] = start, [2r + 1] = end; every header
//                       slot at or past the range count is zeroed; writes
//                       the sorted keys back as 64-bit keys
//   k_vb_tail           the unused tail: keys and ids all ones, its run as
//                       the last range, the other headers zeroed
//                       (voxelbvh_find_range_starts.slang,
//                       voxelbvh_scatter_range_headers.slang)
//
// Float arithmetic: every operation is one IEEE round-to-nearest intrinsic in
// the order the shaders write it (no contraction), so the keys are the same
// bits as the C restatement's.  Values the shaders recompute per corner
// (the per-axis voxel-to-world coordinates, the products of a corner's
// coordinates with the rotation) are computed once per cell (and, in
// k_vb_ijkl, once per row of cells) and reused: the same operations on the
// same operands.
#include <cuda_runtime.h>

#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

namespace
{

constexpr int VB_THREADS = 256;
constexpr int VB_TILE = 2048; // keys per range tile (8 per thread)
constexpr float VB_CELL_LIMIT = 65536.f;
// a level whose cell box exceeds this is reported (VOX_ERR_RANGE) instead of
// searched: it bounds the search, and no Gaussian whose box is its own
// ellipsoid's reaches it (more than 8 of its cells overlap long before)
constexpr int64_t VB_MAX_CELLS = 1ll << 24;

__device__ __forceinline__ uint32_t vb_fkey(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float vb_funkey(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct VbGauss
{
    float mu[3];
    float R[3][3]; // forward rotation rows; the inverse is the transpose
    float e[3];    // scale * local_scale
    float inv[3];  // 1 / (local_scale * scale)
};

__device__ __forceinline__ void vb_load(const VoxelBvhParams& P, int64_t g, VbGauss& G)
{
    for (int a = 0; a < 3; a++)
        G.mu[a] = P.means[3 * g + a];
    const float w = P.quats[4 * g + 0], x = P.quats[4 * g + 1], y = P.quats[4 * g + 2], z = P.quats[4 * g + 3];
    float s[3];
    for (int a = 0; a < 3; a++)
        s[a] = P.scales[3 * g + a];
    const float op = P.opac[g];
    const float o = 0.01f > op ? 0.01f : op;
    const float ls = __fsqrt_rn(__fmul_rn(2.f, vox_logf(__fdiv_rn(o, 0.01f))));
    G.R[0][0] = __fsub_rn(1.f, __fmul_rn(2.f, __fadd_rn(__fmul_rn(y, y), __fmul_rn(z, z))));
    G.R[0][1] = __fmul_rn(2.f, __fsub_rn(__fmul_rn(x, y), __fmul_rn(z, w)));
    G.R[0][2] = __fmul_rn(2.f, __fadd_rn(__fmul_rn(x, z), __fmul_rn(y, w)));
    G.R[1][0] = __fmul_rn(2.f, __fadd_rn(__fmul_rn(x, y), __fmul_rn(z, w)));
    G.R[1][1] = __fsub_rn(1.f, __fmul_rn(2.f, __fadd_rn(__fmul_rn(x, x), __fmul_rn(z, z))));
    G.R[1][2] = __fmul_rn(2.f, __fsub_rn(__fmul_rn(y, z), __fmul_rn(x, w)));
    G.R[2][0] = __fmul_rn(2.f, __fsub_rn(__fmul_rn(x, z), __fmul_rn(y, w)));
    G.R[2][1] = __fmul_rn(2.f, __fadd_rn(__fmul_rn(y, z), __fmul_rn(x, w)));
    G.R[2][2] = __fsub_rn(1.f, __fmul_rn(2.f, __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y))));
    for (int a = 0; a < 3; a++)
    {
        G.e[a] = __fmul_rn(s[a], ls);
        G.inv[a] = __fdiv_rn(1.f, __fmul_rn(ls, s[a]));
    }
}

// p' = [p 1] T (row vector), sums left to right
__device__ __forceinline__ float vb_xf(const float* T, float p0, float p1, float p2, int c)
{
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p0, T[c]), __fmul_rn(p1, T[4 + c])), __fmul_rn(p2, T[8 + c])),
                     T[12 + c]);
}

__device__ __forceinline__ bool vb_finite(float x)
{
    return (__float_as_uint(x) & 0x7f800000u) != 0x7f800000u;
}

// transformed 8-corner box of the local_scale cube; minima / maxima as keys.
// Returns false when a corner is not finite (the keys then cover the finite
// corners only): the caller reports an error, since NaN has no place in the
// order the keys encode.
__device__ __forceinline__ bool vb_box_keys(const VoxelBvhParams& P, const VbGauss& G, uint32_t kmn[3], uint32_t kmx[3])
{
    bool finite = true;
    float pr[3][3]; // pr[c][a] = e[a] * R[c][a]; the -e corner's product is its negation
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int a = 0; a < 3; a++)
            pr[c][a] = __fmul_rn(G.e[a], G.R[c][a]);
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        kmn[a] = 0xffffffffu;
        kmx[a] = 0u;
    }
#pragma unroll
    for (int v = 0; v < 8; v++)
    {
        float wp[3];
#pragma unroll
        for (int c = 0; c < 3; c++)
        {
            const float t0 = (v & 1) ? pr[c][0] : -pr[c][0];
            const float t1 = (v & 2) ? pr[c][1] : -pr[c][1];
            const float t2 = (v & 4) ? pr[c][2] : -pr[c][2];
            wp[c] = __fadd_rn(__fadd_rn(__fadd_rn(t0, t1), t2), G.mu[c]);
        }
        float tp[3];
        if (P.has_xform)
        {
#pragma unroll
            for (int c = 0; c < 3; c++)
                tp[c] = vb_xf(P.t, wp[0], wp[1], wp[2], c);
        }
        else
        {
#pragma unroll
            for (int c = 0; c < 3; c++)
                tp[c] = wp[c];
        }
#pragma unroll
        for (int a = 0; a < 3; a++)
        {
            if (!vb_finite(tp[a]))
            {
                finite = false;
                continue;
            }
            const uint32_t k = vb_fkey(tp[a]);
            kmn[a] = k < kmn[a] ? k : kmn[a];
            kmx[a] = k > kmx[a] ? k : kmx[a];
        }
    }
    return finite;
}

// Voxel-to-world coordinate of one cell boundary on axis a:
// (v - offset) / scale, v = the boundary's voxel coordinate.
__device__ __forceinline__ float vb_lp(const float w2v[4], float v, int a)
{
    return __fdiv_rn(__fsub_rn(v, w2v[a]), w2v[3]);
}

// voxel_ellipsoid_overlap (voxelbvh_gaussians_to_ijkl.slang:25-109) of the
// cells of edge 2^level in the cell box [lo, hi], in the shader's i, j, k
// loop order.  Counts overlapping cells and stops at `limit`; EMIT also
// stores the keys of the first 8.  Per corner the arithmetic is the shader's;
// what a corner shares with its neighbours is computed once: the boundary
// coordinates of an axis (cell k's upper boundary is cell k + 1's lower one,
// the same float: (float)(k + st) == (float)k + (float)st below 2^24), the
// products with the inverse rotation, and the i-j part of each corner's sum.
template <bool EMIT, bool XF>
__device__ __forceinline__ uint32_t vb_scan_level(const VoxelBvhParams& P, const VbGauss& G, const float w2v[4],
                                                  const int lo[3], const int hi[3], uint32_t level, uint32_t limit,
                                                  uint64_t key[8])
{
    const int msk = ~((1 << level) - 1), st = 1 << level;
    const float step = (float)(1u << level);
    uint32_t count = 0;
    for (int i = lo[0] & msk; i <= (hi[0] & msk); i += st)
    {
        const float pi[2] = { vb_lp(w2v, (float)i, 0), vb_lp(w2v, __fadd_rn((float)i, step), 0) };
        for (int j = lo[1] & msk; j <= (hi[1] & msk); j += st)
        {
            const float pj[2] = { vb_lp(w2v, (float)j, 1), vb_lp(w2v, __fadd_rn((float)j, step), 1) };
            // no transform: s01[r][b0][b1] = (pi - mu0) R[0][r] + (pj - mu1) R[1][r]
            // transform:    s01[c][b0][b1] = pi T[c] + pj T[4 + c]
            float s01[3][2][2];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int b0 = 0; b0 < 2; b0++)
#pragma unroll
                    for (int b1 = 0; b1 < 2; b1++)
                    {
                        if (XF)
                            s01[r][b0][b1] = __fadd_rn(__fmul_rn(pi[b0], P.ti[r]), __fmul_rn(pj[b1], P.ti[4 + r]));
                        else
                            s01[r][b0][b1] = __fadd_rn(__fmul_rn(__fsub_rn(pi[b0], G.mu[0]), G.R[0][r]),
                                                       __fmul_rn(__fsub_rn(pj[b1], G.mu[1]), G.R[1][r]));
                    }
            // without a transform a corner's row value is fl(fl(s01 + z term) inv_r); rounded
            // addition and a positive finite multiplier are monotone, so the minimum
            // (maximum) over the 8 corners is that expression over the smallest
            // (largest) s01 and z term - the shader's 8-corner result, bit for bit (a tie
            // differs at most in the sign of a zero, which the test compares with zero)
            const bool mono = !XF && G.inv[0] > 0.f && G.inv[1] > 0.f && G.inv[2] > 0.f &&
                              G.inv[0] < __int_as_float(0x7f800000) && G.inv[1] < __int_as_float(0x7f800000) &&
                              G.inv[2] < __int_as_float(0x7f800000);
            float smin[3], smax[3];
#pragma unroll
            for (int r = 0; r < 3; r++)
            {
                smin[r] = fminf(fminf(s01[r][0][0], s01[r][0][1]), fminf(s01[r][1][0], s01[r][1][1]));
                smax[r] = fmaxf(fmaxf(s01[r][0][0], s01[r][0][1]), fmaxf(s01[r][1][0], s01[r][1][1]));
            }
            int k = lo[2] & msk;
            float pk0 = vb_lp(w2v, (float)k, 2);
            for (; k <= (hi[2] & msk); k += st)
            {
                const float pk1 = vb_lp(w2v, __fadd_rn((float)k, step), 2);
                const float pk[2] = { pk0, pk1 };
                pk0 = pk1;
                float vmin[3] = { 0.f, 0.f, 0.f }, vmax[3] = { 0.f, 0.f, 0.f };
                if (mono)
                {
#pragma unroll
                    for (int r = 0; r < 3; r++)
                    {
                        const float za = __fmul_rn(__fsub_rn(pk[0], G.mu[2]), G.R[2][r]);
                        const float zb = __fmul_rn(__fsub_rn(pk[1], G.mu[2]), G.R[2][r]);
                        vmin[r] = __fmul_rn(__fadd_rn(smin[r], fminf(za, zb)), G.inv[r]);
                        vmax[r] = __fmul_rn(__fadd_rn(smax[r], fmaxf(za, zb)), G.inv[r]);
                    }
                }
                else
#pragma unroll
                for (int v = 0; v < 8; v++)
                {
                    const int b0 = v & 1, b1 = (v >> 1) & 1, b2 = (v >> 2) & 1;
                    float lr[3];
                    if (XF)
                    {
                        float d[3];
#pragma unroll
                        for (int c = 0; c < 3; c++)
                            d[c] = __fsub_rn(
                                __fadd_rn(__fadd_rn(s01[c][b0][b1], __fmul_rn(pk[b2], P.ti[8 + c])), P.ti[12 + c]),
                                G.mu[c]);
#pragma unroll
                        for (int r = 0; r < 3; r++)
                            lr[r] = __fadd_rn(__fadd_rn(__fmul_rn(d[0], G.R[0][r]), __fmul_rn(d[1], G.R[1][r])),
                                              __fmul_rn(d[2], G.R[2][r]));
                    }
                    else
                    {
#pragma unroll
                        for (int r = 0; r < 3; r++)
                            lr[r] = __fadd_rn(s01[r][b0][b1], __fmul_rn(__fsub_rn(pk[b2], G.mu[2]), G.R[2][r]));
                    }
#pragma unroll
                    for (int r = 0; r < 3; r++)
                    {
                        const float x = __fmul_rn(lr[r], G.inv[r]);
                        if (v == 0 || x < vmin[r])
                            vmin[r] = x;
                        if (v == 0 || x > vmax[r])
                            vmax[r] = x;
                    }
                }
                float dist2 = 1.f;
#pragma unroll
                for (int a = 0; a < 3; a++)
                {
                    if (0.f < vmin[a])
                        dist2 = __fsub_rn(dist2, __fmul_rn(vmin[a], vmin[a]));
                    else if (0.f > vmax[a])
                        dist2 = __fsub_rn(dist2, __fmul_rn(vmax[a], vmax[a]));
                }
                if (dist2 > 0.f)
                {
                    if (EMIT)
                    {
                        const uint64_t kv = ((uint64_t)(int64_t)i << 48) | ((uint64_t)(int64_t)j << 32) |
                                            ((uint64_t)(int64_t)k << 16) | (uint64_t)level;
#pragma unroll
                        for (int s = 0; s < 8; s++) // register-resident insert
                            if ((uint32_t)s == count)
                                key[s] = kv;
                    }
                    if (++count >= limit)
                        return count;
                }
            }
        }
    }
    return count;
}

__global__ void k_vb_init(uint32_t* box_keys, int* cell_minmax)
{
    if (threadIdx.x < 3)
        box_keys[threadIdx.x] = 0xff800000u; // key of +inf
    else if (threadIdx.x < 6)
        box_keys[threadIdx.x] = 0x007fffffu; // key of -inf
    if (threadIdx.x < 3)
        cell_minmax[threadIdx.x] = 0x7fffffff;
    else if (threadIdx.x < 6)
        cell_minmax[threadIdx.x] = (int)0x80000000;
}

__global__ void __launch_bounds__(VB_THREADS) k_vb_box(VoxelBvhParams P)
{
    uint32_t mn[3] = { 0xff800000u, 0xff800000u, 0xff800000u }, mx[3] = { 0x007fffffu, 0x007fffffu, 0x007fffffu };
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < P.n; g += (int64_t)gridDim.x * blockDim.x)
    {
        VbGauss G;
        vb_load(P, g, G);
        uint32_t a0[3], a1[3];
        if (!vb_box_keys(P, G, a0, a1))
            atomicOr(P.err, ERR_RANGE);
#pragma unroll
        for (int a = 0; a < 3; a++)
        {
            mn[a] = a0[a] < mn[a] ? a0[a] : mn[a];
            mx[a] = a1[a] > mx[a] ? a1[a] : mx[a];
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const uint32_t wmn = __reduce_min_sync(0xffffffffu, mn[a]);
        const uint32_t wmx = __reduce_max_sync(0xffffffffu, mx[a]);
        if ((threadIdx.x & 31) == 0)
        {
            atomicMin(&P.box_keys[a], wmn);
            atomicMax(&P.box_keys[3 + a], wmx);
        }
    }
}

__device__ __forceinline__ bool vb_cell_ok(float v)
{
    return v >= -VB_CELL_LIMIT && v <= VB_CELL_LIMIT; // false for NaN
}

template <bool XF>
// 3 resident CTAs per SM: 80 registers, faster than the 89 the compiler picks unbounded
// (2 CTAs per SM)
__global__ void __launch_bounds__(VB_THREADS, 3) k_vb_ijkl(VoxelBvhParams P)
{
    // compute_world_to_voxel (voxelbvh_gaussians_to_ijkl.slang:111-118)
    float wmin[3], wmax[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        wmin[a] = vb_funkey(P.box_keys[a]);
        wmax[a] = vb_funkey(P.box_keys[3 + a]);
    }
    if (blockIdx.x == 0 && threadIdx.x < 6)
        P.world_bbox[threadIdx.x] = threadIdx.x < 3 ? wmin[threadIdx.x] : wmax[threadIdx.x - 3];
    const float d0 = __fsub_rn(wmax[0], wmin[0]), d1 = __fsub_rn(wmax[1], wmin[1]), d2 = __fsub_rn(wmax[2], wmin[2]);
    const float dyz = d1 > d2 ? d1 : d2;
    const float dmax = d0 > dyz ? d0 : dyz;
    const float sc = __fdiv_rn((float)(P.resolution - 1u), dmax);
    const float w2v[4] = { __fadd_rn(__fmul_rn(-wmin[0], sc), 0.5f), __fadd_rn(__fmul_rn(-wmin[1], sc), 0.5f),
                           __fadd_rn(__fmul_rn(-wmin[2], sc), 0.5f), sc };

    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P.n)
        return;
    VbGauss G;
    vb_load(P, g, G);
    uint32_t kmn[3], kmx[3];
    bool ok = vb_box_keys(P, G, kmn, kmx);
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const float fl = floorf(__fadd_rn(__fmul_rn(sc, vb_funkey(kmn[a])), w2v[a]));
        const float fh = floorf(__fadd_rn(__fmul_rn(sc, vb_funkey(kmx[a])), w2v[a]));
        ok = ok && vb_cell_ok(fl) && vb_cell_ok(fh);
        lo[a] = (int)fl;
        hi[a] = (int)fh;
    }
    uint64_t key[8] = { ~0ull, ~0ull, ~0ull, ~0ull, ~0ull, ~0ull, ~0ull, ~0ull };
    uint32_t nkeys = 0;
    if (ok)
    {
        // level search (voxelbvh_gaussians_to_ijkl.slang:187-229): only
        // "more than 8 overlap" matters, so a level whose box holds at most 8
        // cells needs no test, and a count stops at 9
        uint32_t level = 11u, last_good = 11u;
        bool bounded = true;
        while (true)
        {
            const int msk = ~((1 << level) - 1);
            int64_t cells = 1;
#pragma unroll
            for (int a = 0; a < 3; a++)
                cells *= (int64_t)(((hi[a] & msk) - (lo[a] & msk)) >> level) + 1;
            if (cells > VB_MAX_CELLS)
            {
                bounded = false;
                break;
            }
            if (cells > 8 && vb_scan_level<false, XF>(P, G, w2v, lo, hi, level, 9u, key) > 8u)
            {
                level = last_good;
                break;
            }
            if (level == 0u)
                break;
            last_good = level;
            level -= 1u;
        }
        // emission: the first 8 overlapping cells in i, j, k loop order
        if (bounded)
            nkeys = vb_scan_level<true, XF>(P, G, w2v, lo, hi, level, 8u, key);
        else
            atomicOr(P.err, ERR_RANGE);
    }
    else
        atomicOr(P.err, ERR_RANGE);
    // range of the emitted cell coordinates (sizes the compressed sort key)
    int cmin[3] = { 0x7fffffff, 0x7fffffff, 0x7fffffff }, cmax[3] = { (int)0x80000000, (int)0x80000000, (int)0x80000000 };
#pragma unroll
    for (int s = 0; s < 8; s++)
        if ((uint32_t)s < nkeys)
        {
            const int c[3] = { (int)(int16_t)(key[s] >> 48), (int)(int16_t)(key[s] >> 32), (int)(int16_t)(key[s] >> 16) };
#pragma unroll
            for (int a = 0; a < 3; a++)
            {
                cmin[a] = min(cmin[a], c[a]);
                cmax[a] = max(cmax[a], c[a]);
            }
        }
    ulonglong2* kd = reinterpret_cast<ulonglong2*>(P.keys + 8 * g);
#pragma unroll
    for (int s = 0; s < 4; s++)
        kd[s] = make_ulonglong2(key[2 * s], key[2 * s + 1]);
    const uint32_t id = (uint32_t)g;
    uint4* idd = reinterpret_cast<uint4*>(P.ids + 8 * g);
    idd[0] = make_uint4(nkeys > 0 ? id : ~0u, nkeys > 1 ? id : ~0u, nkeys > 2 ? id : ~0u, nkeys > 3 ? id : ~0u);
    idd[1] = make_uint4(nkeys > 4 ? id : ~0u, nkeys > 5 ? id : ~0u, nkeys > 6 ? id : ~0u, nkeys > 7 ? id : ~0u);
    const uint32_t active = __activemask();
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const int wmn = __reduce_min_sync(active, cmin[a]), wmx = __reduce_max_sync(active, cmax[a]);
        if ((threadIdx.x & 31) == __ffs(active) - 1)
        {
            if (wmn != 0x7fffffff)
                atomicMin(&P.cell_minmax[a], wmn);
            if (wmx != (int)0x80000000)
                atomicMax(&P.cell_minmax[3 + a], wmx);
        }
    }
}

// ---------------------------------------------------------------------------
// Lane-balanced search: k_vb_setup writes one 96-byte record per Gaussian
// (mean, rotation, 1 / (local_scale * scale), cell box, status) with a thread
// per Gaussian; k_vb_search then runs a persistent loop in which every lane
// tests ONE cell per iteration and, when its Gaussian is done, takes the next
// one (static stride).  Lanes stay busy whatever the per-Gaussian trip counts,
// which differ by orders of magnitude between neighbouring Gaussians.  Same
// tests, same order, same keys as k_vb_ijkl.
constexpr int VB_REC = 24; // floats per record: mu 3, R 9, inv 3, lo 3, hi 3, status 1, pad 2

__global__ void __launch_bounds__(VB_THREADS) k_vb_setup(VoxelBvhParams P)
{
    float wmin[3], wmax[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        wmin[a] = vb_funkey(P.box_keys[a]);
        wmax[a] = vb_funkey(P.box_keys[3 + a]);
    }
    if (blockIdx.x == 0 && threadIdx.x < 6)
        P.world_bbox[threadIdx.x] = threadIdx.x < 3 ? wmin[threadIdx.x] : wmax[threadIdx.x - 3];
    const float d0 = __fsub_rn(wmax[0], wmin[0]), d1 = __fsub_rn(wmax[1], wmin[1]), d2 = __fsub_rn(wmax[2], wmin[2]);
    const float dyz = d1 > d2 ? d1 : d2;
    const float dmax = d0 > dyz ? d0 : dyz;
    const float sc = __fdiv_rn((float)(P.resolution - 1u), dmax);
    const float w2v[3] = { __fadd_rn(__fmul_rn(-wmin[0], sc), 0.5f), __fadd_rn(__fmul_rn(-wmin[1], sc), 0.5f),
                           __fadd_rn(__fmul_rn(-wmin[2], sc), 0.5f) };
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P.n)
        return;
    VbGauss G;
    vb_load(P, g, G);
    uint32_t kmn[3], kmx[3];
    bool ok = vb_box_keys(P, G, kmn, kmx);
    float r[VB_REC];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const float fl = floorf(__fadd_rn(__fmul_rn(sc, vb_funkey(kmn[a])), w2v[a]));
        const float fh = floorf(__fadd_rn(__fmul_rn(sc, vb_funkey(kmx[a])), w2v[a]));
        ok = ok && vb_cell_ok(fl) && vb_cell_ok(fh);
        r[15 + a] = __int_as_float(vb_cell_ok(fl) ? (int)fl : 0);
        r[18 + a] = __int_as_float(vb_cell_ok(fh) ? (int)fh : 0);
        r[a] = G.mu[a];
        r[12 + a] = G.inv[a];
#pragma unroll
        for (int c = 0; c < 3; c++)
            r[3 + 3 * a + c] = G.R[a][c];
    }
    r[21] = ok ? 1.f : 0.f;
    r[22] = 0.f;
    r[23] = 0.f;
    if (!ok)
        atomicOr(P.err, ERR_RANGE);
    float4* dst = reinterpret_cast<float4*>(P.rec + (size_t)VB_REC * g);
#pragma unroll
    for (int q = 0; q < VB_REC / 4; q++)
        dst[q] = make_float4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
}

// voxel_ellipsoid_overlap of one cell (corner arithmetic as in vb_scan_level,
// without the reuse across neighbouring cells)
template <bool XF>
__device__ __forceinline__ bool vb_overlap_cell(const VoxelBvhParams& P, const float* rec, const float w2v[4], int i,
                                                int j, int k, uint32_t level)
{
    const float* mu = rec;
    const float* R = rec + 3; // R[3 * a + r] = G.R[a][r]
    const float* inv = rec + 12;
    const float step = (float)(1u << level);
    const int ijk[3] = { i, j, k };
    float lp[3][2];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const float v0 = (float)ijk[a];
        lp[a][0] = vb_lp(w2v, v0, a);
        lp[a][1] = vb_lp(w2v, __fadd_rn(v0, step), a);
    }
    float q[3][3][2];
    if (!XF)
    {
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
            {
                const float d = __fsub_rn(lp[a][b], mu[a]);
#pragma unroll
                for (int r = 0; r < 3; r++)
                    q[r][a][b] = __fmul_rn(d, R[3 * a + r]);
            }
    }
    float vmin[3] = { 0.f, 0.f, 0.f }, vmax[3] = { 0.f, 0.f, 0.f };
    // Without a transform the corner value of row r is fl(fl(fl(q0 + q1) + q2) inv_r)
    // over one product per axis; rounded addition and a positive finite
    // multiplier are monotone, so the minimum (maximum) over the 8 corners is
    // the same expression over the per-axis minimum (maximum) products - the
    // shader's 8-corner loop's result, bit for bit (a tie differs at most in the
    // sign of a zero, which the test below compares with zero)
    if (!XF && inv[0] > 0.f && inv[1] > 0.f && inv[2] > 0.f && inv[0] < __int_as_float(0x7f800000) &&
        inv[1] < __int_as_float(0x7f800000) && inv[2] < __int_as_float(0x7f800000))
    {
#pragma unroll
        for (int r = 0; r < 3; r++)
        {
            const float lo = __fadd_rn(__fadd_rn(fminf(q[r][0][0], q[r][0][1]), fminf(q[r][1][0], q[r][1][1])),
                                       fminf(q[r][2][0], q[r][2][1]));
            const float hi = __fadd_rn(__fadd_rn(fmaxf(q[r][0][0], q[r][0][1]), fmaxf(q[r][1][0], q[r][1][1])),
                                       fmaxf(q[r][2][0], q[r][2][1]));
            vmin[r] = __fmul_rn(lo, inv[r]);
            vmax[r] = __fmul_rn(hi, inv[r]);
        }
    }
    else
#pragma unroll
    for (int v = 0; v < 8; v++)
    {
        const int b0 = v & 1, b1 = (v >> 1) & 1, b2 = (v >> 2) & 1;
        float lr[3];
        if (XF)
        {
            float d[3];
#pragma unroll
            for (int c = 0; c < 3; c++)
                d[c] = __fsub_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(lp[0][b0], P.ti[c]),
                                                               __fmul_rn(lp[1][b1], P.ti[4 + c])),
                                                     __fmul_rn(lp[2][b2], P.ti[8 + c])),
                                           P.ti[12 + c]),
                                 mu[c]);
#pragma unroll
            for (int r = 0; r < 3; r++)
                lr[r] = __fadd_rn(__fadd_rn(__fmul_rn(d[0], R[r]), __fmul_rn(d[1], R[3 + r])), __fmul_rn(d[2], R[6 + r]));
        }
        else
        {
#pragma unroll
            for (int r = 0; r < 3; r++)
                lr[r] = __fadd_rn(__fadd_rn(q[r][0][b0], q[r][1][b1]), q[r][2][b2]);
        }
#pragma unroll
        for (int r = 0; r < 3; r++)
        {
            const float x = __fmul_rn(lr[r], inv[r]);
            if (v == 0 || x < vmin[r])
                vmin[r] = x;
            if (v == 0 || x > vmax[r])
                vmax[r] = x;
        }
    }
    float dist2 = 1.f;
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        if (0.f < vmin[a])
            dist2 = __fsub_rn(dist2, __fmul_rn(vmin[a], vmin[a]));
        else if (0.f > vmax[a])
            dist2 = __fsub_rn(dist2, __fmul_rn(vmax[a], vmax[a]));
    }
    return dist2 > 0.f;
}

struct VbCursor
{
    int i, j, k, i1, j0, j1, k0, k1, st;
};

__device__ __forceinline__ int64_t vb_level_cells(const int lo[3], const int hi[3], uint32_t level)
{
    const int msk = ~((1 << level) - 1);
    int64_t cells = 1;
#pragma unroll
    for (int a = 0; a < 3; a++)
        cells *= (int64_t)(((hi[a] & msk) - (lo[a] & msk)) >> level) + 1;
    return cells;
}

__device__ __forceinline__ void vb_cursor_start(VbCursor& C, const int lo[3], const int hi[3], uint32_t level)
{
    const int msk = ~((1 << level) - 1);
    C.st = 1 << level;
    C.i = lo[0] & msk;
    C.i1 = hi[0] & msk;
    C.j0 = C.j = lo[1] & msk;
    C.j1 = hi[1] & msk;
    C.k0 = C.k = lo[2] & msk;
    C.k1 = hi[2] & msk;
}

// Position the search at the first level from `level` down that needs a
// test (more than 8 cells: count with limit 9), or at an untested level 0
// (emit).  Levels of at most 8 cells are chosen-so-far without a test.
// Returns false when a level exceeds VB_MAX_CELLS.
__device__ __forceinline__ bool vb_descend(const int lo[3], const int hi[3], uint32_t& level, uint32_t& last_good,
                                           bool& have, bool& emit, VbCursor& C, uint32_t& count, uint64_t cur[8])
{
    while (true)
    {
        const int64_t cells = vb_level_cells(lo, hi, level);
        if (cells > VB_MAX_CELLS)
            return false;
        if (cells > 8 || level == 0u)
        {
            emit = cells <= 8;
            if (emit)
                have = false;
            vb_cursor_start(C, lo, hi, level);
            count = 0;
#pragma unroll
            for (int s = 0; s < 8; s++)
                cur[s] = ~0ull;
            return true;
        }
        have = false;
        last_good = level;
        level -= 1u;
    }
}

template <bool XF>
__global__ void __launch_bounds__(VB_THREADS) k_vb_search(VoxelBvhParams P)
{
    float wmin[3], wmax[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        wmin[a] = vb_funkey(P.box_keys[a]);
        wmax[a] = vb_funkey(P.box_keys[3 + a]);
    }
    const float d0 = __fsub_rn(wmax[0], wmin[0]), d1 = __fsub_rn(wmax[1], wmin[1]), d2 = __fsub_rn(wmax[2], wmin[2]);
    const float dyz = d1 > d2 ? d1 : d2;
    const float dmax = d0 > dyz ? d0 : dyz;
    const float sc = __fdiv_rn((float)(P.resolution - 1u), dmax);
    const float w2v[4] = { __fadd_rn(__fmul_rn(-wmin[0], sc), 0.5f), __fadd_rn(__fmul_rn(-wmin[1], sc), 0.5f),
                           __fadd_rn(__fmul_rn(-wmin[2], sc), 0.5f), sc };

    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x - stride;
    float rec[VB_REC];
    int lo[3] = { 0, 0, 0 }, hi[3] = { 0, 0, 0 };
    uint32_t level = 0, last_good = 0, count = 0, nkeys = 0;
    bool busy = false, have = false, emit = false;
    VbCursor C{};
    uint64_t cur[8];
    int cmin[3] = { 0x7fffffff, 0x7fffffff, 0x7fffffff }, cmax[3] = { (int)0x80000000, (int)0x80000000, (int)0x80000000 };
    while (true)
    {
        int finish = 0; // 1: done with cells, 2: done without (unused slots)
        if (!busy)
        {
            // ---- the lane's next Gaussian
            g += stride;
            if (g >= P.n)
                break;
            const float4* src = reinterpret_cast<const float4*>(P.rec + (size_t)VB_REC * g);
#pragma unroll
            for (int q = 0; q < VB_REC / 4; q++)
            {
                const float4 v = src[q];
                rec[4 * q] = v.x;
                rec[4 * q + 1] = v.y;
                rec[4 * q + 2] = v.z;
                rec[4 * q + 3] = v.w;
            }
#pragma unroll
            for (int a = 0; a < 3; a++)
            {
                lo[a] = __float_as_int(rec[15 + a]);
                hi[a] = __float_as_int(rec[18 + a]);
            }
            level = 11u;
            last_good = 11u;
            have = false;
            nkeys = 0;
            if (rec[21] == 0.f || !vb_descend(lo, hi, level, last_good, have, emit, C, count, cur))
                finish = 2;
            else
                busy = true;
        }
        else
        {
            // ---- one cell of the current level
            if (vb_overlap_cell<XF>(P, rec, w2v, C.i, C.j, C.k, level))
            {
                const uint64_t kv = ((uint64_t)(int64_t)C.i << 48) | ((uint64_t)(int64_t)C.j << 32) |
                                    ((uint64_t)(int64_t)C.k << 16) | (uint64_t)level;
#pragma unroll
                for (int s = 0; s < 8; s++) // register-resident insert
                    if ((uint32_t)s == count)
                        cur[s] = kv;
                count++;
            }
            C.k += C.st;
            if (C.k > C.k1)
            {
                C.k = C.k0;
                C.j += C.st;
                if (C.j > C.j1)
                {
                    C.j = C.j0;
                    C.i += C.st;
                }
            }
            if (C.i > C.i1 || (emit ? count >= 8u : count > 8u))
            {
                // level done; it is the chosen one so far unless it
                // overflows below level 11 (level 11 stays with its first 8)
                if (emit || count <= 8u || level == last_good)
                {
                    ulonglong2* kd = reinterpret_cast<ulonglong2*>(P.keys + 8 * g);
#pragma unroll
                    for (int s = 0; s < 4; s++)
                        kd[s] = make_ulonglong2(cur[2 * s], cur[2 * s + 1]);
                    nkeys = count < 8u ? count : 8u;
                    have = true;
                }
                if (emit)
                    finish = 1;
                else if (count > 8u)
                {
                    level = last_good;
                    if (have)
                        finish = 1;
                    else
                    {
                        // the chosen level was decided untested: emit it
                        emit = true;
                        vb_cursor_start(C, lo, hi, level);
                        count = 0;
#pragma unroll
                        for (int s = 0; s < 8; s++)
                            cur[s] = ~0ull;
                    }
                }
                else if (level == 0u)
                    finish = 1;
                else
                {
                    last_good = level;
                    level -= 1u;
                    if (!vb_descend(lo, hi, level, last_good, have, emit, C, count, cur))
                        finish = 2;
                }
            }
        }
        if (finish != 0)
        {
            if (finish == 2)
            {
                // not finite / out of range / unbounded: unused slots, error
                if (rec[21] != 0.f)
                    atomicOr(P.err, ERR_RANGE);
                ulonglong2* kd = reinterpret_cast<ulonglong2*>(P.keys + 8 * g);
#pragma unroll
                for (int s = 0; s < 4; s++)
                    kd[s] = make_ulonglong2(~0ull, ~0ull);
                nkeys = 0;
            }
            else if (nkeys > 0)
            {
                const int msk = ~((1 << level) - 1);
#pragma unroll
                for (int a = 0; a < 3; a++)
                {
                    cmin[a] = min(cmin[a], lo[a] & msk);
                    cmax[a] = max(cmax[a], hi[a] & msk);
                }
            }
            const uint32_t id = (uint32_t)g;
            uint4* idd = reinterpret_cast<uint4*>(P.ids + 8 * g);
            idd[0] = make_uint4(nkeys > 0 ? id : ~0u, nkeys > 1 ? id : ~0u, nkeys > 2 ? id : ~0u, nkeys > 3 ? id : ~0u);
            idd[1] = make_uint4(nkeys > 4 ? id : ~0u, nkeys > 5 ? id : ~0u, nkeys > 6 ? id : ~0u, nkeys > 7 ? id : ~0u);
            busy = false;
        }
    }
    // every lane gets here (the loop only breaks)
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const int wmn = __reduce_min_sync(0xffffffffu, cmin[a]), wmx = __reduce_max_sync(0xffffffffu, cmax[a]);
        if ((threadIdx.x & 31) == 0)
        {
            if (wmn != 0x7fffffff)
                atomicMin(&P.cell_minmax[a], wmn);
            if (wmx != (int)0x80000000)
                atomicMax(&P.cell_minmax[3 + a], wmx);
        }
    }
}

// starts (key differs from its predecessor) of one 2048-key tile, per thread 8
// consecutive keys
template <class K>
__device__ __forceinline__ uint32_t vb_tile_flags(const K* keys, int64_t N, int64_t i0, uint32_t& first,
                                                  uint32_t& last)
{
    first = 0;
    last = 0;
    if (i0 >= N)
        return 0;
    K prev = i0 > 0 ? keys[i0 - 1] : K(0);
    K cur = keys[i0];
#pragma unroll
    for (int s = 0; s < 8; s++)
    {
        const int64_t i = i0 + s;
        if (i >= N)
            break;
        const K next = i + 1 < N ? keys[i + 1] : K(~cur);
        if (i == 0 || cur != prev)
            first |= 1u << s;
        if (cur != next)
            last |= 1u << s;
        prev = cur;
        cur = next;
    }
    return (uint32_t)__popc(first);
}

template <class K>
__global__ void __launch_bounds__(VB_THREADS) k_vb_range_count(const K* keys, int64_t N, uint64_t* counts)
{
    __shared__ uint32_t s_w[VB_THREADS / 32];
    const int64_t i0 = (int64_t)blockIdx.x * VB_TILE + 8 * threadIdx.x;
    uint32_t f, l;
    uint32_t c = vb_tile_flags(keys, N, i0, f, l);
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0)
        s_w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        uint64_t t = 0;
        for (int w = 0; w < VB_THREADS / 32; w++)
            t += s_w[w];
        counts[blockIdx.x] = t;
    }
}

// 64-bit key of a compressed key (VbRangeParams::bits)
template <class K>
__device__ __forceinline__ uint64_t vb_expand(K c, const VbRangeParams& R)
{
    if ((uint64_t)c == R.sentinel)
        return ~0ull;
    const uint64_t u = (uint64_t)c;
    const uint64_t level = u & 15u;
    const uint64_t k = (u >> 4) & ((1ull << R.bits[2]) - 1);
    const uint64_t j = (u >> (4 + R.bits[2])) & ((1ull << R.bits[1]) - 1);
    const uint64_t i = u >> (4 + R.bits[2] + R.bits[1]);
    return (i << 48) | (j << 32) | (k << 16) | level;
}

// headers [2r] = start, [2r + 1] = end, zeros from the range count on; with
// R.expand the sorted compressed keys are written out as 64-bit keys, and the
// ids copied when the sort left them in its second buffer
template <class K>
__global__ void __launch_bounds__(VB_THREADS) k_vb_range_scatter(const K* keys, int64_t N, const uint64_t* offs,
                                                                   const uint64_t* total, VbRangeParams R)
{
    __shared__ uint64_t s_warp[33];
    const int64_t i0 = (int64_t)blockIdx.x * VB_TILE + 8 * threadIdx.x;
    uint32_t first, last;
    const uint32_t c = vb_tile_flags(keys, N, i0, first, last);
    uint64_t tile_total;
    // inclusive count of starts before this thread's first key, minus one
    const int64_t base = (int64_t)offs[blockIdx.x] + (int64_t)block_excl_scan_u64(c, s_warp, tile_total) - 1;
    const uint64_t nr = *total;
    int64_t r = base;
#pragma unroll
    for (int s = 0; s < 8; s++)
    {
        const int64_t i = i0 + s;
        if (i >= N)
            break;
        if (first & (1u << s))
        {
            r++;
            R.range[2 * r] = (uint32_t)i;
        }
        if (last & (1u << s))
            R.range[2 * r + 1] = (uint32_t)(i + 1);
        if ((uint64_t)i >= nr)
        {
            R.range[2 * i] = 0u;
            R.range[2 * i + 1] = 0u;
        }
        if (R.expand)
            R.keys_out[i] = vb_expand(keys[i], R);
        if (R.ids_src)
            R.ids_out[i] = R.ids_src[i];
    }
}

// Compaction of the used slots before the sort: a Gaussian's used slots are
// the first of its 8 (the unused ones carry key ~0 and id ~0, identical pairs,
// so after a stable sort they simply fill the tail).  The compressed key
// holds i, j, k in bits[0], bits[1], bits[2] bits above a 4-bit level, in the
// order of the 64-bit key for cells in [0, 2^bits).  k_vb_used: each
// Gaussian's used count; k_vb_compress_used: the used slots' compressed keys
// and ids at their scanned positions; k_vb_tail: the tail's keys, ids and
// headers (the unused run [U, N) is the last range).
__global__ void __launch_bounds__(VB_THREADS) k_vb_used(const uint32_t* __restrict__ ids, int64_t count,
                                                        uint32_t* __restrict__ used)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= count)
        return;
    const uint4* p = reinterpret_cast<const uint4*>(ids + 8 * g);
    const uint4 a = p[0], b = p[1];
    used[g] = (uint32_t)(a.x != ~0u) + (a.y != ~0u) + (a.z != ~0u) + (a.w != ~0u) + (b.x != ~0u) + (b.y != ~0u) +
              (b.z != ~0u) + (b.w != ~0u);
}

template <class K>
__global__ void __launch_bounds__(VB_THREADS) k_vb_compress_used(const uint64_t* __restrict__ keys,
                                                                   const uint32_t* __restrict__ ids, int64_t count,
                                                                   const uint32_t* __restrict__ used,
                                                                   const uint32_t* __restrict__ off, VbRangeParams R,
                                                                   K* __restrict__ out_keys, uint32_t* __restrict__ out_ids)
{
    const int64_t N = 8 * count;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t g = t >> 3;
        const uint32_t slot = (uint32_t)(t & 7);
        if (slot >= used[g])
            continue;
        const uint64_t u = keys[t];
        const uint64_t i = (u >> 48) & 0xffffu, j = (u >> 32) & 0xffffu, k = (u >> 16) & 0xffffu, level = u & 15u;
        const int64_t dst = (int64_t)off[g] + slot;
        out_keys[dst] = (K)((((i << R.bits[1] | j) << R.bits[2] | k) << 4) | level);
        out_ids[dst] = ids[t];
    }
}

__global__ void __launch_bounds__(VB_THREADS) k_vb_tail(int64_t U, int64_t N, const uint64_t* __restrict__ nr_used,
                                                        uint64_t* __restrict__ ranges_out, VbRangeParams R)
{
    const uint64_t nr = *nr_used;
    for (int64_t i = U + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    {
        R.keys_out[i] = ~0ull;
        R.ids_out[i] = ~0u;
        if ((uint64_t)i != nr)
        {
            R.range[2 * i] = 0u;
            R.range[2 * i + 1] = 0u;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        R.range[2 * nr] = (uint32_t)U;
        R.range[2 * nr + 1] = (uint32_t)N;
        *ranges_out = nr + 1;
    }
}

} // namespace

void launch_vb_used(const uint32_t* ids, int64_t count, uint32_t* used, cudaStream_t s)
{
    if (count <= 0)
        return;
    k_vb_used<<<(unsigned)((count + VB_THREADS - 1) / VB_THREADS), VB_THREADS, 0, s>>>(ids, count, used);
    count_launch();
}

void launch_vb_compress_used(const uint64_t* keys, const uint32_t* ids, int64_t count, const uint32_t* used,
                             const uint32_t* off, const VbRangeParams& R, void* out_keys, uint32_t* out_ids, int key32,
                             int num_sms, cudaStream_t s)
{
    if (count <= 0)
        return;
    int64_t grid = (8 * count + VB_THREADS - 1) / VB_THREADS;
    const int64_t cap = (int64_t)num_sms * 16;
    if (grid > cap)
        grid = cap;
    if (key32)
        k_vb_compress_used<uint32_t><<<(unsigned)grid, VB_THREADS, 0, s>>>(keys, ids, count, used, off, R,
                                                                           (uint32_t*)out_keys, out_ids);
    else
        k_vb_compress_used<uint64_t><<<(unsigned)grid, VB_THREADS, 0, s>>>(keys, ids, count, used, off, R,
                                                                           (uint64_t*)out_keys, out_ids);
    count_launch();
}

void launch_vb_tail(int64_t U, int64_t N, const uint64_t* nr_used, uint64_t* ranges_out, const VbRangeParams& R,
                    int num_sms, cudaStream_t s)
{
    int64_t grid = (N - U + VB_THREADS - 1) / VB_THREADS;
    const int64_t cap = (int64_t)num_sms * 8;
    if (grid > cap)
        grid = cap;
    if (grid < 1)
        grid = 1;
    k_vb_tail<<<(unsigned)grid, VB_THREADS, 0, s>>>(U, N, nr_used, ranges_out, R);
    count_launch();
}

void launch_vb_init(uint32_t* box_keys, int* cell_minmax, cudaStream_t s)
{
    k_vb_init<<<1, 32, 0, s>>>(box_keys, cell_minmax);
    count_launch();
}

void launch_vb_box(const VoxelBvhParams& P, int num_sms, cudaStream_t s)
{
    if (P.n <= 0)
        return;
    int64_t grid = (P.n + VB_THREADS - 1) / VB_THREADS;
    const int64_t cap = (int64_t)num_sms * 8;
    if (grid > cap)
        grid = cap;
    k_vb_box<<<(unsigned)grid, VB_THREADS, 0, s>>>(P);
    count_launch();
}

void launch_vb_search(const VoxelBvhParams& P, int num_sms, cudaStream_t s)
{
    const int64_t grid1 = P.n > 0 ? (P.n + VB_THREADS - 1) / VB_THREADS : 1;
    k_vb_setup<<<(unsigned)grid1, VB_THREADS, 0, s>>>(P);
    count_launch();
    if (P.n <= 0)
        return;
    int per_sm = 0;
    if (P.has_xform)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vb_search<true>, VB_THREADS, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vb_search<false>, VB_THREADS, 0);
    int64_t grid = (int64_t)num_sms * (per_sm > 0 ? per_sm : 1);
    if (grid > grid1)
        grid = grid1;
    if (P.has_xform)
        k_vb_search<true><<<(unsigned)grid, VB_THREADS, 0, s>>>(P);
    else
        k_vb_search<false><<<(unsigned)grid, VB_THREADS, 0, s>>>(P);
    count_launch();
}

void launch_vb_ijkl(const VoxelBvhParams& P, cudaStream_t s)
{
    // one block even for n = 0: it writes the world box
    const int64_t grid = P.n > 0 ? (P.n + VB_THREADS - 1) / VB_THREADS : 1;
    if (P.has_xform)
        k_vb_ijkl<true><<<(unsigned)grid, VB_THREADS, 0, s>>>(P);
    else
        k_vb_ijkl<false><<<(unsigned)grid, VB_THREADS, 0, s>>>(P);
    count_launch();
}

int64_t vb_range_tiles(int64_t N)
{
    return (N + VB_TILE - 1) / VB_TILE;
}

void launch_vb_range_count(const void* keys, int key32, int64_t N, uint64_t* counts, cudaStream_t s)
{
    const int64_t tiles = vb_range_tiles(N);
    if (tiles == 0)
        return;
    if (key32)
        k_vb_range_count<uint32_t><<<(unsigned)tiles, VB_THREADS, 0, s>>>((const uint32_t*)keys, N, counts);
    else
        k_vb_range_count<uint64_t><<<(unsigned)tiles, VB_THREADS, 0, s>>>((const uint64_t*)keys, N, counts);
    count_launch();
}

void launch_vb_range_scatter(const void* keys, int key32, int64_t N, const uint64_t* offs, const uint64_t* total,
                             const VbRangeParams& R, cudaStream_t s)
{
    const int64_t tiles = vb_range_tiles(N);
    if (tiles == 0)
        return;
    if (key32)
        k_vb_range_scatter<uint32_t><<<(unsigned)tiles, VB_THREADS, 0, s>>>((const uint32_t*)keys, N, offs, total, R);
    else
        k_vb_range_scatter<uint64_t><<<(unsigned)tiles, VB_THREADS, 0, s>>>((const uint64_t*)keys, N, offs, total, R);
    count_launch();
}

} // namespace vox
