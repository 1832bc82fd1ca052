// vox_device.cuh - device-side building blocks of the Gaussian -> node2 path.
//
// Floating-point contract: every operation that decides topology or an RGBA8
// byte is a single IEEE operation with round-to-nearest and no contraction
// (VOX_F* macros -> __f*_rn), so results are bit-identical to the host
// restatement of the reference shaders.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "vox_detmath.h"

namespace vox
{

// ------------------------------------------------------------------------
// node2 layout (nanovdb_editor/PNanoVDBExt.h:49-81), offsets in 64-bit words
// ------------------------------------------------------------------------
constexpr uint32_t N2_OFF_NODE_IDX = 0;
constexpr uint32_t N2_OFF_VALUE_IDX = 1;
__host__ __device__ constexpr uint32_t n2_off_value_prefix(int t)
{
    return t == 0 ? 258u : t == 1 ? 258u : t == 2 ? 34u : 6u;
}
__host__ __device__ constexpr uint32_t n2_off_value_mask(int t)
{
    return t == 0 ? 386u : t == 1 ? 386u : t == 2 ? 50u : 8u;
}
__host__ __device__ constexpr uint32_t n2_off_child_prefix(int t)
{
    return t == 0 ? 898u : t == 1 ? 898u : t == 2 ? 114u : 6u;
}
__host__ __device__ constexpr uint32_t n2_off_child_mask(int t)
{
    return t == 0 ? 1026u : t == 1 ? 1026u : t == 2 ? 130u : 8u;
}
constexpr uint32_t N2_OFF_KEY_PREFIX_ROOT = 1538;
constexpr uint32_t N2_OFF_KEY_MASK_ROOT = 1666;
__host__ __device__ constexpr uint32_t n2_off_children(int t)
{
    return t == 0 ? 2180u : t == 1 ? 1538u : t == 2 ? 194u : 16u;
}
__host__ __device__ constexpr uint64_t n2_node_bytes(int t)
{
    return t == 0 ? 541728ull : t == 1 ? 274464ull : t == 2 ? 34336ull : 128ull;
}
constexpr uint64_t N2_END_KEY = 1ull << 63;

// n = coordinate -> child slot (PNanoVDBExt.h:93-101)
__device__ __forceinline__ uint32_t root_n_of(int32_t x, int32_t y, int32_t z)
{
    return ((((uint32_t)x & 0x1FFFFu) >> 12) << 10) | ((((uint32_t)y & 0x1FFFFu) >> 12) << 5) |
           (((uint32_t)z & 0x1FFFFu) >> 12);
}
// origin (voxel coordinates) of root tile root_n (its low 15 bits)
__device__ __forceinline__ void root_tile_origin(uint32_t rn, int32_t o[3])
{
    int32_t x = (int32_t)((rn >> 10) & 31), y = (int32_t)((rn >> 5) & 31), z = (int32_t)(rn & 31);
    o[0] = (x >= 16 ? x - 32 : x) * 4096;
    o[1] = (y >= 16 ? y - 32 : y) * 4096;
    o[2] = (z >= 16 ? z - 32 : z) * 4096;
}

// root tile index across clouds: cloud << 15 | root_n.  Ranks of touched root
// tiles and lower cells are taken in this order, so the cloud is the most
// significant part of every compact key.
__device__ __forceinline__ uint64_t root_index(uint32_t cloud, int32_t x, int32_t y, int32_t z)
{
    return ((uint64_t)cloud << 15) | root_n_of(x, y, z);
}
__device__ __forceinline__ uint32_t upper_n_of(int32_t x, int32_t y, int32_t z)
{
    return ((((uint32_t)x & 0xFFFu) >> 7) << 10) | ((((uint32_t)y & 0xFFFu) >> 7) << 5) | (((uint32_t)z & 0xFFFu) >> 7);
}
__device__ __forceinline__ uint32_t lower_n_of(int32_t x, int32_t y, int32_t z)
{
    return ((((uint32_t)x & 0x7Fu) >> 3) << 8) | ((((uint32_t)y & 0x7Fu) >> 3) << 4) | (((uint32_t)z & 0x7Fu) >> 3);
}
__device__ __forceinline__ uint32_t leaf_n_of(int32_t x, int32_t y, int32_t z)
{
    return (((uint32_t)x & 7u) << 6) | (((uint32_t)y & 7u) << 3) | ((uint32_t)z & 7u);
}

// rank of bit idx among the set bits of a bitmap with per-word exclusive
// popcount prefixes
__device__ __forceinline__ uint64_t bit_rank(const uint64_t* bits, const uint64_t* prefix, uint64_t idx)
{
    uint64_t w = bits[idx >> 6];
    return prefix[idx >> 6] + (uint64_t)__popcll(w & ((1ull << (idx & 63)) - 1ull));
}

// ------------------------------------------------------------------------
// per-Gaussian record, written once by the prep kernel (128 B, 16B aligned)
// ------------------------------------------------------------------------
struct __align__(16) GaussRec
{
    float4 q0; // pos.xyz, inv_ls = 1/ls
    float4 q1; // rinv[0][0..2], rinv[1][0]
    float4 q2; // rinv[1][1..2], rinv[2][0..1]
    float4 q3; // rinv[2][2], inv_s.xyz = 1/s (clamped scale)
    int4 q4;   // bbox min xyz, valid
    int4 q5;   // bbox range xyz (max + 1 - min), cloud index
    float4 q6; // opacity, ls, e = 1 / (0.1 |s| / voxel_size), |s|
    float4 q7; // rgb, culled (1.f if |s| > cull scale)
};

struct PrepParams
{
    const float* means;   // 3G
    const float* quats;   // 4G, w x y z (raw or normalised)
    const float* scales;  // 3G (log-scale when raw)
    const float* opac;    // G (logit when raw)
    const float* colors;  // 3G RGB (SH0 when raw)
    int64_t count;
    int raw;              // 1: apply the host preprocessing of raster/RasterUtils.cpp:59-117
    int bf16;             // 1: every attribute array holds bfloat16 values (read exactly as float)
    float voxel_size;     // every cloud's voxel size when cloud_vs is null
    float cull_scale;     // > 0
    // batched calls: Gaussians [cloud_start[b], cloud_start[b + 1]) form cloud b
    // with voxel size cloud_vs[b]; null for one cloud
    const int64_t* cloud_start;
    const float* cloud_vs;
    int64_t clouds;
    int64_t g0 = 0, g1 = -1; // the Gaussians [g0, g1) this launch builds (g1 < 0: up to count)
};



// attribute i of an array of float, or of bfloat16 when bf16 (the upper 16 bits
// of a float: the conversion is exact, so every later operation is FP32)
__host__ __device__ __forceinline__ float ld_attr(const float* p, int64_t i, int bf16)
{
    if (bf16)
    {
        const uint32_t u = (uint32_t)reinterpret_cast<const uint16_t*>(p)[i] << 16;
#if defined(__CUDA_ARCH__)
        return __uint_as_float(u);
#else
        float f;
        memcpy(&f, &u, 4);
        return f;
#endif
    }
    return p[i];
}

// dot with the reference's fixed evaluation order (a.x*b.x + a.y*b.y) + a.z*b.z
__device__ __forceinline__ float dot3_rn(float ax, float ay, float az, float bx, float by, float bz)
{
    return VOX_FADD(VOX_FADD(VOX_FMUL(ax, bx), VOX_FMUL(ay, by)), VOX_FMUL(az, bz));
}

__device__ __forceinline__ bool finite_f(float v)
{
    return v == v && VOX_FSUB(v, v) == 0.f;
}

// Builds the record of one Gaussian (gaussian_prim.slang:47-144 and the
// per-Gaussian prologue of gaussian_frag_alloc.slang / gaussian_frag_color.slang).
// Returns the bbox footprint (0 when the Gaussian emits nothing).
__device__ __forceinline__ uint64_t make_record(const PrepParams& P, int64_t g, float vs, GaussRec& R, int32_t bmax[3])
{
    const int h = P.bf16;
    float pos[3] = { ld_attr(P.means, 3 * g + 0, h), ld_attr(P.means, 3 * g + 1, h), ld_attr(P.means, 3 * g + 2, h) };
    float qw = ld_attr(P.quats, 4 * g + 0, h), qx = ld_attr(P.quats, 4 * g + 1, h), qy = ld_attr(P.quats, 4 * g + 2, h),
          qz = ld_attr(P.quats, 4 * g + 3, h);
    float s[3] = { ld_attr(P.scales, 3 * g + 0, h), ld_attr(P.scales, 3 * g + 1, h), ld_attr(P.scales, 3 * g + 2, h) };
    float op = ld_attr(P.opac, g, h);
    float rgb[3] = { ld_attr(P.colors, 3 * g + 0, h), ld_attr(P.colors, 3 * g + 1, h), ld_attr(P.colors, 3 * g + 2, h) };
    if (P.raw)
    {
        // raster/RasterUtils.cpp:59-117
        float ss = VOX_FADD(VOX_FADD(VOX_FADD(VOX_FMUL(qx, qx), VOX_FMUL(qy, qy)), VOX_FMUL(qz, qz)), VOX_FMUL(qw, qw));
        float mi = VOX_FDIV(1.f, VOX_FSQRT(ss));
        qx = VOX_FMUL(qx, mi);
        qy = VOX_FMUL(qy, mi);
        qz = VOX_FMUL(qz, mi);
        qw = VOX_FMUL(qw, mi);
        for (int a = 0; a < 3; a++)
            s[a] = vox_expf_cr(s[a]);
        const float c0 = 0.28209479177387814f;
        for (int a = 0; a < 3; a++)
            rgb[a] = VOX_FADD(VOX_FMUL(c0, rgb[a]), 0.5f);
        op = VOX_FDIV(1.f, VOX_FADD(1.f, vox_expf_cr(-op)));
    }
    const float vs_inv = VOX_FDIV(1.f, vs);

    bool ok = finite_f(op) && finite_f(qx) && finite_f(qy) && finite_f(qz) && finite_f(qw);
    for (int a = 0; a < 3; a++)
        ok = ok && finite_f(pos[a]) && finite_f(s[a]) && s[a] > 0.f;
    float lg = ok ? vox_logf(VOX_FDIV(op, 0.01f)) : 0.f;
    float ls = VOX_FSQRT(VOX_FMUL(2.f, lg));
    const float min_scale = VOX_FMUL(0.125f, vs);
    for (int a = 0; a < 3; a++)
        s[a] = s[a] > min_scale ? s[a] : min_scale;
    ok = ok && lg > 0.f && finite_f(ls);

    // rotation rows (gaussian_prim.slang:83-90); inverse rows are the transpose
    float r[3][3];
    r[0][0] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(qy, qy), VOX_FMUL(qz, qz))));
    r[0][1] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(qx, qy), VOX_FMUL(qz, qw)));
    r[0][2] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(qx, qz), VOX_FMUL(qy, qw)));
    r[1][0] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(qx, qy), VOX_FMUL(qz, qw)));
    r[1][1] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(qx, qx), VOX_FMUL(qz, qz))));
    r[1][2] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(qy, qz), VOX_FMUL(qx, qw)));
    r[2][0] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(qx, qz), VOX_FMUL(qy, qw)));
    r[2][1] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(qy, qz), VOX_FMUL(qx, qw)));
    r[2][2] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(qx, qx), VOX_FMUL(qy, qy))));

    // bbox of the 8 transformed box corners.  Each output coordinate is
    // fl(fl(t0 + t1) + t2) + pos with t_a = +-fl(fl(s_a * ls) * r_ra); rounding
    // is monotone, so the corner minimum / maximum is reached with every
    // t_a = -|.| / +|.|, identical to the reference's 8-corner loop.
    int32_t bmin[3];
    uint64_t footprint = 0;
    if (ok)
    {
        float u[3] = { VOX_FMUL(s[0], ls), VOX_FMUL(s[1], ls), VOX_FMUL(s[2], ls) };
        footprint = 1;
        for (int a = 0; a < 3; a++)
        {
            float m = VOX_FADD(VOX_FADD(fabsf(VOX_FMUL(u[0], r[a][0])), fabsf(VOX_FMUL(u[1], r[a][1]))),
                               fabsf(VOX_FMUL(u[2], r[a][2])));
            float lo = VOX_FMUL(VOX_FSUB(pos[a], m), vs_inv);
            float hi = VOX_FMUL(VOX_FADD(pos[a], m), vs_inv);
            bmin[a] = (int32_t)floorf(lo);
            bmax[a] = (int32_t)floorf(hi);
            footprint *= (uint64_t)(int64_t)(bmax[a] + 1 - bmin[a]);
        }
    }
    else
    {
        bmin[0] = bmin[1] = bmin[2] = 0;
        bmax[0] = bmax[1] = bmax[2] = -1;
    }

    float scale1d = VOX_FSQRT(dot3_rn(s[0], s[1], s[2], s[0], s[1], s[2]));
    float vrs = VOX_FDIV(VOX_FMUL(0.1f, scale1d), vs);
    float e = VOX_FDIV(1.f, vrs);
    float culled = scale1d > P.cull_scale ? 1.f : 0.f;

    R.q0 = make_float4(pos[0], pos[1], pos[2], VOX_FDIV(1.f, ls));
    R.q1 = make_float4(r[0][0], r[1][0], r[2][0], r[0][1]);
    R.q2 = make_float4(r[1][1], r[2][1], r[0][2], r[1][2]);
    R.q3 = make_float4(r[2][2], VOX_FDIV(1.f, s[0]), VOX_FDIV(1.f, s[1]), VOX_FDIV(1.f, s[2]));
    R.q4 = make_int4(bmin[0], bmin[1], bmin[2], ok ? 1 : 0);
    R.q5 = make_int4(bmax[0] + 1 - bmin[0], bmax[1] + 1 - bmin[1], bmax[2] + 1 - bmin[2], 0); // cloud set by the caller
    R.q6 = make_float4(op, ls, e, scale1d);
    R.q7 = make_float4(rgb[0], rgb[1], rgb[2], culled);
    return footprint;
}

__device__ __forceinline__ uint32_t rec_cloud(const GaussRec& R)
{
    return (uint32_t)R.q5.w;
}
// voxel size of the record's cloud
__device__ __forceinline__ float rec_vs(const GaussRec& R, float vs, const float* cloud_vs)
{
    return cloud_vs ? cloud_vs[R.q5.w] : vs;
}

// inverse rotation rows from the record: rinv[row][axis]
struct RInv
{
    float m[3][3];
};
__device__ __forceinline__ RInv rinv_of(const GaussRec& R)
{
    RInv o;
    o.m[0][0] = R.q1.x;
    o.m[0][1] = R.q1.y;
    o.m[0][2] = R.q1.z;
    o.m[1][0] = R.q1.w;
    o.m[1][1] = R.q2.x;
    o.m[1][2] = R.q2.y;
    o.m[2][0] = R.q2.z;
    o.m[2][1] = R.q2.w;
    o.m[2][2] = R.q3.x;
    return o;
}

// Local AABB of a voxel in the Gaussian's unit-sphere space
// (gaussian_frag_alloc.slang:84-131).  The reference transforms the 8 voxel
// corners; every local coordinate is fl(fl(fl(p_x + p_y) + p_z) * inv_ls) * inv_s
// with p_a = fl(c_a * rinv[row][a]) and c_a one of two corner values per axis.
// Rounded addition and multiplication by a positive constant are monotone, so
// the corner minimum (maximum) is the same expression over the per-axis
// minimum (maximum) products - bit-identical to the 8-corner loop.
struct Aabb
{
    float lo[3], hi[3];
};

__device__ __forceinline__ void axis_corners(float vs, float pos, int32_t i, float& c0, float& c1)
{
    float v0 = (float)i;
    float v1 = VOX_FADD(v0, 1.f);
    c0 = VOX_FSUB(VOX_FMUL(v0, vs), pos);
    c1 = VOX_FSUB(VOX_FMUL(v1, vs), pos);
}

// The minimum / maximum of the two corner products.  fminf / fmaxf differ from
// the compare-and-select form only in the sign of a zero on a tie, and every
// consumer squares these bounds or compares them with zero.
__device__ __forceinline__ void minmax_prod(float c0, float c1, float r, float& mn, float& mx)
{
    const float p0 = VOX_FMUL(c0, r), p1 = VOX_FMUL(c1, r);
    mn = fminf(p0, p1);
    mx = fmaxf(p0, p1);
}

__device__ __forceinline__ Aabb voxel_local_aabb(const GaussRec& R, const RInv& M, float vs, int32_t i, int32_t j,
                                                 int32_t k)
{
    float cx0, cx1, cy0, cy1, cz0, cz1;
    axis_corners(vs, R.q0.x, i, cx0, cx1);
    axis_corners(vs, R.q0.y, j, cy0, cy1);
    axis_corners(vs, R.q0.z, k, cz0, cz1);
    const float inv_s[3] = { R.q3.y, R.q3.z, R.q3.w };
    Aabb b;
#pragma unroll
    for (int row = 0; row < 3; row++)
    {
        float xn, xx, yn, yx, zn, zx;
        minmax_prod(cx0, cx1, M.m[row][0], xn, xx);
        minmax_prod(cy0, cy1, M.m[row][1], yn, yx);
        minmax_prod(cz0, cz1, M.m[row][2], zn, zx);
        float lo = VOX_FADD(VOX_FADD(xn, yn), zn);
        float hi = VOX_FADD(VOX_FADD(xx, yx), zx);
        b.lo[row] = VOX_FMUL(VOX_FMUL(lo, R.q0.w), inv_s[row]);
        b.hi[row] = VOX_FMUL(VOX_FMUL(hi, R.q0.w), inv_s[row]);
    }
    return b;
}

// dist2 test of gaussian_frag_alloc.slang:132-162
__device__ __forceinline__ bool aabb_hits_unit_sphere(const Aabb& b)
{
    float d2 = 1.f;
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        if (0.f < b.lo[a])
            d2 = VOX_FSUB(d2, VOX_FMUL(b.lo[a], b.lo[a]));
        else if (0.f > b.hi[a])
            d2 = VOX_FSUB(d2, VOX_FMUL(b.hi[a], b.hi[a]));
    }
    return d2 > 0.f;
}

// Alpha of a passing (voxel, Gaussian) pair (gaussian_frag_color.slang:184-213).
// The reference takes the maximum of op * exp(-ls * |p|^2) over a 4x4x4
// lattice p = w * hi + (1 - w) * lo.  |p|^2 = fl(fl(x^2 + y^2) + z^2) is
// monotone in each per-axis square and exp (vox_expf_cr) is monotone, so the
// maximum is the lattice point with the per-axis smallest square.
// vox_powf(b, e) for 0 <= b <= 1 and finite e > 0, the operations vox_logf /
// vox_expf perform in that domain (the same results): log of a normal b < 1
// (b = 1 - a with a < 1 is at least 2^-24), exp of a non-positive argument.
__device__ __forceinline__ float vox_powf_unit(float b, float e)
{
    if (b == 0.0f)
        return 0.0f;
    if (b == 1.0f)
        return 1.0f;
    // vox_logf(b)
    const uint32_t bits = vox_f2u(b);
    int ex = (int)((bits >> 23) & 0xff) - 127;
    float m = vox_u2f((bits & 0x007fffffu) | 0x3f800000u);
    if (m > VOX_SQRT2_F)
    {
        m = VOX_FMUL(m, 0.5f);
        ex += 1;
    }
    const float t = VOX_FDIV(VOX_FSUB(m, 1.0f), VOX_FADD(m, 1.0f));
    const float t2 = VOX_FMUL(t, t);
    float p = 1.0f / 11.0f;
    p = VOX_FFMA(p, t2, 1.0f / 9.0f);
    p = VOX_FFMA(p, t2, 1.0f / 7.0f);
    p = VOX_FFMA(p, t2, 1.0f / 5.0f);
    p = VOX_FFMA(p, t2, 1.0f / 3.0f);
    p = VOX_FFMA(p, t2, 1.0f);
    const float logm = VOX_FMUL(VOX_FMUL(2.0f, t), p);
    const float ef = (float)ex;
    const float lg = VOX_FADD(VOX_FMUL(ef, VOX_LN2_HI_F), VOX_FADD(VOX_FMUL(ef, VOX_LN2_LO_F), logm));
    // vox_expf(e * lg), argument <= 0
    const float x = VOX_FMUL(e, lg);
    if (x < -87.3f)
        return 0.0f;
    const float kf = VOX_FLOORF(VOX_FADD(VOX_FMUL(x, VOX_INV_LN2_F), 0.5f));
    const float r = VOX_FSUB(VOX_FSUB(x, VOX_FMUL(kf, VOX_LN2_HI_F)), VOX_FMUL(kf, VOX_LN2_LO_F));
    float q = 1.0f / 40320.0f;
    q = VOX_FFMA(q, r, 1.0f / 5040.0f);
    q = VOX_FFMA(q, r, 1.0f / 720.0f);
    q = VOX_FFMA(q, r, 1.0f / 120.0f);
    q = VOX_FFMA(q, r, 1.0f / 24.0f);
    q = VOX_FFMA(q, r, 1.0f / 6.0f);
    q = VOX_FFMA(q, r, 0.5f);
    q = VOX_FFMA(q, r, 1.0f);
    q = VOX_FFMA(q, r, 1.0f);
    const int k = (int)kf;
    const int k1 = k / 2, k2 = k - k1;
    const float s1 = vox_u2f((uint32_t)(k1 + 127) << 23), s2 = vox_u2f((uint32_t)(k2 + 127) << 23);
    return VOX_FMUL(VOX_FMUL(q, s1), s2);
}

// one RGBA8 channel byte of gaussian_frag_color.slang:239-246: clamp to [0, 1], 255 v truncated
__device__ __forceinline__ uint32_t rgba8_byte(float v)
{
    v = v < 1.f ? v : 1.f;
    v = 0.f > v ? 0.f : v;
    return (uint32_t)VOX_FMUL(255.f, v);
}

// Lattice weights w_s = fl(fl(1/3) * s), 1 - w_s rounded (s = 1, 2); s = 0 and
// s = 3 (w = 1 exactly) give p = lo and p = hi.
constexpr float LAT_W1 = 0x1.555556p-2f, LAT_OW1 = 0x1.555554p-1f;
constexpr float LAT_W2 = 0x1.555556p-1f, LAT_OW2 = 0x1.555554p-2f;

// The smallest |p|^2 of the 4x4x4 lattice (gaussian_frag_color.slang:190-197),
// the sum of the per-axis smallest squares
__device__ __forceinline__ float lattice_min_d2(const Aabb& b)
{
    float m[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const float p1 = VOX_FADD(VOX_FMUL(LAT_W1, b.hi[a]), VOX_FMUL(LAT_OW1, b.lo[a]));
        const float p2 = VOX_FADD(VOX_FMUL(LAT_W2, b.hi[a]), VOX_FMUL(LAT_OW2, b.lo[a]));
        const float s0 = VOX_FMUL(b.lo[a], b.lo[a]), s1 = VOX_FMUL(p1, p1), s2 = VOX_FMUL(p2, p2),
                    s3 = VOX_FMUL(b.hi[a], b.hi[a]);
        m[a] = fminf(fminf(s0, s1), fminf(s2, s3)); // squares: no NaN, no signed zero
    }
    return VOX_FADD(VOX_FADD(m[0], m[1]), m[2]);
}

// alpha from the lattice minimum d (gaussian_frag_color.slang:197-213)
__device__ __forceinline__ float alpha_of_d2(const GaussRec& R, float d)
{
    float a = VOX_FMUL(R.q6.x, vox_expf_cr(-VOX_FMUL(R.q6.y, d)));
    a = a > 0.f ? a : 0.f;
    a = VOX_FSUB(1.f, vox_powf_unit(VOX_FSUB(1.f, a), R.q6.z));
    if (R.q7.w != 0.f)
        a = 0.f;
    return a;
}

__device__ __forceinline__ float pair_alpha(const GaussRec& R, const Aabb& b)
{
    return alpha_of_d2(R, lattice_min_d2(b));
}

// Per (leaf, Gaussian) constants of the leaf walk, computed once when a chunk
// is staged (leaf_pair_consts).
//
// The float channels' local AABB is anchored at one voxel of the leaf: c =
// o + r0, r0_a = clamp(bmin_a + (range_a >> 1) - o_a, 0, 7) (the leaf voxel
// nearest the centre voxel of the Gaussian's bbox, integer arithmetic).  With d0_a = fma(c_a, vs, -mu_a) (the anchor's
// corner offset, rounded once, so the low bits of mu survive far from the
// origin), k_r = fl(inv_ls inv_s_r) and the scaled voxel steps A_ra =
// fl(fl(vs m_ra) k_r), row r of voxel o + (rx, ry, rz), t_a = r_a - r0_a, is
//   base_r = fl(fl(fma(m_r2, d0_2, fma(m_r0, d0_0, fl(m_r1 d0_1)))) k_r)
//   lo0_r  = fl(fl(fl(base_r + min(A_r0, 0)) + min(A_r1, 0)) + min(A_r2, 0))
//   W_r    = fl(fl(|A_r0| + |A_r1|) + |A_r2|)
//   lo_r   = fma(t_z, A_r2, fma(t_y, A_r1, fma(t_x, A_r0, lo0_r))),  hi_r = fl(lo_r + W_r)
// (the lower corner of each axis is the one picked by the sign of the step).
// Every rounding is relative to the local magnitudes E_a = |d0_a| + 8 vs
// (|t| <= 7), and near the centre the anchor's offsets are about a voxel, so
// the form is about as accurate as one rounding of each corner offset; a pair
// costs three fma and one add per row.  The oracle's frag_alpha_f evaluates the same operations in
// the same order.
//
// dab_r bounds how far the reference's local AABB (voxel_local_aabb) and this
// one can differ in the leaf, apart from the per-pair 2^-20 B_r term added in
// alpha_byte_bound: per axis the reference's corner offset fl(fl(v vs) -
// mu) is within 0.5 ulp(W) + 0.5 ulp(Cm) of exact (W, Cm: the largest |v vs|
// and |v vs - mu| over the leaf's corners), its products and two sums add at
// most 3 2^-24 sum_a |m_ra| Cm_a <= 2^-21 sum_a |m_ra| Cm_a; this form's d0
// rounding adds 0.5 ulp(E_a), its other roundings (the chain 3, k and base 2,
// the steps' 3 times |t| <= 7 with 8 vs <= E, lo0 3, the per-voxel fma 3, W and
// the hi sum about 1.3, in units of 2^-24 sum_a |m_ra| E_a) at most
// 2^-20 sum_a |m_ra| E_a; all scaled by il is_r.  dab_r also carries the
// roundings proportional to the bound magnitude (the sum and scalings of the
// reference, the lattice points): 2^-20 2 Bl_r, Bl_r = il is_r sum_a |m_ra|
// Cm_a bounding every bound's magnitude in the leaf.  So per row this AABB,
// and its four lattice points, are within dab_r of the reference's for every
// voxel of the leaf.  The leaf test (leaf_test_chunk) classifies voxels from
// it, Delta = sum_r dab_r giving its thresholds lo_t / hi_t.
struct LeafPairConst
{
    float lo0[3], W[3]; // per row: the scaled lower bound of the anchor voxel, the scaled voxel width
    float A[3][3];      // A[r][a]: the scaled step of one voxel along axis a
    float dab[3];       // per row: the reference / float-channel AABB difference bound
    float lo_t, hi_t;   // the linear z classification: certain pass below lo_t, certain fail above hi_t
    uint32_t r0;        // the anchor voxel in the leaf: r0_x | r0_y << 8 | r0_z << 16
};

// the anchor of the float channels' AABB along one axis (leaf origin o)
// (bbox minimum bmin, extent range = max + 1 - min)
__host__ __device__ __forceinline__ int32_t anchor_of(int32_t bmin, int32_t range, int32_t o)
{
    const int32_t r = bmin + (range >> 1) - o;
    return r < 0 ? 0 : r > 7 ? 7 : r;
}

// unit in the last place of |x| (a float), 0 for 0
__device__ __forceinline__ float ulp_of(float x)
{
    return __uint_as_float(__float_as_uint(fabsf(x)) & 0x7f800000u) * 0x1p-23f;
}

__device__ __forceinline__ LeafPairConst leaf_pair_consts(const GaussRec& R, float vs, const int32_t o[3])
{
    LeafPairConst c;
    const float mu[3] = { R.q0.x, R.q0.y, R.q0.z };
    const float il = R.q0.w;
    const float is[3] = { R.q3.y, R.q3.z, R.q3.w };
    const RInv M = rinv_of(R);
    float d0[3], Gr[3], G[3], Cm[3];
    c.r0 = 0;
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const int32_t r0 = anchor_of((&R.q4.x)[a], (&R.q5.x)[a], o[a]);
        c.r0 |= (uint32_t)r0 << (8 * a);
        d0[a] = VOX_FFMA((float)(o[a] + r0), vs, -mu[a]);
        const float w0 = (float)o[a] * vs, w1 = (float)(o[a] + 8) * vs;
        const float W = fmaxf(fabsf(w0), fabsf(w1)) * (1.f + 0x1p-20f);
        Cm[a] = fmaxf(fabsf(w0 - mu[a]), fabsf(w1 - mu[a])) * (1.f + 0x1p-20f);
        Gr[a] = 0.5f * ulp_of(W) + 0.5f * ulp_of(Cm[a]) + 0x1p-21f * Cm[a];
        const float E = (fabsf(d0[a]) + 8.f * vs) * (1.f + 0x1p-20f);
        G[a] = Gr[a] + 0.5f * ulp_of(E) + 0x1p-20f * E;
    }
    float Dl = 0.f;
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        const float k = VOX_FMUL(il, is[r]);
        const float base =
            VOX_FMUL(VOX_FFMA(M.m[r][2], d0[2], VOX_FFMA(M.m[r][0], d0[0], VOX_FMUL(M.m[r][1], d0[1]))), k);
#pragma unroll
        for (int a = 0; a < 3; a++)
            c.A[r][a] = VOX_FMUL(VOX_FMUL(vs, M.m[r][a]), k);
        c.lo0[r] = VOX_FADD(VOX_FADD(VOX_FADD(base, fminf(c.A[r][0], 0.f)), fminf(c.A[r][1], 0.f)),
                            fminf(c.A[r][2], 0.f));
        c.W[r] = VOX_FADD(VOX_FADD(fabsf(c.A[r][0]), fabsf(c.A[r][1])), fabsf(c.A[r][2]));
        const float s = (1.f + 0x1p-20f) * il * is[r];
        const float m0 = fabsf(M.m[r][0]), m1 = fabsf(M.m[r][1]), m2 = fabsf(M.m[r][2]);
        const float Bl = s * (m0 * Cm[0] + m1 * Cm[1] + m2 * Cm[2]);
        // with the scalings' and lattice points' roundings, 2^-20 B_r <= 2^-20 2 Bl_r
        c.dab[r] = s * (m0 * G[0] + m1 * G[1] + m2 * G[2]) + 0x1p-20f * 2.f * Bl;
        Dl += c.dab[r];
    }
    Dl *= 1.f + 0x1p-20f;
    if (Dl <= 0.0625f) // false for NaN
    {
        c.lo_t = 1.f - (2.f * Dl + 0x1p-19f);
        c.hi_t = 1.f + (2.f * Dl + Dl * Dl + 0x1p-18f);
    }
    else
    {
        c.lo_t = -1.f; // every voxel takes the reference test
        c.hi_t = __int_as_float(0x7f800000);
    }
    return c;
}

// the float channels' local AABB of voxel o + (rx, ry, rz) from the leaf's constants (r0: the packed anchor)
__device__ __forceinline__ Aabb stable_leaf_aabb(const float lo0[3], const float W[3], const float A[3][3], uint32_t r0,
                                                 int32_t rx, int32_t ry, int32_t rz)
{
    const float fx = (float)(rx - (int32_t)(r0 & 255u)), fy = (float)(ry - (int32_t)((r0 >> 8) & 255u)),
                fz = (float)(rz - (int32_t)(r0 >> 16));
    Aabb b;
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        b.lo[r] = VOX_FFMA(fz, A[r][2], VOX_FFMA(fy, A[r][1], VOX_FFMA(fx, A[r][0], lo0[r])));
        b.hi[r] = VOX_FADD(b.lo[r], W[r]);
    }
    return b;
}

// Alpha of the float density / colour channels from their local AABB
// (stable_leaf_aabb): the lattice points lo + w (hi - lo), float exp / pow
// (vox_expf_ch / vox_powf_ch: about 2 ulp, no division).  The oracle's
// frag_alpha_f evaluates the same operations in the same order.  Also keeps
// what alpha_byte_bound needs: the lattice minimum d, op exp(-ls d) and the
// smallest lattice square per axis.
struct AlphaF
{
    float a1;   // the channel's alpha
    float d;    // smallest lattice |p|^2
    float a;    // op exp(-ls d), before the opacity transform
    float m[3]; // the smallest lattice square per axis
};
__device__ __forceinline__ AlphaF pair_alpha_f_ex(const GaussRec& R, const Aabb& b)
{
    AlphaF f;
    float m[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
    {
        const float dd = VOX_FSUB(b.hi[a], b.lo[a]);
        const float p1 = VOX_FFMA(dd, 0x1.555556p-2f, b.lo[a]), p2 = VOX_FFMA(dd, 0x1.555556p-1f, b.lo[a]);
        const float s0 = VOX_FMUL(b.lo[a], b.lo[a]), s1 = VOX_FMUL(p1, p1), s2 = VOX_FMUL(p2, p2),
                    s3 = VOX_FMUL(b.hi[a], b.hi[a]);
        m[a] = fminf(fminf(s0, s1), fminf(s2, s3)); // squares: no NaN, no signed zero
        f.m[a] = m[a];
    }
    f.d = VOX_FADD(VOX_FADD(m[0], m[1]), m[2]);
    float a = VOX_FMUL(R.q6.x, vox_expf_ch(-VOX_FMUL(R.q6.y, f.d)));
    a = a > 0.f ? a : 0.f;
    f.a = a;
    a = VOX_FSUB(1.f, vox_powf_ch(VOX_FSUB(1.f, a), R.q6.z));
    if (R.q7.w != 0.f)
        a = 0.f;
    f.a1 = a;
    return f;
}
__device__ __forceinline__ float pair_alpha_f(const GaussRec& R, const Aabb& b)
{
    return pair_alpha_f_ex(R, b).a1;
}


// The RGBA8 alpha byte of a passing pair, rgba8_byte(pair_alpha(R, b_ref))
// with b_ref = voxel_local_aabb(...), decided where possible from the float
// channel's alpha f (same formula, evaluated from stable_leaf_aabb).
// Per row the two AABBs' bounds, and so their four lattice points, differ by at
// most D_r = dab_r (leaf_pair_consts: the scalings' and lattice points'
// roundings included).  With m_r
// the float evaluation's smallest lattice square, either evaluation's
// minimizing point is within u_r = sqrt(m_r) + D_r of zero, so the row minima
// differ by at most 2 sqrt(m_r) D_r + D_r^2 + 2^-22 u_r^2 (rounded squares) and
// the lattice minima d by md = sum_r of that (times 1 + 2^-20) + 2^-21 d (the
// two rounded sums); and the
// alpha a' = 1 - (1 - op e^-ls d)^e, whose slope in d is at most
// e ls a_hi (times 1 / (1 - a_hi) when e < 1) for a_hi >= op e^-ls (d - md),
// by at most that slope times md, plus both evaluations' own error: the exps
// within 0.5 and 1.5 ulp (vox_expf_cr, vox_expf_ch) and two roundings of op e
// give |delta a| <= 3.6e-7 a, so the bases 1 - a differ by at most 3.6e-7 a +
// 6e-8; through the pow's slope (e, or e / (1 - a_hi) when e < 1) plus the two
// pows' own errors (within 1.0e-7 and 0.82e-7, tests/test_oracle_float.py) and
// the final roundings (6e-8) that is slope_e (3.6e-7 a + 6e-8) + 3.1e-7, taken
// three times over.  When a' +- that margin falls
// in one byte (rgba8_byte is monotone) the byte is the reference's and
// decided is set; otherwise the caller runs the reference's evaluation
// (ref_alpha_byte).  VOX_CHECK_EMIT=1 compares every decided byte with the
// reference's evaluation.
// an upper bound of sqrt(x) for x >= 0: the hardware approximation (relative
// error far below 2^-20) raised by 2^-18, plus 2^-60 for subnormal inputs
__device__ __forceinline__ float sqrt_upper(float x)
{
    float y;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y * (1.f + 0x1p-18f) + 0x1p-60f;
}

__device__ __forceinline__ uint32_t alpha_byte_bound(const GaussRec& R, const AlphaF& f, const float dab[3],
                                                     bool& decided)
{
    // branch-free (the pairs of a warp take different cases): every quantity is
    // computed and the cases are combined at the end
    float md = 0.f;
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        const float D = dab[r]; // dab_r + 2^-20 B_r, folded per leaf (leaf_pair_consts)
        const float u = sqrt_upper(f.m[r]) + D; // bounds both evaluations' minimizing lattice point
        md += (2.f * u - D) * D + 0x1p-22f * u * u;
    }
    md = md * (1.f + 0x1p-20f) + 0x1p-21f * f.d;
    const float ls = R.q6.y, e = R.q6.z;
    const float x = ls * md;
    const float a_hi = f.a * (1.f + 2.f * x) * (1.f + 1e-6f); // e^x <= 1 + 2x for x <= 1
    // 1 / (1 - a_hi) from the fast reciprocal (within 2 ulp for 1 - a_hi >= 2^-24,
    // as it is when a_hi < 1), raised by 2^-20 so it stays an upper bound
    const float inv = __fdividef(1.f, 1.f - a_hi) * (1.f + 0x1p-20f);
    const float slope_e = e < 1.f ? e * inv : e; // the pow's slope bound
    const float slope = slope_e * ls * a_hi;
    const float delta = 1.25f * slope * md + slope_e * (1.1e-6f * a_hi + 1.8e-7f) + 9.3e-7f;
    const uint32_t lo = rgba8_byte(f.a1 - delta), hi = rgba8_byte(f.a1 + delta);
    const bool culled = R.q7.w != 0.f; // culled by scale: both alphas are 0
    decided = culled || (x < 0.25f && a_hi < 1.f && lo == hi);
    return culled ? 0u : lo;
}

// the reference's RGBA8 alpha byte of voxel (i, j, k) and the record's Gaussian
__device__ __forceinline__ uint32_t ref_alpha_byte(const GaussRec& R, float vs, int32_t i, int32_t j, int32_t k)
{
    return rgba8_byte(pair_alpha(R, voxel_local_aabb(R, rinv_of(R), vs, i, j, k)));
}

// Differentiable channels (VOX_FLAG_DIFFERENTIABLE).  The reference alpha
// (4^3-lattice maximum, opacity transform, cull) jumps where a voxel enters or
// leaves the pair set, so these channels use the centre-sampled kernel
//   K = max(op * exp(-|z|^2 / 2) - 0.01, 0),  z = S^-1 R^T (x - mu),
// x the voxel centre, over the same pairs.  K vanishes on the 0.01-opacity
// ellipsoid the pair test is built on (radius ls = sqrt(2 log(op / 0.01)),
// gaussian_prim.slang:65), so the channels are continuous in every parameter.
// Centre offsets are rounded once from double (stable far from the origin).
constexpr float SMOOTH_TAU = 0.01f;
struct SmoothTerms
{
    float d[3], z[3], E, e;
};
__device__ __forceinline__ float smooth_kernel(const GaussRec& R, const RInv& M, float vs, int32_t x, int32_t y,
                                               int32_t z, SmoothTerms& t)
{
    const int32_t c[3] = { x, y, z };
    const float mu[3] = { R.q0.x, R.q0.y, R.q0.z };
    const float inv_s[3] = { R.q3.y, R.q3.z, R.q3.w };
#pragma unroll
    for (int a = 0; a < 3; a++)
        t.d[a] = (float)VOX_DSUB(VOX_DMUL(VOX_DADD((double)c[a], 0.5), (double)vs), (double)mu[a]);
#pragma unroll
    for (int r = 0; r < 3; r++)
        t.z[r] = VOX_FMUL(dot3_rn(t.d[0], t.d[1], t.d[2], M.m[r][0], M.m[r][1], M.m[r][2]), inv_s[r]);
    const float q = dot3_rn(t.z[0], t.z[1], t.z[2], t.z[0], t.z[1], t.z[2]);
    t.E = vox_expf_cr(VOX_FMUL(-0.5f, q));
    t.e = VOX_FMUL(R.q6.x, t.E);
    return t.e > SMOOTH_TAU ? VOX_FSUB(t.e, SMOOTH_TAU) : 0.f;
}

// Float channels accumulate as exact 64-bit fixed-point sums (2^-32 units):
// every term is rounded once to the grid, so the sum is the same integer in any
// order (shared-memory atomics are deterministic); the total is rounded once to
// float.  Terms are clamped to +-2^30.
constexpr float FX_SCALE = 4294967296.f;          // 2^32
constexpr float FX_INV = 2.3283064365386963e-10f; // 2^-32
constexpr float FX_CLAMP = 1073741824.f;          // 2^30
__device__ __forceinline__ unsigned long long fx_of(float x)
{
    x = x < FX_CLAMP ? x : FX_CLAMP;
    x = x > -FX_CLAMP ? x : -FX_CLAMP;
    return (unsigned long long)__float2ll_rn(VOX_FMUL(x, FX_SCALE));
}
// the same for a term known to lie in [0, 1] (an alpha or a smooth kernel value)
__device__ __forceinline__ unsigned long long fx_of_unit(float x)
{
    return (unsigned long long)__float2ll_rn(VOX_FMUL(x, FX_SCALE));
}
__device__ __forceinline__ float fx_to_float(unsigned long long s)
{
    return VOX_FMUL(__ll2float_rn((long long)s), FX_INV);
}


__device__ __forceinline__ uint32_t pack_rgba8(const GaussRec& R, float a)
{
    float ch[4] = { R.q7.x, R.q7.y, R.q7.z, a };
    uint32_t out = 0;
#pragma unroll
    for (int c = 0; c < 4; c++)
    {
        float v = ch[c] < 1.f ? ch[c] : 1.f;
        v = 0.f > v ? 0.f : v;
        out |= ((uint32_t)VOX_FMUL(255.f, v)) << (8 * c);
    }
    return out;
}

// ------------------------------------------------------------------------
// decoupled look-back status words: [63:56] epoch, [55] inclusive flag,
// [54:0] value.  Epoch 0 means "not yet written in this use".  Values are
// kept mod 2^55: the sort's digit counts, the run counts and the u32 scans
// (whose sums are wanted mod 2^32) stay far below that; the u64 scan, whose
// prefixes may use all 64 bits, uses lookback_exclusive_wide.
// ------------------------------------------------------------------------
constexpr uint64_t LB_VALUE_MASK = (1ull << 55) - 1ull;
constexpr uint64_t LB_INCL = 1ull << 55;
constexpr uint32_t LB_SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p)
{
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Wait control of a look-back, from the 32-bit word after the device error
// word (err[1]): 0 = the default limit of LB_SPIN_LIMIT polls; otherwise bits
// 30:0 hold limit + 1 and bit 31 withholds this call's publications, so every
// successor waits on a word nothing writes.  Set only through
// vox_context_set_wait_limit, to make the bounded waits run out in tests.
struct LbControl
{
    uint32_t limit;
    bool withhold;
};
__device__ __forceinline__ LbControl lb_control(const int* err)
{
    const uint32_t c = ((const volatile uint32_t*)err)[1];
    LbControl o;
    o.withhold = (c >> 31) != 0u;
    o.limit = (c & 0x7fffffffu) ? (c & 0x7fffffffu) - 1u : LB_SPIN_LIMIT;
    return o;
}

// Decoupled look-back over 64-bit status words (epoch << 56 | flag | value).
// lookback_publish stores `aggregate` for `tile` (tile 0: as its inclusive
// prefix); lookback_walk walks the predecessors, returns the exclusive prefix
// and publishes the inclusive one.  Publishing early and walking late (after
// other tile work) lets the predecessors' inclusive prefixes land meanwhile.
// Every wait is bounded; on timeout *err is set and the partial prefix (never
// larger than the true one) is returned, and the host treats the call as failed.
// max_op: combine predecessors by maximum instead of sum (a running-max scan)
__device__ __forceinline__ void lookback_publish(uint64_t* status, uint64_t tile, uint64_t aggregate, uint32_t epoch,
                                                 int* err, size_t stride = 1)
{
    const LbControl ctl = lb_control(err);
    if (ctl.withhold)
        return;
    const uint64_t tag = (uint64_t)epoch << 56;
    st_release_u64(&status[tile * stride], tag | (tile == 0 ? LB_INCL : 0ull) | (aggregate & LB_VALUE_MASK));
}

__device__ __forceinline__ uint64_t lookback_walk(uint64_t* status, uint64_t tile, uint64_t aggregate, uint32_t epoch,
                                                  int* err, size_t stride = 1, bool max_op = false)
{
    if (tile == 0)
        return 0;
    const LbControl ctl = lb_control(err);
    const uint64_t tag = (uint64_t)epoch << 56;
    uint64_t excl = 0;
    int64_t p = (int64_t)tile - 1;
    uint32_t spins = 0;
    while (p >= 0)
    {
        uint64_t s = ld_acquire_u64(&status[(uint64_t)p * stride]);
        if ((s >> 56) != epoch)
        {
            if (++spins > ctl.limit)
            {
                atomicOr(err, 1); // ERR_LOOKBACK
                break;
            }
            __nanosleep(32);
            continue;
        }
        const uint64_t v = s & LB_VALUE_MASK;
        excl = max_op ? (v > excl ? v : excl) : excl + v;
        if (s & LB_INCL)
            break;
        p--;
    }
    const uint64_t incl = max_op ? (aggregate > excl ? aggregate : excl) : excl + aggregate;
    if (!ctl.withhold)
        st_release_u64(&status[tile * stride], tag | LB_INCL | (incl & LB_VALUE_MASK));
    return excl;
}

// publish and walk at once
__device__ __forceinline__ uint64_t lookback_exclusive(uint64_t* status, uint64_t tile, uint64_t aggregate,
                                                       uint32_t epoch, int* err, size_t stride = 1,
                                                       bool max_op = false)
{
    lookback_publish(status, tile, aggregate, epoch, err, stride);
    return lookback_walk(status, tile, aggregate, epoch, err, stride, max_op);
}

// The same walk for sums that may use all 64 bits (the prefix is exact mod
// 2^64, as uint64 addition is).  Per tile four words: the aggregate's low and
// high halves, then the inclusive prefix's, each word (epoch << 32) | half.
// Every word is written once per use, so two halves that both carry the
// current epoch belong to the same value: a reader can never combine halves
// of different values.
__device__ __forceinline__ uint64_t lookback_exclusive_wide(uint64_t* status, uint64_t tile, uint64_t aggregate,
                                                            uint32_t epoch, int* err)
{
    const LbControl ctl = lb_control(err);
    const uint64_t tag = (uint64_t)epoch << 32;
    uint64_t* mine = status + 4 * tile;
    if (tile > 0 && !ctl.withhold)
    {
        st_release_u64(mine + 0, tag | (aggregate & 0xffffffffull));
        st_release_u64(mine + 1, tag | (aggregate >> 32));
    }
    uint64_t excl = 0;
    int64_t p = (int64_t)tile - 1;
    uint32_t spins = 0;
    while (p >= 0)
    {
        const uint64_t* w = status + 4 * (uint64_t)p;
        const uint64_t il = ld_acquire_u64(w + 2), ih = ld_acquire_u64(w + 3);
        if ((il >> 32) == epoch && (ih >> 32) == epoch)
        {
            excl += (ih << 32) | (il & 0xffffffffull);
            break;
        }
        const uint64_t al = ld_acquire_u64(w + 0), ah = ld_acquire_u64(w + 1);
        if ((al >> 32) == epoch && (ah >> 32) == epoch)
        {
            excl += (ah << 32) | (al & 0xffffffffull);
            p--;
            continue;
        }
        if (++spins > ctl.limit)
        {
            atomicOr(err, 1); // ERR_LOOKBACK
            break;
        }
        __nanosleep(32);
    }
    const uint64_t incl = excl + aggregate;
    if (!ctl.withhold)
    {
        st_release_u64(mine + 2, tag | (incl & 0xffffffffull));
        st_release_u64(mine + 3, tag | (incl >> 32));
    }
    return excl;
}

// ------------------------------------------------------------------------
// warp / block scans
// ------------------------------------------------------------------------
__device__ __forceinline__ uint64_t warp_incl_scan_u64(uint64_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        uint64_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o)
            v += t;
    }
    return v;
}

// Block-wide exclusive scan of one u64 per thread (blockDim.x a multiple of
// 32, <= 1024).  s_warp must hold 33 words.  All threads must call it.
__device__ __forceinline__ uint64_t block_excl_scan_u64(uint64_t v, uint64_t* s_warp, uint64_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    uint64_t incl = warp_incl_scan_u64(v);
    if (lane == 31)
        s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0)
    {
        uint64_t w = lane < nwarps ? s_warp[lane] : 0;
        uint64_t wi = warp_incl_scan_u64(w);
        if (lane < nwarps)
            s_warp[lane] = wi - w;
        if (lane == nwarps - 1)
            s_warp[32] = wi;
    }
    __syncthreads();
    total = s_warp[32];
    uint64_t r = s_warp[warp] + incl - v;
    __syncthreads();
    return r;
}

// device error word bits
constexpr int ERR_LOOKBACK = 1;
constexpr int ERR_RANGE = 2;      // voxel coordinate outside [-65536, 65535]
constexpr int ERR_FOOTPRINT = 4;  // one Gaussian's bbox above 2^31 fragments
constexpr int ERR_CAPACITY = 8;   // pair buffer too small (host retries)
constexpr int ERR_ORDER = 16;     // keys found out of order after the sort
constexpr int ERR_BOUNDS = 32;    // an index check failed; the access was skipped

} // namespace vox
