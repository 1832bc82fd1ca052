/*
 * vox_oracle.c - CPU restatement of the reference's Gaussian -> node2 path.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * bench's CPU-baseline leg as the checker.  Never part of the product path.
 *
 * Every function restates the reference file:line it follows; the shader
 * arithmetic is written literally (8 corners, 64 alpha samples) so that it is
 * independent of the product kernels' optimised formulation.  Floating-point
 * evaluation order: one IEEE operation at a time, no FMA (built with
 * -ffp-contract=off); dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z; the shader's
 * exp is vox_expf_cr (monotone), log and pow are vox_logf / vox_powf, all from
 * vox_detmath.h.
 */
#include "vox_oracle.h"
#include "vox_detmath.h"

#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* node2 layout constants (nanovdb_editor/PNanoVDBExt.h:49-81)              */
/* ------------------------------------------------------------------------ */
static const uint32_t N2_OFF_VALUE_PREFIX[4] = { 258, 258, 34, 6 };
static const uint32_t N2_OFF_VALUE_MASK[4] = { 386, 386, 50, 8 };
static const uint32_t N2_OFF_CHILD_PREFIX[4] = { 898, 898, 114, 6 };
static const uint32_t N2_OFF_CHILD_MASK[4] = { 1026, 1026, 130, 8 };
static const uint32_t N2_OFF_KEY_PREFIX_ROOT = 1538;
static const uint32_t N2_OFF_KEY_MASK_ROOT = 1666;
static const uint32_t N2_OFF_CHILDREN[4] = { 2180, 1538, 194, 16 };
static const uint32_t N2_MAX_SIZE[4] = { 541728, 274464, 34336, 128 };
static const uint32_t N2_IJK_MASK[4] = { 0x1FFFF, 0xFFF, 0x7F, 0x7 };
static const uint32_t N2_FANOUT_BITS[4] = { 5, 5, 4, 3 };
static const uint32_t N2_TILEDIM_BITS[4] = { 12, 7, 3, 0 };
static const uint32_t N2_FANOUT[4] = { 32768, 32768, 4096, 512 };
static const uint64_t N2_END_KEY = 1ull << 63;

/* PNanoVDBExt.h:93-101 */
static uint32_t n2_coord_to_n(int type, int32_t x, int32_t y, int32_t z)
{
    uint32_t m = N2_IJK_MASK[type], t = N2_TILEDIM_BITS[type], b = N2_FANOUT_BITS[type];
    return ((((uint32_t)x & m) >> t) << (b + b)) | ((((uint32_t)y & m) >> t) << b) | (((uint32_t)z & m) >> t);
}

/* hierarchical order key: root_n | upper_n | lower_n | leaf_n (51 bits) */
uint64_t ov_hier_key(int32_t i, int32_t j, int32_t k)
{
    return ((uint64_t)n2_coord_to_n(0, i, j, k) << 36) | ((uint64_t)n2_coord_to_n(1, i, j, k) << 21) |
           ((uint64_t)n2_coord_to_n(2, i, j, k) << 9) | (uint64_t)n2_coord_to_n(3, i, j, k);
}

/* ------------------------------------------------------------------------ */
/* A2 preprocessing: raster/RasterUtils.cpp:59-117                           */
/* ------------------------------------------------------------------------ */
void ov_preprocess(int64_t n, const float* quat_raw, const float* log_scale, const float* opacity_logit,
                   const float* sh0, float* quat_out, float* scale_out, float* opacity_out, float* color_out)
{
    for (int64_t p = 0; p < n; p++)
    {
        /* :61-73 quaternion stored w,x,y,z */
        float x = quat_raw[4 * p + 1], y = quat_raw[4 * p + 2], z = quat_raw[4 * p + 3], w = quat_raw[4 * p + 0];
        float ss = VOX_FADD(VOX_FADD(VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(y, y)), VOX_FMUL(z, z)), VOX_FMUL(w, w));
        float magn_inv = VOX_FDIV(1.f, VOX_FSQRT(ss));
        quat_out[4 * p + 1] = VOX_FMUL(x, magn_inv);
        quat_out[4 * p + 2] = VOX_FMUL(y, magn_inv);
        quat_out[4 * p + 3] = VOX_FMUL(z, magn_inv);
        quat_out[4 * p + 0] = VOX_FMUL(w, magn_inv);
        /* :81-88 */
        for (int a = 0; a < 3; a++)
            scale_out[3 * p + a] = vox_expf_cr(log_scale[3 * p + a]);
        /* :95-105 */
        const float c0 = 0.28209479177387814f;
        for (int a = 0; a < 3; a++)
            color_out[3 * p + a] = VOX_FADD(VOX_FMUL(c0, sh0[3 * p + a]), 0.5f);
        /* :112-117 */
        opacity_out[p] = VOX_FDIV(1.f, VOX_FADD(1.f, vox_expf_cr(-opacity_logit[p])));
    }
}

/* ------------------------------------------------------------------------ */
/* per-Gaussian setup shared by gaussian_prim / frag_alloc / frag_color      */
/* ------------------------------------------------------------------------ */
typedef struct
{
    float pos[3];
    float q[4]; /* x, y, z, w as the shader reads them (gaussian_prim.slang:53-56) */
    float s[3]; /* clamped scale */
    float op;
    float ls;
    float rgb[3];
    int valid;
    int32_t bmin[3], bmax[3];
    uint64_t footprint;
} prim_t;

static float dot3(const float* a, const float* b)
{
    return VOX_FADD(VOX_FADD(VOX_FMUL(a[0], b[0]), VOX_FMUL(a[1], b[1])), VOX_FMUL(a[2], b[2]));
}

/* rotation rows, gaussian_prim.slang:83-90 (forward) */
static void rot_rows(const float* q, float r[3][3])
{
    float x = q[0], y = q[1], z = q[2], w = q[3];
    r[0][0] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(y, y), VOX_FMUL(z, z))));
    r[0][1] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(x, y), VOX_FMUL(z, w)));
    r[0][2] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, z), VOX_FMUL(y, w)));
    r[1][0] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, y), VOX_FMUL(z, w)));
    r[1][1] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(z, z))));
    r[1][2] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(y, z), VOX_FMUL(x, w)));
    r[2][0] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(x, z), VOX_FMUL(y, w)));
    r[2][1] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(y, z), VOX_FMUL(x, w)));
    r[2][2] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(y, y))));
}
/* inverse rows, gaussian_frag_alloc.slang:106-114 */
static void rot_inv_rows(const float* q, float r[3][3])
{
    float x = q[0], y = q[1], z = q[2], w = q[3];
    r[0][0] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(y, y), VOX_FMUL(z, z))));
    r[0][1] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, y), VOX_FMUL(z, w)));
    r[0][2] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(x, z), VOX_FMUL(y, w)));
    r[1][0] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(x, y), VOX_FMUL(z, w)));
    r[1][1] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(z, z))));
    r[1][2] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(y, z), VOX_FMUL(x, w)));
    r[2][0] = VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, z), VOX_FMUL(y, w)));
    r[2][1] = VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(y, z), VOX_FMUL(x, w)));
    r[2][2] = VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(y, y))));
}

static int ov_isfinite(float v)
{
    return v == v && v - v == 0.f;
}

/* gaussian_prim.slang:47-144.  Gaussians whose opacity is not above the 0.01
 * cutoff (sqrt(2 log(op/0.01)) undefined or zero) emit nothing: a deliberate
 * fix of the reference's NaN cutoff radius for those inputs. */
static void prim_setup(prim_t* P, const float* mean, const float* quat_wxyz, const float* scale, float opacity,
                       const float* color, float vs)
{
    float vs_inv = VOX_FDIV(1.f, vs); /* GridBuild.cpp:780 */
    P->pos[0] = mean[0];
    P->pos[1] = mean[1];
    P->pos[2] = mean[2];
    P->q[0] = quat_wxyz[1];
    P->q[1] = quat_wxyz[2];
    P->q[2] = quat_wxyz[3];
    P->q[3] = quat_wxyz[0];
    P->op = opacity;
    if (color)
    {
        P->rgb[0] = color[0];
        P->rgb[1] = color[1];
        P->rgb[2] = color[2];
    }
    int ok = ov_isfinite(opacity);
    for (int a = 0; a < 3; a++)
        ok = ok && ov_isfinite(mean[a]) && ov_isfinite(scale[a]) && scale[a] > 0.f;
    for (int a = 0; a < 4; a++)
        ok = ok && ov_isfinite(quat_wxyz[a]);
    float lg = ok ? vox_logf(VOX_FDIV(opacity, 0.01f)) : 0.f;
    P->ls = VOX_FSQRT(VOX_FMUL(2.f, lg));
    const float min_scale = VOX_FMUL(0.125f, vs); /* :67-68 */
    for (int a = 0; a < 3; a++)
        P->s[a] = scale[a] > min_scale ? scale[a] : min_scale;
    P->valid = ok && lg > 0.f && ov_isfinite(P->ls);
    P->footprint = 0;
    if (!P->valid)
    {
        P->bmin[0] = P->bmin[1] = P->bmin[2] = 0;
        P->bmax[0] = P->bmax[1] = P->bmax[2] = -1;
        return;
    }
    float r[3][3];
    rot_rows(P->q, r);
    for (int v = 0; v < 8; v++)
    {
        float c[3];
        c[0] = (v & 1) ? 1.f : -1.f;
        c[1] = (v & 2) ? 1.f : -1.f;
        c[2] = (v & 4) ? 1.f : -1.f;
        for (int a = 0; a < 3; a++)
        {
            c[a] = VOX_FMUL(c[a], P->s[a]);
            c[a] = VOX_FMUL(c[a], P->ls);
        }
        float p[3] = { dot3(c, r[0]), dot3(c, r[1]), dot3(c, r[2]) };
        int32_t ijk[3];
        for (int a = 0; a < 3; a++)
        {
            p[a] = VOX_FADD(p[a], P->pos[a]);
            ijk[a] = (int32_t)floorf(VOX_FMUL(p[a], vs_inv));
        }
        for (int a = 0; a < 3; a++)
        {
            if (v == 0 || ijk[a] < P->bmin[a])
                P->bmin[a] = ijk[a];
            if (v == 0 || ijk[a] > P->bmax[a])
                P->bmax[a] = ijk[a];
        }
    }
    P->footprint = (uint64_t)(P->bmax[0] + 1 - P->bmin[0]) * (uint64_t)(P->bmax[1] + 1 - P->bmin[1]) *
                   (uint64_t)(P->bmax[2] + 1 - P->bmin[2]);
}

/* gaussian_frag_alloc.slang:84-162: returns 1 when dist2 > 0 */
static int frag_test(const prim_t* P, const float rinv[3][3], float vs, const int32_t* ijk, float* vmin, float* vmax)
{
    float inv_ls = VOX_FDIV(1.f, P->ls);
    float inv_s[3] = { VOX_FDIV(1.f, P->s[0]), VOX_FDIV(1.f, P->s[1]), VOX_FDIV(1.f, P->s[2]) };
    for (int v = 0; v < 8; v++)
    {
        float vp[3] = { (float)ijk[0], (float)ijk[1], (float)ijk[2] };
        if (v & 1)
            vp[0] = VOX_FADD(vp[0], 1.f);
        if (v & 2)
            vp[1] = VOX_FADD(vp[1], 1.f);
        if (v & 4)
            vp[2] = VOX_FADD(vp[2], 1.f);
        float lp[3];
        for (int a = 0; a < 3; a++)
            lp[a] = VOX_FSUB(VOX_FMUL(vp[a], vs), P->pos[a]);
        float l[3] = { dot3(lp, rinv[0]), dot3(lp, rinv[1]), dot3(lp, rinv[2]) };
        for (int a = 0; a < 3; a++)
        {
            l[a] = VOX_FMUL(l[a], inv_ls);
            l[a] = VOX_FMUL(l[a], inv_s[a]);
            if (v == 0 || l[a] < vmin[a])
                vmin[a] = l[a];
            if (v == 0 || l[a] > vmax[a])
                vmax[a] = l[a];
        }
    }
    float dist2 = 1.f;
    for (int a = 0; a < 3; a++)
    {
        if (0.f < vmin[a])
            dist2 = VOX_FSUB(dist2, VOX_FMUL(vmin[a], vmin[a]));
        else if (0.f > vmax[a])
            dist2 = VOX_FSUB(dist2, VOX_FMUL(vmax[a], vmax[a]));
    }
    return dist2 > 0.f;
}

/* gaussian_frag_color.slang:184-217: alpha after the opacity transform and
 * the cull, plus the packed RGBA8 */
static uint32_t frag_rgba(const prim_t* P, float vs, float cull_scale, const float* vmin, const float* vmax,
                          float* alpha_out)
{
    float a = 0.f;
    const float third = VOX_FDIV(1.f, 3.f);
    for (int s = 0; s < 64; s++)
    {
        float w[3] = { VOX_FMUL(third, (float)((s >> 4) & 3)), VOX_FMUL(third, (float)((s >> 2) & 3)),
                       VOX_FMUL(third, (float)(s & 3)) };
        float lp[3];
        for (int c = 0; c < 3; c++)
            lp[c] = VOX_FADD(VOX_FMUL(w[c], vmax[c]), VOX_FMUL(VOX_FSUB(1.f, w[c]), vmin[c]));
        float d = dot3(lp, lp);
        float v = VOX_FMUL(P->op, vox_expf_cr(-VOX_FMUL(P->ls, d)));
        a = v > a ? v : a;
    }
    float scale1d = VOX_FSQRT(dot3(P->s, P->s));
    float vrs = VOX_FDIV(VOX_FMUL(0.1f, scale1d), vs);
    a = VOX_FSUB(1.f, vox_powf(VOX_FSUB(1.f, a), VOX_FDIV(1.f, vrs)));
    float cull = cull_scale > 0.f ? cull_scale : 0.05f;
    if (scale1d > cull)
        a = 0.f;
    *alpha_out = a;
    float ch[4] = { P->rgb[0], P->rgb[1], P->rgb[2], a };
    uint32_t out = 0;
    for (int c = 0; c < 4; c++)
    {
        float v = ch[c] < 1.f ? ch[c] : 1.f;
        v = 0.f > v ? 0.f : v;
        out |= ((uint32_t)VOX_FMUL(255.f, v)) << (8 * c);
    }
    return out;
}

/* The float channels sum as exact 64-bit fixed-point integers in units of
 * 2^-32: each term rounded once to the grid (round to nearest even, clamped to
 * +-2^30), the total rounded once to float.  The integer sum does not depend
 * on the order of the terms; the device adds them with shared-memory atomics. */
#define FX_SCALE 4294967296.f          /* 2^32 */
#define FX_INV 2.3283064365386963e-10f /* 2^-32 */
#define FX_CLAMP 1073741824.f          /* 2^30 */
static int64_t fx_of(float x)
{
    x = x < FX_CLAMP ? x : FX_CLAMP;
    x = x > -FX_CLAMP ? x : -FX_CLAMP;
    return (int64_t)llrintf(VOX_FMUL(x, FX_SCALE));
}
static float fx_to_float(int64_t s)
{
    return VOX_FMUL((float)s, FX_INV);
}

/* Float density / colour channels (this build's F-mode output; the reference
 * has only RGBA8).  The alpha of gaussian_frag_color.slang:184-217 - local
 * AABB of the voxel, maximum over the 4x4x4 lattice, opacity transform, cull -
 * in a numerically stable float form, leaf-relative:
 *   the anchor c = o + r0, o the origin of the voxel's 8^3 leaf, r0_a =
 *     clamp(bmin_a + ((bmax_a + 1 - bmin_a) >> 1) - o_a, 0, 7) (the leaf voxel
 *     nearest the bbox's centre voxel); d0_a = fma(c_a, vs, -mu_a), the anchor corner's offset rounded
 *     once (fl(fl(v vs) - mu) loses the low bits of mu far from the origin);
 *     k_r = fl(inv_ls inv_s_r);
 *   per row r the scaled voxel steps A_ra = fl(fl(vs m_ra) k_r), the leaf
 *     origin's row base_r = fl(fl(fma(m_r2, d0_2, fma(m_r0, d0_0, fl(m_r1 d0_1)))) k_r),
 *     lo0_r = base_r + min(A_r0, 0) + min(A_r1, 0) + min(A_r2, 0) and
 *     W_r = |A_r0| + |A_r1| + |A_r2| (sums left to right, rounded);
 *   for the voxel at r = (rx, ry, rz) in its leaf, t = r - r0: lo_r =
 *     fma(t_z, A_r2, fma(t_y, A_r1, fma(t_x, A_r0, lo0_r))), hi_r = fl(lo_r + W_r);
 *   lattice points lo + w (hi - lo), w = 0, 1/3, 2/3, 1; the maximum of the
 *     decreasing exp is at the per-axis smallest square;
 *   float exp / pow (vox_expf_ch, vox_powf_ch).
 * The device evaluates the same operations in the same order (leaf_pair_consts,
 * stable_leaf_aabb); the signs of zero sums may differ, which the squares hide. */
static float frag_alpha_f(const prim_t* P, const float rinv[3][3], float vs, const int32_t* ijk, float cull_scale)
{
    const float inv_ls = VOX_FDIV(1.f, P->ls);
    float d0[3], rel[3];
    for (int a = 0; a < 3; a++)
    {
        const int32_t o = ijk[a] - (ijk[a] & 7);
        const int32_t rc = P->bmin[a] + ((P->bmax[a] + 1 - P->bmin[a]) >> 1) - o;
        const int32_t r0 = rc < 0 ? 0 : rc > 7 ? 7 : rc;
        d0[a] = VOX_FFMA((float)(o + r0), vs, -P->pos[a]);
        rel[a] = (float)((ijk[a] & 7) - r0);
    }
    float m[3];
    for (int r = 0; r < 3; r++)
    {
        const float* w = rinv[r];
        const float k = VOX_FMUL(inv_ls, VOX_FDIV(1.f, P->s[r]));
        const float base = VOX_FMUL(VOX_FFMA(w[2], d0[2], VOX_FFMA(w[0], d0[0], VOX_FMUL(w[1], d0[1]))), k);
        float A[3];
        for (int a = 0; a < 3; a++)
            A[a] = VOX_FMUL(VOX_FMUL(vs, w[a]), k);
        const float lo0 = VOX_FADD(VOX_FADD(VOX_FADD(base, A[0] < 0.f ? A[0] : 0.f), A[1] < 0.f ? A[1] : 0.f),
                                   A[2] < 0.f ? A[2] : 0.f);
        const float W = VOX_FADD(VOX_FADD(fabsf(A[0]), fabsf(A[1])), fabsf(A[2]));
        const float lo = VOX_FFMA(rel[2], A[2], VOX_FFMA(rel[1], A[1], VOX_FFMA(rel[0], A[0], lo0)));
        const float hi = VOX_FADD(lo, W);
        const float dd = VOX_FSUB(hi, lo);
        const float p1 = VOX_FFMA(dd, 0x1.555556p-2f, lo), p2 = VOX_FFMA(dd, 0x1.555556p-1f, lo);
        float best = VOX_FMUL(lo, lo);
        const float s1 = VOX_FMUL(p1, p1), s2 = VOX_FMUL(p2, p2), s3 = VOX_FMUL(hi, hi);
        best = s1 < best ? s1 : best;
        best = s2 < best ? s2 : best;
        best = s3 < best ? s3 : best;
        m[r] = best;
    }
    const float d = VOX_FADD(VOX_FADD(m[0], m[1]), m[2]);
    float a = VOX_FMUL(P->op, vox_expf_ch(-VOX_FMUL(P->ls, d)));
    a = a > 0.f ? a : 0.f;
    const float scale1d = VOX_FSQRT(dot3(P->s, P->s));
    const float vrs = VOX_FDIV(VOX_FMUL(0.1f, scale1d), vs);
    a = VOX_FSUB(1.f, vox_powf_ch(VOX_FSUB(1.f, a), VOX_FDIV(1.f, vrs)));
    const float cull = cull_scale > 0.f ? cull_scale : 0.05f;
    if (scale1d > cull)
        a = 0.f;
    return a;
}

/* FP64 restatement of the same alpha (lattice of 64 samples, cull), computed
 * from the float inputs in double with the C library's exp/log/pow. */
static double frag_alpha64(const prim_t* P, double vs, double cull_scale, const int32_t* ijk)
{
    double q[4] = { P->q[0], P->q[1], P->q[2], P->q[3] };
    double x = q[0], y = q[1], z = q[2], w = q[3];
    double r[3][3] = { { 1 - 2 * (y * y + z * z), 2 * (x * y + z * w), 2 * (x * z - y * w) },
                       { 2 * (x * y - z * w), 1 - 2 * (x * x + z * z), 2 * (y * z + x * w) },
                       { 2 * (x * z + y * w), 2 * (y * z - x * w), 1 - 2 * (x * x + y * y) } };
    double ls = sqrt(2.0 * log((double)P->op / 0.01));
    double s[3] = { P->s[0], P->s[1], P->s[2] };
    double vmin[3], vmax[3];
    for (int v = 0; v < 8; v++)
    {
        double lp[3] = { (ijk[0] + ((v & 1) ? 1 : 0)) * vs - P->pos[0], (ijk[1] + ((v & 2) ? 1 : 0)) * vs - P->pos[1],
                         (ijk[2] + ((v & 4) ? 1 : 0)) * vs - P->pos[2] };
        for (int a = 0; a < 3; a++)
        {
            double l = (lp[0] * r[a][0] + lp[1] * r[a][1] + lp[2] * r[a][2]) / ls / s[a];
            if (v == 0 || l < vmin[a])
                vmin[a] = l;
            if (v == 0 || l > vmax[a])
                vmax[a] = l;
        }
    }
    double al = 0.0;
    for (int sidx = 0; sidx < 64; sidx++)
    {
        double wv[3] = { ((sidx >> 4) & 3) / 3.0, ((sidx >> 2) & 3) / 3.0, (sidx & 3) / 3.0 };
        double d = 0.0;
        for (int c = 0; c < 3; c++)
        {
            double t = wv[c] * vmax[c] + (1.0 - wv[c]) * vmin[c];
            d += t * t;
        }
        double v = (double)P->op * exp(-ls * d);
        al = v > al ? v : al;
    }
    double scale1d = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    double vrs = 0.1 * scale1d / vs;
    al = 1.0 - pow(1.0 - al, 1.0 / vrs);
    /* the cull decision follows the float pass so both see the same pair set */
    float s1f = VOX_FSQRT(dot3(P->s, P->s));
    float cullf = cull_scale > 0 ? (float)cull_scale : 0.05f;
    if (s1f > cullf)
        al = 0.0;
    return al;
}

int ov_prim_bbox(const float* mean, const float* quat_wxyz, const float* scale, float opacity, float voxel_size,
                 int32_t* bbox6, uint64_t* footprint)
{
    prim_t P;
    prim_setup(&P, mean, quat_wxyz, scale, opacity, NULL, voxel_size);
    for (int a = 0; a < 3; a++)
    {
        bbox6[a] = P.bmin[a];
        bbox6[3 + a] = P.bmax[a];
    }
    *footprint = P.footprint;
    return P.valid;
}

int ov_frag_test(const float* mean, const float* quat_wxyz, const float* scale, float opacity, float voxel_size,
                 const int32_t* ijk, float* vmin3, float* vmax3)
{
    prim_t P;
    prim_setup(&P, mean, quat_wxyz, scale, opacity, NULL, voxel_size);
    if (!P.valid)
        return 0;
    float rinv[3][3];
    rot_inv_rows(P.q, rinv);
    return frag_test(&P, rinv, voxel_size, ijk, vmin3, vmax3);
}

uint32_t ov_frag_rgba(const float* mean, const float* quat_wxyz, const float* scale, float opacity,
                      const float* color, float voxel_size, float cull_scale, const int32_t* ijk, float* alpha_out)
{
    prim_t P;
    prim_setup(&P, mean, quat_wxyz, scale, opacity, color, voxel_size);
    float rinv[3][3], vmin[3], vmax[3];
    rot_inv_rows(P.q, rinv);
    frag_test(&P, rinv, voxel_size, ijk, vmin, vmax);
    return frag_rgba(&P, voxel_size, cull_scale, vmin, vmax, alpha_out);
}

/* ------------------------------------------------------------------------ */
/* incremental node2 build (raster/GridBuild.cpp:361-506 +                   */
/* grid_build_{set_masks,count_new,scatter_new,finalize}.slang)              */
/* ------------------------------------------------------------------------ */
typedef struct
{
    int type;
    int32_t parent;
    uint32_t n;
    int32_t origin[3];
    int32_t* child;     /* dense child node index per n (-1 none); non-leaf */
    uint64_t* vmask;    /* leaf value mask (8 words) */
} node_t;

typedef struct
{
    /* inputs */
    int64_t G;
    float vs, cull;
    int skip_f64; /* timing runs: only the float outputs the product computes */
    int smooth;   /* OV_MODE_SMOOTH: differentiable density / colour channels */
    prim_t* prims;
    /* pairs in emission (Gaussian-major) order, later sorted */
    uint64_t* keys;
    uint32_t* ids;
    int32_t* pijk; /* ijk per pair, emission order */
    int64_t P, Pcap;
    /* tree */
    node_t* nodes;
    int64_t nn, ncap;
    /* results */
    int64_t counts[OV_COUNT_N];
    uint8_t* node2;
    int64_t node2_bytes;
    uint64_t* value_idx_node; /* per node */
    int64_t V;
    int32_t* vox_ijk;
    uint64_t* vox_vidx;
    uint32_t* rgba;
    float* dens;
    float* col;
    double* dens64;
    double* col64;
    int32_t bbox[6];
} ov_state_t;

static int32_t new_node(ov_state_t* S, int type, int32_t parent, uint32_t n, const int32_t* origin)
{
    if (S->nn == S->ncap)
    {
        S->ncap = S->ncap ? 2 * S->ncap : 1024;
        S->nodes = (node_t*)realloc(S->nodes, sizeof(node_t) * S->ncap);
    }
    node_t* N = &S->nodes[S->nn];
    N->type = type;
    N->parent = parent;
    N->n = n;
    N->origin[0] = origin[0];
    N->origin[1] = origin[1];
    N->origin[2] = origin[2];
    N->child = NULL;
    N->vmask = NULL;
    if (type < 3)
    {
        N->child = (int32_t*)malloc(sizeof(int32_t) * N2_FANOUT[type]);
        for (uint32_t i = 0; i < N2_FANOUT[type]; i++)
            N->child[i] = -1;
    }
    else
    {
        N->vmask = (uint64_t*)calloc(8, sizeof(uint64_t));
    }
    return (int32_t)(S->nn++);
}

typedef struct
{
    int32_t node;
    uint32_t n;
    int32_t ijk[3];
} mark_t;

static int mark_cmp(const void* a, const void* b)
{
    const mark_t* x = (const mark_t*)a;
    const mark_t* y = (const mark_t*)b;
    if (x->node != y->node)
        return x->node < y->node ? -1 : 1;
    if (x->n != y->n)
        return x->n < y->n ? -1 : 1;
    return 0;
}

/* one fragment window: levels root -> upper -> lower -> leaf (GridBuild.cpp:412-505).
 * New children are appended in (parent node_idx, n) order, which is the order
 * grid_build_scatter_new.slang:107-170 allocates them in. */
static void insert_window(ov_state_t* S, const int32_t* ijk, int64_t count)
{
    mark_t* marks = (mark_t*)malloc(sizeof(mark_t) * (count ? count : 1));
    for (int level = 0; level < 3; level++)
    {
        int64_t m = 0;
        for (int64_t f = 0; f < count; f++)
        {
            const int32_t* c = &ijk[3 * f];
            int32_t node = 0;
            for (int t = 0; t < level; t++)
                node = S->nodes[node].child[n2_coord_to_n(t, c[0], c[1], c[2])];
            uint32_t n = n2_coord_to_n(level, c[0], c[1], c[2]);
            if (S->nodes[node].child[n] < 0)
            {
                marks[m].node = node;
                marks[m].n = n;
                marks[m].ijk[0] = c[0];
                marks[m].ijk[1] = c[1];
                marks[m].ijk[2] = c[2];
                m++;
            }
        }
        qsort(marks, (size_t)m, sizeof(mark_t), mark_cmp);
        for (int64_t i = 0; i < m; i++)
        {
            if (i > 0 && marks[i].node == marks[i - 1].node && marks[i].n == marks[i - 1].n)
                continue;
            uint32_t tile = 1u << N2_TILEDIM_BITS[level]; /* child covers 2^tiledim voxels per axis */
            int32_t origin[3];
            for (int a = 0; a < 3; a++)
                origin[a] = marks[i].ijk[a] & ~(int32_t)(tile - 1u);
            int32_t child = new_node(S, level + 1, marks[i].node, marks[i].n, origin);
            S->nodes[marks[i].node].child[marks[i].n] = child;
        }
    }
    /* leaf value bits */
    for (int64_t f = 0; f < count; f++)
    {
        const int32_t* c = &ijk[3 * f];
        int32_t node = 0;
        for (int t = 0; t < 3; t++)
            node = S->nodes[node].child[n2_coord_to_n(t, c[0], c[1], c[2])];
        uint32_t n = n2_coord_to_n(3, c[0], c[1], c[2]);
        S->nodes[node].vmask[n >> 6] |= 1ull << (n & 63);
    }
    free(marks);
}

/* ------------------------------------------------------------------------ */
/* threaded fragment test for one window                                     */
/* ------------------------------------------------------------------------ */
typedef struct
{
    ov_state_t* S;
    const int64_t* pidx;      /* prim index per prim in batch */
    const uint64_t* off;      /* exclusive fragment offset within batch */
    int64_t nprim;
    uint64_t f0, f1;          /* fragment range of this worker */
    int32_t* out_ijk;
    uint32_t* out_id;
    int64_t out_n, out_cap;
} wjob_t;

static int64_t upper_bound_u64(const uint64_t* a, int64_t n, uint64_t v)
{
    int64_t lo = 0, hi = n;
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

static void* window_worker(void* arg)
{
    wjob_t* J = (wjob_t*)arg;
    ov_state_t* S = J->S;
    if (J->f0 >= J->f1)
        return NULL;
    /* prim containing fragment f0: last prim with off <= f0 (zero-footprint prims are skipped) */
    int64_t p = upper_bound_u64(J->off, J->nprim, J->f0) - 1;
    uint64_t f = J->f0;
    while (f < J->f1 && p < J->nprim)
    {
        const prim_t* P = &S->prims[J->pidx[p]];
        uint64_t pend = J->off[p] + P->footprint;
        if (P->footprint == 0 || f >= pend)
        {
            p++;
            continue;
        }
        float rinv[3][3];
        rot_inv_rows(P->q, rinv);
        int32_t Ry = P->bmax[1] + 1 - P->bmin[1], Rz = P->bmax[2] + 1 - P->bmin[2];
        uint64_t stop = pend < J->f1 ? pend : J->f1;
        for (; f < stop; f++)
        {
            int32_t r = (int32_t)(f - J->off[p]);
            /* gaussian_frag_alloc.slang:55-58 */
            int32_t ijk[3] = { r / (Rz * Ry) + P->bmin[0], (r / Rz) % Ry + P->bmin[1], r % Rz + P->bmin[2] };
            float vmin[3], vmax[3];
            if (frag_test(P, rinv, S->vs, ijk, vmin, vmax))
            {
                if (J->out_n == J->out_cap)
                {
                    J->out_cap = J->out_cap ? 2 * J->out_cap : 4096;
                    J->out_ijk = (int32_t*)realloc(J->out_ijk, sizeof(int32_t) * 3 * J->out_cap);
                    J->out_id = (uint32_t*)realloc(J->out_id, sizeof(uint32_t) * J->out_cap);
                }
                memcpy(&J->out_ijk[3 * J->out_n], ijk, 12);
                J->out_id[J->out_n] = (uint32_t)J->pidx[p];
                J->out_n++;
            }
        }
        p++;
    }
    return NULL;
}

/* stable LSD radix sort of (key, id) by key, 11-bit digits */
static void radix_sort_pairs(uint64_t* keys, uint32_t* ids, int64_t n, int key_bits)
{
    uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
    uint32_t* i2 = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    int64_t* hist = (int64_t*)malloc(sizeof(int64_t) * 2048);
    for (int sh = 0; sh < key_bits; sh += 11)
    {
        memset(hist, 0, sizeof(int64_t) * 2048);
        for (int64_t i = 0; i < n; i++)
            hist[(keys[i] >> sh) & 2047]++;
        int64_t s = 0;
        for (int d = 0; d < 2048; d++)
        {
            int64_t c = hist[d];
            hist[d] = s;
            s += c;
        }
        for (int64_t i = 0; i < n; i++)
        {
            int64_t dst = hist[(keys[i] >> sh) & 2047]++;
            k2[dst] = keys[i];
            i2[dst] = ids[i];
        }
        memcpy(keys, k2, sizeof(uint64_t) * n);
        memcpy(ids, i2, sizeof(uint32_t) * n);
    }
    free(k2);
    free(i2);
    free(hist);
}


/* ------------------------------------------------------------------------ */
/* VoxelBVH Gaussian ingestion (raster/VoxelBVH.cpp:1225-1435): per Gaussian  */
/* the finest power-of-two cell level at which at most 8 cells overlap it,   */
/* and those cells as 64-bit keys i << 48 | j << 32 | k << 16 | level; keys  */
/* sorted stably, then the [start, end) range of every distinct key.  Inputs */
/* are activated (normalised quaternions w,x,y,z, scales, opacities).  The   */
/* float arithmetic follows the shaders literally, left to right:            */
/* voxelbvh_gaussians_bbox_reduce1/2.slang, voxelbvh_gaussians_to_ijkl.slang */
/* (:25-250), voxelbvh_find_range_starts.slang, voxelbvh_scatter_range_      */
/* headers.slang.  T / Tinv: 16 floats, rows x y z w of the reference's      */
/* pnanovdb_camera_mat_t, applied to row vectors (p' = [p 1] T, the shader's */
/* mul(float4(p, 1), transform) with the transposed constant read back       */
/* column-major, VoxelBVH.cpp:1285-1291); NULL = identity.  World-box        */
/* minima and maxima order -0 below +0 (a total order, as a deterministic    */
/* device reduction has it).  A non-finite box corner, or a box that maps    */
/* beyond +-65536 voxels, is an error (-1), where the shaders' result is     */
/* undefined.                                                                */
/* ------------------------------------------------------------------------ */
static void vb_xform(const float* T, const float p[3], float out[3])
{
    if (!T)
    {
        out[0] = p[0];
        out[1] = p[1];
        out[2] = p[2];
        return;
    }
    for (int c = 0; c < 3; c++)
        out[c] = VOX_FADD(VOX_FADD(VOX_FADD(VOX_FMUL(p[0], T[c]), VOX_FMUL(p[1], T[4 + c])), VOX_FMUL(p[2], T[8 + c])),
                          T[12 + c]);
}

/* float -> uint32 whose unsigned order is the float order, -0 below +0 */
static uint32_t vb_fkey(float f)
{
    const uint32_t u = vox_f2u(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

static float vb_fmin(float a, float b)
{
    return vb_fkey(a) < vb_fkey(b) ? a : b;
}

static float vb_fmax(float a, float b)
{
    return vb_fkey(a) > vb_fkey(b) ? a : b;
}

static float vb_local_scale(float opacity)
{
    const float o = 0.01f > opacity ? 0.01f : opacity; /* max(0.01, opacity) */
    return VOX_FSQRT(VOX_FMUL(2.f, vox_logf(VOX_FDIV(o, 0.01f))));
}

/* the transformed 8-corner box of the 1-sigma * local_scale cube; returns 0
 * when a corner is not finite (an error for the caller) */
static int vb_gauss_aabb(const float* mean, const float* q_wxyz, const float* scale, float opacity, const float* T,
                          float mn[3], float mx[3])
{
    const float x = q_wxyz[1], y = q_wxyz[2], z = q_wxyz[3], w = q_wxyz[0];
    const float ls = vb_local_scale(opacity);
    const float r0[3] = { VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(y, y), VOX_FMUL(z, z)))),
                          VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(x, y), VOX_FMUL(z, w))),
                          VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, z), VOX_FMUL(y, w))) };
    const float r1[3] = { VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, y), VOX_FMUL(z, w))),
                          VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(z, z)))),
                          VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(y, z), VOX_FMUL(x, w))) };
    const float r2[3] = { VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(x, z), VOX_FMUL(y, w))),
                          VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(y, z), VOX_FMUL(x, w))),
                          VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(y, y)))) };
    const float* rr[3] = { r0, r1, r2 };
    for (int a = 0; a < 3; a++)
    {
        mn[a] = vox_u2f(0x7f800000u);
        mx[a] = -vox_u2f(0x7f800000u);
    }
    for (int v = 0; v < 8; v++)
    {
        float cp[3];
        for (int a = 0; a < 3; a++)
        {
            const float e = VOX_FMUL(scale[a], ls);
            cp[a] = ((v >> a) & 1) ? e : -e;
        }
        float wp[3];
        for (int c = 0; c < 3; c++)
            wp[c] = VOX_FADD(VOX_FADD(VOX_FADD(VOX_FMUL(cp[0], rr[c][0]), VOX_FMUL(cp[1], rr[c][1])),
                                      VOX_FMUL(cp[2], rr[c][2])),
                             mean[c]);
        float tp[3];
        vb_xform(T, wp, tp);
        for (int a = 0; a < 3; a++)
        {
            if (!isfinite(tp[a]))
                return 0;
            mn[a] = vb_fmin(tp[a], mn[a]);
            mx[a] = vb_fmax(tp[a], mx[a]);
        }
    }
    return 1;
}

/* voxel_ellipsoid_overlap of voxelbvh_gaussians_to_ijkl.slang:25-109 */
static int vb_overlap(const float* mean, const float* q_wxyz, const float* scale, float opacity, const float w2v[4],
                      const int32_t ijk[3], uint32_t level, const float* Tinv)
{
    const float x = q_wxyz[1], y = q_wxyz[2], z = q_wxyz[3], w = q_wxyz[0];
    const float ls = vb_local_scale(opacity);
    const float i0[3] = { VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(y, y), VOX_FMUL(z, z)))),
                          VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, y), VOX_FMUL(z, w))),
                          VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(x, z), VOX_FMUL(y, w))) };
    const float i1[3] = { VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(x, y), VOX_FMUL(z, w))),
                          VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(z, z)))),
                          VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(y, z), VOX_FMUL(x, w))) };
    const float i2[3] = { VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, z), VOX_FMUL(y, w))),
                          VOX_FMUL(2.f, VOX_FSUB(VOX_FMUL(y, z), VOX_FMUL(x, w))),
                          VOX_FSUB(1.f, VOX_FMUL(2.f, VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(y, y)))) };
    const float* ii[3] = { i0, i1, i2 };
    const float step = (float)(1u << level);
    float vmin[3] = { 0, 0, 0 }, vmax[3] = { 0, 0, 0 };
    for (int v = 0; v < 8; v++)
    {
        float vp[3];
        for (int a = 0; a < 3; a++)
        {
            vp[a] = (float)ijk[a];
            if ((v >> a) & 1)
                vp[a] = VOX_FADD(vp[a], step);
        }
        float lp[3];
        for (int a = 0; a < 3; a++)
            lp[a] = VOX_FDIV(VOX_FSUB(vp[a], w2v[a]), w2v[3]);
        float tp[3];
        vb_xform(Tinv, lp, tp);
        for (int a = 0; a < 3; a++)
            tp[a] = VOX_FSUB(tp[a], mean[a]);
        float lr[3];
        for (int r = 0; r < 3; r++)
            lr[r] = VOX_FADD(VOX_FADD(VOX_FMUL(tp[0], ii[r][0]), VOX_FMUL(tp[1], ii[r][1])), VOX_FMUL(tp[2], ii[r][2]));
        for (int a = 0; a < 3; a++)
        {
            lr[a] = VOX_FMUL(lr[a], VOX_FDIV(1.f, VOX_FMUL(ls, scale[a])));
            if (v == 0 || lr[a] < vmin[a])
                vmin[a] = lr[a];
            if (v == 0 || lr[a] > vmax[a])
                vmax[a] = lr[a];
        }
    }
    float dist2 = 1.f;
    for (int a = 0; a < 3; a++)
    {
        if (0.f < vmin[a])
            dist2 = VOX_FSUB(dist2, VOX_FMUL(vmin[a], vmin[a]));
        else if (0.f > vmax[a])
            dist2 = VOX_FSUB(dist2, VOX_FMUL(vmax[a], vmax[a]));
    }
    return dist2 > 0.f;
}

/* keys of Gaussian g (voxelbvh_gaussians_to_ijkl.slang main); 0 = error */
static int vb_gauss_keys(int64_t g, const float* means, const float* opacities, const float* quats_wxyz,
                         const float* scales, const float* T, const float* Tinv, float sc, const float w2v[4],
                         uint64_t* ijkl, uint32_t* prim_id)
{
    const float* mu = &means[3 * g];
    const float* q = &quats_wxyz[4 * g];
    const float* s = &scales[3 * g];
    const float op = opacities[g];
    float mn[3], mx[3];
    if (!vb_gauss_aabb(mu, q, s, op, T, mn, mx))
        return 0;
    int32_t lo[3], hi[3];
    for (int a = 0; a < 3; a++)
    {
        const float fl = floorf(VOX_FADD(VOX_FMUL(sc, mn[a]), w2v[a]));
        const float fh = floorf(VOX_FADD(VOX_FMUL(sc, mx[a]), w2v[a]));
        /* cells beyond +-65536 (non-finite input, zero-size world box):
         * an error, as the device reports it, not an unbounded search */
        if (!(fl >= -65536.f && fl <= 65536.f && fh >= -65536.f && fh <= 65536.f))
            return 0;
        lo[a] = (int32_t)fl;
        hi[a] = (int32_t)fh;
    }
    uint32_t level = 11u, last_good = 11u;
    while (level < 12u)
    {
        const int32_t msk = ~((1 << level) - 1), st = 1 << level;
        /* a level of more than 2^24 cells: an error, not a search (the
         * device bounds its search the same way) */
        int64_t cells = 1;
        for (int a = 0; a < 3; a++)
            cells *= (int64_t)(((hi[a] & msk) - (lo[a] & msk)) >> level) + 1;
        if (cells > (1ll << 24))
            return 0;
        uint32_t count = 0;
        for (int32_t i = lo[0] & msk; i <= (hi[0] & msk); i += st)
            for (int32_t j = lo[1] & msk; j <= (hi[1] & msk); j += st)
                for (int32_t k = lo[2] & msk; k <= (hi[2] & msk); k += st)
                {
                    const int32_t c[3] = { i, j, k };
                    count += (uint32_t)vb_overlap(mu, q, s, op, w2v, c, level, Tinv);
                }
        if (count > 8u)
        {
            level = last_good;
            break;
        }
        if (level == 0u)
            break;
        last_good = level;
        level -= 1u;
    }
    uint32_t sub = 0;
    {
        const int32_t msk = ~((1 << level) - 1), st = 1 << level;
        for (int32_t i = lo[0] & msk; i <= (hi[0] & msk); i += st)
            for (int32_t j = lo[1] & msk; j <= (hi[1] & msk); j += st)
                for (int32_t k = lo[2] & msk; k <= (hi[2] & msk); k += st)
                {
                    const int32_t c[3] = { i, j, k };
                    if (sub < 8u && vb_overlap(mu, q, s, op, w2v, c, level, Tinv))
                    {
                        ijkl[8 * g + sub] = ((uint64_t)(int64_t)i << 48) | ((uint64_t)(int64_t)j << 32) |
                                            ((uint64_t)(int64_t)k << 16) | (uint64_t)level;
                        prim_id[8 * g + sub] = (uint32_t)g;
                        sub++;
                    }
                }
    }
    for (; sub < 8u; sub++)
    {
        ijkl[8 * g + sub] = ~0ull;
        prim_id[8 * g + sub] = ~0u;
    }

    return 1;
}

typedef struct
{
    int64_t g0, g1;
    const float *means, *opacities, *quats, *scales, *T, *Tinv;
    float sc, w2v[4];
    uint64_t* ijkl;
    uint32_t* prim_id;
    float mn[3], mx[3];
    int err;
} vbjob_t;

static void* vb_box_worker(void* arg)
{
    vbjob_t* J = (vbjob_t*)arg;
    for (int a = 0; a < 3; a++)
    {
        J->mn[a] = vox_u2f(0x7f800000u);
        J->mx[a] = -vox_u2f(0x7f800000u);
    }
    for (int64_t g = J->g0; g < J->g1; g++)
    {
        float mn[3], mx[3];
        if (!vb_gauss_aabb(&J->means[3 * g], &J->quats[4 * g], &J->scales[3 * g], J->opacities[g], J->T, mn, mx))
        {
            J->err = 1;
            return NULL;
        }
        for (int a = 0; a < 3; a++)
        {
            J->mn[a] = vb_fmin(mn[a], J->mn[a]);
            J->mx[a] = vb_fmax(mx[a], J->mx[a]);
        }
    }
    return NULL;
}

static void* vb_keys_worker(void* arg)
{
    vbjob_t* J = (vbjob_t*)arg;
    for (int64_t g = J->g0; g < J->g1 && !J->err; g++)
        if (!vb_gauss_keys(g, J->means, J->opacities, J->quats, J->scales, J->T, J->Tinv, J->sc, J->w2v, J->ijkl,
                           J->prim_id))
            J->err = 1;
    return NULL;
}

int64_t ov_voxelbvh_ijkl(int64_t n, const float* means, const float* opacities, const float* quats_wxyz,
                         const float* scales, uint32_t resolution, const float* T, const float* Tinv,
                         uint64_t* ijkl, uint32_t* prim_id, uint32_t* range, float* world_bbox, int nthreads)
{
    if (nthreads < 1)
        nthreads = 1;
    if ((int64_t)nthreads > n)
        nthreads = n > 0 ? (int)n : 1;
    vbjob_t* jobs = (vbjob_t*)calloc((size_t)nthreads, sizeof(vbjob_t));
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int t = 0; t < nthreads; t++)
    {
        vbjob_t* J = &jobs[t];
        J->g0 = n * t / nthreads;
        J->g1 = n * (t + 1) / nthreads;
        J->means = means;
        J->opacities = opacities;
        J->quats = quats_wxyz;
        J->scales = scales;
        J->T = T;
        J->Tinv = Tinv;
        J->ijkl = ijkl;
        J->prim_id = prim_id;
    }
    /* world bbox (bbox_reduce1/2): minima / maxima in a total order, so the
     * split over threads does not change the result */
    for (int t = 0; t < nthreads; t++)
        pthread_create(&th[t], NULL, vb_box_worker, &jobs[t]);
    int err = 0;
    float wmin[3], wmax[3];
    for (int a = 0; a < 3; a++)
    {
        wmin[a] = vox_u2f(0x7f800000u);
        wmax[a] = -vox_u2f(0x7f800000u);
    }
    for (int t = 0; t < nthreads; t++)
    {
        pthread_join(th[t], NULL);
        err |= jobs[t].err;
        for (int a = 0; a < 3; a++)
        {
            wmin[a] = vb_fmin(jobs[t].mn[a], wmin[a]);
            wmax[a] = vb_fmax(jobs[t].mx[a], wmax[a]);
        }
    }
    if (err)
    {
        free(jobs);
        free(th);
        return -1;
    }
    for (int a = 0; a < 3; a++)
    {
        world_bbox[a] = wmin[a];
        world_bbox[3 + a] = wmax[a];
    }
    /* compute_world_to_voxel */
    const float d[3] = { VOX_FSUB(wmax[0], wmin[0]), VOX_FSUB(wmax[1], wmin[1]), VOX_FSUB(wmax[2], wmin[2]) };
    const float dyz = d[1] > d[2] ? d[1] : d[2];
    const float dmax = d[0] > dyz ? d[0] : dyz;
    const float sc = VOX_FDIV((float)(resolution - 1u), dmax);
    const float w2v[4] = { VOX_FADD(VOX_FMUL(-wmin[0], sc), 0.5f), VOX_FADD(VOX_FMUL(-wmin[1], sc), 0.5f),
                           VOX_FADD(VOX_FMUL(-wmin[2], sc), 0.5f), sc };
    for (int t = 0; t < nthreads; t++)
    {
        jobs[t].sc = sc;
        for (int a = 0; a < 4; a++)
            jobs[t].w2v[a] = w2v[a];
        pthread_create(&th[t], NULL, vb_keys_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++)
    {
        pthread_join(th[t], NULL);
        err |= jobs[t].err;
    }
    free(jobs);
    free(th);
    if (err)
        return -1;
    const int64_t nv = 8 * n;
    /* stable sort by the full 64-bit key */
    radix_sort_pairs(ijkl, prim_id, nv, 64);
    /* ranges: [start, end) of every distinct key, at the key's rank; the rest 0 */
    memset(range, 0, sizeof(uint32_t) * 2 * (size_t)nv);
    int64_t r = -1;
    for (int64_t i = 0; i < nv; i++)
    {
        if (i == 0 || ijkl[i] != ijkl[i - 1])
        {
            r++;
            range[2 * r] = (uint32_t)i;
        }
        if (i + 1 == nv || ijkl[i] != ijkl[i + 1])
            range[2 * r + 1] = (uint32_t)(i + 1);
    }
    return r + 1;
}

/* ------------------------------------------------------------------------ */
/* Differentiable (smooth) channels.  The reference's alpha (max over a 4^3  */
/* lattice, opacity transform, cull) is discontinuous at the pair-set        */
/* boundary and piecewise in every parameter, so the differentiable channels */
/* use the centre-sampled kernel                                             */
/*   K = max(op * exp(-|S^-1 R^T (x - mu)|^2 / 2) - 0.01, 0)                 */
/* over the same pair set: K vanishes where the voxel centre leaves the      */
/* 0.01-opacity ellipsoid the reference test is built on (its radius         */
/* ls = sqrt(2 log(op / 0.01)), gaussian_prim.slang:65), so the channel is   */
/* continuous.  density = sum K, colour = sum K * rgb (premultiplied).       */
/* ------------------------------------------------------------------------ */
#define OV_SMOOTH_TAU 0.01f
#define OV_SH_C0 0.28209479177387814

/* float kernel, bit-identical to the device: centre offsets rounded once
 * from double, u = dot(d, rinv row), z = u * (1 / s), |z|^2 in dot order */
static float smooth_k_f32(const prim_t* P, const float rinv[3][3], float vs, const int32_t* ijk)
{
    float d[3];
    for (int a = 0; a < 3; a++)
        d[a] = (float)(((double)ijk[a] + 0.5) * (double)vs - (double)P->pos[a]);
    float z[3];
    for (int r = 0; r < 3; r++)
        z[r] = VOX_FMUL(dot3(d, rinv[r]), VOX_FDIV(1.f, P->s[r]));
    float q = dot3(z, z);
    float e = VOX_FMUL(P->op, vox_expf_cr(VOX_FMUL(-0.5f, q)));
    return e > OV_SMOOTH_TAU ? VOX_FSUB(e, OV_SMOOTH_TAU) : 0.f;
}

typedef struct
{
    double mu[3];
    double q[4];  /* x, y, z, w after normalisation (raw inputs) */
    double qnorm; /* |q| of the raw quaternion (1 for activated inputs) */
    double R[3][3];
    double s[3], s_act[3];
    int clamped[3];
    double op, rgb[3];
    int raw;
} g64_t;

static void g64_rot(g64_t* g)
{
    double x = g->q[0], y = g->q[1], z = g->q[2], w = g->q[3];
    g->R[0][0] = 1 - 2 * (y * y + z * z);
    g->R[0][1] = 2 * (x * y - z * w);
    g->R[0][2] = 2 * (x * z + y * w);
    g->R[1][0] = 2 * (x * y + z * w);
    g->R[1][1] = 1 - 2 * (x * x + z * z);
    g->R[1][2] = 2 * (y * z - x * w);
    g->R[2][0] = 2 * (x * z - y * w);
    g->R[2][1] = 2 * (y * z + x * w);
    g->R[2][2] = 1 - 2 * (x * x + y * y);
}

/* FP64 Gaussian from the caller's parameters: raw = (quaternion as given,
 * log-scale, opacity logit, SH0) as raster/RasterUtils.cpp:59-117 activates
 * them; otherwise (normalised quaternion, scale, opacity, rgb). */
static void g64_setup(g64_t* g, const double* mean, const double* q_wxyz, const double* scale, double opac,
                      const double* col, int raw, double vs)
{
    g->raw = raw;
    for (int a = 0; a < 3; a++)
        g->mu[a] = mean[a];
    double x = q_wxyz[1], y = q_wxyz[2], z = q_wxyz[3], w = q_wxyz[0];
    double n = raw ? sqrt(x * x + y * y + z * z + w * w) : 1.0;
    g->qnorm = n;
    g->q[0] = x / n;
    g->q[1] = y / n;
    g->q[2] = z / n;
    g->q[3] = w / n;
    g64_rot(g);
    const double min_scale = 0.125 * vs;
    for (int a = 0; a < 3; a++)
    {
        g->s_act[a] = raw ? exp(scale[a]) : scale[a];
        g->clamped[a] = !(g->s_act[a] > min_scale);
        g->s[a] = g->clamped[a] ? min_scale : g->s_act[a];
    }
    g->op = raw ? 1.0 / (1.0 + exp(-opac)) : opac;
    for (int c = 0; c < 3; c++)
        g->rgb[c] = raw ? OV_SH_C0 * col[c] + 0.5 : col[c];
}

/* FP64 Gaussian from the float activated record (value comparison only) */
static void g64_from_prim(g64_t* g, const prim_t* P)
{
    g->raw = 0;
    for (int a = 0; a < 3; a++)
    {
        g->mu[a] = P->pos[a];
        g->s[a] = g->s_act[a] = P->s[a];
        g->clamped[a] = 0;
    }
    for (int a = 0; a < 4; a++)
        g->q[a] = P->q[a];
    g->qnorm = 1.0;
    g64_rot(g);
    g->op = P->op;
    for (int c = 0; c < 3; c++)
        g->rgb[c] = P->rgb[c];
}

typedef struct
{
    double d[3], z[3], E, e;
} smooth_terms_t;

static double smooth64(const g64_t* g, double vs, const int32_t* ijk, smooth_terms_t* t)
{
    double d[3], z[3], q = 0.0;
    for (int a = 0; a < 3; a++)
        d[a] = ((double)ijk[a] + 0.5) * vs - g->mu[a];
    for (int r = 0; r < 3; r++)
    {
        double u = g->R[0][r] * d[0] + g->R[1][r] * d[1] + g->R[2][r] * d[2];
        z[r] = u / g->s[r];
        q += z[r] * z[r];
    }
    double E = exp(-0.5 * q), e = g->op * E;
    if (t)
    {
        memcpy(t->d, d, sizeof(d));
        memcpy(t->z, z, sizeof(z));
        t->E = E;
        t->e = e;
    }
    return e > (double)OV_SMOOTH_TAU ? e - (double)OV_SMOOTH_TAU : 0.0;
}

/* ------------------------------------------------------------------------ */
/* values: gaussian_frag_color.slang:182-246 (R mode, max of packed RGBA8)   */
/* plus the float density / colour sums in (key, id) order                   */
/* ------------------------------------------------------------------------ */
typedef struct
{
    ov_state_t* S;
    const int64_t* vstart; /* pair start per voxel (V + 1 entries) */
    int64_t v0, v1;
} vjob_t;

static void* values_worker(void* arg)
{
    vjob_t* J = (vjob_t*)arg;
    ov_state_t* S = J->S;
    for (int64_t v = J->v0; v < J->v1; v++)
    {
        uint64_t vi = S->vox_vidx[v];
        const int32_t* ijk = &S->vox_ijk[3 * v];
        uint32_t rgba = 0;
        int64_t dfx = 0, cfx[3] = { 0, 0, 0 };
        double dsum64 = 0.0, csum64[3] = { 0.0, 0.0, 0.0 };
        for (int64_t p = J->vstart[v]; p < J->vstart[v + 1]; p++)
        {
            const prim_t* P = &S->prims[S->ids[p]];
            float rinv[3][3], vmin[3], vmax[3], a;
            rot_inv_rows(P->q, rinv);
            frag_test(P, rinv, S->vs, ijk, vmin, vmax);
            float a8;
            uint32_t c = frag_rgba(P, S->vs, S->cull, vmin, vmax, &a8);
            rgba = c > rgba ? c : rgba; /* InterlockedMax, :239-246 */
            if (S->smooth)
            {
                float k = smooth_k_f32(P, rinv, S->vs, ijk);
                dfx += fx_of(k);
                for (int ch = 0; ch < 3; ch++)
                    cfx[ch] += fx_of(VOX_FMUL(k, P->rgb[ch]));
                if (!S->skip_f64)
                {
                    g64_t g;
                    g64_from_prim(&g, P);
                    double k64 = smooth64(&g, (double)S->vs, ijk, NULL);
                    dsum64 += k64;
                    for (int ch = 0; ch < 3; ch++)
                        csum64[ch] += k64 * g.rgb[ch];
                }
                continue;
            }
            a = frag_alpha_f(P, rinv, S->vs, ijk, S->cull);
            dfx += fx_of(a);
            for (int ch = 0; ch < 3; ch++)
                cfx[ch] += fx_of(VOX_FMUL(a, P->rgb[ch]));
            double a64 = S->skip_f64 ? 0.0 : frag_alpha64(P, (double)S->vs, (double)S->cull, ijk);
            dsum64 += a64;
            for (int ch = 0; ch < 3; ch++)
                csum64[ch] += a64 * (double)P->rgb[ch];
        }
        const float dsum = fx_to_float(dfx);
        const float csum[3] = { fx_to_float(cfx[0]), fx_to_float(cfx[1]), fx_to_float(cfx[2]) };
        S->rgba[vi] = rgba;
        S->dens[vi] = dsum;
        S->dens64[vi] = dsum64;
        for (int ch = 0; ch < 3; ch++)
        {
            if (S->smooth)
            {
                /* premultiplied colour: linear in the per-pair weights */
                S->col[3 * vi + ch] = csum[ch];
                S->col64[3 * vi + ch] = csum64[ch];
                continue;
            }
            S->col[3 * vi + ch] = dsum > 0.f ? VOX_FDIV(csum[ch], dsum) : 0.f;
            S->col64[3 * vi + ch] = dsum64 > 0.0 ? csum64[ch] / dsum64 : 0.0;
        }
    }
    return NULL;
}

static int popc64(uint64_t x)
{
    return __builtin_popcountll(x);
}

/* mask prefix sums, grid_build_count_new.slang:49-88: field (w & 3) of word
 * (w >> 2) holds popcount(mask[0 .. w-1]); field 0 of word 0 holds the total. */
static void write_prefix(uint64_t* words, const uint64_t* mask, uint32_t nwords)
{
    uint64_t sum = 0;
    for (uint32_t w = 0; w < nwords; w++)
    {
        sum += (uint64_t)popc64(mask[w]);
        uint32_t wi = (w + 1) & (nwords - 1);
        uint64_t* dst = &words[wi >> 2];
        *dst &= ~(0xFFFFull << ((wi & 3) * 16));
        *dst |= (sum & 0xFFFF) << ((wi & 3) * 16);
    }
}

static void serialize(ov_state_t* S)
{
    int64_t nn = S->nn;
    uint64_t* addr = (uint64_t*)malloc(sizeof(uint64_t) * nn);
    uint64_t total = 0;
    for (int64_t i = 0; i < nn; i++)
    {
        addr[i] = total;
        total += N2_MAX_SIZE[S->nodes[i].type];
    }
    S->node2_bytes = (int64_t)total;
    S->node2 = (uint8_t*)calloc(total, 1);
    S->value_idx_node = (uint64_t*)malloc(sizeof(uint64_t) * nn);
    uint64_t vsum = 2; /* two background values, grid_build_count_new.slang:103-106 */
    for (int64_t i = 0; i < nn; i++)
    {
        S->value_idx_node[i] = vsum;
        if (S->nodes[i].type == 3)
            for (int w = 0; w < 8; w++)
                vsum += (uint64_t)popc64(S->nodes[i].vmask[w]);
    }
    for (int64_t i = 0; i < nn; i++)
    {
        node_t* N = &S->nodes[i];
        uint64_t* W = (uint64_t*)(S->node2 + addr[i]);
        int t = N->type;
        W[0] = (uint64_t)i;
        W[1] = S->value_idx_node[i];
        if (t == 3)
        {
            memcpy(&W[N2_OFF_VALUE_MASK[3]], N->vmask, 64);
            write_prefix(&W[N2_OFF_VALUE_PREFIX[3]], N->vmask, 8);
            continue;
        }
        uint32_t fan = N2_FANOUT[t], nw = fan >> 6;
        uint64_t* cm = &W[N2_OFF_CHILD_MASK[t]];
        for (uint32_t n = 0; n < fan; n++)
            if (N->child[n] >= 0)
                cm[n >> 6] |= 1ull << (n & 63);
        write_prefix(&W[N2_OFF_CHILD_PREFIX[t]], cm, nw);
        uint64_t* ch = &W[N2_OFF_CHILDREN[t]];
        if (t == 0)
        {
            for (uint32_t e = 0; e < 2u * fan; e++)
                ch[e] = N2_END_KEY; /* GridBuild.cpp:178-183 */
        }
        uint32_t rank = 0;
        for (uint32_t n = 0; n < fan; n++)
            if (N->child[n] >= 0)
                ch[rank++] = addr[N->child[n]] - addr[i];
        if (t == 0)
        {
            /* keys, grid_build_blindmetadata.slang:104-201 */
            uint64_t* km = &W[N2_OFF_KEY_MASK_ROOT];
            memcpy(km, cm, 8 * nw);
            write_prefix(&W[N2_OFF_KEY_PREFIX_ROOT], km, nw);
            uint32_t child_count = rank, kidx = 0;
            for (uint32_t n = 0; n < fan; n++)
            {
                if (N->child[n] < 0)
                    continue;
                int32_t x = (int32_t)(((n >> 10) & 0x1F) << 12), y = (int32_t)(((n >> 5) & 0x1F) << 12),
                        z = (int32_t)((n & 0x1F) << 12);
                const int32_t half = 65536;
                x = x >= half ? x - 2 * half : x;
                y = y >= half ? y - 2 * half : y;
                z = z >= half ? z - 2 * half : z;
                uint64_t key = (uint64_t)((uint32_t)z >> 12) | ((uint64_t)((uint32_t)y >> 12) << 21) |
                               ((uint64_t)((uint32_t)x >> 12) << 42);
                ch[child_count + kidx++] = key;
            }
        }
    }
    free(addr);
}

void* ov_run(int64_t n, const float* means, const float* quats_wxyz, const float* scales, const float* colors,
             const float* opacities, float voxel_size, float cull_scale, int window_mode, int nthreads)
{
    if (nthreads < 1)
        nthreads = 1;
    ov_state_t* S = (ov_state_t*)calloc(1, sizeof(ov_state_t));
    S->G = n;
    S->vs = voxel_size;
    S->cull = cull_scale;
    S->skip_f64 = (window_mode & OV_MODE_NO_F64) != 0;
    S->smooth = (window_mode & OV_MODE_SMOOTH) != 0;
    window_mode &= OV_MODE_WINDOWS;
    S->prims = (prim_t*)malloc(sizeof(prim_t) * (n ? n : 1));
    int64_t valid = 0;
    uint64_t F = 0;
    for (int64_t g = 0; g < n; g++)
    {
        prim_setup(&S->prims[g], &means[3 * g], &quats_wxyz[4 * g], &scales[3 * g], opacities[g],
                   colors ? &colors[3 * g] : NULL, voxel_size);
        valid += S->prims[g].valid;
        F += S->prims[g].footprint;
        if (S->prims[g].valid)
        {
            for (int a = 0; a < 3; a++)
                if (S->prims[g].bmin[a] < -65536 || S->prims[g].bmax[a] > 65535)
                    S->counts[OV_ERROR] = 1; /* root key range, grid_build_blindmetadata.slang:182-192 */
            if (S->prims[g].footprint >= (1ull << 31))
                S->counts[OV_ERROR] = 2;
        }
    }
    S->counts[OV_G] = n;
    S->counts[OV_G_VALID] = valid;
    S->counts[OV_F] = (int64_t)F;
    if (S->counts[OV_ERROR])
        return S;

    int32_t origin0[3] = { 0, 0, 0 };
    new_node(S, 0, -1, 0, origin0);

    int64_t batch = window_mode ? OV_PRIM_BATCH : (n ? n : 1);
    uint64_t wsize = window_mode ? OV_WINDOW : ~0ull;
    int64_t windows = 0;
    int64_t* pidx = (int64_t*)malloc(sizeof(int64_t) * (batch ? batch : 1));
    uint64_t* off = (uint64_t*)malloc(sizeof(uint64_t) * (batch ? batch : 1));
    wjob_t* jobs = (wjob_t*)calloc((size_t)nthreads, sizeof(wjob_t));
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    for (int64_t b0 = 0; b0 < n; b0 += batch)
    {
        int64_t nb = (n - b0) < batch ? (n - b0) : batch;
        uint64_t fsum = 0;
        for (int64_t p = 0; p < nb; p++)
        {
            pidx[p] = b0 + p;
            off[p] = fsum;
            fsum += S->prims[b0 + p].footprint;
        }
        for (uint64_t w0 = 0, w1 = 0; w0 < fsum; w0 = w1)
        {
            w1 = (fsum - w0) < wsize ? fsum : w0 + wsize;
            uint64_t span = w1 - w0;
            for (int t = 0; t < nthreads; t++)
            {
                jobs[t].S = S;
                jobs[t].pidx = pidx;
                jobs[t].off = off;
                jobs[t].nprim = nb;
                jobs[t].f0 = w0 + span * (uint64_t)t / (uint64_t)nthreads;
                jobs[t].f1 = w0 + span * (uint64_t)(t + 1) / (uint64_t)nthreads;
                jobs[t].out_n = 0;
                pthread_create(&th[t], NULL, window_worker, &jobs[t]);
            }
            int64_t wcount = 0;
            for (int t = 0; t < nthreads; t++)
            {
                pthread_join(th[t], NULL);
                wcount += jobs[t].out_n;
            }
            int32_t* wijk = (int32_t*)malloc(sizeof(int32_t) * 3 * (wcount ? wcount : 1));
            int64_t pos = 0;
            if (S->P + wcount > S->Pcap)
            {
                S->Pcap = (S->P + wcount) * 2;
                S->keys = (uint64_t*)realloc(S->keys, sizeof(uint64_t) * S->Pcap);
                S->ids = (uint32_t*)realloc(S->ids, sizeof(uint32_t) * S->Pcap);
            }
            for (int t = 0; t < nthreads; t++)
            {
                for (int64_t i = 0; i < jobs[t].out_n; i++)
                {
                    const int32_t* c = &jobs[t].out_ijk[3 * i];
                    memcpy(&wijk[3 * pos], c, 12);
                    S->keys[S->P + pos] = ov_hier_key(c[0], c[1], c[2]);
                    S->ids[S->P + pos] = jobs[t].out_id[i];
                    pos++;
                }
            }
            S->P += wcount;
            insert_window(S, wijk, wcount);
            free(wijk);
            windows++;
        }
    }
    for (int t = 0; t < nthreads; t++)
    {
        free(jobs[t].out_ijk);
        free(jobs[t].out_id);
    }
    free(jobs);
    free(pidx);
    free(off);

    radix_sort_pairs(S->keys, S->ids, S->P, 51);

    /* voxel runs in key order */
    int64_t V = 0;
    for (int64_t p = 0; p < S->P; p++)
        if (p == 0 || S->keys[p] != S->keys[p - 1])
            V++;
    S->V = V;
    int64_t* vstart = (int64_t*)malloc(sizeof(int64_t) * (V + 1));
    S->vox_ijk = (int32_t*)malloc(sizeof(int32_t) * 3 * (V ? V : 1));
    S->vox_vidx = (uint64_t*)malloc(sizeof(uint64_t) * (V ? V : 1));

    serialize(S);

    int64_t vi = 0;
    for (int64_t p = 0; p < S->P; p++)
    {
        if (p == 0 || S->keys[p] != S->keys[p - 1])
            vstart[vi++] = p;
    }
    vstart[V] = S->P;
    /* ijk back from a pair: recompute from the Gaussian's emission is not
     * needed; decode the hierarchical key through the tree instead */
    for (int64_t v = 0; v < V; v++)
    {
        uint64_t key = S->keys[vstart[v]];
        uint32_t rn = (uint32_t)(key >> 36) & 0x7FFF, un = (uint32_t)(key >> 21) & 0x7FFF,
                 ln = (uint32_t)(key >> 9) & 0xFFF, vn = (uint32_t)key & 0x1FF;
        int32_t up = S->nodes[0].child[rn];
        int32_t lo = S->nodes[up].child[un];
        int32_t lf = S->nodes[lo].child[ln];
        node_t* L = &S->nodes[lf];
        int32_t* c = &S->vox_ijk[3 * v];
        c[0] = L->origin[0] + (int32_t)((vn >> 6) & 7);
        c[1] = L->origin[1] + (int32_t)((vn >> 3) & 7);
        c[2] = L->origin[2] + (int32_t)(vn & 7);
        uint64_t below = 0;
        for (uint32_t w = 0; w < (vn >> 6); w++)
            below += (uint64_t)popc64(L->vmask[w]);
        below += (uint64_t)popc64(L->vmask[vn >> 6] & ((1ull << (vn & 63)) - 1ull));
        S->vox_vidx[v] = S->value_idx_node[lf] + below;
    }

    int64_t value_count = 2 + V;
    S->rgba = (uint32_t*)calloc((size_t)value_count, sizeof(uint32_t));
    S->dens = (float*)calloc((size_t)value_count, sizeof(float));
    S->col = (float*)calloc((size_t)value_count * 3, sizeof(float));
    S->dens64 = (double*)calloc((size_t)value_count, sizeof(double));
    S->col64 = (double*)calloc((size_t)value_count * 3, sizeof(double));
    vjob_t* vj = (vjob_t*)malloc(sizeof(vjob_t) * nthreads);
    for (int t = 0; t < nthreads; t++)
    {
        vj[t].S = S;
        vj[t].vstart = vstart;
        vj[t].v0 = V * t / nthreads;
        vj[t].v1 = V * (t + 1) / nthreads;
        pthread_create(&th[t], NULL, values_worker, &vj[t]);
    }
    for (int t = 0; t < nthreads; t++)
        pthread_join(th[t], NULL);
    free(vj);
    free(th);
    free(vstart);

    /* bbox of active voxels (grid_build_compute_bbox.slang) */
    for (int a = 0; a < 3; a++)
    {
        S->bbox[a] = 0x7FFFFFFF;
        S->bbox[3 + a] = (int32_t)0x80000000;
    }
    for (int64_t v = 0; v < V; v++)
        for (int a = 0; a < 3; a++)
        {
            int32_t c = S->vox_ijk[3 * v + a];
            S->bbox[a] = c < S->bbox[a] ? c : S->bbox[a];
            S->bbox[3 + a] = c > S->bbox[3 + a] ? c : S->bbox[3 + a];
        }

    int64_t cnt[4] = { 0, 0, 0, 0 };
    for (int64_t i = 0; i < S->nn; i++)
        cnt[S->nodes[i].type]++;
    S->counts[OV_P] = S->P;
    S->counts[OV_V] = V;
    S->counts[OV_UPPER] = cnt[1];
    S->counts[OV_LOWER] = cnt[2];
    S->counts[OV_LEAF] = cnt[3];
    S->counts[OV_VALUE_COUNT] = value_count;
    S->counts[OV_NODE2_BYTES] = S->node2_bytes;
    S->counts[OV_WINDOWS] = windows;
    return S;
}

void ov_destroy(void* h)
{
    ov_state_t* S = (ov_state_t*)h;
    if (!S)
        return;
    for (int64_t i = 0; i < S->nn; i++)
    {
        free(S->nodes[i].child);
        free(S->nodes[i].vmask);
    }
    free(S->nodes);
    free(S->prims);
    free(S->keys);
    free(S->ids);
    free(S->pijk);
    free(S->node2);
    free(S->value_idx_node);
    free(S->vox_ijk);
    free(S->vox_vidx);
    free(S->rgba);
    free(S->dens);
    free(S->col);
    free(S->dens64);
    free(S->col64);
    free(S);
}

void ov_counts(void* h, int64_t* out)
{
    ov_state_t* S = (ov_state_t*)h;
    memcpy(out, S->counts, sizeof(S->counts));
}

int64_t ov_node2_bytes(void* h, uint8_t* dst)
{
    ov_state_t* S = (ov_state_t*)h;
    if (dst && S->node2)
        memcpy(dst, S->node2, (size_t)S->node2_bytes);
    return S->node2_bytes;
}

void ov_pairs(void* h, uint64_t* keys, uint32_t* ids)
{
    ov_state_t* S = (ov_state_t*)h;
    memcpy(keys, S->keys, sizeof(uint64_t) * S->P);
    memcpy(ids, S->ids, sizeof(uint32_t) * S->P);
}

void ov_values(void* h, uint32_t* rgba8, float* density, float* color, double* density64, double* color64)
{
    ov_state_t* S = (ov_state_t*)h;
    int64_t vc = 2 + S->V;
    if (rgba8)
        memcpy(rgba8, S->rgba, sizeof(uint32_t) * vc);
    if (density)
        memcpy(density, S->dens, sizeof(float) * vc);
    if (color)
        memcpy(color, S->col, sizeof(float) * 3 * vc);
    if (density64)
        memcpy(density64, S->dens64, sizeof(double) * vc);
    if (color64)
        memcpy(color64, S->col64, sizeof(double) * 3 * vc);
}

void ov_voxels(void* h, int32_t* ijk, uint64_t* value_idx)
{
    ov_state_t* S = (ov_state_t*)h;
    memcpy(ijk, S->vox_ijk, sizeof(int32_t) * 3 * S->V);
    memcpy(value_idx, S->vox_vidx, sizeof(uint64_t) * S->V);
}

void ov_bbox(void* h, int32_t* out6)
{
    ov_state_t* S = (ov_state_t*)h;
    memcpy(out6, S->bbox, sizeof(S->bbox));
}

void ov_node_table(void* h, int32_t* type, int32_t* parent, int32_t* n_in_parent, int32_t* origin3)
{
    ov_state_t* S = (ov_state_t*)h;
    for (int64_t i = 0; i < S->nn; i++)
    {
        type[i] = S->nodes[i].type;
        parent[i] = S->nodes[i].parent;
        n_in_parent[i] = (int32_t)S->nodes[i].n;
        memcpy(&origin3[3 * i], S->nodes[i].origin, 12);
    }
}

/* ------------------------------------------------------------------------ */
/* FP64 adjoint of the smooth channels and the per-Gaussian FP64 loss used  */
/* for finite differences.                                                   */
/* ------------------------------------------------------------------------ */
int64_t ov_lookup(void* h, int32_t i, int32_t j, int32_t k)
{
    ov_state_t* S = (ov_state_t*)h;
    if (!S || S->nn == 0 || i < -65536 || i > 65535 || j < -65536 || j > 65535 || k < -65536 || k > 65535)
        return -1;
    uint64_t key = ov_hier_key(i, j, k);
    uint32_t rn = (uint32_t)(key >> 36) & 0x7FFF, un = (uint32_t)(key >> 21) & 0x7FFF,
             ln = (uint32_t)(key >> 9) & 0xFFF, vn = (uint32_t)key & 0x1FF;
    int32_t up = S->nodes[0].child[rn];
    if (up < 0)
        return -1;
    int32_t lo = S->nodes[up].child[un];
    if (lo < 0)
        return -1;
    int32_t lf = S->nodes[lo].child[ln];
    if (lf < 0)
        return -1;
    const node_t* L = &S->nodes[lf];
    if (!((L->vmask[vn >> 6] >> (vn & 63)) & 1ull))
        return -1;
    uint64_t below = 0;
    for (uint32_t w = 0; w < (vn >> 6); w++)
        below += (uint64_t)popc64(L->vmask[w]);
    below += (uint64_t)popc64(L->vmask[vn >> 6] & ((1ull << (vn & 63)) - 1ull));
    return (int64_t)(S->value_idx_node[lf] + below);
}

/* chain the per-Gaussian sums to the caller's parameters */
static void g64_finalize(const g64_t* g, const double U[3], const double W[3], const double Q[3][3], double dop,
                         const double drgb[3], double* d_mean, double* d_quat_wxyz, double* d_scale, double* d_opac,
                         double* d_col)
{
    for (int a = 0; a < 3; a++)
        d_mean[a] = -(g->R[a][0] * U[0] + g->R[a][1] * U[1] + g->R[a][2] * U[2]);
    for (int r = 0; r < 3; r++)
    {
        double ds = g->clamped[r] ? 0.0 : -W[r] / g->s[r];
        d_scale[r] = g->raw ? ds * g->s_act[r] : ds;
    }
    /* u_r = sum_a R[a][r] d_a, so dL/dR[a][r] = Q[r][a] */
    double G[3][3];
    for (int a = 0; a < 3; a++)
        for (int r = 0; r < 3; r++)
            G[a][r] = Q[r][a];
    double x = g->q[0], y = g->q[1], z = g->q[2], w = g->q[3];
    double dx = 2 * y * (G[0][1] + G[1][0]) + 2 * z * (G[0][2] + G[2][0]) + 2 * w * (G[2][1] - G[1][2]) -
                4 * x * (G[1][1] + G[2][2]);
    double dy = 2 * x * (G[0][1] + G[1][0]) + 2 * w * (G[0][2] - G[2][0]) + 2 * z * (G[1][2] + G[2][1]) -
                4 * y * (G[0][0] + G[2][2]);
    double dz = 2 * w * (G[1][0] - G[0][1]) + 2 * x * (G[0][2] + G[2][0]) + 2 * y * (G[1][2] + G[2][1]) -
                4 * z * (G[0][0] + G[1][1]);
    double dw = 2 * z * (G[1][0] - G[0][1]) + 2 * y * (G[0][2] - G[2][0]) + 2 * x * (G[2][1] - G[1][2]);
    if (g->raw)
    {
        /* q_n = q / |q| */
        double dot = x * dx + y * dy + z * dz + w * dw;
        dx = (dx - x * dot) / g->qnorm;
        dy = (dy - y * dot) / g->qnorm;
        dz = (dz - z * dot) / g->qnorm;
        dw = (dw - w * dot) / g->qnorm;
    }
    d_quat_wxyz[0] = dw;
    d_quat_wxyz[1] = dx;
    d_quat_wxyz[2] = dy;
    d_quat_wxyz[3] = dz;
    *d_opac = g->raw ? dop * g->op * (1.0 - g->op) : dop;
    for (int c = 0; c < 3; c++)
        d_col[c] = g->raw ? OV_SH_C0 * drgb[c] : drgb[c];
}

int ov_smooth_grad64(void* h, const float* means, const float* quats_wxyz, const float* scales, const float* opacities,
                     const float* colors, int raw, const double* grad_density, const double* grad_color,
                     double* d_means, double* d_quats, double* d_scales, double* d_opacities, double* d_colors)
{
    ov_state_t* S = (ov_state_t*)h;
    if (!S || S->counts[OV_ERROR])
        return -1;
    const int64_t G = S->G;
    double* acc = (double*)calloc((size_t)(G ? G : 1) * 19, sizeof(double));
    const double vs = (double)S->vs;
    int64_t v = -1;
    for (int64_t p = 0; p < S->P; p++)
    {
        if (p == 0 || S->keys[p] != S->keys[p - 1])
            v++;
        const uint32_t gid = S->ids[p];
        const int32_t* ijk = &S->vox_ijk[3 * v];
        const uint64_t vi = S->vox_vidx[v];
        double mean[3], q[4], sc[3], col[3];
        for (int a = 0; a < 3; a++)
        {
            mean[a] = means[3 * gid + a];
            sc[a] = scales[3 * gid + a];
            col[a] = colors[3 * gid + a];
        }
        for (int a = 0; a < 4; a++)
            q[a] = quats_wxyz[4 * gid + a];
        g64_t g;
        g64_setup(&g, mean, q, sc, (double)opacities[gid], col, raw, vs);
        smooth_terms_t t;
        double K = smooth64(&g, vs, ijk, &t);
        if (!(t.e > (double)OV_SMOOTH_TAU))
            continue;
        double* A = &acc[19 * (int64_t)gid];
        const double gd = grad_density ? grad_density[vi] : 0.0;
        double gc[3] = { 0.0, 0.0, 0.0 };
        if (grad_color)
            for (int c = 0; c < 3; c++)
                gc[c] = grad_color[3 * vi + c];
        const double GK = gd + gc[0] * g.rgb[0] + gc[1] * g.rgb[1] + gc[2] * g.rgb[2];
        A[0] += GK * t.E; /* dop */
        for (int r = 0; r < 3; r++)
        {
            double dz = -GK * t.e * t.z[r];
            double du = dz / g.s[r];
            A[1 + r] += du;           /* U */
            A[4 + r] += dz * t.z[r];  /* W */
            for (int a = 0; a < 3; a++)
                A[7 + 3 * r + a] += du * t.d[a]; /* Q[r][a] */
        }
        for (int c = 0; c < 3; c++)
            A[16 + c] += K * gc[c];
    }
    for (int64_t gid = 0; gid < G; gid++)
    {
        const double* A = &acc[19 * gid];
        double mean[3], q[4], sc[3], col[3];
        for (int a = 0; a < 3; a++)
        {
            mean[a] = means[3 * gid + a];
            sc[a] = scales[3 * gid + a];
            col[a] = colors[3 * gid + a];
        }
        for (int a = 0; a < 4; a++)
            q[a] = quats_wxyz[4 * gid + a];
        g64_t g;
        g64_setup(&g, mean, q, sc, (double)opacities[gid], col, raw, vs);
        double Q[3][3];
        for (int r = 0; r < 3; r++)
            for (int a = 0; a < 3; a++)
                Q[r][a] = A[7 + 3 * r + a];
        g64_finalize(&g, &A[1], &A[4], (const double(*)[3])Q, A[0], &A[16], &d_means[3 * gid], &d_quats[4 * gid],
                     &d_scales[3 * gid], &d_opacities[gid], &d_colors[3 * gid]);
    }
    free(acc);
    return 0;
}

/* L_g(theta) = sum over voxels of grad_density * K + grad_color . K rgb for one
 * Gaussian given in FP64 (theta = mean[3], quat wxyz[4], scale[3], opacity,
 * colour[3]); every voxel of the kernel's support box is visited, so the
 * value does not depend on the pair set. */
double ov_smooth_loss64(void* h, const double* theta, int raw, const double* grad_density, const double* grad_color)
{
    ov_state_t* S = (ov_state_t*)h;
    const double vs = (double)S->vs;
    g64_t g;
    g64_setup(&g, &theta[0], &theta[3], &theta[7], theta[10], &theta[11], raw, vs);
    if (!(g.op > (double)OV_SMOOTH_TAU))
        return 0.0;
    const double ls2 = 2.0 * log(g.op / (double)OV_SMOOTH_TAU);
    int32_t lo[3], hi[3];
    for (int a = 0; a < 3; a++)
    {
        double ext = 0.0;
        for (int r = 0; r < 3; r++)
            ext += g.R[a][r] * g.R[a][r] * g.s[r] * g.s[r];
        ext = sqrt(ls2 * ext);
        lo[a] = (int32_t)floor((g.mu[a] - ext) / vs) - 1;
        hi[a] = (int32_t)floor((g.mu[a] + ext) / vs) + 1;
    }
    double L = 0.0;
    int32_t ijk[3];
    for (ijk[0] = lo[0]; ijk[0] <= hi[0]; ijk[0]++)
        for (ijk[1] = lo[1]; ijk[1] <= hi[1]; ijk[1]++)
            for (ijk[2] = lo[2]; ijk[2] <= hi[2]; ijk[2]++)
            {
                double K = smooth64(&g, vs, ijk, NULL);
                if (K == 0.0)
                    continue;
                int64_t vi = ov_lookup(h, ijk[0], ijk[1], ijk[2]);
                if (vi < 0)
                    continue;
                double t = grad_density ? grad_density[vi] : 0.0;
                if (grad_color)
                    t += grad_color[3 * vi] * g.rgb[0] + grad_color[3 * vi + 1] * g.rgb[1] +
                         grad_color[3 * vi + 2] * g.rgb[2];
                L += K * t;
            }
    return L;
}

/* The float channels' exp / log / pow (vox_expf_ch, vox_logf_ch, vox_powf_ch)
 * on arrays, for their accuracy test against double precision. */
void ov_chan_math(int64_t n, const float* x, const float* b, const float* e, float* exp_out, float* log_out,
                  float* pow_out)
{
    for (int64_t i = 0; i < n; i++)
    {
        exp_out[i] = vox_expf_ch(x[i]);
        log_out[i] = vox_logf_ch(b[i]);
        pow_out[i] = vox_powf_ch(b[i], e[i]);
    }
}
