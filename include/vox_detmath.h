/*
 * vox_detmath.h - deterministic transcendental functions for the Gaussian
 * voxelization path.
 *
 * Every function here is built only from correctly rounded IEEE-754
 * operations (+, -, *, /, sqrt, the fused multiply-add fma, floor, integer bit
 * manipulation) evaluated one at a time with round-to-nearest; no compiler
 * contraction.  The same source therefore produces bit-identical results on
 * the host (gcc/g++ with -ffp-contract=off, fma() from the C library) and on
 * the device (nvcc, where the VOX_F* / VOX_D* macros map to the __f*_rn /
 * __d*_rn / __fma*_rn intrinsics that are never contracted).
 *
 * Two families:
 *   vox_exp_d / vox_log_d  double precision, ~1e-16 relative; rounded to
 *                          float they give the correctly rounded float result
 *                          in all but double-rounding tie cases, which also
 *                          makes them monotone.  Used for the host-side
 *                          preprocessing the reference runs with the C
 *                          library's expf (raster/RasterUtils.cpp:81-117) and
 *                          for the exp inside the 64-sample alpha maximum
 *                          (raster/shaders/gaussian_frag_color.slang:190-197).
 *   vox_logf / vox_powf / vox_expf
 *                          single precision, <= 3 ulp; used for the cutoff
 *                          radius sqrt(2 log(op / 0.01)) and the opacity
 *                          transform pow(1 - a, 1 / s) (gaussian_prim.slang:65,
 *                          gaussian_frag_color.slang:199-202), whose log/pow the
 *                          reference leaves to the Vulkan driver.
 *
 * Method (standard, from the mathematics):
 *   exp(x) = 2^k * exp(r), k = round(x / ln2), r = x - k ln2 (ln2 split in a
 *            float-exact high part and a low part), exp(r) by its Taylor series
 *            (Horner form with fused multiply-adds).
 *   log(x) = e ln2 + 2 atanh((m - 1) / (m + 1)), x = m 2^e, m in [sqrt(1/2), sqrt(2)),
 *            atanh by its odd power series.
 */
#ifndef VOX_DETMATH_H
#define VOX_DETMATH_H

#include <stdint.h>

#if defined(__CUDACC__)
#define VOX_HD static __host__ __device__ __forceinline__
#else
#define VOX_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define VOX_FADD(a, b) __fadd_rn((a), (b))
#define VOX_FSUB(a, b) __fsub_rn((a), (b))
#define VOX_FMUL(a, b) __fmul_rn((a), (b))
#define VOX_FDIV(a, b) __fdiv_rn((a), (b))
#define VOX_FSQRT(a) __fsqrt_rn((a))
#define VOX_DADD(a, b) __dadd_rn((a), (b))
#define VOX_DSUB(a, b) __dsub_rn((a), (b))
#define VOX_DMUL(a, b) __dmul_rn((a), (b))
#define VOX_DDIV(a, b) __ddiv_rn((a), (b))
#define VOX_DSQRT(a) __dsqrt_rn((a))
#define VOX_DFMA(a, b, c) __fma_rn((a), (b), (c))
#define VOX_FFMA(a, b, c) __fmaf_rn((a), (b), (c))
#define VOX_FLOORF(a) floorf((a))
#define VOX_FLOORD(a) floor((a))
#else
#include <math.h>
#include <string.h>
#define VOX_FADD(a, b) ((float)((float)(a) + (float)(b)))
#define VOX_FSUB(a, b) ((float)((float)(a) - (float)(b)))
#define VOX_FMUL(a, b) ((float)((float)(a) * (float)(b)))
#define VOX_FDIV(a, b) ((float)((float)(a) / (float)(b)))
#define VOX_FSQRT(a) sqrtf((a))
#define VOX_DADD(a, b) ((double)(a) + (double)(b))
#define VOX_DSUB(a, b) ((double)(a) - (double)(b))
#define VOX_DMUL(a, b) ((double)(a) * (double)(b))
#define VOX_DDIV(a, b) ((double)(a) / (double)(b))
#define VOX_DSQRT(a) sqrt((a))
/* IEEE fused multiply-add: correctly rounded on host and device alike */
#define VOX_DFMA(a, b, c) fma((a), (b), (c))
#define VOX_FFMA(a, b, c) fmaf((a), (b), (c))
#define VOX_FLOORF(a) floorf((a))
#define VOX_FLOORD(a) floor((a))
#endif

VOX_HD uint64_t vox_d2u(double x)
{
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
#endif
}
VOX_HD double vox_u2d(uint64_t u)
{
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, 8);
    return x;
#endif
}
VOX_HD uint32_t vox_f2u(float x)
{
#if defined(__CUDA_ARCH__)
    return (uint32_t)__float_as_uint(x);
#else
    uint32_t u;
    memcpy(&u, &x, 4);
    return u;
#endif
}
VOX_HD float vox_u2f(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float x;
    memcpy(&x, &u, 4);
    return x;
#endif
}

/* ln 2 = 0.693147180559945309417232121458...; the high part is ln 2 rounded to
 * float (24 significant bits) so k * hi is exact for |k| < 2^29. */
#define VOX_LN2_D 0.6931471805599453094
#define VOX_INV_LN2_D 1.4426950408889634074
#define VOX_LN2_HI_D 0.693147182464599609375 /* (float)ln2 */
#define VOX_SQRT2_D 1.4142135623730950488

/* 2^k for k in [-1022, 1023] as an exact double */
VOX_HD double vox_pow2_d(int k)
{
    return vox_u2d((uint64_t)(k + 1023) << 52);
}

/* exp(x) in double. Finite results for x in [-708, 709]; 0 / +inf outside. */
VOX_HD double vox_exp_d(double x)
{
    if (!(x == x))
        return x;
    if (x > 709.0)
        return vox_u2d(0x7ff0000000000000ull);
    if (x < -708.0)
        return 0.0;
    double kd = VOX_FLOORD(VOX_DADD(VOX_DMUL(x, VOX_INV_LN2_D), 0.5));
    const double ln2_lo = VOX_LN2_D - VOX_LN2_HI_D; /* exact: both within a factor 2 */
    double r = VOX_DSUB(VOX_DSUB(x, VOX_DMUL(kd, VOX_LN2_HI_D)), VOX_DMUL(kd, ln2_lo));
    /* sum_{n=0}^{13} r^n / n!, Horner with fused multiply-adds; |r| <= 0.3466,
     * truncation r^14 / 14! < 5e-18 (below double rounding) */
    double p = 1.0 / 6227020800.0;
    p = VOX_DFMA(p, r, 1.0 / 479001600.0);
    p = VOX_DFMA(p, r, 1.0 / 39916800.0);
    p = VOX_DFMA(p, r, 1.0 / 3628800.0);
    p = VOX_DFMA(p, r, 1.0 / 362880.0);
    p = VOX_DFMA(p, r, 1.0 / 40320.0);
    p = VOX_DFMA(p, r, 1.0 / 5040.0);
    p = VOX_DFMA(p, r, 1.0 / 720.0);
    p = VOX_DFMA(p, r, 1.0 / 120.0);
    p = VOX_DFMA(p, r, 1.0 / 24.0);
    p = VOX_DFMA(p, r, 1.0 / 6.0);
    p = VOX_DFMA(p, r, 0.5);
    p = VOX_DFMA(p, r, 1.0);
    p = VOX_DFMA(p, r, 1.0);
    int k = (int)kd;
    if (k < -1000)
    {
        /* two exact scalings keep the intermediate normal */
        return VOX_DMUL(VOX_DMUL(p, vox_pow2_d(k + 600)), vox_pow2_d(-600));
    }
    return VOX_DMUL(p, vox_pow2_d(k));
}

/* natural log in double for finite x > 0 (x <= 0 -> -inf / NaN). */
VOX_HD double vox_log_d(double x)
{
    if (!(x > 0.0))
        return (x == 0.0) ? -vox_u2d(0x7ff0000000000000ull) : vox_u2d(0x7ff8000000000000ull);
    if (x == vox_u2d(0x7ff0000000000000ull))
        return x;
    int e = 0;
    if (x < 2.2250738585072014e-308)
    {
        x = VOX_DMUL(x, 18014398509481984.0); /* 2^54, exact */
        e = -54;
    }
    uint64_t bits = vox_d2u(x);
    e += (int)((bits >> 52) & 0x7ff) - 1023;
    double m = vox_u2d((bits & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    if (m > VOX_SQRT2_D)
    {
        m = VOX_DMUL(m, 0.5);
        e += 1;
    }
    double t = VOX_DDIV(VOX_DSUB(m, 1.0), VOX_DADD(m, 1.0));
    double t2 = VOX_DMUL(t, t);
    /* atanh(t)/t = sum t^(2n)/(2n+1), n = 0..11; |t| <= 0.1716, truncation < 1e-19 */
    double p = 1.0 / 23.0;
    p = VOX_DFMA(p, t2, 1.0 / 21.0);
    p = VOX_DFMA(p, t2, 1.0 / 19.0);
    p = VOX_DFMA(p, t2, 1.0 / 17.0);
    p = VOX_DFMA(p, t2, 1.0 / 15.0);
    p = VOX_DFMA(p, t2, 1.0 / 13.0);
    p = VOX_DFMA(p, t2, 1.0 / 11.0);
    p = VOX_DFMA(p, t2, 1.0 / 9.0);
    p = VOX_DFMA(p, t2, 1.0 / 7.0);
    p = VOX_DFMA(p, t2, 1.0 / 5.0);
    p = VOX_DFMA(p, t2, 1.0 / 3.0);
    p = VOX_DFMA(p, t2, 1.0);
    double logm = VOX_DMUL(VOX_DMUL(2.0, t), p);
    double ed = (double)e;
    const double ln2_lo = VOX_LN2_D - VOX_LN2_HI_D;
    return VOX_DADD(VOX_DMUL(ed, VOX_LN2_HI_D), VOX_DADD(VOX_DMUL(ed, ln2_lo), logm));
}

/* float-valued, (almost always) correctly rounded exp/log through double */
VOX_HD float vox_expf_cr(float x)
{
    return (float)vox_exp_d((double)x);
}
VOX_HD float vox_logf_cr(float x)
{
    return (float)vox_log_d((double)x);
}

/* ------------------------- single precision family ------------------------- */

#define VOX_LN2_HI_F 0.693145751953125f /* 0x1.62e4p-1: 17 significant bits */
#define VOX_LN2_LO_F 1.4286068203094172321e-06f
#define VOX_INV_LN2_F 1.44269504088896341f
#define VOX_SQRT2_F 1.41421356237309505f

/* exp(x) in float, |rel err| <= ~3 ulp for x in [-87, 88]. */
VOX_HD float vox_expf(float x)
{
    if (!(x == x))
        return x;
    if (x > 88.7f)
        return vox_u2f(0x7f800000u);
    if (x < -87.3f)
        return 0.0f;
    float kf = VOX_FLOORF(VOX_FADD(VOX_FMUL(x, VOX_INV_LN2_F), 0.5f));
    float r = VOX_FSUB(VOX_FSUB(x, VOX_FMUL(kf, VOX_LN2_HI_F)), VOX_FMUL(kf, VOX_LN2_LO_F));
    /* sum_{n=0}^{8} r^n/n!, |r| <= 0.347 */
    float p = 1.0f / 40320.0f;
    p = VOX_FFMA(p, r, 1.0f / 5040.0f);
    p = VOX_FFMA(p, r, 1.0f / 720.0f);
    p = VOX_FFMA(p, r, 1.0f / 120.0f);
    p = VOX_FFMA(p, r, 1.0f / 24.0f);
    p = VOX_FFMA(p, r, 1.0f / 6.0f);
    p = VOX_FFMA(p, r, 0.5f);
    p = VOX_FFMA(p, r, 1.0f);
    p = VOX_FFMA(p, r, 1.0f);
    int k = (int)kf;
    /* k in [-126, 128]; split the scaling so each factor is a normal float */
    int k1 = k / 2;
    int k2 = k - k1;
    float s1 = vox_u2f((uint32_t)(k1 + 127) << 23);
    float s2 = vox_u2f((uint32_t)(k2 + 127) << 23);
    return VOX_FMUL(VOX_FMUL(p, s1), s2);
}

/* natural log in float for finite x > 0, |abs err| <= ~2 ulp of the result scale. */
VOX_HD float vox_logf(float x)
{
    if (!(x > 0.0f))
        return (x == 0.0f) ? -vox_u2f(0x7f800000u) : vox_u2f(0x7fc00000u);
    if (x == vox_u2f(0x7f800000u))
        return x;
    int e = 0;
    if (x < 1.17549435e-38f)
    {
        x = VOX_FMUL(x, 16777216.0f); /* 2^24, exact */
        e = -24;
    }
    uint32_t bits = vox_f2u(x);
    e += (int)((bits >> 23) & 0xff) - 127;
    float m = vox_u2f((bits & 0x007fffffu) | 0x3f800000u);
    if (m > VOX_SQRT2_F)
    {
        m = VOX_FMUL(m, 0.5f);
        e += 1;
    }
    float t = VOX_FDIV(VOX_FSUB(m, 1.0f), VOX_FADD(m, 1.0f));
    float t2 = VOX_FMUL(t, t);
    float p = 1.0f / 11.0f;
    p = VOX_FFMA(p, t2, 1.0f / 9.0f);
    p = VOX_FFMA(p, t2, 1.0f / 7.0f);
    p = VOX_FFMA(p, t2, 1.0f / 5.0f);
    p = VOX_FFMA(p, t2, 1.0f / 3.0f);
    p = VOX_FFMA(p, t2, 1.0f);
    float logm = VOX_FMUL(VOX_FMUL(2.0f, t), p);
    float ef = (float)e;
    return VOX_FADD(VOX_FMUL(ef, VOX_LN2_HI_F), VOX_FADD(VOX_FMUL(ef, VOX_LN2_LO_F), logm));
}

/* b^e for b >= 0, e > 0: exp(e * log(b)); 0^e = 0. */
VOX_HD float vox_powf(float b, float e)
{
    if (b == 0.0f)
        return 0.0f;
    if (b == 1.0f)
        return 1.0f;
    return vox_expf(VOX_FMUL(e, vox_logf(b)));
}

/* The float density / colour channels' exp and pow: the same functions to
 * about 2 ulp at a lower cost (their domain is x <= 0 and b in [0, 1]; the
 * RGBA8 path keeps vox_expf_cr / vox_powf, which the reference's outputs pin).
 * Coefficients: polynomials fitted here for relative error (iteratively
 * reweighted least squares on Chebyshev nodes), rounded to float. */

/* exp(x) for finite x <= 0 (0 below -87.3): x = k ln2 + r, |r| <= ln2 / 2,
 * e^r by a degree-6 polynomial (relative error 2.1e-9 before rounding), one
 * exact scaling by 2^k (k >= -126). */
VOX_HD float vox_expf_ch(float x)
{
    const float xc = x > -87.3f ? x : -87.3f;
    const float kf = VOX_FLOORF(VOX_FADD(VOX_FMUL(xc, VOX_INV_LN2_F), 0.5f));
    const float r = VOX_FSUB(VOX_FSUB(xc, VOX_FMUL(kf, VOX_LN2_HI_F)), VOX_FMUL(kf, VOX_LN2_LO_F));
    float p = 0.001384272240102291f;
    p = VOX_FFMA(p, r, 0.008374955505132675f);
    p = VOX_FFMA(p, r, 0.041668057441711426f);
    p = VOX_FFMA(p, r, 0.1666642129421234f);
    p = VOX_FFMA(p, r, 0.4999999403953552f);
    p = VOX_FFMA(p, r, 1.0f);
    p = VOX_FFMA(p, r, 1.0f);
    const float y = VOX_FMUL(p, vox_u2f((uint32_t)((int)kf + 127) << 23));
    return x < -87.3f ? 0.0f : y;
}

/* log(b) for normal b in (0, 1]: b = 2^e m with m in [sqrt(1/2), sqrt(2)),
 * log m = f Q(f) with f = m - 1 (exact) and Q of degree 9 (relative error
 * 4.2e-9 before rounding): no division. */
VOX_HD float vox_logf_ch(float b)
{
    const uint32_t bits = vox_f2u(b);
    int ex = (int)((bits >> 23) & 0xff) - 127;
    float m = vox_u2f((bits & 0x007fffffu) | 0x3f800000u);
    const int up = m > VOX_SQRT2_F;
    m = up ? VOX_FMUL(m, 0.5f) : m;
    ex += up;
    const float f = VOX_FSUB(m, 1.0f);
    float q = -0.07633855938911438f;
    q = VOX_FFMA(q, f, 0.1292378008365631f);
    q = VOX_FFMA(q, f, -0.1324782371520996f);
    q = VOX_FFMA(q, f, 0.1417929232120514f);
    q = VOX_FFMA(q, f, -0.16608239710330963f);
    q = VOX_FFMA(q, f, 0.2000207006931305f);
    q = VOX_FFMA(q, f, -0.2500161826610565f);
    q = VOX_FFMA(q, f, 0.33333325386047363f);
    q = VOX_FFMA(q, f, -0.49999988079071045f);
    q = VOX_FFMA(q, f, 1.0f);
    const float logm = VOX_FMUL(f, q);
    const float ef = (float)ex;
    return VOX_FADD(VOX_FMUL(ef, VOX_LN2_HI_F), VOX_FADD(VOX_FMUL(ef, VOX_LN2_LO_F), logm));
}

/* b^e for b in [0, 1] and finite e > 0: exp(e log b); 0^e = 0, 1^e = 1 */
VOX_HD float vox_powf_ch(float b, float e)
{
    const float y = vox_expf_ch(VOX_FMUL(e, vox_logf_ch(b > 0.0f ? b : 1.0f)));
    return b == 0.0f ? 0.0f : (b == 1.0f ? 1.0f : y);
}

#endif /* VOX_DETMATH_H */
