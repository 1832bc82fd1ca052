// vox_backward.cu - adjoint of the differentiable channels.
//
// Forward (VOX_FLAG_DIFFERENTIABLE, smooth_kernel in vox_device.cuh), per pair
// (Gaussian g, voxel v) of the reference's pair set
// (gaussian_frag_alloc.slang:84-162):
//   d = x_v - mu,  u = R^T d,  z_r = u_r / s_r,  E = exp(-|z|^2 / 2),
//   e = op E,  K = max(e - 0.01, 0),
//   density[v] += K,  colour[v] += K rgb.
// Given dL/d density and dL/d colour (value-indexed), with
// GK = dL/d density[v] + dL/d colour[v] . rgb, a pair with e > 0.01 adds
//   dL/d op  += GK E
//   dL/d z_r  = -GK e z_r,   dL/d u_r = dL/d z_r / s_r
//   U_r += dL/d u_r,  W_r += dL/d z_r z_r,  Q[r][a] += dL/d u_r d_a
//   dL/d rgb += K dL/d colour[v]
// and per Gaussian dL/d mu = -R U, dL/d s_r = -W_r / s_r, dL/d R[a][r] = Q[r][a],
// chained through the rotation of gaussian_prim.slang:83-90, the quaternion
// normalisation, exp, the sigmoid and SH0 of raster/RasterUtils.cpp:59-117.
//
// k_bwd_pairs walks the pair list in emission order, which is sorted by
// Gaussian id, so the pairs of one Gaussian are contiguous: each warp owns a
// contiguous range, keeps the 19 per-Gaussian sums in registers, and reduces
// them across the warp once per Gaussian segment.  A segment that lies wholly
// inside one warp's range is stored; one cut by a range boundary is added with
// FP64 atomics.  Nothing is stored per pair.
#include <cstdio>
#include <cuda_runtime.h>

#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

constexpr int BWD_BLOCK = 256;
constexpr int BWD_RANGE = 1024; // pairs per warp
constexpr unsigned FULL = 0xffffffffu;

template <class K>
__device__ __forceinline__ void pair_adjoint(const BwdParams& B, uint64_t key, uint32_t gid, float (&c)[BWD_NACC])
{
    const uint32_t lr = (uint32_t)(key >> 21), ln = (uint32_t)(key >> 9) & 4095u, vn = (uint32_t)key & 511u;
    const uint32_t lo = B.rank_to_lower[lr];
    const uint32_t l = B.leaf_slot[(uint64_t)lo * 4096u + ln];
    const uint64_t* m = B.leaf_mask + 8ull * l;
    uint64_t below = 0;
    for (uint32_t w = 0; w < (vn >> 6); w++)
        below += (uint64_t)__popcll(m[w]);
    below += (uint64_t)__popcll(m[vn >> 6] & ((1ull << (vn & 63)) - 1ull));
    // value index in the value-concatenated upstream arrays (clouds back to back)
    const uint64_t vi = B.value_base[B.leaf_cloud[l]] + B.leaf_vidx[l] + below;
    const int32_t x = B.lower_origin[3 * lo + 0] + (int32_t)((ln >> 8) & 15) * 8 + (int32_t)(vn >> 6);
    const int32_t y = B.lower_origin[3 * lo + 1] + (int32_t)((ln >> 4) & 15) * 8 + (int32_t)((vn >> 3) & 7);
    const int32_t z = B.lower_origin[3 * lo + 2] + (int32_t)(ln & 15) * 8 + (int32_t)(vn & 7);
    const GaussRec R = B.recs[gid];
    const RInv M = rinv_of(R);
    SmoothTerms t;
    const float Kw = smooth_kernel(R, M, rec_vs(R, B.voxel_size, B.cloud_vs), x, y, z, t);
    if (!(t.e > SMOOTH_TAU))
        return;
    const float gd = B.grad_density ? B.grad_density[vi] : 0.f;
    float gc[3] = { 0.f, 0.f, 0.f };
    if (B.grad_color)
    {
        gc[0] = B.grad_color[3 * vi + 0];
        gc[1] = B.grad_color[3 * vi + 1];
        gc[2] = B.grad_color[3 * vi + 2];
    }
    const float GK = gd + gc[0] * R.q7.x + gc[1] * R.q7.y + gc[2] * R.q7.z;
    const float inv_s[3] = { R.q3.y, R.q3.z, R.q3.w };
    c[0] = GK * t.E;
#pragma unroll
    for (int r = 0; r < 3; r++)
    {
        const float dz = -GK * t.e * t.z[r];
        const float du = dz * inv_s[r];
        c[1 + r] = du;
        c[4 + r] = dz * t.z[r];
#pragma unroll
        for (int a = 0; a < 3; a++)
            c[7 + 3 * r + a] = du * t.d[a];
    }
    c[16] = Kw * gc[0];
    c[17] = Kw * gc[1];
    c[18] = Kw * gc[2];
}

__device__ __forceinline__ void bwd_flush(double* dst, float (&a)[BWD_NACC], bool exclusive, int lane)
{
#pragma unroll
    for (int i = 0; i < BWD_NACC; i++)
    {
        float v = a[i];
#pragma unroll
        for (int o = 16; o; o >>= 1)
            v += __shfl_xor_sync(FULL, v, o);
        a[i] = 0.f;
        if (lane == 0)
        {
            if (exclusive)
                dst[i] = (double)v;
            else
                atomicAdd(&dst[i], (double)v);
        }
    }
}

template <class K>
__global__ void __launch_bounds__(BWD_BLOCK) k_bwd_pairs(BwdParams B)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * BWD_BLOCK + threadIdx.x) >> 5;
    const int64_t r0 = warp * BWD_RANGE;
    if (r0 >= B.P)
        return; // uniform per warp
    const int64_t r1 = min(B.P, r0 + (int64_t)BWD_RANGE);
    const K* keys = (const K*)B.keys;
    float acc[BWD_NACC];
#pragma unroll
    for (int i = 0; i < BWD_NACC; i++)
        acc[i] = 0.f;
    uint32_t cur = B.ids[r0];
    bool head = r0 == 0 || B.ids[r0 - 1] != cur;
    for (int64_t base = r0; base < r1; base += 32)
    {
        const int64_t p = base + lane;
        const bool valid = p < r1;
        const uint32_t gid = valid ? B.ids[p] : 0xFFFFFFFFu;
        float c[BWD_NACC];
#pragma unroll
        for (int i = 0; i < BWD_NACC; i++)
            c[i] = 0.f;
        if (valid && gid < (uint64_t)B.G)
            pair_adjoint<K>(B, (uint64_t)keys[p], gid, c);
        // one pass per Gaussian present in this chunk (at most 32)
        bool pend = valid;
        while (true)
        {
            if (pend && gid == cur)
            {
#pragma unroll
                for (int i = 0; i < BWD_NACC; i++)
                    acc[i] += c[i];
                pend = false;
            }
            const unsigned later = __ballot_sync(FULL, pend);
            if (!later)
                break;
            // the segment of `cur` ends inside this range
            if (cur < (uint64_t)B.G)
                bwd_flush(B.acc + (uint64_t)cur * BWD_NACC, acc, head, lane);
            cur = __shfl_sync(FULL, gid, __ffs(later) - 1);
            head = true;
        }
    }
    const bool tail = r1 == B.P || B.ids[r1] != cur;
    if (cur < (uint64_t)B.G)
        bwd_flush(B.acc + (uint64_t)cur * BWD_NACC, acc, head && tail, lane);
}

// per Gaussian: chain the FP64 sums to the caller's parameters
__global__ void __launch_bounds__(256) k_bwd_finalize(BwdFinalParams F)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= F.G)
        return;
    double a[BWD_NACC];
    bool any = false;
    if (F.partials)
    {
        // the Gaussian's (leaf, Gaussian) pairs are emission indices [e0, e1)
        const uint64_t c0 = F.lcol_off[g], c1 = g + 1 < F.G ? F.lcol_off[g + 1] : F.NLC;
        const uint64_t e0 = c0 < F.NLC ? F.lc_off[c0] : F.Q, e1 = c1 < F.NLC ? F.lc_off[c1] : F.Q;
        for (int i = 0; i < BWD_NACC; i++)
            a[i] = 0.0;
        for (uint64_t e = e0; e < e1; e++)
            for (int i = 0; i < BWD_NACC; i++)
                a[i] += (double)F.partials[e * BWD_NACC + i];
        for (int i = 0; i < BWD_NACC; i++)
            any = any || a[i] != 0.0;
    }
    else
    {
        const double* A = F.acc + BWD_NACC * g;
        for (int i = 0; i < BWD_NACC; i++)
        {
            a[i] = A[i];
            any = any || a[i] != 0.0;
        }
    }
    float dmu[3] = { 0.f, 0.f, 0.f }, dq[4] = { 0.f, 0.f, 0.f, 0.f }, ds[3] = { 0.f, 0.f, 0.f }, dop = 0.f,
          dc[3] = { 0.f, 0.f, 0.f };
    if (any)
    {
        const float vsf = rec_vs(F.recs[g], F.voxel_size, F.cloud_vs);
        const double vs = (double)vsf;
        // rotation of the quaternion as the forward used it (normalised for raw inputs)
        double x = F.quats[4 * g + 1], y = F.quats[4 * g + 2], z = F.quats[4 * g + 3], w = F.quats[4 * g + 0];
        const double n = F.raw ? sqrt(x * x + y * y + z * z + w * w) : 1.0;
        x /= n;
        y /= n;
        z /= n;
        w /= n;
        double R[3][3];
        R[0][0] = 1 - 2 * (y * y + z * z);
        R[0][1] = 2 * (x * y - z * w);
        R[0][2] = 2 * (x * z + y * w);
        R[1][0] = 2 * (x * y + z * w);
        R[1][1] = 1 - 2 * (x * x + z * z);
        R[1][2] = 2 * (y * z - x * w);
        R[2][0] = 2 * (x * z - y * w);
        R[2][1] = 2 * (y * z + x * w);
        R[2][2] = 1 - 2 * (x * x + y * y);
        const double* U = &a[1];
        const double* W = &a[4];
        for (int k = 0; k < 3; k++)
            dmu[k] = (float)(-(R[k][0] * U[0] + R[k][1] * U[1] + R[k][2] * U[2]));
        const float min_scale = VOX_FMUL(0.125f, vsf);
        for (int r = 0; r < 3; r++)
        {
            const float in = F.scales[3 * g + r];
            const float sf = F.raw ? vox_expf_cr(in) : in; // the forward's clamp decision
            const bool clamped = !(sf > min_scale);
            const double s_act = F.raw ? exp((double)in) : (double)in;
            const double s = clamped ? 0.125 * vs : s_act;
            const double d = clamped ? 0.0 : -W[r] / s;
            ds[r] = (float)(F.raw ? d * s_act : d);
        }
        double G[3][3];
        for (int k = 0; k < 3; k++)
            for (int r = 0; r < 3; r++)
                G[k][r] = a[7 + 3 * r + k];
        double dx = 2 * y * (G[0][1] + G[1][0]) + 2 * z * (G[0][2] + G[2][0]) + 2 * w * (G[2][1] - G[1][2]) -
                    4 * x * (G[1][1] + G[2][2]);
        double dy = 2 * x * (G[0][1] + G[1][0]) + 2 * w * (G[0][2] - G[2][0]) + 2 * z * (G[1][2] + G[2][1]) -
                    4 * y * (G[0][0] + G[2][2]);
        double dz = 2 * w * (G[1][0] - G[0][1]) + 2 * x * (G[0][2] + G[2][0]) + 2 * y * (G[1][2] + G[2][1]) -
                    4 * z * (G[0][0] + G[1][1]);
        double dw = 2 * z * (G[1][0] - G[0][1]) + 2 * y * (G[0][2] - G[2][0]) + 2 * x * (G[2][1] - G[1][2]);
        if (F.raw)
        {
            const double dot = x * dx + y * dy + z * dz + w * dw;
            dx = (dx - x * dot) / n;
            dy = (dy - y * dot) / n;
            dz = (dz - z * dot) / n;
            dw = (dw - w * dot) / n;
        }
        dq[0] = (float)dw;
        dq[1] = (float)dx;
        dq[2] = (float)dy;
        dq[3] = (float)dz;
        if (F.raw)
        {
            const double op = 1.0 / (1.0 + exp(-(double)F.opacities[g]));
            dop = (float)(a[0] * op * (1.0 - op));
            for (int c = 0; c < 3; c++)
                dc[c] = (float)(0.28209479177387814 * a[16 + c]);
        }
        else
        {
            dop = (float)a[0];
            for (int c = 0; c < 3; c++)
                dc[c] = (float)a[16 + c];
        }
    }
    if (F.d_means)
        for (int k = 0; k < 3; k++)
            F.d_means[3 * g + k] = dmu[k];
    if (F.d_quats)
        for (int k = 0; k < 4; k++)
            F.d_quats[4 * g + k] = dq[k];
    if (F.d_scales)
        for (int k = 0; k < 3; k++)
            F.d_scales[3 * g + k] = ds[k];
    if (F.d_opacities)
        F.d_opacities[g] = dop;
    if (F.d_colors)
        for (int k = 0; k < 3; k++)
            F.d_colors[3 * g + k] = dc[k];
}

void launch_bwd_pairs(const BwdParams& B, int key64, cudaStream_t s)
{
    if (B.P <= 0)
        return;
    const int64_t warps = (B.P + BWD_RANGE - 1) / BWD_RANGE;
    const int64_t blocks = (warps + (BWD_BLOCK / 32) - 1) / (BWD_BLOCK / 32);
    if (key64)
        { k_bwd_pairs<uint64_t><<<(unsigned)blocks, BWD_BLOCK, 0, s>>>(B); count_launch(); }
    else
        { k_bwd_pairs<uint32_t><<<(unsigned)blocks, BWD_BLOCK, 0, s>>>(B); count_launch(); }
}

void launch_bwd_finalize(const BwdFinalParams& F, cudaStream_t s)
{
    if (F.G <= 0)
        return;
    { k_bwd_finalize<<<(unsigned)((F.G + 255) / 256), 256, 0, s>>>(F); count_launch(); }
}

} // namespace vox
