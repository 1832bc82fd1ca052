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
// k_leaf_backward (vox_leaf.cu) replays the forward leaf walk: per candidate
// leaf and Gaussian, the terms above summed over the leaf's voxels (a block
// reduction) are stored by the pair's emission index; k_bwd_finalize sums a
// Gaussian's partials (its emission indices are contiguous) in FP64 and
// chains them.  No atomics, nothing stored per voxel pair.
#include <cstdio>
#include <cuda_runtime.h>

#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

// per Gaussian: chain the FP64 sums to the caller's parameters
__global__ void __launch_bounds__(256) k_bwd_finalize(BwdFinalParams F)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= F.G)
        return;
    double a[BWD_NACC];
    bool any = false;
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
    float dmu[3] = { 0.f, 0.f, 0.f }, dq[4] = { 0.f, 0.f, 0.f, 0.f }, ds[3] = { 0.f, 0.f, 0.f }, dop = 0.f,
          dc[3] = { 0.f, 0.f, 0.f };
    if (any)
    {
        const float vsf = rec_vs(F.recs[g], F.voxel_size, F.cloud_vs);
        const double vs = (double)vsf;
        // rotation of the quaternion as the forward used it (normalised for raw inputs)
        double x = ld_attr(F.quats, 4 * g + 1, F.bf16), y = ld_attr(F.quats, 4 * g + 2, F.bf16), z = ld_attr(F.quats, 4 * g + 3, F.bf16), w = ld_attr(F.quats, 4 * g + 0, F.bf16);
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
            const float in = ld_attr(F.scales, 3 * g + r, F.bf16);
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
            const double op = 1.0 / (1.0 + exp(-(double)ld_attr(F.opacities, g, F.bf16)));
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

void launch_bwd_finalize(const BwdFinalParams& F, cudaStream_t s)
{
    if (F.G <= 0)
        return;
    { k_bwd_finalize<<<(unsigned)((F.G + 255) / 256), 256, 0, s>>>(F); count_launch(); }
}

} // namespace vox
