// vox_optim.cu - the update step of the BF16 fitting loop: Adam over the
// voxelizer's attribute arrays, FP32 master copies and moments, bfloat16
// attributes out, one pass.  Elementwise and HBM-bound (30 bytes per
// parameter: 16 read, 14 written); grid-stride over the SMs.
#include <cmath>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "pnanovdb_b200.h"
#include "vox_internal.h"

namespace vox
{

__global__ void __launch_bounds__(256) k_adam_bf16(float* __restrict__ master, float* __restrict__ m, float* __restrict__ v,
                                                    const float* __restrict__ grad, __nv_bfloat16* __restrict__ out,
                                                    int64_t n, float lr_t, float beta1, float beta2, float eps_t)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        const float g = grad[i];
        const float mi = beta1 * m[i] + (1.f - beta1) * g;
        const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
        // lr (m / c1) / (sqrt(v / c2) + eps) = lr_t m / (sqrt(v) + eps_t), lr_t = lr sqrt(c2) / c1, eps_t = eps sqrt(c2)
        const float p = master[i] - lr_t * mi / (sqrtf(vi) + eps_t);
        m[i] = mi;
        v[i] = vi;
        master[i] = p;
        out[i] = __float2bfloat16_rn(p);
    }
}

} // namespace vox

extern "C" int vox_adam_bf16(float* master, float* m, float* v, const float* grad, uint16_t* out_bf16, int64_t n,
                             float lr, float beta1, float beta2, float eps, int64_t step, void* stream)
{
    if (n < 0 || (n > 0 && (!master || !m || !v || !grad || !out_bf16)) || step < 1 || !(beta1 >= 0.f && beta1 < 1.f) ||
        !(beta2 >= 0.f && beta2 < 1.f))
        return VOX_ERR_ARGS;
    if (n == 0)
        return VOX_OK;
    const double c1 = 1.0 - pow((double)beta1, (double)step), c2 = 1.0 - pow((double)beta2, (double)step);
    const float lr_t = (float)((double)lr * sqrt(c2) / c1), eps_t = (float)((double)eps * sqrt(c2));
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t blocks = (n + 255) / 256;
    if (blocks > (int64_t)sms * 8)
        blocks = (int64_t)sms * 8;
    vox::k_adam_bf16<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(master, m, v, grad, (__nv_bfloat16*)out_bf16, n, lr_t,
                                                                          beta1, beta2, eps_t);
    vox::count_launch();
    return cudaGetLastError() == cudaSuccess ? VOX_OK : VOX_ERR_CUDA;
}
