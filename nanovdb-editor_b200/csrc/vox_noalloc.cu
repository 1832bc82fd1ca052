// vox_noalloc.cu - a scan entry point that allocates no device memory.
//
// vox_global_scan_u64 keeps its look-back words in context buffers it grows
// with cudaMalloc.  Some callers cannot let a library allocate: hosts whose
// device memory is owned by their own allocator (a framework's caching pool
// holding the free memory, where an extra cudaMalloc can fail or fragment the
// pool) and loops where the implicit device synchronisation of cudaMalloc /
// cudaFree is not acceptable.  This variant keeps its scratch in a fixed
// file-scope device array instead, so the caller only passes inputs, outputs
// and a stream.
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "pnanovdb_b200.h"
#include "vox_device.cuh"
#include "vox_internal.h"

using namespace vox;

namespace
{

// Scratch of the look-back scan: one status word per 2048-element tile for up
// to VOX_NOALLOC_SCAN_MAX elements, then the tile counter and the error word.
// 8195 words = 64 KiB; every GPU that loads the library holds it until exit.
constexpr int64_t kMaxTiles = (VOX_NOALLOC_SCAN_MAX + 2047) / 2048;
constexpr int64_t kStatusWords = kMaxTiles + 1;
constexpr int64_t kScratchWords = kStatusWords + 2;

static __device__ __align__(256) uint64_t g_scan_scratch[kScratchWords];

std::mutex g_setup_mutex;
uint64_t* g_scratch_addr[64] = {};

// Device address of g_scan_scratch on the current device.  In host code the
// symbol is only a host-side stand-in, so the address must come from
// cudaGetSymbolAddress, once per device, with that device current.
uint64_t* scratch_on_current_device(int* device_out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    {
        cudaGetLastError();
        return nullptr;
    }
    *device_out = dev;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev])
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            fprintf(stderr, "[pnanovdb_b200] vox_global_scan_u64_noalloc: cudaGetSymbolAddress failed on device %d: %s\n",
                    dev, cudaGetErrorString(e));
            return nullptr;
        }
        g_scratch_addr[dev] = (uint64_t*)p;
    }
    return g_scratch_addr[dev];
}

} // namespace

extern "C" int vox_global_scan_u64_noalloc(const uint64_t* d_in, uint64_t* d_out, int64_t n, int inclusive,
                                           uint64_t* d_total, void* stream)
{
    if (n < 0 || (n > 0 && (!d_in || !d_out)) || !d_total)
        return VOX_ERR_ARGS;
    if (n > VOX_NOALLOC_SCAN_MAX)
    {
        fprintf(stderr,
                "[pnanovdb_b200] vox_global_scan_u64_noalloc: %lld elements exceed the fixed scratch limit of %lld; "
                "use vox_global_scan_u64\n",
                (long long)n, (long long)VOX_NOALLOC_SCAN_MAX);
        return VOX_ERR_SIZE;
    }
    int dev = 0;
    uint64_t* scratch = scratch_on_current_device(&dev);
    if (!scratch)
        return VOX_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    // The array keeps the previous call's contents: clear the status words,
    // the tile counter and the error word this call uses.
    const int64_t tiles = (n + 2047) / 2048;
    uint64_t* status = scratch;
    uint32_t* counter = (uint32_t*)(scratch + kStatusWords);
    int* err = (int*)(scratch + kStatusWords + 1);
    cudaMemsetAsync(status, 0, sizeof(uint64_t) * (size_t)(tiles + 1), s);
    cudaMemsetAsync(scratch + kStatusWords, 0, sizeof(uint64_t) * 2, s);
    scan_exclusive_u64(d_in, d_out, n, inclusive ? 2 : 0, d_total, status, 1u, counter, err, 0, s);
    int host_err = 0;
    cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
    {
        fprintf(stderr, "[pnanovdb_b200] vox_global_scan_u64_noalloc: %s\n", cudaGetErrorString(e));
        return VOX_ERR_CUDA;
    }
    return host_err ? VOX_ERR_TIMEOUT : VOX_OK;
}
