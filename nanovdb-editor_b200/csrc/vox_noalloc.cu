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

#include <cuda_runtime.h>

#include "pnanovdb_b200.h"
#include "vox_device.cuh"
#include "vox_internal.h"

using namespace vox;

namespace
{

// Scratch of the look-back scan: four status words per 2048-element tile for
// up to VOX_NOALLOC_SCAN_MAX elements (the 64-bit look-back of the u64 scan),
// then the tile counter and the error word: 32,774 words = 256 KiB + 48 B,
// which every GPU that loads the library holds until exit.
constexpr int64_t kMaxTiles = (VOX_NOALLOC_SCAN_MAX + 2047) / 2048;
constexpr int64_t kStatusWords = 4 * (kMaxTiles + 1);
constexpr int64_t kScratchWords = kStatusWords + 2;

static __device__ __align__(256) uint64_t g_scan_scratch[kScratchWords];

// Device address of g_scan_scratch on the current device.  In host code the
// symbol is only a host-side stand-in, so the address must come from
// cudaGetSymbolAddress with that device current.  It is looked up on every
// call (cheap after the first, which loads the module on the device): a
// cached address would go stale if the caller reset the device in between.
uint64_t* scratch_on_current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
    {
        cudaGetLastError();
        return nullptr;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        fprintf(stderr, "[pnanovdb_b200] vox_global_scan_u64_noalloc: cudaGetSymbolAddress failed on device %d: %s\n",
                dev, cudaGetErrorString(e));
        return nullptr;
    }
    return (uint64_t*)p;
}

int cuda_failed(cudaError_t e)
{
    fprintf(stderr, "[pnanovdb_b200] vox_global_scan_u64_noalloc: %s\n", cudaGetErrorString(e));
    return VOX_ERR_CUDA;
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
    uint64_t* scratch = scratch_on_current_device();
    if (!scratch)
        return VOX_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    // The array keeps the previous call's contents: clear the status words,
    // the tile counter and the error word (with its wait control) this call uses.
    const int64_t tiles = (n + 2047) / 2048;
    uint64_t* status = scratch;
    uint32_t* counter = (uint32_t*)(scratch + kStatusWords);
    int* err = (int*)(scratch + kStatusWords + 1);
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint64_t) * 4 * (size_t)(tiles + 1), s);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(scratch + kStatusWords, 0, sizeof(uint64_t) * 2, s);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return cuda_failed(e);
    }
    scan_exclusive_u64(d_in, d_out, n, inclusive ? 2 : 0, d_total, status, 1u, counter, err, 0, s);
    // a launch-configuration error or a bad stream handle surfaces here, not in the synchronisation
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_failed(e);
    int host_err = 0;
    e = cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return cuda_failed(e);
    }
    return host_err ? VOX_ERR_TIMEOUT : VOX_OK;
}
