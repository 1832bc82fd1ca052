// vox_dropin.cu - the reference-compatible function tables:
// pnanovdb_get_raster() (raster/Raster.cpp:822-840, RasterUtils.cpp) and a
// headless pnanovdb_get_compute() whose array functions follow
// nanovdb_editor/putil/Compute.h:838-843.  Every raster entry is a thin
// wrapper over vox_voxelize / vox_voxelize_host.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "pnanovdb_b200.h"

// ------------------------------------------------------------- queue / device
// A queue is a CUDA device plus its own voxelization context (one stream and
// its buffers), created on the queue's first raster call.  The reference's
// callers are editor worker threads, each with its own queue
// (editor/PipelineRuntime.cpp:416-427), so calls on different queues run
// concurrently; the per-queue mutex only serialises callers that share a queue.
struct pnanovdb_compute_queue_t
{
    int device = 0;
    std::mutex mu;
    vox_context_t* vox = nullptr;
};
struct pnanovdb_compute_device_t
{
    int index = 0;
    pnanovdb_compute_queue_t* queue = nullptr;         // get_device_queue
    pnanovdb_compute_queue_t* compute_queue = nullptr; // get_compute_queue
};

struct pnanovdb_raster_context_t
{
    vox_context_t* vox;
    std::mutex mu;
};

struct pnanovdb_raster_gaussian_data_t
{
    int64_t n = 0;
    std::vector<float> means, quats, scales, colors, opacities; // activated
    float cull_scale = 0.05f;
    int raw = 0;          // attributes still in the on-disk convention (VOX_FLAG_RAW_INPUTS)
    float* dev = nullptr; // device copy after upload_gaussian_data
    int device = 0;
};

static int queue_device(pnanovdb_compute_queue_t* q)
{
    return q ? q->device : 0;
}

static void log_err(const char* msg)
{
    fprintf(stderr, "[pnanovdb_b200] %s\n", msg);
}

// Table entries run their bodies through this: no C++ exception (an allocation
// failure, say) crosses the C ABI; it is logged and the entry's failure value
// returned, as the reference's entries report errors (log + FALSE / NULL).
template <class R, class F>
static R no_throw(const char* entry, R fail, F&& body)
{
    try
    {
        return body();
    }
    catch (const std::bad_alloc&)
    {
        fprintf(stderr, "[pnanovdb_b200] %s: out of host memory\n", entry);
    }
    catch (const std::exception& e)
    {
        fprintf(stderr, "[pnanovdb_b200] %s: %s\n", entry, e.what());
    }
    catch (...)
    {
        fprintf(stderr, "[pnanovdb_b200] %s: unexpected error\n", entry);
    }
    return fail;
}

// callers that pass no queue share one default queue per device
constexpr int MAX_DEVICES = 64;
static pnanovdb_compute_queue_t g_default_queue[MAX_DEVICES];

static pnanovdb_compute_queue_t* resolve_queue(pnanovdb_compute_queue_t* q)
{
    if (q)
        return q;
    return &g_default_queue[0];
}

// the queue's context; the caller holds q->mu
static vox_context_t* queue_context(pnanovdb_compute_queue_t* q)
{
    if (!q->vox)
        q->vox = vox_context_create(q->device);
    return q->vox;
}

// cull scale from gaussian_frag_color's parameter block (gaussian_frag_color.slang:205-213)
static float cull_from_params(pnanovdb_compute_array_t** shader_params_arrays)
{
    if (!shader_params_arrays)
        return 0.05f;
    pnanovdb_compute_array_t* a = shader_params_arrays[PNANOVDB_RASTER_SHADER_GAUSSIAN_FRAG_COLOR];
    if (!a || !a->data || a->element_size * a->element_count < 8)
        return 0.05f;
    float cull;
    uint32_t use_default;
    memcpy(&cull, a->data, 4);
    memcpy(&use_default, (const char*)a->data + 4, 4);
    if (use_default || cull == 0.f)
        return 0.05f;
    return cull;
}

// The reference's table entries return the reference's node order: node_idx,
// node2 addresses and value indices of its window-by-window build.
constexpr uint32_t DROPIN_ORDER = VOX_FLAG_WINDOW_ORDER;

// ------------------------------------------------------------------ arrays
// Grids returned to the caller live in page-locked host memory so the
// device-to-host copy runs at link speed.  Page-locking is slow, so blocks
// come back to a small pool when the caller destroys the array and the next
// result of a similar size reuses them.
namespace
{
std::mutex g_pin_mutex;
std::unordered_map<void*, size_t> g_pinned;           // live page-locked blocks -> capacity
std::vector<std::pair<void*, size_t>> g_pin_free;     // pooled blocks
constexpr size_t PIN_POOL_MAX = 4;                    // blocks kept for reuse

void* pinned_alloc(size_t bytes)
{
    std::lock_guard<std::mutex> lock(g_pin_mutex);
    size_t best = (size_t)-1;
    for (size_t i = 0; i < g_pin_free.size(); i++)
        if (g_pin_free[i].second >= bytes && g_pin_free[i].second <= 2 * bytes + 4096 &&
            (best == (size_t)-1 || g_pin_free[i].second < g_pin_free[best].second))
            best = i;
    if (best != (size_t)-1)
    {
        auto blk = g_pin_free[best];
        g_pin_free.erase(g_pin_free.begin() + (long)best);
        g_pinned[blk.first] = blk.second;
        return blk.first;
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocPortable) != cudaSuccess)
    {
        cudaGetLastError();
        return nullptr;
    }
    g_pinned[p] = bytes ? bytes : 1;
    return p;
}

// returns true when p was a pooled page-locked block
bool pinned_release(void* p)
{
    std::lock_guard<std::mutex> lock(g_pin_mutex);
    auto it = g_pinned.find(p);
    if (it == g_pinned.end())
        return false;
    g_pin_free.emplace_back(it->first, it->second);
    g_pinned.erase(it);
    if (g_pin_free.size() > PIN_POOL_MAX)
    {
        cudaFreeHost(g_pin_free.front().first);
        g_pin_free.erase(g_pin_free.begin());
    }
    return true;
}
} // namespace

static pnanovdb_compute_array_t* PNANOVDB_ABI array_create(size_t element_size, pnanovdb_uint64_t element_count,
                                                           const void* data)
{
    pnanovdb_compute_array_t* a = (pnanovdb_compute_array_t*)calloc(1, sizeof(pnanovdb_compute_array_t));
    if (!a)
        return nullptr;
    size_t bytes = element_size * element_count;
    a->data = malloc(bytes ? bytes : 1);
    if (!a->data)
    {
        free(a);
        return nullptr;
    }
    if (data && bytes)
        memcpy(a->data, data, bytes);
    else if (bytes)
        memset(a->data, 0, bytes);
    a->element_size = element_size;
    a->element_count = element_count;
    return a;
}
static void PNANOVDB_ABI array_destroy(pnanovdb_compute_array_t* a)
{
    if (!a)
        return;
    if (!pinned_release(a->data))
        free(a->data);
    free(a);
}

// an array whose contents the caller fills at once (page-locked, not cleared)
static pnanovdb_compute_array_t* array_create_pinned(size_t element_size, pnanovdb_uint64_t element_count)
{
    pnanovdb_compute_array_t* a = (pnanovdb_compute_array_t*)calloc(1, sizeof(pnanovdb_compute_array_t));
    if (!a)
        return nullptr;
    a->data = pinned_alloc(element_size * element_count);
    if (!a->data)
    {
        free(a);
        return nullptr;
    }
    a->element_size = element_size;
    a->element_count = element_count;
    return a;
}
static void* PNANOVDB_ABI array_map(pnanovdb_compute_array_t* a)
{
    return a ? a->data : nullptr;
}
static void PNANOVDB_ABI array_unmap(pnanovdb_compute_array_t*)
{
}
static pnanovdb_compute_array_t* PNANOVDB_ABI array_duplicate(pnanovdb_compute_array_t* a)
{
    return a ? array_create(a->element_size, a->element_count, a->data) : nullptr;
}
static pnanovdb_compute_array_t* PNANOVDB_ABI load_grid(const char* path)
{
    FILE* f = fopen(path, "rb");
    if (!f)
        return nullptr;
    fseek(f, 0, SEEK_END);
    long bytes = ftell(f);
    fseek(f, 0, SEEK_SET);
    pnanovdb_compute_array_t* a = array_create(4, (uint64_t)(bytes + 3) / 4, nullptr);
    if (a && fread(a->data, 1, (size_t)bytes, f) != (size_t)bytes)
    {
        array_destroy(a);
        a = nullptr;
    }
    fclose(f);
    return a;
}
static pnanovdb_bool_t PNANOVDB_ABI save_grid(pnanovdb_compute_array_t* a, const char* path)
{
    if (!a || !path)
        return PNANOVDB_FALSE;
    FILE* f = fopen(path, "wb");
    if (!f)
        return PNANOVDB_FALSE;
    size_t bytes = a->element_size * a->element_count;
    bool ok = fwrite(a->data, 1, bytes, f) == bytes;
    fclose(f);
    return ok ? PNANOVDB_TRUE : PNANOVDB_FALSE;
}

// ---------------------------------------------------------- device interface
static int g_manager_token = 0;
static void* PNANOVDB_ABI dev_create_manager(pnanovdb_bool_t)
{
    return &g_manager_token;
}
static void PNANOVDB_ABI dev_destroy_manager(void*)
{
}
static pnanovdb_bool_t PNANOVDB_ABI dev_enumerate(void*, pnanovdb_uint32_t index, void*)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess)
    {
        cudaGetLastError();
        return PNANOVDB_FALSE;
    }
    return (int)index < n ? PNANOVDB_TRUE : PNANOVDB_FALSE;
}
static pnanovdb_compute_queue_t* new_queue(int device)
{
    pnanovdb_compute_queue_t* q = new pnanovdb_compute_queue_t();
    q->device = device;
    return q;
}
static void delete_queue(pnanovdb_compute_queue_t* q)
{
    if (!q)
        return;
    if (q->vox)
        vox_context_destroy(q->vox);
    delete q;
}
// desc: pnanovdb_compute_device_desc_t (nanovdb_editor/putil/Compute.h:503-508),
// whose first field is the device index
static pnanovdb_compute_device_t* PNANOVDB_ABI dev_create(void*, const void* desc)
{
    return no_throw<pnanovdb_compute_device_t*>("create_device", nullptr, [&]() -> pnanovdb_compute_device_t* {
        uint32_t index = 0;
        if (desc)
            memcpy(&index, desc, sizeof(index));
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || (int)index >= n)
        {
            cudaGetLastError();
            log_err("create_device: no such CUDA device");
            return nullptr;
        }
        pnanovdb_compute_device_t* d = new pnanovdb_compute_device_t();
        d->index = (int)index;
        d->queue = new_queue((int)index);
        d->compute_queue = new_queue((int)index);
        return d;
    });
}
static void PNANOVDB_ABI dev_destroy(void*, pnanovdb_compute_device_t* d)
{
    if (!d)
        return;
    delete_queue(d->queue);
    delete_queue(d->compute_queue);
    delete d;
}
static pnanovdb_compute_queue_t* PNANOVDB_ABI dev_queue(const pnanovdb_compute_device_t* d)
{
    return d ? d->queue : nullptr;
}
static pnanovdb_compute_queue_t* PNANOVDB_ABI dev_compute_queue(const pnanovdb_compute_device_t* d)
{
    return d ? d->compute_queue : nullptr;
}
static int PNANOVDB_ABI dev_flush(pnanovdb_compute_queue_t*, pnanovdb_uint64_t* flushed, void*, void*)
{
    if (flushed)
        *flushed = 0;
    return 0;
}
static void PNANOVDB_ABI dev_wait_idle(pnanovdb_compute_queue_t* q)
{
    if (q)
    {
        std::lock_guard<std::mutex> lock(q->mu);
        if (q->vox)
        {
            cudaStreamSynchronize((cudaStream_t)vox_context_stream(q->vox));
            return;
        }
    }
    cudaSetDevice(queue_device(q));
    cudaDeviceSynchronize();
}
static pnanovdb_uint32_t PNANOVDB_ABI dev_index(const pnanovdb_compute_device_t* d)
{
    return d ? (pnanovdb_uint32_t)d->index : 0u;
}

// ------------------------------------------------------------------- raster
static pnanovdb_raster_context_t* PNANOVDB_ABI r_create_context(const pnanovdb_compute_t*,
                                                                  pnanovdb_compute_queue_t* queue)
{
    return no_throw<pnanovdb_raster_context_t*>("create_context", nullptr, [&]() -> pnanovdb_raster_context_t* {
        vox_context_t* v = vox_context_create(queue_device(queue));
        if (!v)
            return nullptr;
        pnanovdb_raster_context_t* c = new pnanovdb_raster_context_t();
        c->vox = v;
        return c;
    });
}
static void PNANOVDB_ABI r_destroy_context(const pnanovdb_compute_t*, pnanovdb_compute_queue_t*,
                                           pnanovdb_raster_context_t* c)
{
    if (!c)
        return;
    vox_context_destroy(c->vox);
    delete c;
}

static bool copy_floats(std::vector<float>& dst, pnanovdb_compute_array_t* a, int64_t count)
{
    if (!a || !a->data || a->element_size != 4 || (int64_t)a->element_count < count)
        return false;
    dst.assign((const float*)a->data, (const float*)a->data + count);
    return true;
}

// raster/RasterContext.cpp:92-229: copies the caller's arrays (activated
// attributes; colours from `colors`, else from sh_0 as c0 * sh_0 + 0.5)
static pnanovdb_raster_gaussian_data_t* PNANOVDB_ABI r_create_gaussian_data(
    const pnanovdb_compute_t*, pnanovdb_compute_queue_t* queue, pnanovdb_raster_context_t*,
    pnanovdb_compute_array_t* means, pnanovdb_compute_array_t* quaternions, pnanovdb_compute_array_t* scales,
    pnanovdb_compute_array_t* colors, pnanovdb_compute_array_t* sh_0, pnanovdb_compute_array_t*,
    pnanovdb_compute_array_t* opacities, pnanovdb_compute_array_t** shader_params_arrays,
    pnanovdb_raster_shader_params_t*)
{
    return no_throw<pnanovdb_raster_gaussian_data_t*>("create_gaussian_data", nullptr, [&]() -> pnanovdb_raster_gaussian_data_t* {
        if (!means || means->element_size != 4)
        {
            log_err("create_gaussian_data: means must be float32");
            return nullptr;
        }
        std::unique_ptr<pnanovdb_raster_gaussian_data_t> d(new pnanovdb_raster_gaussian_data_t());
        d->n = (int64_t)(means->element_count / 3);
        d->device = queue_device(queue);
        bool ok = copy_floats(d->means, means, 3 * d->n) && copy_floats(d->quats, quaternions, 4 * d->n) &&
                  copy_floats(d->scales, scales, 3 * d->n) && copy_floats(d->opacities, opacities, d->n);
        if (ok && colors)
            ok = copy_floats(d->colors, colors, 3 * d->n);
        else if (ok && sh_0)
        {
            ok = copy_floats(d->colors, sh_0, 3 * d->n);
            for (auto& c : d->colors)
                c = 0.28209479177387814f * c + 0.5f;
        }
        else
            ok = false;
        if (!ok)
        {
            log_err("create_gaussian_data: attribute arrays must be float32 with 3/4/3/3/1 values per Gaussian");
            return nullptr;
        }
        d->cull_scale = cull_from_params(shader_params_arrays);
        return d.release();
    });
}

// the device copy of the attributes, one allocation: means, quats, scales, opacities, colours
static void PNANOVDB_ABI r_upload_gaussian_data(const pnanovdb_compute_t*, pnanovdb_compute_queue_t*,
                                                pnanovdb_raster_context_t*, pnanovdb_raster_gaussian_data_t* d)
{
    if (!d)
        return;
    cudaSetDevice(d->device);
    if (d->dev)
        cudaFree(d->dev);
    d->dev = nullptr;
    const int64_t n = d->n;
    const size_t floats = (size_t)n * 14;
    if (cudaMalloc(&d->dev, floats * 4 + 4) != cudaSuccess)
    {
        cudaGetLastError();
        log_err("upload_gaussian_data: cudaMalloc failed");
        d->dev = nullptr;
        return;
    }
    bool ok = cudaMemcpy(d->dev, d->means.data(), 12 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(d->dev + 3 * n, d->quats.data(), 16 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(d->dev + 7 * n, d->scales.data(), 12 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(d->dev + 10 * n, d->opacities.data(), 4 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(d->dev + 11 * n, d->colors.data(), 12 * n, cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok)
    {
        cudaGetLastError();
        log_err("upload_gaussian_data: host to device copy failed");
        cudaFree(d->dev);
        d->dev = nullptr;
    }
}

static void PNANOVDB_ABI r_destroy_gaussian_data(const pnanovdb_compute_t*, pnanovdb_compute_queue_t*,
                                                 pnanovdb_raster_gaussian_data_t* d)
{
    if (!d)
        return;
    if (d->dev)
    {
        cudaSetDevice(d->device);
        cudaFree(d->dev);
    }
    delete d;
}

static void PNANOVDB_ABI r_raster_gaussian_2d(const pnanovdb_compute_t*, pnanovdb_compute_queue_t*,
                                              pnanovdb_raster_context_t*, pnanovdb_raster_gaussian_data_t*, void*,
                                              pnanovdb_uint32_t, pnanovdb_uint32_t, const void*, const void*,
                                              const pnanovdb_raster_shader_params_t*, pnanovdb_uint32_t)
{
    log_err("raster_gaussian_2d: the screen-space splatting path is not provided by this library");
}

// raster/Raster.cpp:420-558: uploaded Gaussians -> the reference's output, the
// node2 tree and its RGBA8 values (vox_copy_grid_rgba8), written to the
// caller's device buffer of word_count 32-bit words.  A void entry: failures
// are logged, as the reference's are.
static void PNANOVDB_ABI r_raster_gaussian_3d(const pnanovdb_compute_t*, pnanovdb_compute_queue_t*,
                                              pnanovdb_raster_context_t* ctx, float voxel_size,
                                              pnanovdb_raster_gaussian_data_t* d, pnanovdb_compute_buffer_t* out,
                                              pnanovdb_uint64_t word_count, void*)
{
    if (!ctx || !d || !out || !out->device_ptr)
    {
        log_err("raster_gaussian_3d: missing context, data or output buffer");
        return;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (!d->dev)
        r_upload_gaussian_data(nullptr, nullptr, ctx, d);
    if (!d->dev)
        return;
    vox_gaussians_t g;
    const int64_t n = d->n;
    g.count = n;
    g.means = d->dev;
    g.quats = d->dev + 3 * n;
    g.scales = d->dev + 7 * n;
    g.opacities = d->dev + 10 * n;
    g.colors = d->dev + 11 * n;
    void* grid = nullptr;
    uint64_t bytes = 0;
    if (vox_voxelize(ctx->vox, &g, voxel_size, d->cull_scale, (d->raw ? VOX_FLAG_RAW_INPUTS : 0u) | DROPIN_ORDER,
                     &grid, &bytes) != VOX_OK)
    {
        log_err((std::string("raster_gaussian_3d: ") + vox_last_error(ctx->vox)).c_str());
        return;
    }
    uint64_t cap = word_count * 4ull;
    if (out->size_bytes && out->size_bytes < cap)
        cap = out->size_bytes;
    const int rc = vox_copy_grid_rgba8(ctx->vox, out->device_ptr, cap, &bytes);
    if (rc == VOX_ERR_SIZE)
        log_err("raster_gaussian_3d: output buffer too small for the node2 grid and its RGBA8 values");
    else if (rc != VOX_OK)
        log_err((std::string("raster_gaussian_3d: ") + vox_last_error(ctx->vox)).c_str());
}

// voxelizes host arrays on the queue's context; the result is what the
// reference's host entries return: the node2 tree and its RGBA8 values
static pnanovdb_compute_array_t* run_host(pnanovdb_compute_queue_t* queue, const vox_gaussians_t* g, float voxel_size,
                                          float cull, uint32_t flags, pnanovdb_profiler_report_t report, void* userdata,
                                          const char* entry)
{
    pnanovdb_compute_queue_t* q = resolve_queue(queue);
    std::lock_guard<std::mutex> lock(q->mu);
    vox_context_t* v = queue_context(q);
    if (!v)
    {
        fprintf(stderr, "[pnanovdb_b200] %s: cannot create a CUDA context on device %d\n", entry, q->device);
        return nullptr;
    }
    uint64_t bytes = 0;
    if (vox_voxelize_host(v, g, voxel_size, cull, flags, nullptr, 0, &bytes) != VOX_OK ||
        vox_copy_grid_rgba8(v, nullptr, 0, &bytes) != VOX_OK)
    {
        fprintf(stderr, "[pnanovdb_b200] %s: %s\n", entry, vox_last_error(v));
        return nullptr;
    }
    pnanovdb_compute_array_t* a = array_create_pinned(4, (bytes + 3) / 4);
    if (!a)
    {
        fprintf(stderr, "[pnanovdb_b200] %s: out of page-locked host memory\n", entry);
        return nullptr;
    }
    if (vox_copy_grid_rgba8(v, a->data, 4 * a->element_count, &bytes) != VOX_OK)
    {
        fprintf(stderr, "[pnanovdb_b200] %s: %s\n", entry, vox_last_error(v));
        array_destroy(a);
        return nullptr;
    }
    if (report)
    {
        vox_stats_t st;
        vox_get_stats(v, &st);
        pnanovdb_compute_profiler_entry_t e[5] = { { "prep", 0.f, st.ms_prep * 1e-3f },
                                                   { "emit", 0.f, st.ms_emit * 1e-3f },
                                                   { "sort", 0.f, st.ms_sort * 1e-3f },
                                                   { "build", 0.f, st.ms_build * 1e-3f },
                                                   { "accumulate", 0.f, st.ms_accumulate * 1e-3f } };
        report(userdata, 0, 5, e);
    }
    return a;
}

static pnanovdb_compute_array_t* PNANOVDB_ABI r_raster_to_nanovdb(
    const pnanovdb_compute_t*, pnanovdb_compute_queue_t* queue, float voxel_size, pnanovdb_compute_array_t* means,
    pnanovdb_compute_array_t* quaternions, pnanovdb_compute_array_t* scales, pnanovdb_compute_array_t* colors,
    pnanovdb_compute_array_t* sh_0, pnanovdb_compute_array_t* sh_n, pnanovdb_compute_array_t* opacities,
    pnanovdb_compute_array_t** shader_params_arrays, pnanovdb_profiler_report_t profiler_report, void* userdata)
{
    return no_throw<pnanovdb_compute_array_t*>("raster_to_nanovdb", nullptr, [&]() -> pnanovdb_compute_array_t* {
        pnanovdb_raster_gaussian_data_t* d = r_create_gaussian_data(nullptr, queue, nullptr, means, quaternions, scales,
                                                                    colors, sh_0, sh_n, opacities, shader_params_arrays,
                                                                    nullptr);
        if (!d)
            return nullptr;
        std::unique_ptr<pnanovdb_raster_gaussian_data_t, void (*)(pnanovdb_raster_gaussian_data_t*)> hold(
            d, [](pnanovdb_raster_gaussian_data_t* x) { r_destroy_gaussian_data(nullptr, nullptr, x); });
        vox_gaussians_t g;
        g.count = d->n;
        g.means = d->means.data();
        g.quats = d->quats.data();
        g.scales = d->scales.data();
        g.opacities = d->opacities.data();
        g.colors = d->colors.data();
        return run_host(queue, &g, voxel_size, d->cull_scale, DROPIN_ORDER, profiler_report, userdata,
                        "raster_to_nanovdb");
    });
}

// raster/RasterUtils.cpp:400-415
static pnanovdb_bool_t PNANOVDB_ABI r_from_arrays(pnanovdb_raster_t*, const pnanovdb_compute_t*,
                                                  pnanovdb_compute_queue_t* queue, float voxel_size,
                                                  pnanovdb_compute_array_t** arrays, pnanovdb_uint32_t count,
                                                  pnanovdb_compute_array_t** out)
{
    if (!out || !arrays || count < 5u)
        return PNANOVDB_FALSE;
    *out = nullptr;
    return no_throw<pnanovdb_bool_t>("raster_to_nanovdb_from_arrays", PNANOVDB_FALSE, [&]() -> pnanovdb_bool_t {
        pnanovdb_compute_array_t *m = arrays[0], *o = arrays[1], *q = arrays[2], *s = arrays[3], *c = arrays[4];
        if (!m || !o || !q || !s || !c || m->element_size != 4 || o->element_size != 4 || q->element_size != 4 ||
            s->element_size != 4 || c->element_size != 4)
        {
            log_err("raster_to_nanovdb_from_arrays: arrays must be float32 [means, opacities, quaternions, scales, sh_0]");
            return PNANOVDB_FALSE;
        }
        const int64_t n = (int64_t)(m->element_count / 3);
        if ((int64_t)o->element_count < n || (int64_t)q->element_count < 4 * n || (int64_t)s->element_count < 3 * n ||
            (int64_t)c->element_count < 3 * n)
        {
            log_err("raster_to_nanovdb_from_arrays: attribute counts do not match means");
            return PNANOVDB_FALSE;
        }
        // raw inputs: the reference preprocesses them on the host in place
        // (RasterUtils.cpp:59-117); here the same arithmetic runs inside the prep
        // kernel and the caller's arrays are left untouched.
        vox_gaussians_t g;
        g.count = n;
        g.means = (const float*)m->data;
        g.quats = (const float*)q->data;
        g.scales = (const float*)s->data;
        g.opacities = (const float*)o->data;
        g.colors = (const float*)c->data;
        *out = run_host(queue, &g, voxel_size, 0.05f, VOX_FLAG_RAW_INPUTS | DROPIN_ORDER, nullptr, nullptr,
                        "raster_to_nanovdb_from_arrays");
        return *out ? PNANOVDB_TRUE : PNANOVDB_FALSE;
    });
}

static pnanovdb_bool_t PNANOVDB_ABI r_create_from_arrays(pnanovdb_raster_t*, const pnanovdb_compute_t*,
                                                         pnanovdb_compute_queue_t*, pnanovdb_compute_array_t**,
                                                         pnanovdb_uint32_t, pnanovdb_raster_gaussian_data_t**,
                                                         pnanovdb_raster_shader_params_t*,
                                                         pnanovdb_raster_context_t**);
static pnanovdb_bool_t PNANOVDB_ABI r_raster_file(pnanovdb_raster_t*, const pnanovdb_compute_t*,
                                                  pnanovdb_compute_queue_t*, const char*, float,
                                                  pnanovdb_compute_array_t**, pnanovdb_raster_gaussian_data_t**,
                                                  pnanovdb_raster_context_t**, pnanovdb_compute_array_t**,
                                                  pnanovdb_raster_shader_params_t*, pnanovdb_profiler_report_t,
                                                  void*);

static pnanovdb_bool_t PNANOVDB_ABI r_create_from_desc(pnanovdb_raster_t*, const pnanovdb_compute_t*,
                                                       pnanovdb_compute_queue_t*, const void*, const char*,
                                                       pnanovdb_raster_gaussian_data_t**,
                                                       pnanovdb_raster_shader_params_t*, pnanovdb_raster_context_t**)
{
    log_err("create_gaussian_data_from_desc: editor descriptors are not provided by this library");
    return PNANOVDB_FALSE;
}

#include "vox_npz.inl"

#include "vox_detmath.h"

namespace
{

// the reference's host activation of file arrays in ijkl_from_gaussians_file
// (raster/VoxelBVH.cpp:1474-1503): quaternions (w x y z) scaled by
// 1 / sqrt(x^2 + y^2 + z^2 + w^2), scales exp, opacities 1 / (1 + exp(-x)),
// one IEEE operation at a time; exp is vox_expf_cr (correctly rounded but
// for ties), the same exp the raster path's preprocessing uses
void vb_activate_host(int64_t n, float* quats, float* scales, float* opac)
{
    for (int64_t p = 0; p < n; p++)
    {
        const float x = quats[4 * p + 1], y = quats[4 * p + 2], z = quats[4 * p + 3], w = quats[4 * p + 0];
        const float ss = VOX_FADD(VOX_FADD(VOX_FADD(VOX_FMUL(x, x), VOX_FMUL(y, y)), VOX_FMUL(z, z)), VOX_FMUL(w, w));
        const float inv = VOX_FDIV(1.f, VOX_FSQRT(ss));
        quats[4 * p + 1] = VOX_FMUL(x, inv);
        quats[4 * p + 2] = VOX_FMUL(y, inv);
        quats[4 * p + 3] = VOX_FMUL(z, inv);
        quats[4 * p + 0] = VOX_FMUL(w, inv);
        for (int a = 0; a < 3; a++)
            scales[3 * p + a] = vox_expf_cr(scales[3 * p + a]);
        opac[p] = VOX_FDIV(1.f, VOX_FADD(1.f, vox_expf_cr(-opac[p])));
    }
}

} // namespace

static int vb_file_body(vox_context_t* ctx, const char* filename, uint32_t resolution, const float* transform,
                        pnanovdb_compute_array_t** ijkl_out, pnanovdb_compute_array_t** prim_id_out,
                        pnanovdb_compute_array_t** range_out, pnanovdb_compute_array_t** world_bbox_out,
                        pnanovdb_compute_array_t** gaussian_arrays_out, uint32_t gaussian_array_count)
{
    if (!ctx || !filename || !ijkl_out || !prim_id_out || !range_out || !world_bbox_out)
        return VOX_ERR_ARGS;
    *ijkl_out = *prim_id_out = *range_out = *world_bbox_out = nullptr;
    std::vector<NpzArray> arrays;
    std::string why;
    if (!read_gaussian_file(filename, arrays, why, true))
    {
        log_err((std::string("ijkl_from_gaussians_file: failed to load '") + filename + "': " + why).c_str());
        return VOX_ERR_ARGS;
    }
    // means, opacities, quaternions, scales, sh_0, sh_n (the reference's names and order)
    const char* names[6] = { "means", "opacities", "quaternions", "scales", "sh_0", "sh_n" };
    FloatBuf* a[6] = {};
    for (int i = 0; i < 6; i++)
        for (auto& x : arrays)
            if (x.name == names[i])
                a[i] = &x.data;
    for (int i = 0; i < 4; i++)
        if (!a[i])
        {
            log_err((std::string("ijkl_from_gaussians_file: '") + filename + "' has no array '" + names[i] + "'").c_str());
            return VOX_ERR_ARGS;
        }
    const int64_t n = (int64_t)a[1]->size(); // gaussian_count = opacities (VoxelBVH.cpp:1458)
    if ((int64_t)a[0]->size() < 3 * n || (int64_t)a[2]->size() < 4 * n || (int64_t)a[3]->size() < 3 * n)
    {
        log_err("ijkl_from_gaussians_file: attribute counts do not match the opacities");
        return VOX_ERR_ARGS;
    }
    vb_activate_host(n, a[2]->data(), a[3]->data(), a[1]->data());

    // device copies on the context's stream, outputs back to page-locked arrays
    cudaStream_t s = (cudaStream_t)vox_context_stream(ctx);
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t b_means = 12 * (size_t)n, b_op = 4 * (size_t)n, b_q = 16 * (size_t)n, b_s = 12 * (size_t)n;
    const size_t b_k = 64 * (size_t)n, b_id = 32 * (size_t)n, b_r = 64 * (size_t)n, b_box = 24;
    const size_t total = al(b_means) + al(b_op) + al(b_q) + al(b_s) + al(b_k) + al(b_id) + al(b_r) + al(b_box);
    char* base = nullptr;
    if (cudaMalloc(&base, total) != cudaSuccess)
    {
        cudaGetLastError();
        log_err("ijkl_from_gaussians_file: out of device memory");
        return VOX_ERR_MEMORY;
    }
    char* p = base;
    float* d_means = (float*)p;
    p += al(b_means);
    float* d_op = (float*)p;
    p += al(b_op);
    float* d_q = (float*)p;
    p += al(b_q);
    float* d_s = (float*)p;
    p += al(b_s);
    uint64_t* d_k = (uint64_t*)p;
    p += al(b_k);
    uint32_t* d_id = (uint32_t*)p;
    p += al(b_id);
    uint32_t* d_r = (uint32_t*)p;
    p += al(b_r);
    float* d_box = (float*)p;
    cudaMemcpyAsync(d_means, a[0]->data(), b_means, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_op, a[1]->data(), b_op, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_q, a[2]->data(), b_q, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_s, a[3]->data(), b_s, cudaMemcpyHostToDevice, s);
    int rc = vox_voxelbvh_ijkl_from_gaussians(ctx, d_means, d_op, d_q, d_s, n, resolution, transform, d_k, d_id, d_r,
                                              d_box, nullptr);
    pnanovdb_compute_array_t* out[4] = { array_create_pinned(8, 8 * (uint64_t)n), array_create_pinned(4, 8 * (uint64_t)n),
                                         array_create_pinned(8, 8 * (uint64_t)n), array_create_pinned(4, 6) };
    if (rc == VOX_OK && !(out[0] && out[1] && out[2] && out[3]))
        rc = VOX_ERR_MEMORY;
    if (rc == VOX_OK)
    {
        cudaMemcpyAsync(out[0]->data, d_k, b_k, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(out[1]->data, d_id, b_id, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(out[2]->data, d_r, b_r, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(out[3]->data, d_box, b_box, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess)
            rc = VOX_ERR_CUDA;
    }
    cudaFree(base);
    if (rc != VOX_OK)
    {
        for (auto* x : out)
            array_destroy(x);
        return rc;
    }
    *ijkl_out = out[0];
    *prim_id_out = out[1];
    *range_out = out[2];
    *world_bbox_out = out[3];
    // the activated arrays, as the reference hands them back
    if (gaussian_arrays_out)
        for (uint32_t i = 0; i < gaussian_array_count && i < 6; i++)
            gaussian_arrays_out[i] = a[i] ? array_create(4, a[i]->size(), a[i]->data()) : array_create(4, 0, nullptr);
    return VOX_OK;
}

extern "C" {

int vox_voxelbvh_ijkl_from_gaussians_file(vox_context_t* ctx, const char* filename, uint32_t resolution,
                                          const float* transform, pnanovdb_compute_array_t** ijkl_out,
                                          pnanovdb_compute_array_t** prim_id_out, pnanovdb_compute_array_t** range_out,
                                          pnanovdb_compute_array_t** world_bbox_out,
                                          pnanovdb_compute_array_t** gaussian_arrays_out,
                                          uint32_t gaussian_array_count)
{
    return no_throw<int>("ijkl_from_gaussians_file", VOX_ERR_MEMORY, [&]() {
        return vb_file_body(ctx, filename, resolution, transform, ijkl_out, prim_id_out, range_out, world_bbox_out,
                            gaussian_arrays_out, gaussian_array_count);
    });
}

pnanovdb_compute_t* pnanovdb_get_compute(void)
{
    static pnanovdb_compute_t t;
    static bool init = false;
    if (!init)
    {
        memset(&t, 0, sizeof(t));
        t.device_interface.create_device_manager = dev_create_manager;
        t.device_interface.destroy_device_manager = dev_destroy_manager;
        t.device_interface.enumerate_devices = dev_enumerate;
        t.device_interface.create_device = dev_create;
        t.device_interface.destroy_device = dev_destroy;
        t.device_interface.get_device_queue = dev_queue;
        t.device_interface.get_compute_queue = dev_compute_queue;
        t.device_interface.flush = dev_flush;
        t.device_interface.wait_idle = dev_wait_idle;
        t.device_interface.get_device_index = dev_index;
        t.load_nanovdb = load_grid;
        t.save_nanovdb = save_grid;
        t.create_array = array_create;
        t.destroy_array = array_destroy;
        t.map_array = array_map;
        t.unmap_array = array_unmap;
        t.duplicate_array = array_duplicate;
        init = true;
    }
    return &t;
}

pnanovdb_compute_device_interface_t* pnanovdb_get_compute_device_interface(uint32_t)
{
    return &pnanovdb_get_compute()->device_interface;
}

pnanovdb_compute_shader_interface_t* pnanovdb_get_compute_shader_interface(void)
{
    return &pnanovdb_get_compute()->shader_interface;
}

pnanovdb_fileformat_t* pnanovdb_get_fileformat(void)
{
    static pnanovdb_fileformat_t t = { nullptr, ff_can_load_file, ff_load_file, nullptr };
    return &t;
}

pnanovdb_raster_t* pnanovdb_get_raster(void)
{
    static pnanovdb_raster_t r;
    static bool init = false;
    if (!init)
    {
        memset(&r, 0, sizeof(r));
        r.compute = pnanovdb_get_compute();
        r.create_context = r_create_context;
        r.destroy_context = r_destroy_context;
        r.create_gaussian_data = r_create_gaussian_data;
        r.upload_gaussian_data = r_upload_gaussian_data;
        r.destroy_gaussian_data = r_destroy_gaussian_data;
        r.raster_gaussian_2d = r_raster_gaussian_2d;
        r.raster_gaussian_3d = r_raster_gaussian_3d;
        r.raster_to_nanovdb = r_raster_to_nanovdb;
        r.raster_file = r_raster_file;
        r.raster_to_nanovdb_from_arrays = r_from_arrays;
        r.create_gaussian_data_from_arrays = r_create_from_arrays;
        r.create_gaussian_data_from_desc = r_create_from_desc;
        init = true;
    }
    return &r;
}

} // extern "C"
