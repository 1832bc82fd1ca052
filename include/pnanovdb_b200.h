/*
 * pnanovdb_b200.h - C ABI of the B200 Gaussian -> NanoVDB (node2) voxelizer.
 *
 * Drop-in boundary: libpnanovdbcompute.so exports pnanovdb_get_raster() and
 * pnanovdb_get_compute(), whose tables are layout-compatible with the
 * reference's pnanovdb_raster_t (nanovdb_editor/putil/Raster.h:58-174) and
 * pnanovdb_compute_t (nanovdb_editor/putil/Compute.h:784-853), so the
 * reference's ctypes binding (pymodule/nanovdb_editor/raster.py:14-168,
 * compute.py:109-217) binds them unchanged.  Vulkan handles are replaced by
 * headless CUDA ones: a queue is a CUDA stream on one device and a
 * pnanovdb_compute_buffer_t is a device pointer plus a size.
 *
 * Below the drop-in table are the library's own vox_* entry points (device
 * pointers in, node2 grid out), which the table is built on and which the
 * Python autograd path calls directly.
 *
 * Calling convention: cdecl (PNANOVDB_ABI is empty on Linux,
 * nanovdb_editor/putil/Reflect.h:28-32).  No exceptions cross this boundary;
 * failures return PNANOVDB_FALSE / NULL / a negative vox status and log.
 */
#ifndef PNANOVDB_B200_H
#define PNANOVDB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef PNANOVDB_ABI
#define PNANOVDB_ABI
#endif
#ifndef PNANOVDB_API
#define PNANOVDB_API __attribute__((visibility("default")))
#endif

typedef uint32_t pnanovdb_uint32_t;
typedef uint64_t pnanovdb_uint64_t;
typedef int32_t pnanovdb_int32_t;
typedef int32_t pnanovdb_bool_t; /* bound as c_int32 by raster.py:126 */
#define PNANOVDB_TRUE 1
#define PNANOVDB_FALSE 0

/* --------------------------------------------------------------- arrays -- */
/* nanovdb_editor/putil/Compute.h:765-771 */
typedef struct pnanovdb_compute_array_t
{
    void* data;
    pnanovdb_uint64_t element_size;
    pnanovdb_uint64_t element_count;
    const char* filepath;
} pnanovdb_compute_array_t;

/* headless device buffer (replaces the opaque Vulkan buffer of
 * nanovdb_editor/putil/Compute.h:101) */
typedef struct pnanovdb_compute_buffer_t
{
    void* device_ptr;
    pnanovdb_uint64_t size_bytes;
} pnanovdb_compute_buffer_t;

/* a queue: one CUDA stream on one device (replaces Compute.h's Vulkan queue) */
typedef struct pnanovdb_compute_queue_t pnanovdb_compute_queue_t;
typedef struct pnanovdb_compute_device_t pnanovdb_compute_device_t;

/* nanovdb_editor/putil/Compute.h:546-551, :561-564 */
typedef struct pnanovdb_compute_profiler_entry_t
{
    const char* label;
    float cpu_delta_time;
    float gpu_delta_time;
} pnanovdb_compute_profiler_entry_t;
typedef void(PNANOVDB_ABI* pnanovdb_profiler_report_t)(void* userdata, pnanovdb_uint64_t capture_id,
                                                       pnanovdb_uint32_t num_entries,
                                                       pnanovdb_compute_profiler_entry_t* entries);

/* ------------------------------------------------------ compute table -- */
/* Layout of nanovdb_editor/putil/Compute.h:566-661: 1 + 33 pointers.  The
 * entries this library implements are named; the rest are NULL. */
typedef struct pnanovdb_compute_device_interface_t
{
    const void* interface_pnanovdb_reflect_data_type;
    void* (PNANOVDB_ABI* create_device_manager)(pnanovdb_bool_t enable_validation_on_debug_build);
    void(PNANOVDB_ABI* destroy_device_manager)(void* manager);
    pnanovdb_bool_t(PNANOVDB_ABI* enumerate_devices)(void* manager, pnanovdb_uint32_t device_index, void* p_desc);
    pnanovdb_compute_device_t*(PNANOVDB_ABI* create_device)(void* manager, const void* desc);
    void(PNANOVDB_ABI* destroy_device)(void* manager, pnanovdb_compute_device_t* device);
    void* reserved_get_memory_stats;
    void* reserved_semaphore[4];
    pnanovdb_compute_queue_t*(PNANOVDB_ABI* get_device_queue)(const pnanovdb_compute_device_t* device);
    pnanovdb_compute_queue_t*(PNANOVDB_ABI* get_compute_queue)(const pnanovdb_compute_device_t* device);
    int(PNANOVDB_ABI* flush)(pnanovdb_compute_queue_t* queue, pnanovdb_uint64_t* flushed_frame, void* wait_semaphore,
                             void* signal_semaphore);
    void* reserved_frames[2];
    void(PNANOVDB_ABI* wait_idle)(pnanovdb_compute_queue_t* queue);
    void* reserved_interface[2];
    void* reserved_swapchain[5];
    void* reserved_encoder[6];
    void* reserved_profiler[3];
    pnanovdb_uint32_t(PNANOVDB_ABI* get_device_index)(const pnanovdb_compute_device_t* device);
} pnanovdb_compute_device_interface_t;

/* nanovdb_editor/putil/Compute.h:734-745 */
typedef struct pnanovdb_compute_shader_interface_t
{
    const void* interface_pnanovdb_reflect_data_type;
    void* reserved[3];
} pnanovdb_compute_shader_interface_t;

/* nanovdb_editor/putil/Compute.h:784-853 */
typedef struct pnanovdb_compute_t
{
    const void* interface_pnanovdb_reflect_data_type;
    void* module;
    const void* compiler;
    pnanovdb_compute_shader_interface_t shader_interface;
    pnanovdb_compute_device_interface_t device_interface;
    pnanovdb_compute_array_t*(PNANOVDB_ABI* load_nanovdb)(const char* filepath);
    pnanovdb_bool_t(PNANOVDB_ABI* save_nanovdb)(pnanovdb_compute_array_t* array, const char* filepath);
    void* reserved_shader[5]; /* create_shader_context .. dispatch_shader */
    void* reserved_dispatch[2];
    pnanovdb_compute_array_t*(PNANOVDB_ABI* create_array)(size_t element_size, pnanovdb_uint64_t element_count,
                                                          const void* data);
    void(PNANOVDB_ABI* destroy_array)(pnanovdb_compute_array_t* array);
    void*(PNANOVDB_ABI* map_array)(pnanovdb_compute_array_t* array);
    void(PNANOVDB_ABI* unmap_array)(pnanovdb_compute_array_t* array);
    void* reserved_print_range;
    void* reserved_from_image;
    pnanovdb_compute_array_t*(PNANOVDB_ABI* duplicate_array)(pnanovdb_compute_array_t* array);
} pnanovdb_compute_t;

/* ------------------------------------------------------- raster table -- */
typedef struct pnanovdb_raster_context_t pnanovdb_raster_context_t;
typedef struct pnanovdb_raster_gaussian_data_t pnanovdb_raster_gaussian_data_t;

/* nanovdb_editor/putil/Raster.h:26-34 */
typedef struct pnanovdb_raster_shader_params_t
{
    float eps2d;
    float min_radius_2d;
    pnanovdb_uint32_t tile_size;
    pnanovdb_int32_t sh_degree_override;
    pnanovdb_uint32_t sh_stride_rgbrgbrgb_override;
    const void* data_type;
    const char* name;
} pnanovdb_raster_shader_params_t;

/* index of gaussian_frag_color's parameter block in shader_params_arrays
 * (nanovdb_editor/putil/Raster.h:216-235); its first two 32-bit words are
 * cull_scale (float) and use_default (bool32), gaussian_frag_color.slang:21-28 */
#define PNANOVDB_RASTER_SHADER_GAUSSIAN_FRAG_COLOR 1

/* nanovdb_editor/putil/Raster.h:58-174, field order preserved */
typedef struct pnanovdb_raster_t
{
    const void* interface_pnanovdb_reflect_data_type;
    const pnanovdb_compute_t* compute;
    pnanovdb_raster_context_t*(PNANOVDB_ABI* create_context)(const pnanovdb_compute_t* compute,
                                                             pnanovdb_compute_queue_t* queue);
    void(PNANOVDB_ABI* destroy_context)(const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue,
                                        pnanovdb_raster_context_t* context);
    pnanovdb_raster_gaussian_data_t*(PNANOVDB_ABI* create_gaussian_data)(
        const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue, pnanovdb_raster_context_t* context,
        pnanovdb_compute_array_t* means, pnanovdb_compute_array_t* quaternions, pnanovdb_compute_array_t* scales,
        pnanovdb_compute_array_t* colors, pnanovdb_compute_array_t* sh_0, pnanovdb_compute_array_t* sh_n,
        pnanovdb_compute_array_t* opacities, pnanovdb_compute_array_t** shader_params_arrays,
        pnanovdb_raster_shader_params_t* raster_params);
    void(PNANOVDB_ABI* upload_gaussian_data)(const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue,
                                             pnanovdb_raster_context_t* context, pnanovdb_raster_gaussian_data_t* data);
    void(PNANOVDB_ABI* destroy_gaussian_data)(const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue,
                                              pnanovdb_raster_gaussian_data_t* data);
    void(PNANOVDB_ABI* raster_gaussian_2d)(const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue,
                                           pnanovdb_raster_context_t* context, pnanovdb_raster_gaussian_data_t* data,
                                           void* color_2d, pnanovdb_uint32_t image_width,
                                           pnanovdb_uint32_t image_height, const void* view, const void* projection,
                                           const pnanovdb_raster_shader_params_t* shader_params,
                                           pnanovdb_uint32_t composite);
    void(PNANOVDB_ABI* raster_gaussian_3d)(const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue,
                                           pnanovdb_raster_context_t* context, float voxel_size,
                                           pnanovdb_raster_gaussian_data_t* data,
                                           pnanovdb_compute_buffer_t* nanovdb_out,
                                           pnanovdb_uint64_t nanovdb_word_count, void* userdata);
    pnanovdb_compute_array_t*(PNANOVDB_ABI* raster_to_nanovdb)(
        const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue, float voxel_size,
        pnanovdb_compute_array_t* means, pnanovdb_compute_array_t* quaternions, pnanovdb_compute_array_t* scales,
        pnanovdb_compute_array_t* colors, pnanovdb_compute_array_t* sh_0, pnanovdb_compute_array_t* sh_n,
        pnanovdb_compute_array_t* opacities, pnanovdb_compute_array_t** shader_params_arrays,
        pnanovdb_profiler_report_t profiler_report, void* userdata);
    pnanovdb_bool_t(PNANOVDB_ABI* raster_file)(struct pnanovdb_raster_t* raster, const pnanovdb_compute_t* compute,
                                               pnanovdb_compute_queue_t* queue, const char* filename,
                                               float voxel_size, pnanovdb_compute_array_t** nanovdb_arr,
                                               pnanovdb_raster_gaussian_data_t** gaussian_data,
                                               pnanovdb_raster_context_t** raster_context,
                                               pnanovdb_compute_array_t** shader_params_arrays,
                                               pnanovdb_raster_shader_params_t* raster_params,
                                               pnanovdb_profiler_report_t profiler_report, void* userdata);
    pnanovdb_bool_t(PNANOVDB_ABI* raster_to_nanovdb_from_arrays)(struct pnanovdb_raster_t* raster,
                                                                 const pnanovdb_compute_t* compute,
                                                                 pnanovdb_compute_queue_t* queue, float voxel_size,
                                                                 pnanovdb_compute_array_t** arrays_gaussian,
                                                                 pnanovdb_uint32_t array_count,
                                                                 pnanovdb_compute_array_t** out_nanovdb_arr);
    pnanovdb_bool_t(PNANOVDB_ABI* create_gaussian_data_from_arrays)(
        struct pnanovdb_raster_t* raster, const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue,
        pnanovdb_compute_array_t** arrays_gaussian, pnanovdb_uint32_t array_count,
        pnanovdb_raster_gaussian_data_t** gaussian_data, pnanovdb_raster_shader_params_t* raster_params,
        pnanovdb_raster_context_t** raster_context);
    pnanovdb_bool_t(PNANOVDB_ABI* create_gaussian_data_from_desc)(
        struct pnanovdb_raster_t* raster, const pnanovdb_compute_t* compute, pnanovdb_compute_queue_t* queue,
        const void* desc, const char* name, pnanovdb_raster_gaussian_data_t** gaussian_data,
        pnanovdb_raster_shader_params_t* raster_params, pnanovdb_raster_context_t** raster_context);
} pnanovdb_raster_t;

/* replaces raster/Raster.cpp:822-840 */
PNANOVDB_API pnanovdb_raster_t* pnanovdb_get_raster(void);
/* replaces the compute table the reference builds in compute/Compute.cpp */
PNANOVDB_API pnanovdb_compute_t* pnanovdb_get_compute(void);
/* the device interface inside that table (vulkan/PublicDeviceVulkan.cpp:114,
 * declared at nanovdb_editor/putil/Compute.h:705): a CUDA device and its
 * queues, whatever `api` asks for (0 = Vulkan is the only value the
 * reference defines) */
PNANOVDB_API pnanovdb_compute_device_interface_t* pnanovdb_get_compute_device_interface(uint32_t api);
/* the shader interface inside that table (compute/ComputeShader.cpp:173,
 * Compute.h:758): no Slang shaders here, every entry is NULL */
PNANOVDB_API pnanovdb_compute_shader_interface_t* pnanovdb_get_compute_shader_interface(void);

/* ------------------------------------------------------- file formats -- */
/* Layout of pnanovdb_fileformat_t (nanovdb_editor/putil/FileFormat.h:19-36,
 * without the optional e57 entry).  load_file fills out_arrays[i] with the
 * float32 array named array_names[i] ("means", "opacities", "quaternions",
 * "scales", "sh_0", "sh_n", "colors"; NULL when the file has none), each freed
 * with the compute table's destroy_array, and returns FALSE when the file
 * cannot be read or lacks one of the arrays (fileformat/FileFormat.cpp:87-205,
 * :754-800).  Formats: .npz (stored or deflated entries; an "sh" array of
 * shape (G, K, 3) stands for sh_0 / sh_n) and binary .ply. */
typedef struct pnanovdb_fileformat_t
{
    void* interface_pnanovdb_reflect_data_type;
    pnanovdb_bool_t(PNANOVDB_ABI* can_load_file)(const char* filename);
    pnanovdb_bool_t(PNANOVDB_ABI* load_file)(const char* filename, pnanovdb_uint32_t array_count,
                                             const char** array_names, pnanovdb_compute_array_t** out_arrays);
    void* module;
} pnanovdb_fileformat_t;

/* replaces fileformat/FileFormat.cpp:803-811 (libpnanovdbfileformat) */
PNANOVDB_API pnanovdb_fileformat_t* pnanovdb_get_fileformat(void);

/* ------------------------------------------------------ grid container -- */
/* The grid buffer this library produces.  The reference returns a NanoVDB
 * grid whose GridData/TreeData headers come from PNanoVDB.h, which the
 * reference does not vendor; this header stands in for them and everything
 * from node2_offset on is the reference's node2 layout: the root node
 * (541728 B) followed by every node at its node2 maximum size in node_idx
 * order (upper 274464 B, lower 34336 B, leaf 128 B; PNanoVDBExt.h:49-64),
 * child links as byte offsets relative to the parent.  The blind data that
 * grid_build_blindmetadata.slang appends follow: the bbox (two int32x3,
 * inclusive voxel coordinates) and per-value arrays indexed by value index
 * (two background slots first): RGBA8 as the reference computes it, float
 * density = sum of per-pair alpha (an exact 64-bit fixed-point sum of the
 * terms rounded to 2^-32, rounded once to float, so independent of order),
 * and Vec3f colour = alpha-weighted mean RGB.  density_offset = color_offset
 * = 0 marks a grid copied without the float channels. */
#define VOX_GRID_MAGIC 0x32454E58564F5642ull /* "BVOXNE2" */
#define VOX_GRID_HEADER_BYTES 256u

typedef struct vox_grid_header_t
{
    uint64_t magic;
    uint32_t version;
    uint32_t header_bytes;
    uint64_t grid_bytes;
    uint64_t node2_offset;
    uint64_t node2_bytes;
    uint32_t upper_count;
    uint32_t lower_count;
    uint32_t leaf_count;
    uint32_t node_order; /* 0: one fragment window, 1: reference 256K x 8M windows */
    uint64_t value_count; /* 2 + active voxels */
    uint64_t bbox_offset;
    uint64_t rgba8_offset;
    uint64_t density_offset;
    uint64_t color_offset;
    float voxel_size;
    int32_t bbox[6];
    uint32_t pad0;
    uint64_t pair_count;
    uint64_t candidate_count;
    uint8_t reserved[256 - 144];
} vox_grid_header_t;

/* --------------------------------------------------- vox_* entry points -- */
typedef struct vox_context_t vox_context_t;

/* flags for vox_voxelize */
#define VOX_FLAG_RAW_INPUTS 1u     /* log scales, logit opacities, raw quaternions, SH0 colours */
#define VOX_FLAG_WINDOW_ORDER 2u   /* node_idx order of the reference's fragment windows */
/* differentiable channels: density = sum over the pairs of
 * K = max(op exp(-|S^-1 R^T (x - mu)|^2 / 2) - 0.01, 0) at the voxel centre x,
 * colour = sum K rgb (premultiplied); RGBA8 stays the reference's
 * (gaussian_frag_color.slang:182-246).  Keeps what vox_backward needs. */
#define VOX_FLAG_DIFFERENTIABLE 4u
/* every attribute array holds bfloat16 values (2 bytes each, same layouts);
 * they are read exactly as float and all arithmetic stays FP32 / FP64 (the
 * batched fitting loop's storage format; no counterpart in the reference) */
#define VOX_FLAG_BF16_INPUTS 8u

/* status codes */
#define VOX_OK 0
#define VOX_ERR_ARGS -1
#define VOX_ERR_CUDA -2
#define VOX_ERR_MEMORY -3
#define VOX_ERR_RANGE -4      /* voxel coordinate outside [-65536, 65535] */
#define VOX_ERR_FOOTPRINT -5  /* one Gaussian covers >= 2^31 candidate voxels */
#define VOX_ERR_TIMEOUT -6    /* a bounded device wait expired */
#define VOX_ERR_SIZE -7       /* caller buffer too small */

typedef struct vox_gaussians_t
{
    const float* means;     /* [n][3] */
    const float* quats;     /* [n][4] w, x, y, z */
    const float* scales;    /* [n][3] (log scales with VOX_FLAG_RAW_INPUTS) */
    const float* opacities; /* [n] (logits with VOX_FLAG_RAW_INPUTS) */
    const float* colors;    /* [n][3] RGB (SH0 coefficients with VOX_FLAG_RAW_INPUTS) */
    int64_t count;
} vox_gaussians_t;

typedef struct vox_stats_t
{
    int64_t gaussians, candidates, pairs, voxels, uppers, lowers, leaves, value_count;
    int64_t grid_bytes;
    int32_t key_bits;
    int32_t sort_passes;
    float ms_prep, ms_emit, ms_sort, ms_build, ms_accumulate, ms_total;
    int64_t kernel_launches; /* kernels this library launched in the call */
    float ms_backward;       /* last vox_backward */
    int32_t sort_shape;      /* the sort's tuned candidate: 0-4 onesweep tile shapes, 5-9 the same as three-kernel passes */
    int64_t leaf_pairs;      /* (leaf, Gaussian) pairs sorted */
    int64_t candidate_leaves; /* leaves walked (some end up empty) */
    /* last vox_voxelbvh_ijkl_from_gaussians */
    float ms_vb_keys;     /* world box + level search + keys */
    float ms_vb_sort;     /* key compression + radix sort */
    float ms_vb_ranges;   /* range headers + 64-bit key write-back */
    int32_t vb_sort_bits; /* key bits sorted (compressed key width, or 64) */
    int64_t vb_launches;  /* kernels launched by that call */
    /* the online tuner's choices (variants give identical results) */
    int32_t walk_ctas_per_sm; /* leaf walk: resident CTAs per SM it ran with */
    int32_t vb_search;        /* VoxelBVH level search: 0 lane-balanced, 1 thread per Gaussian */
} vox_stats_t;

/* One context per caller thread; it owns a CUDA stream on `device` and a
 * device arena that grows to the largest workload seen. */
PNANOVDB_API vox_context_t* vox_context_create(int device);
PNANOVDB_API void vox_context_destroy(vox_context_t* ctx);
PNANOVDB_API void* vox_context_stream(vox_context_t* ctx);
PNANOVDB_API const char* vox_last_error(vox_context_t* ctx);

/* Bounded device waits.  The single-pass scans, the onesweep sort and the run
 * detection wait on their predecessor tiles (decoupled look-back); every such
 * wait gives up after a bounded number of polls, records the failure and lets
 * the kernel finish, and the call returns VOX_ERR_TIMEOUT with the context
 * still usable.  This sets that bound for later calls on ctx: max_polls polls
 * per wait (VOX_WAIT_DEFAULT restores the default of 2^22 polls of >= 32 ns);
 * withhold_publication != 0 also stops those calls' tiles from publishing, so
 * every wait runs out - a test of the error path (no counterpart in the
 * reference, whose Vulkan dispatches have no inter-workgroup waits). */
#define VOX_WAIT_DEFAULT 0xffffffffu
PNANOVDB_API int vox_context_set_wait_limit(vox_context_t* ctx, uint32_t max_polls, int withhold_publication);

/* Voxelizes device-resident Gaussians (the path of raster_gaussian_3d,
 * raster/Raster.cpp:420-558).  On success *grid (device) points at the
 * context-owned grid buffer (valid until the next call) and *grid_bytes is
 * its size.  cull_scale <= 0 selects 0.05 (gaussian_frag_color.slang:205). */
PNANOVDB_API int vox_voxelize(vox_context_t* ctx, const vox_gaussians_t* gaussians, float voxel_size,
                              float cull_scale, uint32_t flags, void** grid, uint64_t* grid_bytes);

/* Same from host arrays, with the grid copied to host memory (`out`,
 * `out_capacity` bytes); copies are counted in the call. */
PNANOVDB_API int vox_voxelize_host(vox_context_t* ctx, const vox_gaussians_t* gaussians, float voxel_size,
                                   float cull_scale, uint32_t flags, void* out, uint64_t out_capacity,
                                   uint64_t* grid_bytes);

/* Batched form: `clouds` independent clouds in one call, cloud b = Gaussians
 * [cloud_start[b], cloud_start[b + 1]) of `gaussians` with its own voxel size
 * voxel_sizes[b] (host arrays, clouds + 1 and clouds entries).  The cloud
 * index is the most significant part of every sort key, so one emit / sort /
 * build / accumulate chain serves all clouds.  *grids (device, context-owned)
 * holds one self-contained grid per cloud, cloud b at byte offset
 * grid_offsets[b] (host, clouds + 1 entries, the last = total bytes); each is
 * laid out exactly as the single-cloud grid.  value_offsets (host, clouds + 1,
 * may be NULL) receives where each cloud's values start when the clouds'
 * value arrays are concatenated (the layout of vox_backward's upstream arrays
 * after a batched call). */
#define VOX_MAX_CLOUDS 4096
PNANOVDB_API int vox_voxelize_batch(vox_context_t* ctx, const vox_gaussians_t* gaussians, int64_t clouds,
                                    const int64_t* cloud_start, const float* voxel_sizes, float cull_scale,
                                    uint32_t flags, void** grids, uint64_t* grid_offsets, uint64_t* value_offsets);

/* Copies the grid of the last vox_voxelize / vox_voxelize_host call to host
 * or device memory (`capacity` bytes). */
PNANOVDB_API int vox_copy_grid(vox_context_t* ctx, void* out, uint64_t capacity);

/* The part of the last single-cloud grid that the reference's raster entries
 * return (raster/Raster.cpp:636-668: node2 tree and RGBA8 values): header,
 * node2 region, bbox and RGBA8 array, copied to host or device memory; the
 * copied header has grid_bytes = *bytes and density_offset = color_offset = 0
 * (the float channels stay in the context's grid, vox_copy_grid).  With
 * out = NULL only *bytes is set.  The drop-in raster entries return this. */
PNANOVDB_API int vox_copy_grid_rgba8(vox_context_t* ctx, void* out, uint64_t capacity, uint64_t* bytes);

/* Sorted (voxel, Gaussian) pairs of the last vox_voxelize call: hierarchical
 * 64-bit keys (root_n << 36 | upper_n << 21 | lower_n << 9 | leaf_n) and
 * Gaussian ids, in (key, id) order, copied to host memory. */
PNANOVDB_API int vox_copy_pairs(vox_context_t* ctx, uint64_t* keys, uint32_t* ids, int64_t capacity);

PNANOVDB_API void vox_get_stats(vox_context_t* ctx, vox_stats_t* out);

/* Coordinates (i, j, k) of the active voxels of the last call, row r for value
 * index r (clouds' value arrays back to back after a batched call; the two
 * background rows of every cloud are not written), to DEVICE memory
 * d_ijk [capacity][3], capacity >= the total value count. */
PNANOVDB_API int vox_voxel_coords(vox_context_t* ctx, int32_t* d_ijk, int64_t capacity);

/* Adjoint of the differentiable channels of the context's last call, which
 * must have been a successful vox_voxelize with VOX_FLAG_DIFFERENTIABLE (the
 * reference has no adjoint; this differentiates the forward above).
 * `gaussians`: the forward's inputs (device).  grad_density [value_count] and
 * grad_color [value_count][3] are dL/d channel, indexed like the grid's
 * channels (either may be NULL = zero).  Outputs (device, any may be NULL):
 * dL/d means [n][3], quats [n][4] (w, x, y, z), scales [n][3], opacities [n],
 * colors [n][3], with respect to the inputs as given (with VOX_FLAG_RAW_INPUTS:
 * the raw quaternion before normalisation, log scales, opacity logits, SH0). */
PNANOVDB_API int vox_backward(vox_context_t* ctx, const vox_gaussians_t* gaussians, const float* grad_density,
                              const float* grad_color, float* grad_means, float* grad_quats, float* grad_scales,
                              float* grad_opacities, float* grad_colors);

/* ---------------------------------------------------- parallel primitives --
 * The primitives the path is built on, on device pointers, ordered on the
 * context's stream and synchronised before returning. */

/* replaces pnanovdb_parallel_primitives_t::global_scan_uint64
 * (nanovdb_editor/putil/ParallelPrimitives.h:41-47, raster/ParallelPrimitives.cpp:151-310):
 * scan of n u64 values d_in -> d_out (may alias), inclusive when `inclusive`
 * is non-zero (the reference's scan is inclusive), else exclusive; *d_total
 * (device) receives the sum. */
PNANOVDB_API int vox_global_scan_u64(vox_context_t* ctx, const uint64_t* d_in, uint64_t* d_out, int64_t n,
                                     int inclusive, uint64_t* d_total);

/* replaces pnanovdb_parallel_primitives_t::global_scan
 * (nanovdb_editor/putil/ParallelPrimitives.h:33-39, raster/ParallelPrimitives.cpp:276-286):
 * scan of n uint32 values, sums wrapping mod 2^32, inclusive when `inclusive`
 * is non-zero (the reference's), else exclusive; *d_total (device, may be
 * NULL) receives the sum mod 2^32.  The reference's dispatch_count repeats
 * the same scan and has no counterpart. */
PNANOVDB_API int vox_global_scan_u32(vox_context_t* ctx, const uint32_t* d_in, uint32_t* d_out, int64_t n,
                                     int inclusive, uint32_t* d_total);

/* replaces pnanovdb_parallel_primitives_t::global_scan_max
 * (ParallelPrimitives.h:49-55, ParallelPrimitives.cpp:300-310): inclusive
 * running maximum of n uint32 values. */
PNANOVDB_API int vox_global_scan_max_u32(vox_context_t* ctx, const uint32_t* d_in, uint32_t* d_out, int64_t n);

/* replaces pnanovdb_parallel_primitives_t::radix_sort
 * (ParallelPrimitives.h:57-64, ParallelPrimitives.cpp:347-525): stable sort
 * of n (32-bit key, 32-bit value) device pairs in place by key bits
 * [0, key_bit_count); higher key bits take no part in the order. */
PNANOVDB_API int vox_radix_sort_u32(vox_context_t* ctx, uint32_t* d_keys, uint32_t* d_vals, int64_t n,
                                    uint32_t key_bit_count);

/* replaces pnanovdb_parallel_primitives_t::radix_sort_dual_key
 * (ParallelPrimitives.h:66-75, ParallelPrimitives.cpp:527-683), the tile sort
 * of raster_gaussian_2d (raster/Raster2D.cpp:495-506): stable sort of n
 * (low key, high key, value) uint32 triples in place by (high key bits
 * [0, key_high_bit_count), low key bits [0, key_low_bit_count)). */
PNANOVDB_API int vox_radix_sort_dual_key(vox_context_t* ctx, uint32_t* d_keys_low, uint32_t* d_keys_high,
                                         uint32_t* d_vals, int64_t n, uint32_t key_low_bit_count,
                                         uint32_t key_high_bit_count);

/* replaces pnanovdb_parallel_primitives_t::radix_sort_key64
 * (nanovdb_editor/putil/ParallelPrimitives.h:77-84, raster/ParallelPrimitives.cpp:685-869):
 * stable sort of n (64-bit key, 32-bit value) device pairs in place by key
 * bits [0, key_bit_count); higher key bits take no part in the order. */
PNANOVDB_API int vox_radix_sort_key64(vox_context_t* ctx, uint64_t* d_keys, uint32_t* d_vals, int64_t n,
                                      uint32_t key_bit_count);

/* ------------------------------------------------ VoxelBVH ingestion -- */

/* replaces ijkl_from_gaussians (raster/VoxelBVH.cpp:1225-1435; the device
 * half of ijkl_from_gaussians_file, :1437-1575, after its host activation):
 * for `count` activated Gaussians on the device (means [count][3], opacities
 * [count], quaternions [count][4] as w x y z, scales [count][3]; the
 * reference's sh0 / shn buffers play no part in this step):
 *   d_world_bbox [6]      the box of every Gaussian's transformed
 *                         sqrt(2 ln(max(op, 0.01) / 0.01))-sigma cube
 *                         (min xyz, max xyz);
 *   d_ijkl [8 count]      per Gaussian the cells of the finest level
 *                         (0..11, cells of edge 2^level in a grid of
 *                         `resolution` voxels over the box's longest side)
 *                         at which at most 8 cells overlap its ellipsoid, as
 *                         i << 48 | j << 32 | k << 16 | level, unused slots
 *                         ~0; sorted (stable) with
 *   d_prim_id [8 count]   the Gaussian index of each key (~0 for unused);
 *   d_range [16 count]    [2 r] = first, [2 r + 1] = one past the last sorted
 *                         position of the r-th distinct key, zeros after the
 *                         last range;
 *   *range_count (host, may be NULL) the number of ranges.
 * `transform` (host, 16 floats or NULL for the identity) is the reference's
 * transform_floats: the rows x y z w of a pnanovdb_camera_mat_t applied to row
 * vectors, p' = [p 1] M; its inverse is taken in double precision
 * (vox_voxelbvh_transform_inverse) and rounded to float.  count <= 2^29 - 1
 * (8 count positions index in 32 bits), 1 <= resolution <= 4096 (the
 * reference's PNANOVDB_VOXELBVH_MAX_RESOLUTION), d_ijkl and
 * d_prim_id 16-byte aligned.  A Gaussian whose box is not finite or maps
 * outside [-65536, 65536] voxels (a zero-size world box) returns
 * VOX_ERR_RANGE; the outputs are then undefined.  Ordered on the context's stream; returns after completion. */
PNANOVDB_API int vox_voxelbvh_ijkl_from_gaussians(vox_context_t* ctx, const float* d_means, const float* d_opacities,
                                                  const float* d_quats, const float* d_scales, int64_t count,
                                                  uint32_t resolution, const float* transform, uint64_t* d_ijkl,
                                                  uint32_t* d_prim_id, uint32_t* d_range, float* d_world_bbox,
                                                  int64_t* range_count);

/* replaces ijkl_from_gaussians_file (raster/VoxelBVH.cpp:1437-1575): loads
 * `filename` (.npz or binary Gaussian-splat .ply; arrays means, opacities,
 * quaternions, scales, and sh_0 / sh_n when present), activates them on the
 * host as the reference does (normalised quaternions, exp scales, sigmoid
 * opacities), runs vox_voxelbvh_ijkl_from_gaussians and returns page-locked
 * host arrays: *ijkl_out (8-byte elements, 8 per Gaussian), *prim_id_out
 * (4-byte, 8 per Gaussian), *range_out (8-byte [start, end) pairs, 8 per
 * Gaussian), *world_bbox_out (6 floats), and in gaussian_arrays_out (up to
 * gaussian_array_count of the 6, may be NULL) the activated arrays.  Release
 * each with pnanovdb_get_compute()->destroy_array. */
PNANOVDB_API int vox_voxelbvh_ijkl_from_gaussians_file(vox_context_t* ctx, const char* filename, uint32_t resolution,
                                                       const float* transform, pnanovdb_compute_array_t** ijkl_out,
                                                       pnanovdb_compute_array_t** prim_id_out,
                                                       pnanovdb_compute_array_t** range_out,
                                                       pnanovdb_compute_array_t** world_bbox_out,
                                                       pnanovdb_compute_array_t** gaussian_arrays_out,
                                                       uint32_t gaussian_array_count);

/* The inverse vox_voxelbvh_ijkl_from_gaussians applies for `m` (16 floats,
 * host): Gauss-Jordan elimination with partial pivoting in double precision,
 * rounded to float.  The reference inverts in float by cofactor expansion
 * (nanovdb_editor/putil/Camera.h:316), so the two may differ in the last
 * bits.  VOX_ERR_ARGS for a singular or non-finite matrix. */
PNANOVDB_API int vox_voxelbvh_transform_inverse(const float* m, float* inv);

/* One Adam step (Kingma & Ba) on n parameters stored in bfloat16 for the
 * voxelizer with FP32 master copies: with t the 1-based step,
 *   m = b1 m + (1 - b1) g,  v = b2 v + (1 - b2) g^2,
 *   master -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps),
 *   out_bf16 = master rounded to nearest even,
 * all in one pass over device arrays, ordered on `stream` (cudaStream_t, may
 * be 0), asynchronous.  No counterpart in the reference (it has no training
 * loop); it closes the forward / adjoint / update step of the BF16 fitting
 * loop without a round trip through another library. */
PNANOVDB_API int vox_adam_bf16(float* master, float* m, float* v, const float* grad, uint16_t* out_bf16, int64_t n,
                               float lr, float beta1, float beta2, float eps, int64_t step, void* stream);

/* Scan that allocates nothing.  No counterpart in the reference.
 *
 * Same result as vox_global_scan_u64 (exact mod 2^64), for callers that cannot
 * let a library allocate device memory: hosts whose device memory is owned by
 * their own allocator (a framework's caching pool holding the free memory,
 * where an extra cudaMalloc can fail or fragment it) and loops where the
 * implicit device synchronisation of cudaMalloc / cudaFree is not acceptable.
 * It needs no vox_context_t and calls no cudaMalloc, cudaFree or other
 * allocating routine: its look-back scratch is a fixed 256 KiB device array
 * inside the library (held by every GPU that loads the library until exit),
 * which limits n to VOX_NOALLOC_SCAN_MAX; larger n returns VOX_ERR_SIZE.
 *
 * Each call looks up that array's address on the current device, so the
 * first call on a device also loads the library's kernels there.  All calls
 * share the one array and it keeps the last call's contents (each call clears
 * what it uses first): calls whose work overlaps on the GPU (concurrent
 * streams or threads) race and must be serialised by the caller.  The call is
 * ordered on `stream` (cudaStream_t, may be 0) and synchronises it before
 * returning (it reads the device error word back), so it cannot be recorded
 * into a stream capture. */
#define VOX_NOALLOC_SCAN_MAX (1ll << 24)
PNANOVDB_API int vox_global_scan_u64_noalloc(const uint64_t* d_in, uint64_t* d_out, int64_t n, int inclusive,
                                             uint64_t* d_total, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PNANOVDB_B200_H */
