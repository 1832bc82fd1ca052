/*
 * vox_oracle.h - CPU restatement of nanovdb-editor's Gaussian -> node2 grid
 * voxelization ("raster3d") path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product path and the timed CPU baseline; the product never links it.
 *
 * Parity status: the per-Gaussian / per-fragment arithmetic is pinned against
 * the reference's own shader sources compiled as C++ on this machine
 * (oracle/ref_shaders, outputs under oracle/_ref); the node2 byte layout is
 * pinned by the reference's own node2 accessors (PNanoVDBExt.h) compiled
 * against the bytes this oracle writes.  The incremental window-by-window
 * topology build itself has no golden vectors in the reference (its only
 * raster3d test asserts element_count > 0), so that part is checked through
 * the invariants the reference states: every Gaussian mean's voxel is active
 * (raster/Raster.cpp:777-815), sort monotonicity + checksum
 * (raster/ParallelPrimitives.cpp:910-968), value index == leaf value_idx +
 * local index (nanovdb_editor/putil/Convert.h:315-415), element_count > 0
 * for the 32-Gaussian pytest case (pytests/test_pipelines.py:313-336).
 */
#ifndef VOX_ORACLE_H
#define VOX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OV_PRIM_BATCH 262144u      /* raster/Raster.cpp:443 */
#define OV_WINDOW 8388608ull       /* raster/Raster.cpp:444 */

/* counters returned by ov_counts() */
enum
{
    OV_G = 0,        /* Gaussians */
    OV_G_VALID,      /* Gaussians that emit fragments */
    OV_F,            /* candidate bbox fragments */
    OV_P,            /* passing (voxel, Gaussian) pairs */
    OV_V,            /* active voxels */
    OV_UPPER,        /* upper nodes */
    OV_LOWER,        /* lower nodes */
    OV_LEAF,         /* leaf nodes */
    OV_VALUE_COUNT,  /* 2 + V */
    OV_NODE2_BYTES,  /* bytes of the node2 region (root + nodes) */
    OV_WINDOWS,      /* reference fragment windows that held fragments */
    OV_ERROR,        /* 0 = ok */
    OV_COUNT_N
};

/* A2: raster/RasterUtils.cpp:31-136 (does NOT modify its inputs) */
void ov_preprocess(int64_t n, const float* quat_raw, const float* log_scale, const float* opacity_logit,
                   const float* sh0, float* quat_out, float* scale_out, float* opacity_out, float* color_out);

/* mode bits of ov_run */
#define OV_MODE_WINDOWS 1 /* reference 256K-prim x 8M-fragment windows (else one window) */
#define OV_MODE_NO_F64 2  /* skip the FP64 values (timed CPU-baseline runs) */
#define OV_MODE_SMOOTH 4  /* differentiable channels: density = sum of
                             K = max(op exp(-|S^-1 R^T (x - mu)|^2 / 2) - 0.01, 0)
                             at voxel centres over the pair set, colour = sum K rgb */

/* Full forward.  window_mode 1 = reference 256K-prim x 8M-fragment windows,
 * 0 = one window (canonical hierarchical node order).  cull_scale <= 0 selects
 * the shader default 0.05 (gaussian_frag_color.slang:205-213). */
void* ov_run(int64_t n, const float* means, const float* quats_wxyz, const float* scales, const float* colors,
             const float* opacities, float voxel_size, float cull_scale, int window_mode, int nthreads);
void ov_destroy(void* h);
void ov_counts(void* h, int64_t* out);
/* the float channels' exp / log / pow on arrays (accuracy test) */
void ov_chan_math(int64_t n, const float* x, const float* b, const float* e, float* exp_out, float* log_out,
                  float* pow_out);
int64_t ov_node2_bytes(void* h, uint8_t* dst); /* node2 region starting at the root */
void ov_pairs(void* h, uint64_t* keys, uint32_t* ids); /* sorted by (hierarchical key, Gaussian id) */
void ov_values(void* h, uint32_t* rgba8, float* density, float* color, double* density64, double* color64);
void ov_voxels(void* h, int32_t* ijk, uint64_t* value_idx); /* active voxels in key order */
void ov_bbox(void* h, int32_t* out6);
void ov_node_table(void* h, int32_t* type, int32_t* parent, int32_t* n_in_parent, int32_t* origin3);

/* per-Gaussian bbox / footprint (gaussian_prim.slang:47-144) */
int ov_prim_bbox(const float* mean, const float* quat_wxyz, const float* scale, float opacity, float voxel_size,
                 int32_t* bbox6, uint64_t* footprint);
/* per-fragment test (gaussian_frag_alloc.slang:43-176): returns 1 if the voxel passes */
int ov_frag_test(const float* mean, const float* quat_wxyz, const float* scale, float opacity, float voxel_size,
                 const int32_t* ijk, float* vmin3, float* vmax3);
/* per-fragment packed RGBA8 and alpha (gaussian_frag_color.slang:182-217) */
uint32_t ov_frag_rgba(const float* mean, const float* quat_wxyz, const float* scale, float opacity,
                      const float* color, float voxel_size, float cull_scale, const int32_t* ijk, float* alpha_out);

uint64_t ov_hier_key(int32_t i, int32_t j, int32_t k);

/* value index of an active voxel, -1 when inactive */
int64_t ov_lookup(void* h, int32_t i, int32_t j, int32_t k);
/* FP64 adjoint of the smooth channels over the pair set: gradients of
 * L = sum_v grad_density[v] density[v] + grad_color[v] . colour[v] with respect
 * to the inputs as given (raw = 1: quaternion before normalisation, log-scale,
 * opacity logit, SH0 - raster/RasterUtils.cpp:59-117; raw = 0: activated
 * values).  grad arrays are indexed by value index (2 + V entries). */
int ov_smooth_grad64(void* h, const float* means, const float* quats_wxyz, const float* scales, const float* opacities,
                     const float* colors, int raw, const double* grad_density, const double* grad_color,
                     double* d_means, double* d_quats, double* d_scales, double* d_opacities, double* d_colors);
/* FP64 contribution of one Gaussian (theta = mean[3], quat wxyz[4], scale[3],
 * opacity, colour[3], raw as above) to L, summed over its kernel's support */
double ov_smooth_loss64(void* h, const double* theta, int raw, const double* grad_density, const double* grad_color);

/* VoxelBVH Gaussian ingestion (raster/VoxelBVH.cpp:1225-1435), activated
 * inputs; outputs sized 8 n (range: 2 x 8 n); returns the number of ranges,
 * or -1 when a Gaussian's box maps outside [-65536, 65536] voxels.
 * T / Tinv: 16 floats (rows of pnanovdb_camera_mat_t) for row vectors,
 * p' = [p 1] T, or NULL for the identity. */
int64_t ov_voxelbvh_ijkl(int64_t n, const float* means, const float* opacities, const float* quats_wxyz,
                         const float* scales, uint32_t resolution, const float* T, const float* Tinv,
                         uint64_t* ijkl, uint32_t* prim_id, uint32_t* range, float* world_bbox, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
