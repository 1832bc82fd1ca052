/*
 * ref_driver.cpp - runs the reference's own raster shaders, compiled as C++,
 * on the host: one call per dispatch, every (group, thread) invocation in
 * order.  TEST INFRASTRUCTURE ONLY (builds oracle/_ref/libref_shaders.so from
 * the shader files of the reference checkout; nothing here ships).
 *
 * Shaders wrapped (raster/shaders/...):
 *   gaussian_prim.slang                 per-Gaussian bbox + footprint
 *   fanout_scatter_prim_idxs.slang      window fan-out, scatter of first slots
 *   fanout_compute_fragment_idxs.slang  window fan-out, raster index per slot
 *   gaussian_frag_alloc.slang           fragment test -> ijk or 0x7FFFFFFF
 *   gaussian_frag_color.slang           alpha / RGBA8 of a passing fragment
 *   voxelbvh/voxelbvh_gaussians_to_ijkl.slang  per-Gaussian level and cells
 *   voxelbvh/voxelbvh_find_range_starts.slang, voxelbvh_scatter_range_headers.slang
 *                                       range headers of the sorted keys
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "vox_detmath.h"

#define VOX_REF_GROUP 256u

namespace sh_prim
{
#include "slang_compat.h"
#include "gaussian_prim.inc"
}
namespace sh_scatter
{
#include "slang_compat.h"
#include "fanout_scatter_prim_idxs.inc"
}
namespace sh_fragidx
{
#include "slang_compat.h"
#include "fanout_compute_fragment_idxs.inc"
}
namespace sh_alloc
{
#include "slang_compat.h"
#include "gaussian_frag_alloc.inc"
}
namespace sh_color
{
#include "slang_compat.h"
#include "pnanovdb_capture.h"
#include "gaussian_frag_color.inc"
}

namespace sh_vbijkl
{
#include "slang_compat.h"
#include "voxelbvh_gaussians_to_ijkl.inc"
}

namespace sh_vbstarts
{
#include "slang_compat.h"
#include "voxelbvh_find_range_starts.inc"
}
namespace sh_vbscatter
{
#include "slang_compat.h"
#include "voxelbvh_scatter_range_headers.inc"
}

template <class C>
static void set_constants(C& c, uint32_t prim_batch_size, uint32_t ijk_batch_size, uint64_t wmin, uint64_t wmax,
                          uint32_t prim_begin, uint32_t prim_count, float vs)
{
    memset(&c, 0, sizeof(c));
    c.prim_batch_size = prim_batch_size;
    c.ijk_batch_size = ijk_batch_size;
    c.fragment_window_min = wmin;
    c.fragment_window_max = wmax;
    c.global_prim_begin_idx = prim_begin;
    c.global_prim_count = prim_count;
    c.voxel_size = vs;
    c.voxel_size_inv = 1.f / vs; /* raster/GridBuild.cpp:780 */
}

extern "C" {

/* gaussian_prim over one prim batch */
void ref_gaussian_prim(uint32_t prim_batch_size, uint32_t prim_begin, uint32_t prim_count, float vs,
                       const float* means, const float* quats, const float* scales, const float* opac,
                       uint64_t* counts_out, int32_t* bbox_out)
{
    using namespace sh_prim;
    set_constants(constants, prim_batch_size, 0, 0, 0, prim_begin, prim_count, vs);
    positions_in.p = (uint*)means;
    quaterions_in.p = (uint*)quats;
    scales_in.p = (uint*)scales;
    opacities_in.p = (uint*)opac;
    fragment_counts_out.p = counts_out;
    prim_bbox_out.p = (uint*)bbox_out;
    uint32_t groups = (prim_batch_size + VOX_REF_GROUP - 1) / VOX_REF_GROUP;
    for (uint32_t g = 0; g < groups; g++)
        for (uint32_t t = 0; t < VOX_REF_GROUP; t++)
        {
            uint3 gi = { g, 0, 0 }, ti = { t, 0, 0 };
            main(gi, ti);
        }
}

/* one fragment window: clear + scatter + max-scan + fragment idxs
 * (raster/GridBuild.cpp:830-942).  The max-scan is ParallelPrimitives'
 * global_scan_max: an inclusive running maximum. */
void ref_fanout(uint32_t prim_batch_size, uint32_t ijk_batch_size, uint64_t wmin, const uint64_t* counts,
                const uint64_t* scan_counts, uint32_t* scatter_tmp, uint32_t* prim_idxs, uint32_t* raster_idxs)
{
    memset(scatter_tmp, 0, sizeof(uint32_t) * ijk_batch_size); /* fanout_clear_prim_idxs.slang */
    {
        using namespace sh_scatter;
        set_constants(constants, prim_batch_size, ijk_batch_size, wmin, wmin + ijk_batch_size, 0, 0, 1.f);
        fragment_counts_in.p = (uint64_t*)counts;
        scan_fragment_counts_in.p = (uint64_t*)scan_counts;
        prim_idxs_out.p = scatter_tmp;
        uint32_t groups = (prim_batch_size + VOX_REF_GROUP - 1) / VOX_REF_GROUP;
        for (uint32_t g = 0; g < groups; g++)
            for (uint32_t t = 0; t < VOX_REF_GROUP; t++)
            {
                uint3 gi = { g, 0, 0 }, ti = { t, 0, 0 };
                main(gi, ti);
            }
    }
    uint32_t run = 0;
    for (uint32_t i = 0; i < ijk_batch_size; i++)
    {
        run = scatter_tmp[i] > run ? scatter_tmp[i] : run;
        prim_idxs[i] = run;
    }
    {
        using namespace sh_fragidx;
        set_constants(constants, prim_batch_size, ijk_batch_size, wmin, wmin + ijk_batch_size, 0, 0, 1.f);
        fragment_counts_in.p = (uint64_t*)counts;
        scan_fragment_counts_in.p = (uint64_t*)scan_counts;
        prim_idxs_in.p = prim_idxs;
        prim_raster_idxs_out.p = raster_idxs;
        uint32_t groups = (ijk_batch_size + VOX_REF_GROUP - 1) / VOX_REF_GROUP;
        for (uint32_t g = 0; g < groups; g++)
            for (uint32_t t = 0; t < VOX_REF_GROUP; t++)
            {
                uint3 gi = { g, 0, 0 }, ti = { t, 0, 0 };
                main(gi, ti);
            }
    }
}

/* gaussian_frag_alloc over one window; ijks_out must be pre-filled by the
 * caller (slots with raster idx ~0 are left untouched, as in the shader) */
void ref_frag_alloc(uint32_t ijk_batch_size, uint32_t prim_begin, float vs, const float* means, const float* quats,
                    const float* scales, const float* opac, const uint32_t* prim_idxs, const uint32_t* raster_idxs,
                    const int32_t* bboxes, int32_t* ijk_dst)
{
    using namespace sh_alloc;
    set_constants(constants, 0, ijk_batch_size, 0, 0, prim_begin, 0, vs);
    positions_in.p = (uint*)means;
    quaterions_in.p = (uint*)quats;
    scales_in.p = (uint*)scales;
    opacities_in.p = (uint*)opac;
    prim_idxs_in.p = (uint*)prim_idxs;
    prim_raster_idxs_in.p = (uint*)raster_idxs;
    prim_bboxs_in.p = (uint*)bboxes;
    ijks_out.p = (uint*)ijk_dst;
    uint32_t groups = (ijk_batch_size + VOX_REF_GROUP - 1) / VOX_REF_GROUP;
    for (uint32_t g = 0; g < groups; g++)
        for (uint32_t t = 0; t < VOX_REF_GROUP; t++)
        {
            uint3 gi = { g, 0, 0 }, ti = { t, 0, 0 };
            main(gi, ti);
        }
}

/* gaussian_frag_color over one window; rgba_out[slot] receives the slot's
 * packed RGBA8 (0 for empty or failing slots) */
void ref_frag_color(uint32_t ijk_batch_size, uint32_t prim_begin, float vs, float cull_scale, int use_default,
                    const float* means, const float* quats, const float* scales, const float* opac,
                    const float* colors, const uint32_t* prim_idxs, const uint32_t* raster_idxs,
                    const int32_t* bboxes, uint32_t* rgba_out)
{
    using namespace sh_color;
    set_constants(constants, 0, ijk_batch_size, 0, 0, prim_begin, 0, vs);
    memset(&shader_params, 0, sizeof(shader_params));
    shader_params.cull_scale = cull_scale;
    shader_params.use_default = use_default != 0;
    positions_in.p = (uint*)means;
    quaterions_in.p = (uint*)quats;
    scales_in.p = (uint*)scales;
    opacities_in.p = (uint*)opac;
    colors_in.p = (uint*)colors;
    prim_idxs_in.p = (uint*)prim_idxs;
    prim_raster_idxs_in.p = (uint*)raster_idxs;
    prim_bboxs_in.p = (uint*)bboxes;
    memset(rgba_out, 0, sizeof(uint32_t) * ijk_batch_size);
    buf.p = (uint2*)rgba_out; /* slot s -> byte offset 4 s -> word s */
    uint32_t groups = (ijk_batch_size + VOX_REF_GROUP - 1) / VOX_REF_GROUP;
    for (uint32_t g = 0; g < groups; g++)
        for (uint32_t t = 0; t < VOX_REF_GROUP; t++)
        {
            uint3 gi = { g, 0, 0 }, ti = { t, 0, 0 };
            g_capture_slot = (uint64_t)g * VOX_REF_GROUP + t;
            main(gi, ti);
        }
}

/* voxelbvh_gaussians_to_ijkl over all Gaussians (raster/VoxelBVH.cpp:1355-1372)
 * given the reduced world box bbox6 (min xyz, max xyz).  T / Tinv: 16 floats,
 * the logical float4x4 the shader reads (rows of the caller's matrix; the
 * host uploads its transpose and the shaders read constants column-major,
 * compiler/SlangCompiler.cpp:298-299, nanovdb_editor/putil/Compiler.h:134),
 * NULL = identity.  keys / ids hold 8 x 256 x ceil(n / 256) entries: the
 * shader writes the unused-slot sentinel for every thread of the last group. */
void ref_voxelbvh_to_ijkl(uint32_t n, uint32_t resolution, const float* means, const float* opac, const float* quats,
                          const float* scales, const float* T, const float* Tinv, const float* bbox6, uint64_t* keys,
                          uint32_t* ids)
{
    using namespace sh_vbijkl;
    memset(&constants, 0, sizeof(constants));
    constants.point_count = n;
    constants.workgroup_count = (n + 255u) / 256u;
    constants.voxel_count = 8u * n;
    constants.voxel_workgroup_count = (constants.voxel_count + 255u) / 256u;
    constants.resolution = resolution;
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++)
        {
            constants.transform.m[r][c] = T ? T[4 * r + c] : (r == c ? 1.f : 0.f);
            constants.transform_inv.m[r][c] = Tinv ? Tinv[4 * r + c] : (r == c ? 1.f : 0.f);
        }
    means_in.p = (float*)means;
    opacities_in.p = (float*)opac;
    quats_in.p = (float*)quats;
    scales_in.p = (float*)scales;
    bbox_in.p = (float*)bbox6;
    keys_out.p = keys;
    bbox_ids_out.p = ids;
    for (uint32_t g = 0; g < constants.workgroup_count; g++)
        for (uint32_t t = 0; t < VOX_REF_GROUP; t++)
        {
            uint3 gi = { g, 0, 0 }, ti = { t, 0, 0 };
            main(gi, ti);
        }
}

/* range headers of n sorted keys (raster/VoxelBVH.cpp:1380-1431): range
 * starts, the inclusive uint32 global_scan of them, the header scatter.
 * headers: 2 n words; starts / scan: n words of scratch each. */
void ref_voxelbvh_ranges(uint32_t n, const uint64_t* keys, uint32_t* starts, uint32_t* scan, uint32_t* headers)
{
    const uint32_t groups = (n + VOX_REF_GROUP - 1) / VOX_REF_GROUP;
    {
        using namespace sh_vbstarts;
        memset(&constants, 0, sizeof(constants));
        constants.voxel_count = n;
        constants.voxel_workgroup_count = groups;
        keys_in.p = (uint64_t*)keys;
        range_starts_out.p = starts;
        range_headers_out.p = headers;
        for (uint32_t g = 0; g < groups; g++)
            for (uint32_t t = 0; t < VOX_REF_GROUP; t++)
            {
                uint3 gi = { g, 0, 0 }, ti = { t, 0, 0 };
                main(gi, ti);
            }
    }
    uint32_t run = 0; /* global_scan: inclusive, uint32 */
    for (uint32_t i = 0; i < n; i++)
    {
        run += starts[i];
        scan[i] = run;
    }
    {
        using namespace sh_vbscatter;
        memset(&constants, 0, sizeof(constants));
        constants.voxel_count = n;
        constants.voxel_workgroup_count = groups;
        keys_in.p = (uint64_t*)keys;
        range_starts_in.p = starts;
        range_scan_in.p = scan;
        range_headers_out.p = headers;
        for (uint32_t g = 0; g < groups; g++)
            for (uint32_t t = 0; t < VOX_REF_GROUP; t++)
            {
                uint3 gi = { g, 0, 0 }, ti = { t, 0, 0 };
                main(gi, ti);
            }
    }
}

} /* extern "C" */
