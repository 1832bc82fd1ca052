/*
 * ref_gridbuild.cpp - the reference's topology build, run on the host with its
 * own shaders compiled as C++: raster_gaussian_3d's first pass
 * (raster/Raster.cpp:420-510) - prim batches, fragment windows, and per
 * window grid_build (raster/GridBuild.cpp:361-506: per tree level
 * grid_build_set_masks, grid_build_count_new, an inclusive global scan,
 * grid_build_scatter_new, grid_build_finalize) - then grid_build_finalize
 * (GridBuild.cpp:508-650: grid_build_blindmetadata, grid_build_compute_bbox
 * from the leaves up).  The result is the node2 region (root first, nodes at
 * their node2 maximum sizes in allocation order), the node counts, the value
 * count and the bbox, for comparison with the CPU oracle and the CUDA path.
 *
 * Host steps restated from the reference (not shaders): the node2 part of
 * empty_grid_generate (GridBuild.cpp:126-192: zeroed root, every root child
 * slot set to the end key), the fan-out window loop (GridBuild.cpp:654-700:
 * ceil(fragments / window) windows per prim batch) and ParallelPrimitives'
 * inclusive uint32 global_scan.
 *
 * TEST INFRASTRUCTURE ONLY (part of oracle/_ref/libref_shaders.so).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "vox_detmath.h"

namespace gb
{
#include "slang_compat.h"
#include "pnanovdb_gridbuild.h"
#include "PNanoVDBExt.inc"
} // namespace gb

/* gb_fiber_switch(save_sp, load_sp): pushes the callee-saved registers, saves
 * the stack pointer, loads the other fiber's and pops its registers */
asm(R"(
    .text
    .globl gb_fiber_switch
    .type gb_fiber_switch, @function
gb_fiber_switch:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
    .size gb_fiber_switch, .-gb_fiber_switch
)");

namespace gb_init
{
using namespace gb;
#include "grid_build_init.inc"
}
namespace gb_masks
{
using namespace gb;
#include "grid_build_set_masks.inc"
}
namespace gb_count
{
using namespace gb;
#include "grid_build_count_new.inc"
}
namespace gb_scatter
{
using namespace gb;
#include "grid_build_scatter_new.inc"
}
namespace gb_final
{
using namespace gb;
#include "grid_build_finalize.inc"
}
namespace gb_blind
{
using namespace gb;
#include "grid_build_blindmetadata.inc"
}
namespace gb_bbox
{
using namespace gb;
#include "grid_build_compute_bbox.inc"
}

extern "C" {
void ref_gaussian_prim(uint32_t prim_batch_size, uint32_t prim_begin, uint32_t prim_count, float vs,
                       const float* means, const float* quats, const float* scales, const float* opac,
                       uint64_t* counts_out, int32_t* bbox_out);
void ref_fanout(uint32_t prim_batch_size, uint32_t ijk_batch_size, uint64_t wmin, const uint64_t* counts,
                const uint64_t* scan_counts, uint32_t* scatter_tmp, uint32_t* prim_idxs, uint32_t* raster_idxs);
void ref_frag_alloc(uint32_t ijk_batch_size, uint32_t prim_begin, float vs, const float* means, const float* quats,
                    const float* scales, const float* opac, const uint32_t* prim_idxs, const uint32_t* raster_idxs,
                    const int32_t* bboxes, int32_t* ijk_dst);
}

namespace
{

/* the constants block every grid-build shader declares (GridBuild.cpp:375-395) */
struct GbConstants
{
    uint32_t workgroup_count, max_node_count, buf_word_count, point_count, empty_grid_word_count, active_node_type,
        child_node_type;
};

constexpr uint32_t WORKGROUPS = 4096u;             /* constants.workgroup_count */
constexpr uint32_t MAX_NODES = 2u * 1024u * 1024u; /* constants.max_node_count */
constexpr uint64_t ROOT_OFFSET = 4096u;            /* where this host places the root */
constexpr uint64_t ROOT_BYTES = 541728u, UPPER_BYTES = 274464u, LOWER_BYTES = 34336u, LEAF_BYTES = 128u;

struct Build
{
    std::vector<gb::uint2> buf; /* the grid buffer in 64-bit words */
    std::vector<uint32_t> node_addresses, node_types, new_child_counts, scan_new, bboxes;
    GbConstants c;
    int64_t windows = 0;
    uint64_t region_bytes = 0;
    int32_t bbox[6] = { 0, 0, 0, 0, 0, 0 };
};
Build g_b;

uint64_t nodes_end()
{
    const gb::GbTreeFields& t = gb::g_tree_fields;
    return ROOT_OFFSET + ROOT_BYTES + (uint64_t)t.count_upper * UPPER_BYTES + (uint64_t)t.count_lower * LOWER_BYTES +
           (uint64_t)t.count_leaf * LEAF_BYTES;
}

uint32_t node_count()
{
    const gb::GbTreeFields& t = gb::g_tree_fields;
    return 1u + t.count_upper + t.count_lower + t.count_leaf;
}

void ensure_bytes(uint64_t bytes)
{
    const size_t words = (size_t)((bytes + 7) / 8);
    if (g_b.buf.size() < words)
        g_b.buf.resize(words + words / 2 + 1024);
}

template <class C>
void set_constants(C& dst)
{
    memcpy(&dst, &g_b.c, sizeof(GbConstants));
    static_assert(sizeof(C) == sizeof(GbConstants), "constants layout");
}

void level_types(uint32_t level, uint32_t& active, uint32_t& child)
{
    active = level == 0 ? 0u : level == 1 ? 1u : level == 2 ? 2u : 3u;
    child = level == 0 ? 1u : level == 1 ? 2u : 3u;
}

/* the empty grid's node2 part (GridBuild.cpp:126-192) and grid_build_init */
void reset()
{
    g_b.buf.assign((size_t)((ROOT_OFFSET + ROOT_BYTES) / 8) + 1024, gb::uint2(0u, 0u));
    gb::g_tree_fields = gb::GbTreeFields{ ROOT_OFFSET, 0u, 0u, 0u, 0u };
    const uint64_t root_idx64 = ROOT_OFFSET / 8;
    for (uint32_t n = 0; n < 2u * 32768u; n++)
        g_b.buf[root_idx64 + 2180u + n] = gb::uint2(0u, 0x80000000u); /* pnanovdb_node2_end_key */
    g_b.node_addresses.assign(MAX_NODES, 0u);
    g_b.node_types.assign(MAX_NODES, 0u);
    g_b.new_child_counts.assign(MAX_NODES, 0u);
    g_b.scan_new.assign(MAX_NODES, 0u);
    g_b.bboxes.assign((size_t)MAX_NODES * 6u, 0u);
    memset(&g_b.c, 0, sizeof(g_b.c));
    g_b.c.workgroup_count = WORKGROUPS;
    g_b.c.max_node_count = MAX_NODES;
    g_b.windows = 0;
    {
        using namespace gb_init;
        set_constants(constants);
        buf.p = g_b.buf.data();
        node_addresses.p = g_b.node_addresses.data();
        node_types.p = g_b.node_types.data();
        gb::gb_run_flat((MAX_NODES + 255u) / 256u, [](uint32_t g, uint32_t t) { main(gb::uint3(g, 0, 0), gb::uint3(t, 0, 0)); });
    }
}

/* one window of fragments: GridBuild.cpp:361-506 */
void grid_build(const int32_t* ijk, uint32_t point_count)
{
    for (uint32_t level = 0; level < 4; level++)
    {
        level_types(level, g_b.c.active_node_type, g_b.c.child_node_type);
        g_b.c.point_count = point_count;
        {
            using namespace gb_masks;
            set_constants(constants);
            point_ijk_in.p = (gb::uint*)ijk;
            buf.p = g_b.buf.data();
            gb::gb_run_flat((point_count + 255u) / 256u,
                            [](uint32_t g, uint32_t t) { main(gb::uint3(g, 0, 0), gb::uint3(t, 0, 0)); });
        }
        const uint32_t nodes = node_count();
        const uint32_t groups = nodes < WORKGROUPS ? nodes : WORKGROUPS; /* later groups find no node */
        {
            using namespace gb_count;
            set_constants(constants);
            node_addresses.p = g_b.node_addresses.data();
            node_types.p = g_b.node_types.data();
            buf.p = g_b.buf.data();
            new_child_counts.p = g_b.new_child_counts.data();
            gb::gb_run_groups(groups, [](uint32_t g, uint32_t t) { main(gb::uint3(g, 0, 0), gb::uint3(t, 0, 0)); });
        }
        /* ParallelPrimitives global_scan: inclusive, uint32 */
        uint32_t run = 0;
        for (uint32_t i = 0; i < nodes; i++)
        {
            run += g_b.new_child_counts[i];
            g_b.scan_new[i] = run;
        }
        if (g_b.c.active_node_type != g_b.c.child_node_type)
        {
            const uint64_t child_bytes = g_b.c.child_node_type == 1 ? UPPER_BYTES : g_b.c.child_node_type == 2 ? LOWER_BYTES : LEAF_BYTES;
            ensure_bytes(nodes_end() + (uint64_t)run * child_bytes + 64);
        }
        {
            using namespace gb_scatter;
            set_constants(constants);
            new_child_counts.p = g_b.new_child_counts.data();
            scan_new_child_counts.p = g_b.scan_new.data();
            buf.p = g_b.buf.data();
            node_addresses.p = g_b.node_addresses.data();
            node_types.p = g_b.node_types.data();
            gb::gb_run_groups(groups, [](uint32_t g, uint32_t t) { main(gb::uint3(g, 0, 0), gb::uint3(t, 0, 0)); });
        }
        {
            using namespace gb_final;
            set_constants(constants);
            new_child_counts.p = g_b.new_child_counts.data();
            scan_new_child_counts.p = g_b.scan_new.data();
            buf.p = g_b.buf.data();
            gb::gb_run_flat(1u, [](uint32_t g, uint32_t t) { main(gb::uint3(g, 0, 0), gb::uint3(t, 0, 0)); });
        }
    }
}

/* GridBuild.cpp:508-650 */
void finalize()
{
    g_b.c.active_node_type = 3u;
    g_b.c.child_node_type = 3u;
    {
        using namespace gb_blind;
        set_constants(constants);
        new_child_counts.p = g_b.new_child_counts.data();
        scan_new_child_counts.p = g_b.scan_new.data();
        buf.p = g_b.buf.data();
        gb::gb_run_groups(1u, [](uint32_t g, uint32_t t) { main(gb::uint3(g, 0, 0), gb::uint3(t, 0, 0)); });
    }
    /* the blind bbox value: a record after the node region */
    const uint64_t end = nodes_end();
    ensure_bytes(end + 64);
    gb::g_tree_fields.blind_value0 = end;
    const uint32_t nodes = node_count();
    const uint32_t groups = nodes < WORKGROUPS ? nodes : WORKGROUPS;
    for (uint32_t level = 3; level < 4; level--)
    {
        level_types(level, g_b.c.active_node_type, g_b.c.child_node_type);
        if (level == 3)
            g_b.c.child_node_type = 3u;
        using namespace gb_bbox;
        set_constants(constants);
        node_addresses.p = g_b.node_addresses.data();
        node_types.p = g_b.node_types.data();
        buf.p = g_b.buf.data();
        bboxes.p = g_b.bboxes.data();
        gb::gb_run_groups(groups, [](uint32_t g, uint32_t t) { main(gb::uint3(g, 0, 0), gb::uint3(t, 0, 0)); });
    }
    memcpy(g_b.bbox, (const char*)g_b.buf.data() + end, sizeof(g_b.bbox));
    g_b.region_bytes = end - ROOT_OFFSET;
}

} // namespace

extern "C" {

/* The reference's topology build of one cloud (activated attributes) in
 * prim batches of prim_batch Gaussians and fragment windows of ijk_batch
 * slots (the reference's defaults: 256K and 8M, Raster.cpp:443-444).
 * counts_out: upper, lower, leaf nodes, value count, windows.  Returns the
 * node2 region's size in bytes (ref_node2_copy copies it) or -1. */
int64_t ref_node2_build(int64_t n, const float* means, const float* quats, const float* scales, const float* opac,
                        float vs, uint32_t prim_batch, uint32_t ijk_batch, int64_t* counts_out, int32_t* bbox_out)
{
    if (n < 0 || prim_batch == 0 || ijk_batch == 0 || (ijk_batch & 255u) || (prim_batch & 255u))
        return -1;
    reset();
    std::vector<uint64_t> counts(prim_batch), scan(prim_batch);
    std::vector<int32_t> bbox((size_t)prim_batch * 6);
    std::vector<uint32_t> tmp(ijk_batch), pidx(ijk_batch), ridx(ijk_batch);
    std::vector<int32_t> ijk((size_t)ijk_batch * 3);
    const int64_t batches = (n + prim_batch - 1) / prim_batch;
    for (int64_t b = 0; b < batches; b++)
    {
        const uint32_t begin = (uint32_t)(b * prim_batch);
        ref_gaussian_prim(prim_batch, begin, (uint32_t)n, vs, means, quats, scales, opac, counts.data(), bbox.data());
        uint64_t run = 0;
        for (uint32_t i = 0; i < prim_batch; i++)
        {
            run += counts[i];
            scan[i] = run; /* global_scan_uint64, inclusive */
        }
        const uint64_t windows = (run + ijk_batch - 1) / ijk_batch;
        for (uint64_t w = 0; w < windows; w++)
        {
            ref_fanout(prim_batch, ijk_batch, w * (uint64_t)ijk_batch, counts.data(), scan.data(), tmp.data(), pidx.data(),
                       ridx.data());
            /* slots gaussian_frag_alloc leaves unwritten hold no fragment */
            for (uint32_t s = 0; s < ijk_batch; s++)
            {
                ijk[3 * (size_t)s + 0] = 0;
                ijk[3 * (size_t)s + 1] = 0;
                ijk[3 * (size_t)s + 2] = 0x7FFFFFFF;
            }
            ref_frag_alloc(ijk_batch, begin, vs, means, quats, scales, opac, pidx.data(), ridx.data(), bbox.data(),
                           ijk.data());
            grid_build(ijk.data(), ijk_batch);
            g_b.windows++;
        }
    }
    finalize();
    const gb::GbTreeFields& t = gb::g_tree_fields;
    if (counts_out)
    {
        counts_out[0] = t.count_upper;
        counts_out[1] = t.count_lower;
        counts_out[2] = t.count_leaf;
        counts_out[3] = g_b.scan_new[node_count() - 1u];
        counts_out[4] = g_b.windows;
    }
    if (bbox_out)
        memcpy(bbox_out, g_b.bbox, sizeof(g_b.bbox));
    return (int64_t)g_b.region_bytes;
}

/* the node2 region of the last ref_node2_build (root first) */
int64_t ref_node2_copy(uint8_t* dst, int64_t capacity)
{
    if (capacity < (int64_t)g_b.region_bytes)
        return -1;
    memcpy(dst, (const char*)g_b.buf.data() + ROOT_OFFSET, g_b.region_bytes);
    return (int64_t)g_b.region_bytes;
}

} // extern "C"
