// vox_raster.h - kernel parameter blocks and launchers of vox_raster.cu.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "vox_device.cuh"

namespace vox
{

struct RankTables
{
    const uint64_t* root_bits;    // 512 words: touched root tiles by root_n
    const uint64_t* root_prefix;  // exclusive popcount prefix per word
    const uint64_t* lower_bits;   // roots * 512 words: touched lower cells (root rank, upper_n)
    const uint64_t* lower_prefix;
};

struct RunParams
{
    int64_t P;
    uint32_t* vox_start;    // [V + 1]
    uint32_t* leaf_vstart;  // [L + 1]
    uint32_t* lower_lstart; // [Lo + 1]
    uint32_t* lower_rank;   // [Lo]
    uint64_t* counts;       // V, L, Lo
    uint64_t* status;       // 3 per tile
    uint32_t epoch;
    uint32_t* counter;
    int* err;
    uint64_t lower_cap;     // entries of lower_lstart / lower_rank (heads beyond it are an error)
    uint32_t* vox_leaf;     // [V] leaf index of each voxel
    uint16_t* vox_n;        // [V] leaf_n (position in the leaf) of each voxel
};

// per-cloud layout: every cloud gets its own self-contained grid (header,
// node2 region, bbox, channels) in one output buffer; nodes, leaves and voxels
// of all clouds sit in one array per level, ordered by cloud first
struct CloudParams
{
    int64_t B;                   // clouds
    uint32_t *upper_start, *lower_start, *leaf_start; // [B + 1] first node of each cloud per level
    uint32_t* leaf_cloud;        // [L]
    uint64_t* vstart;            // [B + 1] first voxel (run order) of each cloud
    uint64_t* grid_off;          // [B + 1] byte offset of each cloud's grid; [B] = total bytes
    uint64_t* value_base;        // [B + 1] first value of each cloud in value-concatenated arrays
    uint64_t* node2_bytes;       // [B]
    uint64_t *bbox_off, *rgba_off, *dens_off, *col_off; // [B] byte offsets in the output
    int32_t* bbox;               // [B][6] active-voxel bbox
    const float* cloud_vs;       // [B] or null (voxel_size for every cloud)
    float voxel_size;
    const int64_t* cloud_start;  // [B + 1] Gaussian ranges (device) or null for one cloud
    const uint64_t* frag_off;    // exclusive scan of footprints (candidates per cloud)
    const uint64_t* F_total;
    const uint64_t* cloud_pairs; // [B] passing pairs per cloud (null: one cloud, P)
    int64_t G, P, V;
    uint32_t node_order;
};

struct NodeParams
{
    int64_t Lo, L;
    CloudParams C;
    const uint32_t* lower_rank;
    const uint32_t* lower_cell;   // lower rank -> cell (root rank << 15 | upper_n)
    const uint32_t* root_of_rank; // root rank -> root_n
    const uint32_t* lower_lstart;
    const uint32_t* leaf_vstart;
    const uint32_t* vox_start;
    int32_t* lower_origin;
    uint32_t* lower_upper_n;
    uint32_t* rank_to_lower; // [touched lower cells] lower rank -> lower node index
    uint64_t* upper_head;
    uint64_t* upper_scan;
    uint32_t* lower_parent;
    uint32_t* upper_root_n;
    uint32_t* upper_lostart;
    uint64_t* upper_count;
    uint32_t* leaf_lower;
    uint32_t* leaf_lower_n;
    uint64_t* leaf_mask;
    int32_t* leaf_origin;
    uint64_t *upper_idx, *upper_addr, *upper_vidx;
    uint64_t *lower_idx, *lower_addr, *lower_vidx;
    uint64_t *leaf_idx, *leaf_addr, *leaf_vidx;
};

// per-Gaussian adjoint sums: [0] dL/d op, [1..3] U, [4..6] W, [7..15] Q[r][a], [16..18] dL/d rgb
constexpr int BWD_NACC = 19;

struct BwdFinalParams
{
    const float* partials;    // per-(leaf, Gaussian) partial sums by emission index
    const uint64_t* lcol_off; // [G] first leaf column of each Gaussian
    const uint64_t* lc_off;   // [NLC] first emission index of each leaf column
    uint64_t NLC, Q;
    int64_t G;
    const float *means, *quats, *scales, *opacities, *colors; // the forward's inputs
    int raw;
    int bf16; // the inputs are bfloat16 arrays
    float voxel_size;
    const float* cloud_vs;
    const GaussRec* recs;
    float *d_means, *d_quats, *d_scales, *d_opacities, *d_colors; // any may be null
};

// ---------------------------------------------------------------- leaves --
// (leaf cell, Gaussian) pairs: every Gaussian emits the leaf cells (8^3
// voxels) its ellipsoid may touch, in Gaussian-major order; sorted stably by
// leaf key they give, per candidate leaf, its Gaussians in ascending id.
struct LeafEmitParams
{
    const GaussRec* recs;
    int64_t G;
    const uint64_t* lcol_off; // [G] exclusive scan of per-Gaussian leaf columns (Lx * Ly)
    uint64_t NLC;             // leaf columns
    const int64_t* tile_g0;   // [NLC / 256 + 1] Gaussian of each 256-column tile's first column
    uint64_t* lc_count;       // count pass: pairs per leaf column
    uint32_t* lc_mask;        // count pass writes, write pass reads: leaf-test results of a
                              // column's first 32 leaves (bit lz - lz0)
    const uint64_t* lc_off;   // write pass: exclusive scan of lc_count
    uint32_t* keys;           // leaf key: lower rank << 12 | lower_n
    uint32_t* vals;           // emission index (the sort's value)
    uint32_t* emit_gid;       // Gaussian of each emission index
    uint8_t* emit_flag;       // check mode: 1 = the leaf test culls this pair
    float voxel_size;
    const float* cloud_vs;
    int check;                // emit every bbox leaf, flag the ones the test culls
};

struct LeafPassParams
{
    const GaussRec* recs;
    const uint32_t* vals;      // sorted leaf pairs' emission indices
    const uint32_t* emit_gid;
    const uint32_t* pair_gid;  // sorted leaf pairs' Gaussian ids
    const uint8_t* emit_flag;  // check mode or null
    const uint32_t* cand_key;  // [NCL] candidate leaf keys
    const int4* cand_org;      // [NCL] candidate leaf origins (x, y, z, 0)
    const uint32_t* cand_start;// [NCL + 1] first sorted pair of each candidate
    int64_t NCL;
    const uint32_t* lower_cell;
    const uint32_t* root_of_rank;
    float voxel_size;
    const float* cloud_vs;
    int smooth;
    uint64_t* cand_mask;       // [NCL][8]
    uint32_t* s_rgba;          // staging [NCL * 512]
    float* s_dens;
    float* s_col;              // [NCL * 512][3]
    uint32_t* s_pairs;
    uint64_t* total_pairs;
    int* err;
    // adjoint
    const uint64_t* cand_vbase; // [NCL] value index of each candidate's first voxel
    const float* grad_density;
    const float* grad_color;
    float* partials;            // [emission index][BWD_NACC]
    // reference node order: creation window of each candidate leaf
    int window;
    const uint64_t* frag_off;   // exclusive scan of footprints
    const uint64_t* win_before; // windows of the earlier 256K-Gaussian batches
    uint64_t* cand_wkey;        // [NCL]
    // pair export
    const uint64_t* cand_voff;  // [NCL] first voxel (run order) of each candidate
    const uint64_t* pair_off;   // [V] first pair of each voxel
    void* out_keys;             // compact voxel keys
    uint32_t* out_ids;
    int key64;
};

void launch_leaf_cols(const GaussRec* recs, int64_t G, uint64_t* lcols, cudaStream_t s);
void launch_leaf_emit(const LeafEmitParams& P, const RankTables& T, bool write, cudaStream_t s);
void launch_tile_gauss(const uint64_t* lcol_off, int64_t G, uint64_t NLC, int64_t* tile_g0, cudaStream_t s);
void launch_leaf_heads(const uint32_t* keys, int64_t Q, uint64_t* flags, cudaStream_t s);
void launch_leaf_compact(const uint32_t* keys, const uint32_t* vals, const uint32_t* emit_gid, int64_t Q,
                         const uint64_t* flags, const uint64_t* pos, const uint32_t* lower_cell,
                         const uint32_t* root_of_rank, uint32_t* cand_key, int4* cand_org, uint32_t* cand_start,
                         uint32_t* pair_gid, cudaStream_t s);
// variant 0: 4 resident CTAs per SM (64 registers per thread), 1: 3 CTAs per SM;
// returns the CTAs per SM it ran with
int launch_leaf_pass(const LeafPassParams& P, uint32_t* counter, int num_sms, cudaStream_t s, int variant = 0);
void launch_leaf_backward(const LeafPassParams& P, uint32_t* counter, int num_sms, cudaStream_t s);
void launch_leaf_export(const LeafPassParams& P, uint32_t* counter, int num_sms, cudaStream_t s);
void launch_leaf_popc(const uint64_t* cand_mask, int64_t NCL, uint64_t* counts, cudaStream_t s);
void launch_voxel_keys(const uint64_t* cand_mask, const uint32_t* cand_key, const uint64_t* cand_voff, int64_t NCL,
                       void* vkeys, int key64, uint32_t* vslot, cudaStream_t s);

struct ValueParams
{
    int64_t V;
    const uint32_t* vslot;     // [V] staging slot (candidate * 512 + leaf_n)
    const uint32_t* s_rgba;
    const float* s_dens;
    const float* s_col;
    const uint32_t* s_pairs;
    uint64_t* cloud_pairs;     // [B] passing pairs per cloud, summed here (null: one cloud)
    uint64_t* cand_vbase;      // [NCL]
    const uint32_t* vox_leaf;
    const uint16_t* vox_n;
    uint8_t* out;
};
void launch_values(const ValueParams& A, const NodeParams& N, cudaStream_t s);
void launch_leaf_masks(const NodeParams& N, const uint64_t* cand_mask, const uint32_t* vslot, cudaStream_t s);
void launch_voxel_pairs(int64_t V, const uint32_t* vslot, const uint32_t* s_pairs, uint64_t* vpairs, cudaStream_t s);
void launch_zero_gaps(const NodeParams& N, uint8_t* out, uint64_t grid_bytes, cudaStream_t s);

// the reference's fragment batches and windows (raster/Raster.cpp:443-444)
constexpr int64_t REF_PRIM_BATCH = 262144; // Gaussians per batch (2^18)
constexpr uint64_t REF_WINDOW = 8388608;   // fragments per window

struct WindowOrderParams
{
    uint64_t U;
    const uint32_t *rank_u, *rank_lo, *rank_leaf;   // position in each level's (window, parent, n) order
    const uint64_t *wkey_u, *wkey_lo, *wkey_leaf;   // creation window
    const uint64_t *base_u, *base_lo, *base_leaf, *base_all; // [windows + 1] nodes in earlier windows
    const uint64_t* leaf_voff; // voxels of the leaves before, in node_idx order
    uint64_t V;                // active voxels
};
void launch_batch_windows(const uint64_t* frag_off, const uint64_t* F_total, int64_t G, int64_t nbatch,
                          uint64_t* nwin, cudaStream_t s);
void launch_leaf_wkey(int64_t L, const uint32_t* leaf_vstart, const uint32_t* vslot, const uint64_t* cand_wkey,
                      uint64_t* leaf_wkey, cudaStream_t s);
void launch_run_min(int64_t n, const uint32_t* start, const uint64_t* child, uint64_t* out, cudaStream_t s);
void launch_level_keys(int64_t n, const uint64_t* wkey, const uint32_t* parent, const uint32_t* parent_rank,
                       const uint32_t* nval, uint32_t nmask, uint64_t* keys, uint32_t* vals, uint64_t* wcount,
                       cudaStream_t s);
void launch_level_rank(int64_t n, const uint32_t* sorted_vals, uint32_t* rank, cudaStream_t s);
void launch_leaf_popc_sorted(int64_t L, const uint32_t* sorted_vals, const uint32_t* leaf_vstart, uint64_t* out,
                             cudaStream_t s);
void launch_window_bases(int64_t nw, const uint64_t* cu, const uint64_t* clo, const uint64_t* cleaf, uint64_t* base_u,
                         uint64_t* base_lo, uint64_t* base_leaf, uint64_t* base_all, cudaStream_t s);
void launch_window_place(const WindowOrderParams& W, const NodeParams& N, cudaStream_t s);

void launch_bwd_finalize(const BwdFinalParams& F, cudaStream_t s);

void launch_prep(const PrepParams& P, GaussRec* recs, uint64_t* footprints, uint64_t* root_bits, int* err,
                 cudaStream_t s);
void launch_mark_lower(const GaussRec* recs, int64_t G, const uint64_t* root_bits, const uint64_t* root_prefix,
                       uint64_t* lower_bits, cudaStream_t s);
void launch_invert_bits(const uint64_t* bits, const uint64_t* prefix, int64_t words, uint32_t* out, cudaStream_t s);
void launch_runs(const RunParams& Rp, const void* keys, int key64, cudaStream_t s);
int64_t runs_tile_count(int64_t P);
void launch_lower_info(const NodeParams& N, cudaStream_t s);
void launch_upper_info(const NodeParams& N, cudaStream_t s);
void launch_leaf_tables(const NodeParams& N, const void* keys, int key64, cudaStream_t s);
void launch_leaf_bbox(const NodeParams& N, cudaStream_t s);
void launch_cloud_layout(const NodeParams& N, cudaStream_t s);
void launch_canonical_order(const NodeParams& N, uint64_t U, cudaStream_t s);
void launch_write_nodes(const NodeParams& N, uint64_t U, uint8_t* out, cudaStream_t s);
void launch_write_headers(const NodeParams& N, uint8_t* out, cudaStream_t s);

// VoxelBVH Gaussian ingestion (raster/VoxelBVH.cpp:1225-1435)
struct VoxelBvhParams
{
    const float* means;  // [n][3]
    const float* opac;   // [n]
    const float* quats;  // [n][4] w x y z
    const float* scales; // [n][3]
    int64_t n;
    uint32_t resolution;
    int has_xform;       // 0: identity transform
    float t[16];         // p' = [p 1] t (rows of the caller's matrix)
    float ti[16];        // inverse of t
    uint32_t* box_keys;  // [6] order-preserving keys of the world box (min xyz, max xyz)
    int* cell_minmax;    // [6] min i j k, max i j k over the emitted cells
    float* world_bbox;   // [6] output
    uint64_t* keys;      // [8 n], 16-byte aligned
    uint32_t* ids;       // [8 n], 16-byte aligned
    float* rec;          // [n][24] per-Gaussian search records (lane-balanced search)
    int* err;
};
// sorted-key pass: compressed key layout, range headers, 64-bit key write-back
struct VbRangeParams
{
    int bits[3];         // bits of i, j, k in a compressed key
    uint64_t sentinel;   // compressed key of an unused slot
    int expand;          // write keys_out from the compressed keys
    uint32_t* range;     // [2 N] headers
    uint64_t* keys_out;  // [N] 64-bit keys (expand)
    const uint32_t* ids_src; // sorted ids to copy into ids_out, or null
    uint32_t* ids_out;
};
void launch_vb_init(uint32_t* box_keys, int* cell_minmax, cudaStream_t s);
void launch_vb_box(const VoxelBvhParams& P, int num_sms, cudaStream_t s);
void launch_vb_ijkl(const VoxelBvhParams& P, cudaStream_t s);
void launch_vb_search(const VoxelBvhParams& P, int num_sms, cudaStream_t s);
int64_t vb_range_tiles(int64_t N);
void launch_vb_used(const uint32_t* ids, int64_t count, uint32_t* used, cudaStream_t s);
void launch_vb_compress_used(const uint64_t* keys, const uint32_t* ids, int64_t count, const uint32_t* used,
                             const uint32_t* off, const VbRangeParams& R, void* out_keys, uint32_t* out_ids, int key32,
                             int num_sms, cudaStream_t s);
void launch_vb_tail(int64_t U, int64_t N, const uint64_t* nr_used, uint64_t* ranges_out, const VbRangeParams& R,
                    int num_sms, cudaStream_t s);
void launch_vb_range_count(const void* keys, int key32, int64_t N, uint64_t* counts, cudaStream_t s);
void launch_vb_range_scatter(const void* keys, int key32, int64_t N, const uint64_t* offs, const uint64_t* total,
                             const VbRangeParams& R, cudaStream_t s);

} // namespace vox
