// vox_order.cu - the reference's node order (VOX_FLAG_WINDOW_ORDER).
//
// The reference builds the tree window by window: Gaussians in batches of
// 256K, each batch's bbox fragments in windows of 8M (raster/Raster.cpp:443-444),
// and per window, level by level (upper, lower, leaf), the nodes the window
// creates are appended to one node pool in (parent node_idx, n) order
// (raster/GridBuild.cpp:412-505, grid_build_scatter_new.slang:107-170).
// node_idx is a node's position in that pool, node2 addresses follow node_idx
// order, and every node's value_idx is 2 + the active voxels of the leaves
// before it in node_idx order (so uppers and lowers created in a later window
// carry the count of the earlier windows' leaves).
//
// A node is created in the first window holding a passing fragment of one of
// its voxels.  The leaf walk records that window per candidate leaf (the
// minimum over its passing pairs); lowers and uppers take the minimum over
// their children.  Per level, a sort by (window, parent rank, n) gives each
// node's rank; per-window counts place the levels of a window after the
// nodes of every earlier window.
#include <cstdio>
#include <cuda_runtime.h>

#include "pnanovdb_b200.h"
#include "vox_device.cuh"
#include "vox_internal.h"
#include "vox_raster.h"

namespace vox
{

// windows of each 256K-Gaussian batch: ceil(fragments / 8M)
__global__ void k_batch_windows(const uint64_t* frag_off, const uint64_t* F_total, int64_t G, int64_t nbatch,
                                uint64_t* nwin)
{
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbatch)
        return;
    const int64_t g0 = b * REF_PRIM_BATCH, g1 = min(G, g0 + (int64_t)REF_PRIM_BATCH);
    const uint64_t f0 = frag_off[g0], f1 = g1 < G ? frag_off[g1] : *F_total;
    nwin[b] = (f1 - f0 + REF_WINDOW - 1) / REF_WINDOW;
}

__global__ void k_leaf_wkey(int64_t L, const uint32_t* leaf_vstart, const uint32_t* vslot, const uint64_t* cand_wkey,
                            uint64_t* leaf_wkey)
{
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l < L)
        leaf_wkey[l] = cand_wkey[vslot[leaf_vstart[l]] >> 9];
}

// minimum over the children runs [start[i], start[i + 1])
__global__ void k_run_min(int64_t n, const uint32_t* start, const uint64_t* child, uint64_t* out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    uint64_t m = ~0ull;
    for (uint32_t c = start[i]; c < start[i + 1]; c++)
        m = child[c] < m ? child[c] : m;
    out[i] = m;
}

// sort key of a level: window << 40 | parent rank << 15 | n
__global__ void k_level_keys(int64_t n, const uint64_t* wkey, const uint32_t* parent, const uint32_t* parent_rank,
                             const uint32_t* nval, uint32_t nmask, uint64_t* keys, uint32_t* vals, uint64_t* wcount)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint64_t pr = parent ? (uint64_t)parent_rank[parent[i]] : 0ull;
    keys[i] = (wkey[i] << 40) | (pr << 15) | (uint64_t)(nval[i] & nmask);
    vals[i] = (uint32_t)i;
    atomicAdd((unsigned long long*)&wcount[wkey[i]], 1ull);
}

__global__ void k_level_rank(int64_t n, const uint32_t* sorted_vals, uint32_t* rank)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n)
        rank[sorted_vals[p]] = (uint32_t)p;
}

__global__ void k_leaf_popc_sorted(int64_t L, const uint32_t* sorted_vals, const uint32_t* leaf_vstart,
                                   uint64_t* out)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L)
        return;
    const uint32_t l = sorted_vals[p];
    out[p] = (uint64_t)(leaf_vstart[l + 1] - leaf_vstart[l]);
}

// node_idx, byte address and value index of every node from its level rank and
// the per-window counts (base_* = nodes of each level in earlier windows)
__global__ void k_window_place(WindowOrderParams W, NodeParams N)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t root_sz = n2_node_bytes(0), up_sz = n2_node_bytes(1), lo_sz = n2_node_bytes(2),
                   lf_sz = n2_node_bytes(3);
    const uint64_t base_addr = N.C.grid_off[0] + VOX_GRID_HEADER_BYTES + root_sz;
    // every node's value_idx is 2 + the active voxels of the leaves before it in
    // node_idx order; the uppers and lowers of window w follow the leaves of the
    // earlier windows
    if (t < (int64_t)W.U)
    {
        const uint64_t p = W.rank_u[t], w = W.wkey_u[t];
        N.upper_idx[t] = 1 + W.base_all[w] + (p - W.base_u[w]);
        N.upper_addr[t] = base_addr + p * up_sz + W.base_lo[w] * lo_sz + W.base_leaf[w] * lf_sz;
        N.upper_vidx[t] = 2 + (W.base_leaf[w] < (uint64_t)N.L ? W.leaf_voff[W.base_leaf[w]] : W.V);
    }
    if (t < N.Lo)
    {
        const uint64_t p = W.rank_lo[t], w = W.wkey_lo[t];
        const uint64_t cu = W.base_u[w + 1] - W.base_u[w];
        N.lower_idx[t] = 1 + W.base_all[w] + cu + (p - W.base_lo[w]);
        N.lower_addr[t] = base_addr + W.base_u[w + 1] * up_sz + p * lo_sz + W.base_leaf[w] * lf_sz;
        N.lower_vidx[t] = 2 + (W.base_leaf[w] < (uint64_t)N.L ? W.leaf_voff[W.base_leaf[w]] : W.V);
    }
    if (t < N.L)
    {
        const uint64_t p = W.rank_leaf[t], w = W.wkey_leaf[t];
        const uint64_t cu = W.base_u[w + 1] - W.base_u[w], clo = W.base_lo[w + 1] - W.base_lo[w];
        N.leaf_idx[t] = 1 + W.base_all[w] + cu + clo + (p - W.base_leaf[w]);
        N.leaf_addr[t] = base_addr + W.base_u[w + 1] * up_sz + W.base_lo[w + 1] * lo_sz + p * lf_sz;
        N.leaf_vidx[t] = 2 + W.leaf_voff[p];
    }
}

__global__ void k_window_bases(int64_t nw, const uint64_t* cu, const uint64_t* clo, const uint64_t* cleaf,
                               uint64_t* base_u, uint64_t* base_lo, uint64_t* base_leaf, uint64_t* base_all)
{
    // one thread: the number of windows is small (total fragments / 8M)
    if (blockIdx.x != 0 || threadIdx.x != 0)
        return;
    uint64_t su = 0, slo = 0, sl = 0;
    for (int64_t w = 0; w < nw; w++)
    {
        base_u[w] = su;
        base_lo[w] = slo;
        base_leaf[w] = sl;
        base_all[w] = su + slo + sl;
        su += cu[w];
        slo += clo[w];
        sl += cleaf[w];
    }
    base_u[nw] = su;
    base_lo[nw] = slo;
    base_leaf[nw] = sl;
    base_all[nw] = su + slo + sl;
}

static unsigned blocks_for(int64_t n)
{
    return (unsigned)((n + 255) / 256 > 0 ? (n + 255) / 256 : 1);
}

void launch_batch_windows(const uint64_t* frag_off, const uint64_t* F_total, int64_t G, int64_t nbatch,
                          uint64_t* nwin, cudaStream_t s)
{
    if (nbatch <= 0)
        return;
    { k_batch_windows<<<blocks_for(nbatch), 256, 0, s>>>(frag_off, F_total, G, nbatch, nwin); count_launch(); }
}

void launch_leaf_wkey(int64_t L, const uint32_t* leaf_vstart, const uint32_t* vslot, const uint64_t* cand_wkey,
                      uint64_t* leaf_wkey, cudaStream_t s)
{
    if (L <= 0)
        return;
    { k_leaf_wkey<<<blocks_for(L), 256, 0, s>>>(L, leaf_vstart, vslot, cand_wkey, leaf_wkey); count_launch(); }
}

void launch_run_min(int64_t n, const uint32_t* start, const uint64_t* child, uint64_t* out, cudaStream_t s)
{
    if (n <= 0)
        return;
    { k_run_min<<<blocks_for(n), 256, 0, s>>>(n, start, child, out); count_launch(); }
}

void launch_level_keys(int64_t n, const uint64_t* wkey, const uint32_t* parent, const uint32_t* parent_rank,
                       const uint32_t* nval, uint32_t nmask, uint64_t* keys, uint32_t* vals, uint64_t* wcount,
                       cudaStream_t s)
{
    if (n <= 0)
        return;
    { k_level_keys<<<blocks_for(n), 256, 0, s>>>(n, wkey, parent, parent_rank, nval, nmask, keys, vals, wcount); count_launch(); }
}

void launch_level_rank(int64_t n, const uint32_t* sorted_vals, uint32_t* rank, cudaStream_t s)
{
    if (n <= 0)
        return;
    { k_level_rank<<<blocks_for(n), 256, 0, s>>>(n, sorted_vals, rank); count_launch(); }
}

void launch_leaf_popc_sorted(int64_t L, const uint32_t* sorted_vals, const uint32_t* leaf_vstart, uint64_t* out,
                             cudaStream_t s)
{
    if (L <= 0)
        return;
    { k_leaf_popc_sorted<<<blocks_for(L), 256, 0, s>>>(L, sorted_vals, leaf_vstart, out); count_launch(); }
}

void launch_window_bases(int64_t nw, const uint64_t* cu, const uint64_t* clo, const uint64_t* cleaf, uint64_t* base_u,
                         uint64_t* base_lo, uint64_t* base_leaf, uint64_t* base_all, cudaStream_t s)
{
    { k_window_bases<<<1, 1, 0, s>>>(nw, cu, clo, cleaf, base_u, base_lo, base_leaf, base_all); count_launch(); }
}

void launch_window_place(const WindowOrderParams& W, const NodeParams& N, cudaStream_t s)
{
    const int64_t n = N.L > N.Lo ? N.L : N.Lo;
    if (n <= 0)
        return;
    { k_window_place<<<blocks_for(n), 256, 0, s>>>(W, N); count_launch(); }
}

} // namespace vox
