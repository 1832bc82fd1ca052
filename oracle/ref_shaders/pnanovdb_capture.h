/*
 * pnanovdb_capture.h - the handful of PNanoVDB/node2 calls that
 * gaussian_frag_color.slang makes around its value write, replaced by a
 * capture: the tree walk records nothing and resolves every voxel to a leaf
 * whose value slot is the fragment's own slot, so the shader's
 * InterlockedMax lands in a per-fragment output word.  Only the arithmetic
 * before the write (alpha, cull, RGBA8 packing) is under test here.
 *
 * TEST INFRASTRUCTURE ONLY.  Include inside the shader's namespace, after
 * slang_compat.h.
 */
typedef int3 pnanovdb_coord_t;
typedef uint32_t pnanovdb_uint32_t;
typedef uint64_t pnanovdb_uint64_t;
struct pnanovdb_address_t
{
    uint64_t byte_offset;
};
struct pnanovdb_grid_handle_t
{
    pnanovdb_address_t address;
};
struct pnanovdb_tree_handle_t
{
    pnanovdb_address_t address;
};
struct pnanovdb_root_handle_t
{
    pnanovdb_address_t address;
};
struct pnanovdb_node2_handle_t
{
    uint32_t idx64;
};
#define PNANOVDB_FALSE 0
#define PNANOVDB_NODE2_TYPE_LEAF 3
#define PNANOVDB_REF(x) x

static thread_local uint64_t g_capture_slot = 0;

inline pnanovdb_address_t pnanovdb_address_null()
{
    return pnanovdb_address_t{ 0 };
}
template <class B>
inline pnanovdb_tree_handle_t pnanovdb_grid_get_tree(B&, pnanovdb_grid_handle_t)
{
    return pnanovdb_tree_handle_t{ { 0 } };
}
template <class B>
inline pnanovdb_root_handle_t pnanovdb_tree_get_root(B&, pnanovdb_tree_handle_t)
{
    return pnanovdb_root_handle_t{ { 0 } };
}
template <class B>
inline pnanovdb_address_t pnanovdb_grid_get_gridblindmetadata_value_address(B&, pnanovdb_grid_handle_t, uint32_t)
{
    return pnanovdb_address_t{ 0 };
}
template <class B>
inline void pnanovdb_node2_find_node(B&, pnanovdb_node2_handle_t, pnanovdb_node2_handle_t& node, uint32_t& node_type,
                                     uint32_t& node_n, uint32_t& level, pnanovdb_coord_t)
{
    node.idx64 = 0;
    node_type = PNANOVDB_NODE2_TYPE_LEAF;
    node_n = 0;
    level = 0;
}
template <class B>
inline bool pnanovdb_node2_get_value_mask_bit(B&, pnanovdb_node2_handle_t, uint32_t, uint32_t)
{
    return true;
}
template <class B>
inline uint64_t pnanovdb_node2_get_value_index(B&, pnanovdb_node2_handle_t, uint32_t, uint32_t, int,
                                               pnanovdb_address_t, pnanovdb_address_t)
{
    return g_capture_slot;
}
inline pnanovdb_address_t pnanovdb_address_offset64_product(pnanovdb_address_t a, uint64_t idx, uint32_t mul)
{
    return pnanovdb_address_t{ a.byte_offset + idx * mul };
}
