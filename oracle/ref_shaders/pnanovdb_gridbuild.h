/*
 * pnanovdb_gridbuild.h - what the reference's grid-build shaders
 * (raster/shaders/grid_build_*.slang, workgroup_scan.slang) and the node2 core
 * of nanovdb_editor/PNanoVDBExt.h (its first part, compiled without
 * PNANOVDB_C) need to run as C++ on the host:
 *
 *   - generic primitives: integer types, the portability macros, 64-bit
 *     buffer words (a node2 buffer of uint2 words, low half first), address
 *     arithmetic, bit counts, Interlocked* on a buffer word (the host runs one
 *     shader thread at a time, so a plain read-modify-write is atomic);
 *   - NanoVDB grid / tree header calls, stubbed: the header fields the shaders
 *     read or write (root offset, node counts) live in a side struct, the
 *     blind-metadata setters are no-ops and the blind bbox value lives in a
 *     side record.  No byte layout of NanoVDB's GridData / TreeData /
 *     GridBlindMetaData is reproduced;
 *   - workgroups: 256 shader threads run as cooperative fibers so that
 *     GroupMemoryBarrierWithGroupSync() and `groupshared` memory behave as on
 *     a GPU (every thread reaches the barrier before any continues).
 *
 * TEST INFRASTRUCTURE ONLY (oracle/_ref/libref_shaders.so pins the CPU
 * oracle's topology build to the reference's shaders).  Include inside a
 * namespace, after slang_compat.h; the includer provides <stdint.h>,
 * <stdlib.h> and <string.h> at file scope.
 */

typedef uint32_t pnanovdb_uint32_t;
typedef uint64_t pnanovdb_uint64_t;
typedef int32_t pnanovdb_int32_t;
typedef int64_t pnanovdb_int64_t;
typedef bool pnanovdb_bool_t;
typedef int3 pnanovdb_coord_t;
#define PNANOVDB_TRUE true
#define PNANOVDB_FALSE false

#ifndef PNANOVDB_FORCE_INLINE
#define PNANOVDB_FORCE_INLINE static inline
#define PNANOVDB_STATIC_CONST static const
#define PNANOVDB_STRUCT_TYPEDEF(X)
#define PNANOVDB_INOUT(X) X&
#define PNANOVDB_DEREF(X) X
#define PNANOVDB_REF(X) X
#endif
#define groupshared static

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
struct pnanovdb_gridblindmetadata_handle_t
{
    pnanovdb_address_t address;
};

typedef StructuredBuffer<uint2> pnanovdb_buf_t;

/* -------------------------------------------------------- buffer words -- */
inline uint64_t pnanovdb_read_uint64(pnanovdb_buf_t buf, pnanovdb_address_t a)
{
    const uint2 w = buf[a.byte_offset >> 3];
    return (uint64_t)w.x | ((uint64_t)w.y << 32);
}
inline void pnanovdb_write_uint64(pnanovdb_buf_t buf, pnanovdb_address_t a, uint64_t v)
{
    buf[a.byte_offset >> 3] = uint2((uint)v, (uint)(v >> 32));
}
inline uint32_t pnanovdb_read_uint32(pnanovdb_buf_t buf, pnanovdb_address_t a)
{
    const uint2 w = buf[a.byte_offset >> 3];
    return (a.byte_offset & 4) ? w.y : w.x;
}
inline void pnanovdb_write_uint32(pnanovdb_buf_t buf, pnanovdb_address_t a, uint32_t v)
{
    uint2& w = buf[a.byte_offset >> 3];
    if (a.byte_offset & 4)
        w.y = v;
    else
        w.x = v;
}
inline void pnanovdb_write_coord(pnanovdb_buf_t buf, pnanovdb_address_t a, pnanovdb_coord_t c)
{
    pnanovdb_write_uint32(buf, pnanovdb_address_t{ a.byte_offset + 0 }, (uint32_t)c.x);
    pnanovdb_write_uint32(buf, pnanovdb_address_t{ a.byte_offset + 4 }, (uint32_t)c.y);
    pnanovdb_write_uint32(buf, pnanovdb_address_t{ a.byte_offset + 8 }, (uint32_t)c.z);
}

inline void InterlockedOr(uint& d, uint v)
{
    d |= v;
}
inline void InterlockedOr(uint& d, uint v, uint& old)
{
    old = d;
    d |= v;
}
inline void InterlockedAnd(uint& d, uint v)
{
    d &= v;
}

/* ------------------------------------------------------- addresses, bits -- */
inline pnanovdb_address_t pnanovdb_address_null()
{
    return pnanovdb_address_t{ 0 };
}
inline pnanovdb_address_t pnanovdb_address_offset(pnanovdb_address_t a, uint32_t off)
{
    return pnanovdb_address_t{ a.byte_offset + off };
}
inline pnanovdb_address_t pnanovdb_address_offset64(pnanovdb_address_t a, uint64_t off)
{
    return pnanovdb_address_t{ a.byte_offset + off };
}
inline pnanovdb_address_t pnanovdb_address_offset_product(pnanovdb_address_t a, uint32_t off, uint32_t mul)
{
    return pnanovdb_address_t{ a.byte_offset + (uint64_t)off * mul };
}
inline pnanovdb_address_t pnanovdb_address_offset64_product(pnanovdb_address_t a, uint64_t off, uint32_t mul)
{
    return pnanovdb_address_t{ a.byte_offset + off * mul };
}
inline uint64_t pnanovdb_address_diff(pnanovdb_address_t a, pnanovdb_address_t b)
{
    return a.byte_offset - b.byte_offset;
}
inline uint32_t pnanovdb_uint64_countbits(uint64_t v)
{
    return (uint32_t)__builtin_popcountll(v);
}
inline uint64_t pnanovdb_uint32_as_uint64(uint32_t lo, uint32_t hi)
{
    return (uint64_t)lo | ((uint64_t)hi << 32);
}
inline uint64_t pnanovdb_uint32_as_uint64_low(uint32_t lo)
{
    return (uint64_t)lo;
}
inline int32_t pnanovdb_uint32_as_int32(uint32_t v)
{
    return (int32_t)v;
}
inline uint32_t pnanovdb_uint64_to_uint32_lsr(uint64_t v, uint32_t s)
{
    return (uint32_t)(v >> s);
}

/* ------------------------------------- grid / tree headers (side struct) -- */
struct GbTreeFields
{
    uint64_t root_offset;                        /* root node, bytes from the tree */
    uint32_t count_upper, count_lower, count_leaf;
    uint64_t blind_value0;                       /* address of blind value 0 (the bbox) */
};
static GbTreeFields g_tree_fields;

inline pnanovdb_tree_handle_t pnanovdb_grid_get_tree(pnanovdb_buf_t, pnanovdb_grid_handle_t g)
{
    return pnanovdb_tree_handle_t{ g.address };
}
inline pnanovdb_root_handle_t pnanovdb_tree_get_root(pnanovdb_buf_t, pnanovdb_tree_handle_t t)
{
    return pnanovdb_root_handle_t{ { t.address.byte_offset + g_tree_fields.root_offset } };
}
inline uint64_t pnanovdb_tree_get_node_offset_root(pnanovdb_buf_t, pnanovdb_tree_handle_t)
{
    return g_tree_fields.root_offset;
}
inline uint32_t pnanovdb_tree_get_node_count_upper(pnanovdb_buf_t, pnanovdb_tree_handle_t)
{
    return g_tree_fields.count_upper;
}
inline uint32_t pnanovdb_tree_get_node_count_lower(pnanovdb_buf_t, pnanovdb_tree_handle_t)
{
    return g_tree_fields.count_lower;
}
inline uint32_t pnanovdb_tree_get_node_count_leaf(pnanovdb_buf_t, pnanovdb_tree_handle_t)
{
    return g_tree_fields.count_leaf;
}
inline void pnanovdb_tree_set_node_count_upper(pnanovdb_buf_t, pnanovdb_tree_handle_t, uint32_t v)
{
    g_tree_fields.count_upper = v;
}
inline void pnanovdb_tree_set_node_count_lower(pnanovdb_buf_t, pnanovdb_tree_handle_t, uint32_t v)
{
    g_tree_fields.count_lower = v;
}
inline void pnanovdb_tree_set_node_count_leaf(pnanovdb_buf_t, pnanovdb_tree_handle_t, uint32_t v)
{
    g_tree_fields.count_leaf = v;
}
inline pnanovdb_address_t pnanovdb_grid_get_gridblindmetadata_value_address(pnanovdb_buf_t, pnanovdb_grid_handle_t,
                                                                          uint32_t)
{
    return pnanovdb_address_t{ g_tree_fields.blind_value0 };
}
/* blind metadata headers: not reproduced */
#define PNANOVDB_GRIDBLINDMETADATA_SIZE 0u
#define PNANOVDB_GRID_TYPE_VEC3F 0u
#define PNANOVDB_GRID_TYPE_RGBA8 0u
template <class... A>
inline void pnanovdb_gridblindmetadata_set_data_offset(A...) {}
template <class... A>
inline void pnanovdb_gridblindmetadata_set_value_count(A...) {}
template <class... A>
inline void pnanovdb_gridblindmetadata_set_value_size(A...) {}
template <class... A>
inline void pnanovdb_gridblindmetadata_set_semantic(A...) {}
template <class... A>
inline void pnanovdb_gridblindmetadata_set_data_class(A...) {}
template <class... A>
inline void pnanovdb_gridblindmetadata_set_data_type(A...) {}
template <class... A>
inline void pnanovdb_gridblindmetadata_set_name(A...) {}
template <class... A>
inline void pnanovdb_grid_set_first_gridblindmetadata(A...) {}
template <class... A>
inline void pnanovdb_grid_set_blind_metadata_count(A...) {}
template <class... A>
inline void pnanovdb_grid_set_grid_size(A...) {}

/* -------------------------------------------- workgroups as fibers -------- */
/* A group's 256 threads are fibers on the calling thread, switched by a
 * minimal x86-64 context switch (callee-saved registers and the stack
 * pointer).  The scheduler runs every runnable fiber until it reaches the
 * barrier or returns; when none is runnable it releases the barrier. */
extern "C" void gb_fiber_switch(void** save_sp, void* load_sp);

struct GbGroup
{
    static const int THREADS = 256;
    static const size_t STACK = 128 * 1024;
    void* sched_sp;
    void* sp[THREADS];
    int state[THREADS]; /* 0 runnable, 1 at a barrier, 2 returned */
    int cur;
    char* stacks;
    void (*body)(uint32_t g, uint32_t t);
    uint32_t group;
};
static GbGroup* g_gb_group = nullptr;

inline void GroupMemoryBarrierWithGroupSync()
{
    GbGroup* G = g_gb_group;
    G->state[G->cur] = 1;
    gb_fiber_switch(&G->sp[G->cur], G->sched_sp);
}

static void gb_fiber_entry()
{
    GbGroup* G = g_gb_group;
    G->body(G->group, (uint32_t)G->cur);
    G->state[G->cur] = 2;
    void* dead;
    gb_fiber_switch(&dead, G->sched_sp);
    abort(); /* never resumed */
}

/* runs groups [0, groups) of `body` with workgroup barriers */
static void gb_run_groups(uint32_t groups, void (*body)(uint32_t g, uint32_t t))
{
    static GbGroup G;
    if (!G.stacks)
        G.stacks = (char*)malloc(GbGroup::STACK * GbGroup::THREADS);
    g_gb_group = &G;
    G.body = body;
    for (uint32_t g = 0; g < groups; g++)
    {
        G.group = g;
        for (int t = 0; t < GbGroup::THREADS; t++)
        {
            /* a fresh stack whose first switch "returns" into gb_fiber_entry:
             * six zeroed callee-saved registers, then the entry address, with
             * the entry seeing the stack alignment of a call */
            uintptr_t top = ((uintptr_t)(G.stacks + (size_t)(t + 1) * GbGroup::STACK)) & ~(uintptr_t)15;
            void** s = (void**)(top - 16);
            s[0] = (void*)&gb_fiber_entry;
            s[1] = nullptr;
            void** regs = s - 6;
            for (int r = 0; r < 6; r++)
                regs[r] = nullptr;
            G.sp[t] = (void*)regs;
            G.state[t] = 0;
        }
        for (;;)
        {
            for (int t = 0; t < GbGroup::THREADS; t++)
                if (G.state[t] == 0)
                {
                    G.cur = t;
                    gb_fiber_switch(&G.sched_sp, G.sp[t]);
                }
            bool waiting = false;
            for (int t = 0; t < GbGroup::THREADS; t++)
                if (G.state[t] == 1)
                {
                    G.state[t] = 0;
                    waiting = true;
                }
            if (!waiting)
                break;
        }
    }
}

/* groups without barriers: one thread after another */
static void gb_run_flat(uint32_t groups, void (*body)(uint32_t g, uint32_t t))
{
    for (uint32_t g = 0; g < groups; g++)
        for (uint32_t t = 0; t < 256; t++)
            body(g, t);
}
