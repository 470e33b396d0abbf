// bh.cuh -- Barnes-Hut octree layout shared by the builder and the walks.
//
// The tree is the reference's (gprt-core/src/lib.rs:340-539): a cube root
// around the bounding box, geometric octant splits at the cell centre, a
// cell is a leaf when it holds <= bucket bodies or its width drops below
// min_width, nodes in pre-order with next = self + 1 and an "autorope" to
// the node after the subtree, leaf buckets contiguous in the flat body
// order.  Node records (pre-order index):
//   node_a[i] = (com.x, com.y, com.z, mass)
//   node_b[i] = (autorope, bucket_start, count | LEAF_BIT, bits of width)
//   node_q[i] = traceless quadrupole about the COM (xx, yy, zz, xy, xz, yz, 0, 0)
#pragma once

#include "common.cuh"
#include "sort.cuh"

namespace rtd {

constexpr uint32_t BH_LEAF_BIT = 0x80000000u;
constexpr int BH_MAX_LEVEL = 21;            // octant digits held by a 63-bit path key
constexpr int BH_GROUP = 32;                // bodies per warp-coherent group

struct BhHeader {
    float root_min[3], root_max[3];
    float max_extent, scale;
    float min_b[3];
    uint32_t box[6];          // order-preserving bbox of the positions
    uint32_t lw;              // first level whose width < min_width
    uint32_t n_nodes, n_leaves;
    uint32_t err;
    uint32_t level_count[BH_MAX_LEVEL + 2];
    uint32_t level_off[BH_MAX_LEVEL + 3];
    uint32_t n_groups;        // warp groups of the Plummer walks
    uint32_t max_stack;       // deepest traversal stack seen by a walk
    uint32_t group_counter;   // work queue of the walks (next group to take)
    uint32_t ilog_used;       // interaction-log pages taken by the last logging forward
    uint32_t ilog_need;       // pages its groups needed (pool size for the next one)
};

// Interaction log of a Plummer forward walk: every tile of interactions a
// warp group evaluated (up to 32 (cell or body id, lane mask) entries),
// in evaluation order, in pages of ILOG_PAGE tiles chained per group, so
// that the adjoint replays the same decisions instead of walking the tree
// again.  group[g] = (first page, tiles), tiles = ILOG_NONE when the pool ran
// out before the group ended (that group walks).
constexpr uint32_t ILOG_PAGE = 16;
constexpr uint32_t ILOG_NONE = 0xFFFFFFFFu;
struct IlogView {
    uint2 *entries;     // pages * ILOG_PAGE * 32
    uint8_t *counts;    // pages * ILOG_PAGE: entries | 0x80 for a body tile
    uint32_t *next;     // pages: the group's next page
    uint2 *group;       // per warp group; nullptr = no log (forward) / walk (adjoint)
    uint32_t pages;     // pool capacity
};

// Traversal stack entries per walking warp: the slice each warp owns in a
// stack buffer.  The walks push within stack_entries <= BH_STACK_CAP_MAX
// (rtd_limits_set lowers it; a push beyond it is refused and reported as
// DEVERR_STACK).
constexpr uint32_t BH_STACK_CAP_MAX = 8192;
uint32_t bh_stack_entries();   // the current per-warp limit (capi.cu)

}  // namespace rtd

struct rtd_bh {
    uint64_t n = 0;
    uint32_t bucket = 128;
    float min_width = 1e-5f;
    bool built = false;
    bool plummer_ready = false;   // child table and groups built (Plummer-law walks)
    bool has_quad = false;        // quadrupoles computed
    rtd::DevBuf hdr;
    // build scratch
    rtd::DevBuf mkeys, mkeys_alt, mvals, mvals_alt;   // Morton sort
    rtd::DevBuf pkeys, pkeys_alt, pvals, pvals_alt;   // path-key sort (values: Morton rank)
    rtd::DevBuf lcp, wmin, lam, nn, base, heads, leaf_head, leaf_of;
    rtd::DevBuf fkeys, fkeys_alt, fvals, fvals_alt;   // final regroup sort
    rtd::DevBuf node_start, node_level, level_nodes;
    rtd::SortScratch sort;
    rtd::ScanScratch scan;
    // tree
    rtd::DevBuf order;        // flat order: original index of the i-th body
    rtd::DevBuf fbody;        // float4 (pos, mass) in flat order
    rtd::DevBuf node_a, node_b, node_q;
    // walk structures: child table (8 per node), leaf list, warp groups
    rtd::DevBuf child8, leaf_node, groups, stack;
    uint64_t stack_warps = 0;
    // adjoint scratch
    rtd::DevBuf cell_grad, prefix, gpos_flat, gmass_flat;
    // interaction log (Plummer forward -> adjoint), kept once a backward has
    // followed a forward on this handle; its pool is sized from the last
    // logging forward's need (a pinned copy read when it has landed)
    rtd::DevBuf ilog_entries, ilog_counts, ilog_next, ilog_group;
    uint32_t ilog_pages = 0;
    bool ilog_valid = false;      // the log holds the last forward's decisions
    float ilog_theta = 0.f;
    int ilog_quad = -1;
    bool backward_seen = false;
    uint32_t *ilog_hint = nullptr;   // pinned: pages the last logging forward needed
    cudaEvent_t ilog_ev = nullptr;
    ~rtd_bh();
};

// Device buffers a host-buffer context keeps for barnes_hut! calls.
struct rtd_context_bh {
    rtd_bh bh;
    rtd::DevBuf bodies, pos, mass, out;
};

namespace rtd {

struct BhView {
    const float4 *node_a;
    const uint4 *node_b;
    const float4 *node_q;      // 2 float4 per node
    const float4 *fbody;
    const uint32_t *order;
    const BhHeader *hdr;
    uint64_t n;
    const uint4 *child8;       // 2 uint4 per node: up to 8 children, 0xFFFFFFFF pads
    const uint2 *groups;       // (first flat body, count <= 32)
};

inline BhView bh_view(const rtd_bh *b) {
    return BhView{b->node_a.as<float4>(), b->node_b.as<uint4>(), b->node_q.as<float4>(),
                  b->fbody.as<float4>(), b->order.as<uint32_t>(), b->hdr.as<BhHeader>(), b->n,
                  b->child8.as<uint4>(), b->groups.as<uint2>()};
}

rtd_status bh_build(rtd_bh *b, const float *d_pos, const float *d_mass, uint64_t n,
                    const rtd_bh_params *p, cudaStream_t st);

}  // namespace rtd
