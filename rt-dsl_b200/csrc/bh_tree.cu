// bh_tree.cu -- GPU build of the reference Barnes-Hut octree.
//
// The reference builds recursively on the CPU (gprt-core/src/lib.rs:
// 427-539): Morton-sort the bodies (scale 1023/max_extent from the bbox
// minimum), then split each cell at its centre into up to eight octant
// children (stable partition, children in octant order), stopping at
// <= bucket bodies or width < min_width; COM bottom-up; pre-order flatten.
// The same tree comes out of a flat, data-parallel pipeline here:
//
//   1. bbox -> root cube, Morton codes, stable radix sort (order M)
//   2. per body: the octant path of the first 21 levels, computed with the
//      reference's float operations (centre = (min + max) * 0.5, child box
//      from min/centre/max), packed 3 bits per level into a 63-bit key;
//      stable radix sort of M by that key (order P: every cell contiguous)
//   3. lcp[i]: levels shared by the keys of P-neighbours i, i+1.  A cell at
//      level l around body j holds > bucket bodies iff some window of
//      bucket+1 consecutive bodies containing j shares >= l levels, so a
//      windowed min (over lcp) then max gives each body's leaf level
//   4. the tree nodes starting at body j are the cells of levels
//      lcp[j-1]+1 .. leaf_level[j]; a scan numbers them in pre-order
//   5. flat order F = M stably regrouped by leaf (what the recursive stable
//      partition produces); COM/mass (and quadrupoles) bottom-up, each node
//      summing its bodies or children sequentially in the reference order.
#include <rtdsl.h>

#include "bh.cuh"

namespace rtd {
namespace {

constexpr int BLOCK = 256;

__global__ void bh_hdr_init_kernel(BhHeader *h) {
    for (int a = 0; a < 3; ++a) {
        h->box[a] = 0xFFFFFFFFu;
        h->box[3 + a] = 0u;
    }
    h->err = 0;
    h->max_stack = 0;
    h->n_nodes = 0;
    h->n_leaves = 0;
    for (int l = 0; l < BH_MAX_LEVEL + 2; ++l) h->level_count[l] = 0;
}

__global__ void __launch_bounds__(BLOCK) bh_bbox_kernel(const float *__restrict__ pos, uint64_t n,
                                                        BhHeader *h) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK)
        for (int a = 0; a < 3; ++a) {
            float v = pos[3 * i + a];
            lo[a] = fminf(lo[a], v);
            hi[a] = fmaxf(hi[a], v);
        }
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a) {
            atomicMin(&h->box[a], float_flip(lo[a]));
            atomicMax(&h->box[3 + a], float_flip(hi[a]));
        }
}

// BarnesHutTree::build root (lib.rs:431-443): cube of side max_extent
// around the bbox centre; Morton scale 1023 / max_extent.
__global__ void bh_root_kernel(BhHeader *h, float min_width) {
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a) {
        mn[a] = float_unflip(h->box[a]);
        mx[a] = float_unflip(h->box[3 + a]);
    }
    float ex = __fsub_rn(mx[0], mn[0]), ey = __fsub_rn(mx[1], mn[1]), ez = __fsub_rn(mx[2], mn[2]);
    float me = fmaxf(fmaxf(ex, ey), ez);
    float half = __fdiv_rn(me, 2.0f);
    for (int a = 0; a < 3; ++a) {
        float c = __fmul_rn(__fadd_rn(mn[a], mx[a]), 0.5f);
        h->root_min[a] = __fsub_rn(c, half);
        h->root_max[a] = __fadd_rn(c, half);
        h->min_b[a] = mn[a];
    }
    h->max_extent = me;
    h->scale = me > 0.0f ? __fdiv_rn(1023.0f, me) : 0.0f;
    uint32_t l = 0;
    float w = me;
    while (!(w < min_width) && l < 64) {
        w = __fmul_rn(w, 0.5f);
        ++l;
    }
    h->lw = l;
}

// Rust `f32 as u32`: saturating, NaN -> 0.
__device__ __forceinline__ uint32_t f2u_sat(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

__global__ void __launch_bounds__(BLOCK) bh_morton_kernel(const float *__restrict__ pos, uint64_t n,
                                                          const BhHeader *h,
                                                          uint32_t *__restrict__ keys) {
    const float sc = h->scale;
    const float m0 = h->min_b[0], m1 = h->min_b[1], m2 = h->min_b[2];
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK) {
        uint32_t lx = f2u_sat(__fmul_rn(__fsub_rn(pos[3 * i], m0), sc));
        uint32_t ly = f2u_sat(__fmul_rn(__fsub_rn(pos[3 * i + 1], m1), sc));
        uint32_t lz = f2u_sat(__fmul_rn(__fsub_rn(pos[3 * i + 2], m2), sc));
        keys[i] = morton30(lx, ly, lz);   // expand_bits keeps the low 10 bits (lib.rs:263)
    }
}

// Octant path of one body from the root cube, `levels` levels deep, with
// the reference's centre / child-box arithmetic (lib.rs:363-407).  Also
// returns the cell box at that depth.
__device__ __forceinline__ uint64_t octant_path(float px, float py, float pz, const BhHeader *h,
                                                int levels, float mn[3], float mx[3]) {
    for (int a = 0; a < 3; ++a) { mn[a] = h->root_min[a]; mx[a] = h->root_max[a]; }
    uint64_t key = 0;
    const float p[3] = {px, py, pz};
    for (int l = 1; l <= levels; ++l) {
        uint32_t oct = 0;
        for (int a = 0; a < 3; ++a) {
            float c = __fmul_rn(__fadd_rn(mn[a], mx[a]), 0.5f);
            bool up = p[a] >= c;
            oct |= (up ? 1u : 0u) << a;
            if (up) mn[a] = c;
            else mx[a] = c;
        }
        key |= (uint64_t)oct << (3 * (BH_MAX_LEVEL - l));
    }
    return key;
}

__global__ void __launch_bounds__(BLOCK) bh_path_kernel(const float *__restrict__ pos, uint64_t n,
                                                        const uint32_t *__restrict__ morder,
                                                        const BhHeader *h,
                                                        uint64_t *__restrict__ pkeys) {
    for (uint64_t r = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; r < n;
         r += (uint64_t)gridDim.x * BLOCK) {
        uint32_t b = morder[r];
        float mn[3], mx[3];
        pkeys[r] = octant_path(pos[3 * (uint64_t)b], pos[3 * (uint64_t)b + 1],
                               pos[3 * (uint64_t)b + 2], h, BH_MAX_LEVEL, mn, mx);
    }
}

__device__ __forceinline__ int key_lcp(uint64_t a, uint64_t b) {
    if (a == b) return BH_MAX_LEVEL;
    return (__clzll((long long)(a ^ b)) - 1) / 3;   // bit 63 is always clear
}

__global__ void __launch_bounds__(BLOCK) bh_lcp_kernel(const uint64_t *__restrict__ pk, uint64_t n,
                                                       uint8_t *__restrict__ lcp) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i + 1 < n;
         i += (uint64_t)gridDim.x * BLOCK)
        lcp[i] = (uint8_t)key_lcp(pk[i], pk[i + 1]);
}

// W[a] = min(lcp[a .. a+B-1]): levels shared by the B+1 bodies a..a+B.
__global__ void __launch_bounds__(BLOCK) bh_window_min_kernel(const uint8_t *__restrict__ lcp,
                                                              uint64_t nwin, uint32_t B,
                                                              uint8_t *__restrict__ w) {
    for (uint64_t a = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; a < nwin;
         a += (uint64_t)gridDim.x * BLOCK) {
        uint32_t m = 255;
        for (uint32_t t = 0; t < B; ++t) m = min(m, (uint32_t)lcp[a + t]);
        w[a] = (uint8_t)m;
    }
}

// Leaf level of body j: one past the deepest level at which some window
// containing j holds B+1 bodies, capped by the width stop.
__global__ void __launch_bounds__(BLOCK) bh_lambda_kernel(const uint8_t *__restrict__ w, uint64_t n,
                                                          uint64_t nwin, uint32_t B,
                                                          BhHeader *h, uint8_t *__restrict__ lam) {
    const uint32_t lw = h->lw;
    for (uint64_t j = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * BLOCK) {
        int m = -1;
        if (nwin > 0) {
            uint64_t a0 = j >= B ? j - B : 0;
            uint64_t a1 = j < nwin - 1 ? j : nwin - 1;
            for (uint64_t a = a0; a <= a1; ++a) m = max(m, (int)w[a]);
        }
        uint32_t l = (uint32_t)(m + 1);
        if (l > lw) l = lw;
        if (l > BH_MAX_LEVEL) {   // a cell 21 levels down still too full to be a leaf
            atomicOr(&h->err, DEVERR_DEPTH);
            l = BH_MAX_LEVEL;
        }
        lam[j] = (uint8_t)l;
    }
}

__device__ __forceinline__ int lcp_before(const uint8_t *lcp, uint64_t j) {
    return j == 0 ? -1 : (int)lcp[j - 1];
}

// Nodes starting at body j (levels lcp[j-1]+1 .. lam[j]) and leaf heads.
__global__ void __launch_bounds__(BLOCK) bh_count_kernel(const uint8_t *__restrict__ lcp,
                                                         const uint8_t *__restrict__ lam, uint64_t n,
                                                         uint32_t *__restrict__ nn,
                                                         uint32_t *__restrict__ heads) {
    for (uint64_t j = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * BLOCK) {
        int c = (int)lam[j] - lcp_before(lcp, j);
        nn[j] = c > 0 ? (uint32_t)c : 0u;
        heads[j] = c > 0 ? 1u : 0u;
    }
}

__global__ void __launch_bounds__(BLOCK) bh_nodes_kernel(
    const uint8_t *__restrict__ lcp, const uint8_t *__restrict__ lam,
    const uint32_t *__restrict__ nn, const uint32_t *__restrict__ base,
    const uint32_t *__restrict__ leafidx, uint64_t n, uint32_t *__restrict__ node_start,
    uint8_t *__restrict__ node_level, uint32_t *__restrict__ leaf_head,
    uint32_t *__restrict__ leaf_node, BhHeader *h) {
    for (uint64_t j = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * BLOCK) {
        uint32_t c = nn[j];
        if (!c) continue;
        int l0 = lcp_before(lcp, j) + 1;
        for (uint32_t t = 0; t < c; ++t) {
            node_start[base[j] + t] = (uint32_t)j;
            node_level[base[j] + t] = (uint8_t)(l0 + (int)t);
            atomicAdd(&h->level_count[l0 + t], 1u);
        }
        leaf_head[leafidx[j]] = (uint32_t)j;
        leaf_node[leafidx[j]] = base[j] + c - 1;   // the deepest node starting at j
        (void)lam;
    }
}

// Child table: up to 8 children per internal node (first child = i + 1,
// next sibling = autorope), padded with 0xFFFFFFFF.
__global__ void __launch_bounds__(BLOCK) bh_child_kernel(const BhHeader *h,
                                                         const uint4 *__restrict__ node_b,
                                                         uint4 *__restrict__ child8) {
    const uint32_t n_nodes = h->n_nodes;
    for (uint32_t i = blockIdx.x * BLOCK + threadIdx.x; i < n_nodes; i += gridDim.x * BLOCK) {
        uint32_t c[8];
        for (int k = 0; k < 8; ++k) c[k] = 0xFFFFFFFFu;
        const uint4 b = node_b[i];
        if (!(b.z & BH_LEAF_BIT)) {
            int k = 0;
            for (uint32_t x = i + 1; x < b.x && k < 8; x = node_b[x].x) c[k++] = x;
        }
        child8[2 * i] = make_uint4(c[0], c[1], c[2], c[3]);
        child8[2 * i + 1] = make_uint4(c[4], c[5], c[6], c[7]);
    }
}

// Warp groups for the Plummer walks: runs of sibling leaves (consecutive
// pre-order nodes at the same level) packed greedily up to 32 bodies;
// a leaf of more than 32 bodies is split into chunks of 32.  The run head
// writes, per leaf, the number of groups starting there (gcnt) and the
// body count of a packed group starting there (gsize).
__device__ __forceinline__ bool next_sibling_leaf(const uint32_t *leaf_node, const uint8_t *lvl,
                                                  uint32_t m) {
    return leaf_node[m] == leaf_node[m - 1] + 1 && lvl[leaf_node[m]] == lvl[leaf_node[m - 1]];
}

__global__ void __launch_bounds__(BLOCK) bh_group_plan_kernel(const BhHeader *h,
                                                              const uint32_t *__restrict__ leaf_node,
                                                              const uint8_t *__restrict__ lvl,
                                                              const uint4 *__restrict__ node_b,
                                                              uint32_t *__restrict__ gcnt,
                                                              uint32_t *__restrict__ gsize) {
    const uint32_t nl = h->n_leaves;
    for (uint32_t m = blockIdx.x * BLOCK + threadIdx.x; m < nl; m += gridDim.x * BLOCK) {
        if (m > 0 && next_sibling_leaf(leaf_node, lvl, m)) continue;   // not a run head
        uint32_t open = 0xFFFFFFFFu, acc = 0;
        for (uint32_t t = m; t < nl && (t == m || next_sibling_leaf(leaf_node, lvl, t)); ++t) {
            const uint32_t c = node_b[leaf_node[t]].z & ~BH_LEAF_BIT;
            if (c > (uint32_t)BH_GROUP) {
                if (open != 0xFFFFFFFFu) gsize[open] = acc;
                open = 0xFFFFFFFFu;
                acc = 0;
                gcnt[t] = (c + BH_GROUP - 1) / BH_GROUP;
                gsize[t] = 0;
                continue;
            }
            if (open != 0xFFFFFFFFu && acc + c <= (uint32_t)BH_GROUP) {
                acc += c;
                gcnt[t] = 0;
            } else {
                if (open != 0xFFFFFFFFu) gsize[open] = acc;
                open = t;
                acc = c;
                gcnt[t] = 1;
            }
        }
        if (open != 0xFFFFFFFFu) gsize[open] = acc;
    }
}

__global__ void __launch_bounds__(BLOCK) bh_group_write_kernel(BhHeader *h,
                                                               const uint32_t *__restrict__ leaf_node,
                                                               const uint4 *__restrict__ node_b,
                                                               const uint32_t *__restrict__ gcnt,
                                                               const uint32_t *__restrict__ gsize,
                                                               const uint32_t *__restrict__ goff,
                                                               const uint32_t *__restrict__ gtotal,
                                                               uint2 *__restrict__ groups) {
    const uint32_t nl = h->n_leaves;
    if (blockIdx.x == 0 && threadIdx.x == 0) h->n_groups = *gtotal;
    for (uint32_t m = blockIdx.x * BLOCK + threadIdx.x; m < nl; m += gridDim.x * BLOCK) {
        const uint32_t k = gcnt[m];
        if (!k) continue;
        const uint4 b = node_b[leaf_node[m]];
        const uint32_t s = b.y, c = b.z & ~BH_LEAF_BIT;
        if (c > (uint32_t)BH_GROUP) {
            for (uint32_t t = 0; t < k; ++t) {
                const uint32_t cs = t * BH_GROUP;
                groups[goff[m] + t] = make_uint2(s + cs, min((uint32_t)BH_GROUP, c - cs));
            }
        } else {
            groups[goff[m]] = make_uint2(s, gsize[m]);
        }
    }
}

// Node records: end of each node's body range (leaves: next leaf head;
// internal: first later leaf whose boundary shares < level levels, found
// by a warp scanning 32 leaf boundaries at a time), autorope, counts,
// width of the cell box.  One warp per node.
__global__ void __launch_bounds__(BLOCK) bh_records_kernel(
    const float *__restrict__ pos, const uint32_t *__restrict__ morder,
    const uint32_t *__restrict__ pvals, const uint8_t *__restrict__ lcp,
    const uint32_t *__restrict__ base, const uint32_t *__restrict__ leafidx,
    const uint32_t *__restrict__ leaf_head, const uint32_t *__restrict__ node_start,
    const uint8_t *__restrict__ node_level, uint64_t n, BhHeader *h, uint4 *__restrict__ node_b,
    uint32_t *__restrict__ level_nodes, uint32_t *__restrict__ level_fill) {
    const uint32_t n_nodes = h->n_nodes, n_leaves = h->n_leaves;
    const int lane = threadIdx.x & 31;
    const uint64_t warp0 = ((uint64_t)blockIdx.x * BLOCK + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * BLOCK) >> 5;
    for (uint64_t i = warp0; i < n_nodes; i += nwarps) {
        const uint32_t j = node_start[i];
        const int l = node_level[i];
        const uint32_t m0 = leafidx[j];
        const bool leaf = (i + 1 == n_nodes) || node_start[i + 1] != j;
        uint64_t end = n;
        if (leaf) {
            end = m0 + 1 < n_leaves ? leaf_head[m0 + 1] : n;
        } else {
            for (uint64_t m = (uint64_t)m0 + 1; m < n_leaves; m += 32) {
                uint64_t mm = m + lane;
                bool stop = false;
                uint32_t hh = 0;
                if (mm < n_leaves) {
                    hh = leaf_head[mm];
                    stop = (int)lcp[hh - 1] < l;
                }
                uint32_t bal = __ballot_sync(0xffffffffu, stop);
                if (bal) {
                    end = __shfl_sync(0xffffffffu, hh, __ffs(bal) - 1);
                    break;
                }
            }
        }
        if (lane == 0) {
            uint32_t autorope = end < n ? base[end] : n_nodes;
            // cell box: descend l levels along the path of this cell's first body
            uint32_t b = morder[pvals[j]];
            float mn[3], mx[3];
            octant_path(pos[3 * (uint64_t)b], pos[3 * (uint64_t)b + 1], pos[3 * (uint64_t)b + 2], h,
                        l, mn, mx);
            float w = fmaxf(fmaxf(__fsub_rn(mx[0], mn[0]), __fsub_rn(mx[1], mn[1])),
                            __fsub_rn(mx[2], mn[2]));
            uint32_t cnt = (uint32_t)(end - j);
            node_b[i] = make_uint4(autorope, j, (leaf ? BH_LEAF_BIT : 0u) | cnt, __float_as_uint(w));
            uint32_t slot = atomicAdd(&level_fill[l], 1u);
            level_nodes[h->level_off[l] + slot] = (uint32_t)i;
        }
    }
}

__global__ void bh_level_offsets_kernel(BhHeader *h) {
    uint32_t acc = 0;
    for (int l = 0; l < BH_MAX_LEVEL + 2; ++l) {
        h->level_off[l] = acc;
        acc += h->level_count[l];
    }
    h->level_off[BH_MAX_LEVEL + 2] = acc;
}

__global__ void bh_totals_kernel(BhHeader *h, const uint32_t *nn_total, const uint32_t *leaf_total) {
    h->n_nodes = *nn_total;
    h->n_leaves = *leaf_total;
}

// Leaf position of every P-ordered body, scattered to its Morton rank.
__global__ void __launch_bounds__(BLOCK) bh_leafof_kernel(const uint32_t *__restrict__ leafidx,
                                                          const uint32_t *__restrict__ heads,
                                                          const uint32_t *__restrict__ pvals,
                                                          const uint32_t *__restrict__ morder,
                                                          uint64_t n, uint32_t *__restrict__ fkeys,
                                                          uint32_t *__restrict__ fvals) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK) {
        uint32_t leaf = leafidx[i] + heads[i] - 1u;
        uint32_t r = pvals[i];
        fkeys[r] = leaf;
        fvals[r] = morder[r];
    }
}

__global__ void __launch_bounds__(BLOCK) bh_flat_kernel(const float *__restrict__ pos,
                                                        const float *__restrict__ mass,
                                                        const uint32_t *__restrict__ f, uint64_t n,
                                                        uint32_t *__restrict__ order,
                                                        float4 *__restrict__ fbody) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK) {
        uint32_t b = f[i];
        order[i] = b;
        fbody[i] = make_float4(pos[3 * (uint64_t)b], pos[3 * (uint64_t)b + 1],
                               pos[3 * (uint64_t)b + 2], mass[b]);
    }
}

// compute_com leaves (lib.rs:472-484): sequential sums over the bucket in
// flat order; optional traceless quadrupole about the COM.
__global__ void __launch_bounds__(BLOCK) bh_leaf_com_kernel(const BhHeader *h,
                                                            const uint4 *__restrict__ node_b,
                                                            const float4 *__restrict__ fbody,
                                                            float4 *__restrict__ node_a,
                                                            float4 *__restrict__ node_q, int quad) {
    const uint32_t n_nodes = h->n_nodes;
    for (uint32_t i = blockIdx.x * BLOCK + threadIdx.x; i < n_nodes; i += gridDim.x * BLOCK) {
        uint4 b = node_b[i];
        if (!(b.z & BH_LEAF_BIT)) continue;
        const uint32_t s = b.y, c = b.z & ~BH_LEAF_BIT;
        float tm = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
        for (uint32_t k = 0; k < c; ++k) {
            float4 p = fbody[s + k];
            tm = __fadd_rn(tm, p.w);
            cx = __fadd_rn(cx, __fmul_rn(p.x, p.w));
            cy = __fadd_rn(cy, __fmul_rn(p.y, p.w));
            cz = __fadd_rn(cz, __fmul_rn(p.z, p.w));
        }
        if (tm > 0.0f) { cx = __fdiv_rn(cx, tm); cy = __fdiv_rn(cy, tm); cz = __fdiv_rn(cz, tm); }
        else { cx = cy = cz = 0.0f; }
        node_a[i] = make_float4(cx, cy, cz, tm);
        if (quad) {
            float q[6] = {0, 0, 0, 0, 0, 0};
            for (uint32_t k = 0; k < c; ++k) {
                float4 p = fbody[s + k];
                float dx = p.x - cx, dy = p.y - cy, dz = p.z - cz;
                float r2 = dx * dx + dy * dy + dz * dz;
                q[0] += p.w * (3.f * dx * dx - r2);
                q[1] += p.w * (3.f * dy * dy - r2);
                q[2] += p.w * (3.f * dz * dz - r2);
                q[3] += p.w * 3.f * dx * dy;
                q[4] += p.w * 3.f * dx * dz;
                q[5] += p.w * 3.f * dy * dz;
            }
            node_q[2 * i] = make_float4(q[0], q[1], q[2], q[3]);
            node_q[2 * i + 1] = make_float4(q[4], q[5], 0.f, 0.f);
        }
    }
}

// compute_com internal nodes (lib.rs:487-500), deepest level first: each
// node sums its children in order (child = i+1, next sibling = autorope).
// Quadrupoles combine by the parallel-axis rule.  One block; levels are
// separated by __syncthreads().
__global__ void __launch_bounds__(1024) bh_internal_com_kernel(const BhHeader *h,
                                                               const uint4 *__restrict__ node_b,
                                                               const uint32_t *__restrict__ level_nodes,
                                                               float4 *node_a, float4 *node_q,
                                                               int quad) {
    for (int l = BH_MAX_LEVEL + 1; l >= 0; --l) {
        const uint32_t off = h->level_off[l], cnt = h->level_count[l];
        for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) {
            const uint32_t i = level_nodes[off + t];
            const uint4 b = node_b[i];
            if (b.z & BH_LEAF_BIT) continue;
            float tm = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
            for (uint32_t c = i + 1; c < b.x; c = node_b[c].x) {
                float4 a = node_a[c];
                tm = __fadd_rn(tm, a.w);
                cx = __fadd_rn(cx, __fmul_rn(a.x, a.w));
                cy = __fadd_rn(cy, __fmul_rn(a.y, a.w));
                cz = __fadd_rn(cz, __fmul_rn(a.z, a.w));
            }
            if (tm > 0.0f) { cx = __fdiv_rn(cx, tm); cy = __fdiv_rn(cy, tm); cz = __fdiv_rn(cz, tm); }
            else { cx = cy = cz = 0.0f; }
            node_a[i] = make_float4(cx, cy, cz, tm);
            if (quad) {
                float q[6] = {0, 0, 0, 0, 0, 0};
                for (uint32_t c = i + 1; c < b.x; c = node_b[c].x) {
                    float4 a = node_a[c];
                    float4 q0 = node_q[2 * c], q1 = node_q[2 * c + 1];
                    float dx = a.x - cx, dy = a.y - cy, dz = a.z - cz;
                    float r2 = dx * dx + dy * dy + dz * dz;
                    q[0] += q0.x + a.w * (3.f * dx * dx - r2);
                    q[1] += q0.y + a.w * (3.f * dy * dy - r2);
                    q[2] += q0.z + a.w * (3.f * dz * dz - r2);
                    q[3] += q0.w + a.w * 3.f * dx * dy;
                    q[4] += q1.x + a.w * 3.f * dx * dz;
                    q[5] += q1.y + a.w * 3.f * dy * dz;
                }
                node_q[2 * i] = make_float4(q[0], q[1], q[2], q[3]);
                node_q[2 * i + 1] = make_float4(q[4], q[5], 0.f, 0.f);
            }
        }
        __syncthreads();
    }
}

}  // namespace

rtd_status check_bh_errors(rtd_bh *b, cudaStream_t st);

rtd_status bh_build(rtd_bh *b, const float *d_pos, const float *d_mass, uint64_t n,
                    const rtd_bh_params *p, cudaStream_t st) {
    if (!b) return fail(RTD_ERR_INVALID_ARGUMENT, "bh handle is NULL");
    if (n > 0 && (!d_pos || !d_mass)) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL positions or masses");
    if (n >= (1ull << 30) - 1) return fail(RTD_ERR_INVALID_ARGUMENT, "at most 2^30-2 bodies");
    rtd_bh_params def;
    rtd_bh_params_default(&def);
    if (!p) p = &def;
    if (p->bucket < 1 || p->bucket > 4096) return fail(RTD_ERR_INVALID_ARGUMENT, "bucket must be in [1, 4096]");
    b->built = false;
    b->plummer_ready = false;
    b->has_quad = false;
    b->n = n;
    b->bucket = p->bucket;
    b->min_width = p->min_width;
    const int quad = p->law == RTD_BH_LAW_PLUMMER && p->quadrupole;
    RTD_TRY(b->hdr.reserve(sizeof(BhHeader)));
    BhHeader *h = b->hdr.as<BhHeader>();
    bh_hdr_init_kernel<<<1, 1, 0, st>>>(h);
    RTD_LAUNCH_CHECK();
    if (n == 0) {
        b->built = true;
    b->ilog_valid = false;   // a new tree: the last forward's log no longer applies
        return RTD_OK;
    }
    const uint64_t n1 = n;
    for (DevBuf *d : {&b->mkeys, &b->mkeys_alt, &b->mvals, &b->mvals_alt, &b->pvals, &b->pvals_alt,
                      &b->nn, &b->base, &b->heads, &b->leaf_head, &b->fkeys, &b->fkeys_alt,
                      &b->fvals, &b->fvals_alt, &b->node_start, &b->order, &b->level_nodes,
                      &b->leaf_node})
        RTD_TRY(d->reserve(n1 * 4 + 16));
    RTD_TRY(b->pkeys.reserve(n1 * 8));
    RTD_TRY(b->pkeys_alt.reserve(n1 * 8));
    RTD_TRY(b->lcp.reserve(n1 + 16));
    RTD_TRY(b->wmin.reserve(n1 + 16));
    RTD_TRY(b->lam.reserve(n1 + 16));
    RTD_TRY(b->leaf_of.reserve(n1 + 16));   // node levels (u8)
    RTD_TRY(b->fbody.reserve(n1 * sizeof(float4)));
    RTD_TRY(b->node_a.reserve(n1 * sizeof(float4) + 64));
    RTD_TRY(b->node_b.reserve(n1 * sizeof(uint4) + 64));
    RTD_TRY(b->node_q.reserve(quad ? n1 * 2 * sizeof(float4) + 64 : 64));
    RTD_TRY(b->cell_grad.reserve(64 * sizeof(uint32_t)));   // per-level fill counters (reused)

    const int g = grid_for(n, BLOCK, 148 * 8);
    bh_bbox_kernel<<<grid_for(n, BLOCK, 148 * 4), BLOCK, 0, st>>>(d_pos, n, h);
    RTD_LAUNCH_CHECK();
    bh_root_kernel<<<1, 1, 0, st>>>(h, p->min_width);
    RTD_LAUNCH_CHECK();
    bh_morton_kernel<<<g, BLOCK, 0, st>>>(d_pos, n, h, b->mkeys.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    bool alt = false;
    RTD_TRY(radix_sort_pairs<uint32_t>(b->mkeys.as<uint32_t>(), b->mkeys_alt.as<uint32_t>(),
                                       b->mvals.as<uint32_t>(), b->mvals_alt.as<uint32_t>(), true, n,
                                       0, 30, b->sort, &h->err, st, &alt));
    const uint32_t *morder = alt ? b->mvals_alt.as<uint32_t>() : b->mvals.as<uint32_t>();
    bh_path_kernel<<<g, BLOCK, 0, st>>>(d_pos, n, morder, h, b->pkeys.as<uint64_t>());
    RTD_LAUNCH_CHECK();
    RTD_TRY(radix_sort_pairs<uint64_t>(b->pkeys.as<uint64_t>(), b->pkeys_alt.as<uint64_t>(),
                                       b->pvals.as<uint32_t>(), b->pvals_alt.as<uint32_t>(), true, n,
                                       0, 3 * BH_MAX_LEVEL, b->sort, &h->err, st, &alt));
    const uint64_t *pk = alt ? b->pkeys_alt.as<uint64_t>() : b->pkeys.as<uint64_t>();
    const uint32_t *pvals = alt ? b->pvals_alt.as<uint32_t>() : b->pvals.as<uint32_t>();
    uint8_t *lcp = b->lcp.as<uint8_t>();
    bh_lcp_kernel<<<g, BLOCK, 0, st>>>(pk, n, lcp);
    RTD_LAUNCH_CHECK();
    const uint32_t B = p->bucket;
    const uint64_t nwin = n > B ? n - B : 0;
    if (nwin) {
        bh_window_min_kernel<<<grid_for(nwin, BLOCK, 148 * 8), BLOCK, 0, st>>>(lcp, nwin, B,
                                                                               b->wmin.as<uint8_t>());
        RTD_LAUNCH_CHECK();
    }
    bh_lambda_kernel<<<g, BLOCK, 0, st>>>(b->wmin.as<uint8_t>(), n, nwin, B, h, b->lam.as<uint8_t>());
    RTD_LAUNCH_CHECK();
    bh_count_kernel<<<g, BLOCK, 0, st>>>(lcp, b->lam.as<uint8_t>(), n, b->nn.as<uint32_t>(),
                                         b->heads.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    uint32_t *totals = b->cell_grad.as<uint32_t>();   // [0] nodes, [1] leaves, [2..] level fill
    RTD_TRY(exclusive_scan_u32_32(b->nn.as<uint32_t>(), b->base.as<uint32_t>(), n, totals,
                                  b->scan, &h->err, st));
    // leaf index of each head (exclusive count of heads); the fvals buffer is free until later
    uint32_t *leafidx = b->fkeys_alt.as<uint32_t>();
    RTD_TRY(exclusive_scan_u32_32(b->heads.as<uint32_t>(), leafidx, n, totals + 1, b->scan,
                                  &h->err, st));
    bh_totals_kernel<<<1, 1, 0, st>>>(h, totals, totals + 1);
    RTD_LAUNCH_CHECK();
    uint8_t *node_level = b->leaf_of.as<uint8_t>();
    bh_nodes_kernel<<<g, BLOCK, 0, st>>>(lcp, b->lam.as<uint8_t>(), b->nn.as<uint32_t>(),
                                         b->base.as<uint32_t>(), leafidx, n,
                                         b->node_start.as<uint32_t>(), node_level,
                                         b->leaf_head.as<uint32_t>(), b->leaf_node.as<uint32_t>(), h);
    RTD_LAUNCH_CHECK();
    bh_level_offsets_kernel<<<1, 1, 0, st>>>(h);
    RTD_LAUNCH_CHECK();
    RTD_CUDA(cudaMemsetAsync(totals + 2, 0, (BH_MAX_LEVEL + 2) * sizeof(uint32_t), st));
    bh_records_kernel<<<grid_for(n * 32, BLOCK, 148 * 16), BLOCK, 0, st>>>(
        d_pos, morder, pvals, lcp, b->base.as<uint32_t>(), leafidx, b->leaf_head.as<uint32_t>(),
        b->node_start.as<uint32_t>(), node_level, n, h, b->node_b.as<uint4>(),
        b->level_nodes.as<uint32_t>(), totals + 2);
    RTD_LAUNCH_CHECK();
    // final body order: Morton order stably regrouped by leaf
    bh_leafof_kernel<<<g, BLOCK, 0, st>>>(leafidx, b->heads.as<uint32_t>(), pvals, morder, n,
                                          b->fkeys.as<uint32_t>(), b->fvals.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    int lbits = 1;
    while (lbits < 32 && (1ull << lbits) < n) ++lbits;
    RTD_TRY(radix_sort_pairs<uint32_t>(b->fkeys.as<uint32_t>(), b->mkeys_alt.as<uint32_t>(),
                                       b->fvals.as<uint32_t>(), b->fvals_alt.as<uint32_t>(), false,
                                       n, 0, lbits, b->sort, &h->err, st, &alt));
    const uint32_t *F = alt ? b->fvals_alt.as<uint32_t>() : b->fvals.as<uint32_t>();
    bh_flat_kernel<<<g, BLOCK, 0, st>>>(d_pos, d_mass, F, n, b->order.as<uint32_t>(),
                                        b->fbody.as<float4>());
    RTD_LAUNCH_CHECK();
    bh_leaf_com_kernel<<<g, BLOCK, 0, st>>>(h, b->node_b.as<uint4>(), b->fbody.as<float4>(),
                                            b->node_a.as<float4>(), b->node_q.as<float4>(), quad);
    RTD_LAUNCH_CHECK();
    bh_internal_com_kernel<<<1, 1024, 0, st>>>(h, b->node_b.as<uint4>(),
                                               b->level_nodes.as<uint32_t>(),
                                               b->node_a.as<float4>(), b->node_q.as<float4>(), quad);
    RTD_LAUNCH_CHECK();
    if (p->law == RTD_BH_LAW_PLUMMER) {
        // child table and warp groups for the tiled walks (scratch reuse:
        // mkeys = gsize, mkeys_alt = gcnt, nn = group offsets)
        RTD_TRY(b->child8.reserve(n1 * 2 * sizeof(uint4) + 64));
        RTD_TRY(b->groups.reserve(n1 * sizeof(uint2) + 64));
        bh_child_kernel<<<g, BLOCK, 0, st>>>(h, b->node_b.as<uint4>(), b->child8.as<uint4>());
        RTD_LAUNCH_CHECK();
        uint32_t *gsize = b->mkeys.as<uint32_t>(), *gcnt = b->mkeys_alt.as<uint32_t>();
        RTD_CUDA(cudaMemsetAsync(gcnt, 0, n1 * 4, st));
        bh_group_plan_kernel<<<g, BLOCK, 0, st>>>(h, b->leaf_node.as<uint32_t>(), node_level,
                                                  b->node_b.as<uint4>(), gcnt, gsize);
        RTD_LAUNCH_CHECK();
        // scan over all n slots (leaves beyond n_leaves hold 0)
        RTD_TRY(exclusive_scan_u32_32(gcnt, b->nn.as<uint32_t>(), n, totals + 1, b->scan, &h->err,
                                      st));
        bh_group_write_kernel<<<g, BLOCK, 0, st>>>(h, b->leaf_node.as<uint32_t>(),
                                                   b->node_b.as<uint4>(), gcnt, gsize,
                                                   b->nn.as<uint32_t>(), totals + 1,
                                                   b->groups.as<uint2>());
        RTD_LAUNCH_CHECK();
        b->plummer_ready = true;
        b->has_quad = quad != 0;
    }
    b->built = true;
    b->ilog_valid = false;   // a new tree: the last forward's log no longer applies
    return RTD_OK;
}

}  // namespace rtd
