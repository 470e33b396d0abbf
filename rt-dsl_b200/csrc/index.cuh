// index.cuh -- LBVH index layout shared by the builder and the search kernels.
//
// Points are stored Morton-sorted as float4 (x, y, z, bits of the original
// id): one 128-bit load per candidate.  Internal nodes hold the boxes of
// their two children (64 B, four 128-bit loads).  A child word is either an
// internal-node index or a leaf (first sorted point); the number of points
// below each child is stored beside the words, so a traversal that carries
// a node's first point knows every subtree's contiguous point range.
// The top levels of the tree are copied into a small array that search
// kernels stage in shared memory; child words that point into it carry
// CHILD_TOP.
#pragma once

#include "common.cuh"
#include "sort.cuh"

namespace rtd {

constexpr uint32_t CHILD_LEAF = 0x80000000u;
constexpr uint32_t CHILD_TOP = 0x40000000u;
constexpr uint32_t CHILD_INDEX = 0x3FFFFFFFu;
constexpr uint32_t CHILD_NONE = 0xFFFFFFFFu;
constexpr uint32_t EMPTY_ID = 0xFFFFFFFFu;
constexpr int TOP_LEVELS = 6;
constexpr int TOP_MAX = (1 << TOP_LEVELS) - 1;   // 63 nodes, 4 KB of shared memory

struct __align__(16) BvhNode {
    float4 a;  // lo.x[0] lo.y[0] lo.z[0] hi.x[0]
    float4 b;  // hi.y[0] hi.z[0] lo.x[1] lo.y[1]
    float4 c;  // lo.z[1] hi.x[1] hi.y[1] hi.z[1]
    uint4 d;   // child[0] child[1] count[0] count[1] (points below each child)
};
static_assert(sizeof(BvhNode) == 64, "node is one half cache line");

// Device-resident header of an index (all fields written on the device).
struct IndexHeader {
    uint32_t root;        // child word of the root for search kernels (CHILD_TOP|0 or a leaf)
    uint32_t root_count;  // point count when the root is a leaf
    uint32_t n_internal;  // compact internal nodes
    uint32_t n_top;       // staged top nodes
    uint32_t box[6];      // scene box as order-preserving u32: lo xyz, hi xyz
    uint32_t err;         // DEVERR_* flags
    float r0sq;           // squared initial radius of the last search
    uint64_t total;       // last range-count total
    float nn95_key;       // p95 of the squared 1-NN distance within a 4096-point sample
    uint32_t n_sample;    // points in the radius-seed sample (<= 1000)
    unsigned long long qfp[2];   // query fingerprints of the last range count / fill
};

constexpr int SEED_NN_SAMPLE = 4096;
constexpr int SEED_PCT_POINTS = 1000;
constexpr int SEED_PCT_QUERIES = 100;

}  // namespace rtd

namespace rtd {
// The same order computed against the queries' own box with scratch of its
// own, so that it can run on another stream while an index is being built.
// Device errors land in the scratch header's err word.
struct QueryOrderScratch {
    DevBuf hdr;   // IndexHeader: the query box and err
    DevBuf keys, keys_alt, perm, perm_alt;
    SortScratch sort;
};
}  // namespace rtd

struct rtd_index {
    uint64_t n = 0;
    uint32_t leaf_size = 4;
    int morton_bits = 30;
    int device = 0;
    rtd::DevBuf hdr;        // IndexHeader
    rtd::DevBuf pts;        // float4 * n, Morton order
    rtd::DevBuf nodes;      // BvhNode * (n - 1)
    rtd::DevBuf top;        // BvhNode * TOP_MAX
    // build scratch
    rtd::DevBuf keys, keys_alt, vals, vals_alt;
    rtd::DevBuf k32a, k32b;   // 32-bit top keys of the split sort
    // Karras node flags (1: the node keeps more than leaf_size points),
    // compact indices, the list of kept nodes, and (forest builds) the kept
    // nodes' first and last points by Karras index
    rtd::DevBuf flags, cidx, csel, kfirst, klast;
    rtd::DevBuf pyramid;    // run boxes over the sorted points (2 float4 per run)
    rtd::SortScratch sort;
    rtd::ScanScratch scan;
    // radius-seed data kept from the build: stride samples of the points in
    // input order (<= 1000 + 4096 float4) and the 1-NN scratch; nn_seeded:
    // the sampled 1-NN seed (IndexHeader::nn95_key) has been computed for
    // this build
    rtd::DevBuf sample, seed;
    bool nn_seeded = false;
    // search scratch
    rtd::DevBuf qkeys, qkeys_alt, qperm, qperm_alt;
    const void *skeys = nullptr;   // the points' sorted Morton keys (in keys or keys_alt)
    rtd::DevBuf rcounts, roffsets, rcursor, rpairs_alt, rkeys, rkeys_alt;
    // the count pass's own (query, id) pairs, kept when a buffer from an
    // earlier count is large enough (rspec_cap pairs), and the fill's
    // per-query cursors
    rtd::DevBuf rspec, rqcur, rrec;
    uint64_t rspec_cap = 0, rrec_cap = 0;
    // DBSCAN scratch (rtd_dbscan): counts, pairs, core flags, union-find
    rtd::DevBuf db_counts, db_pairs, db_core, db_parent, db_flag, db_rank, db_nc;
    rtd::ScanScratch db_scan;
    // What the last range count left behind for a fill of the same queries:
    // per-query exclusive offsets (roffsets), the total, and the query order.
    // Cleared by a build and by any other query ordering on this index.
    struct RangeToken {
        bool valid = false;
        const float *q = nullptr;
        uint64_t nq = 0;
        float radius = 0.f;
        uint64_t total = 0;
        const uint32_t *perm = nullptr;
        bool spec = false;   // rspec / rrec hold every pair of that count
        uint64_t spec_pairs = 0, spec_recs = 0;
    } rtoken;
    // Side stream for work that overlaps the build: the radius-seed sample
    // (every build) and rtd_k_nn's query ordering; tree stream: the box
    // pyramid, beside the Karras flags and their scan
    cudaStream_t side_stream = nullptr, tree_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_seed_fork = nullptr,
                ev_seed_join = nullptr, ev_sorted = nullptr, ev_tree_fork = nullptr,
                ev_tree_join = nullptr;
    rtd::DevBuf wpos;       // queries' Morton positions for the window seed
    rtd::DevBuf wide;       // per-warp list slabs of the k > 2048 search
    rtd::QueryOrderScratch qorder;
    // phase timers (rtd_index_profile_*)
    bool prof = false;
    cudaEvent_t ev[8] = {};
    bool ev_set[8] = {};
    void mark(int i, cudaStream_t st) {
        if (!prof) return;
        if (!ev[i] && cudaEventCreate(&ev[i]) != cudaSuccess) { ev[i] = nullptr; return; }
        if (cudaEventRecord(ev[i], st) == cudaSuccess) ev_set[i] = true;
    }
    ~rtd_index() {
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : {ev_fork, ev_join, ev_seed_fork, ev_seed_join, ev_sorted,
                              ev_tree_fork, ev_tree_join})
            if (e) cudaEventDestroy(e);
        if (side_stream) cudaStreamDestroy(side_stream);
        if (tree_stream) cudaStreamDestroy(tree_stream);
    }
};

namespace rtd {
// Event slots of rtd_index::mark.
enum : int { EV_BUILD0 = 0, EV_BUILD_SORTED, EV_BUILD1, EV_SEARCH0, EV_SEEDED, EV_ORDERED,
             EV_SEARCH1 };
}  // namespace rtd

namespace rtd {

// Normalisation of the Morton quantisation: the scene box (per axis) or its
// cube (one extent, the largest).
struct SceneNorm {
    float lo[3], ext[3];
};
__device__ __forceinline__ SceneNorm scene_norm(const IndexHeader *h) {
    SceneNorm s;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float lo = float_unflip(h->box[a]), hi = float_unflip(h->box[3 + a]);
        s.lo[a] = lo;
        // morton.rs:37-39: extent clamped to >= 1e-6
        s.ext[a] = fmaxf(__fsub_rn(hi, lo), 1e-6f);
    }
    return s;
}

// One extent for all three axes (the largest): every Morton bit level then
// halves the same length on each axis, so a flat or elongated cloud is split
// along its long axes first.  With an extent per axis, the top levels of a
// thin sheet's tree would split its thickness and give every node a box
// spanning the whole sheet.
__device__ __forceinline__ SceneNorm scene_norm_cubic(const IndexHeader *h) {
    SceneNorm s = scene_norm(h);
    const float e = fmaxf(s.ext[0], fmaxf(s.ext[1], s.ext[2]));
    s.ext[0] = s.ext[1] = s.ext[2] = e;
    return s;
}

// Arguments the search kernels need from an index.
struct IndexView {
    const float4 *pts;
    const BvhNode *nodes;
    const BvhNode *top;
    const IndexHeader *hdr;
    uint64_t n;
};
inline IndexView view_of(const rtd_index *idx) {
    return IndexView{idx->pts.as<float4>(), idx->nodes.as<BvhNode>(), idx->top.as<BvhNode>(),
                     idx->hdr.as<IndexHeader>(), idx->n};
}

// Karras tree, leaf collapse and child boxes over n keys already sorted
// (idx->pts holds the points in key order; idx->leaf_size set).  With
// ranges, every kept Karras node i also leaves its point range in
// kfirst[i], klast[i] (flags[i] says which nodes are kept).
template <typename K>
rtd_status build_tree_sorted(rtd_index *idx, const K *skeys, uint64_t n, cudaStream_t st,
                             bool ranges = false);

// Query ordering: Morton codes of the queries against the scene box, sorted;
// perm[i] is the i-th query to process.  Returns perm (device) or nullptr
// when ordering is off.
rtd_status order_queries(rtd_index *idx, const float *d_q, uint64_t nq, bool morton,
                         const uint32_t **perm, cudaStream_t stream);

// With chunks > 1 the order is by (chunk, Morton code), chunk c holding the
// queries [ceil(c nq / chunks), ceil((c + 1) nq / chunks)) in caller order,
// so each chunk's processing positions are the same range.
rtd_status order_queries_own(QueryOrderScratch &qs, const float *d_q, uint64_t nq,
                             const uint32_t **perm, cudaStream_t stream, uint32_t chunks = 1);

// A search whose results go to host memory in chunks of the caller's query
// order: chunk c searches on streams[c] (after `fork` on the caller's
// stream) and copies its rows out as soon as it ends, while later chunks
// search; the caller's stream then waits for every chunk (`done`).
constexpr int MAX_CHUNKS = 8;
struct HostChunks {
    uint32_t chunks = 1;
    cudaStream_t streams[MAX_CHUNKS] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t done[MAX_CHUNKS] = {};
    uint32_t *h_ids = nullptr;
    float *h_d2 = nullptr;
};
inline uint64_t chunk_begin(uint64_t nq, uint32_t chunks, uint32_t c) {
    return (c * nq + chunks - 1) / chunks;
}

// Creates the index's side and tree streams and their events on first use.
rtd_status ensure_side_stream(rtd_index *idx);

// The sampled 1-NN seed of the last build (IndexHeader::nn95_key), computed
// on stream st unless it already has been (lbvh.cu).
rtd_status ensure_nn_seed(rtd_index *idx, cudaStream_t st);

// LBVH build over n device points (lbvh.cu).
rtd_status index_build(rtd_index *idx, const float *d_xyz, uint64_t n, const rtd_schedule *s,
                       cudaStream_t st);

// k-NN search (knn.cu); with have_perm the query order is given (perm, or
// nullptr for caller order) instead of computed on the index; wpos, when
// not nullptr, holds the Morton-window positions of the queries in that
// order.
rtd_status knn_search_ex(rtd_index *idx, const float *d_q, uint64_t nq, uint32_t k,
                         const rtd_schedule *sched, uint32_t *d_ids, float *d_d2,
                         cudaStream_t st, bool have_perm, const uint32_t *perm,
                         const uint32_t *wpos, const HostChunks *hc = nullptr);

}  // namespace rtd
