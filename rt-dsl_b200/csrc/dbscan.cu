// dbscan.cu -- DBSCAN on top of the range count and fill passes.
//
// The reference advertises DBSCAN over its push-to-buffer range search
// (README.md:13) without shipping one.  Here:
//   1. count pass over the indexed points themselves (radius eps, the point
//      itself included): core = count >= min_pts;
//   2. fill pass: every (point, neighbour) pair;
//   3. lock-free union-find over core-core pairs, always linking the larger
//      root under the smaller, so each component's root is its smallest
//      core point;
//   4. clusters numbered by a scan over roots in point order (the order of
//      their smallest core point), core points take their root's number;
//   5. a non-core point takes the smallest number among its core neighbours
//      (the first cluster a sequential expansion in point order would reach
//      it with), else noise (-1).
// Labels equal those of the sequential algorithm that expands clusters one
// at a time from core points in index order.
#include <climits>

#include "index.cuh"

namespace rtd {

rtd_status range_count(rtd_index *idx, const float *d_q, uint64_t nq, float r,
                       const rtd_schedule *s, uint32_t *d_counts, uint64_t *h_total,
                       cudaStream_t st);
rtd_status range_fill(rtd_index *idx, const float *d_q, uint64_t nq, float r,
                      const rtd_schedule *s, uint32_t *d_pairs, uint64_t capacity, int sort_pairs,
                      uint64_t *h_written, cudaStream_t st);
rtd_status check_index_errors(rtd_index *idx, cudaStream_t st);

namespace {

constexpr int BLOCK = 256;
constexpr uint32_t UF_LIMIT = 1u << 26;   // steps of one find or one union

__device__ __forceinline__ uint32_t uf_find(uint32_t *parent, uint32_t x, uint32_t *err) {
    // path halving: parents only ever point to smaller indices, so every
    // write moves a pointer to an ancestor and the walk ends at the root
    for (uint32_t it = 0; it < UF_LIMIT; ++it) {
        const uint32_t p = *(volatile uint32_t *)&parent[x];
        if (p == x) return x;
        const uint32_t g = *(volatile uint32_t *)&parent[p];
        if (g != p) atomicMin(&parent[x], g);
        x = g;
    }
    atomicOr(err, DEVERR_TIMEOUT);
    return x;
}

__global__ void dbscan_init_kernel(const uint32_t *__restrict__ counts, uint64_t n,
                                   uint32_t min_pts, uint8_t *__restrict__ core,
                                   uint32_t *__restrict__ parent) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK) {
        core[i] = counts[i] >= min_pts;
        parent[i] = (uint32_t)i;
    }
}

__global__ void dbscan_union_kernel(const uint2 *__restrict__ pairs, uint64_t n_pairs,
                                    const uint8_t *__restrict__ core, uint32_t *parent,
                                    uint32_t *err) {
    for (uint64_t t = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; t < n_pairs;
         t += (uint64_t)gridDim.x * BLOCK) {
        const uint2 pr = pairs[t];
        uint32_t a = pr.x, b = pr.y;
        if (a >= b || !core[a] || !core[b]) continue;   // each core-core edge once
        for (uint32_t it = 0;; ++it) {
            if (it >= UF_LIMIT) {
                atomicOr(err, DEVERR_TIMEOUT);
                break;
            }
            a = uf_find(parent, a, err);
            b = uf_find(parent, b, err);
            if (a == b) break;
            const uint32_t hi = a > b ? a : b, lo = a > b ? b : a;
            if (atomicCAS(&parent[hi], hi, lo) == hi) break;   // linked hi under lo
            a = hi;   // hi gained a parent meanwhile: retry from its new root
            b = lo;
        }
    }
}

// Root flags (core points that are their component's smallest core point).
__global__ void dbscan_roots_kernel(uint64_t n, const uint8_t *__restrict__ core, uint32_t *parent,
                                    uint32_t *__restrict__ flag, uint32_t *err) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK) {
        uint32_t r = 0;
        if (core[i]) {
            const uint32_t root = uf_find(parent, (uint32_t)i, err);
            parent[i] = root;
            r = root == (uint32_t)i;
        }
        flag[i] = r;
    }
}

__global__ void dbscan_core_labels_kernel(uint64_t n, const uint8_t *__restrict__ core,
                                          const uint32_t *__restrict__ parent,
                                          const uint32_t *__restrict__ rank,
                                          int32_t *__restrict__ labels) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK)
        labels[i] = core[i] ? (int32_t)rank[parent[i]] : INT_MAX;
}

__global__ void dbscan_border_kernel(const uint2 *__restrict__ pairs, uint64_t n_pairs,
                                     const uint8_t *__restrict__ core, int32_t *labels) {
    for (uint64_t t = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; t < n_pairs;
         t += (uint64_t)gridDim.x * BLOCK) {
        const uint2 pr = pairs[t];
        if (!core[pr.x] && core[pr.y]) atomicMin(&labels[pr.x], labels[pr.y]);
    }
}

__global__ void dbscan_noise_kernel(uint64_t n, int32_t *labels) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK)
        if (labels[i] == INT_MAX) labels[i] = -1;
}

}  // namespace
}  // namespace rtd

using namespace rtd;

extern "C" rtd_status rtd_dbscan(rtd_index *idx, const float *d_points, uint64_t n, float eps,
                                 uint32_t min_pts, int32_t *d_labels, uint64_t *h_n_clusters,
                                 rtd_stream stream) {
    if (!idx || !idx->hdr.ptr) return fail(RTD_ERR_INVALID_ARGUMENT, "index not built");
    if (idx->n != n) return fail(RTD_ERR_INVALID_ARGUMENT, "the index must be built over these points");
    if (!(eps >= 0.0f)) return fail(RTD_ERR_INVALID_ARGUMENT, "eps must be >= 0");
    if (min_pts < 1) return fail(RTD_ERR_INVALID_ARGUMENT, "min_pts must be >= 1");
    if (h_n_clusters) *h_n_clusters = 0;
    if (n == 0) return RTD_OK;
    if (!d_points || !d_labels) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL device buffer");
    cudaStream_t st = (cudaStream_t)stream;
    // scratch kept on the index and grown only, so repeated calls allocate nothing
    DevBuf &counts = idx->db_counts, &pairs = idx->db_pairs, &core = idx->db_core,
           &parent = idx->db_parent, &flag = idx->db_flag, &rank = idx->db_rank,
           &ncbuf = idx->db_nc;
    RTD_TRY(counts.reserve(n * 4));
    uint64_t total = 0;
    RTD_TRY(range_count(idx, d_points, n, eps, nullptr, counts.as<uint32_t>(), &total, st));
    if (total >= (1ull << 32)) return fail(RTD_ERR_UNSUPPORTED, "more than 2^32 neighbour pairs");
    RTD_TRY(pairs.reserve(total * 8 + 8));
    uint64_t written = 0;
    RTD_TRY(range_fill(idx, d_points, n, eps, nullptr, pairs.as<uint32_t>(), total, 0, &written, st));
    RTD_TRY(core.reserve(n));
    RTD_TRY(parent.reserve(n * 4));
    RTD_TRY(flag.reserve(n * 4));
    RTD_TRY(rank.reserve(n * 4));
    uint32_t *err = &idx->hdr.as<IndexHeader>()->err;
    const int g = grid_for(n, BLOCK, 148 * 8), gp = grid_for(total, BLOCK, 148 * 16);
    dbscan_init_kernel<<<g, BLOCK, 0, st>>>(counts.as<uint32_t>(), n, min_pts, core.as<uint8_t>(),
                                            parent.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    if (total) {
        dbscan_union_kernel<<<gp, BLOCK, 0, st>>>(pairs.as<uint2>(), total, core.as<uint8_t>(),
                                                  parent.as<uint32_t>(), err);
        RTD_LAUNCH_CHECK();
    }
    dbscan_roots_kernel<<<g, BLOCK, 0, st>>>(n, core.as<uint8_t>(), parent.as<uint32_t>(),
                                             flag.as<uint32_t>(), err);
    RTD_LAUNCH_CHECK();
    ScanScratch &scan = idx->db_scan;
    RTD_TRY(ncbuf.reserve(sizeof(uint32_t)));
    uint32_t *d_nc = ncbuf.as<uint32_t>();
    RTD_TRY(exclusive_scan_u32_32(flag.as<uint32_t>(), rank.as<uint32_t>(), n, d_nc, scan, err, st));
    dbscan_core_labels_kernel<<<g, BLOCK, 0, st>>>(n, core.as<uint8_t>(), parent.as<uint32_t>(),
                                                   rank.as<uint32_t>(), d_labels);
    RTD_LAUNCH_CHECK();
    if (total) {
        dbscan_border_kernel<<<gp, BLOCK, 0, st>>>(pairs.as<uint2>(), total, core.as<uint8_t>(),
                                                   d_labels);
        RTD_LAUNCH_CHECK();
    }
    dbscan_noise_kernel<<<g, BLOCK, 0, st>>>(n, d_labels);
    RTD_LAUNCH_CHECK();
    uint32_t nc = 0;
    RTD_CUDA(cudaMemcpyAsync(&nc, d_nc, sizeof(nc), cudaMemcpyDeviceToHost, st));
    RTD_TRY(check_index_errors(idx, st));   // synchronises
    if (h_n_clusters) *h_n_clusters = nc;
    return RTD_OK;
}
