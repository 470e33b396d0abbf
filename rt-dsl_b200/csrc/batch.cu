// batch.cu -- batched exact k-NN over many independent point clouds.
//
// Build: every point gets the key (cloud id << 3B) | Morton_B(point in its
// cloud's box), B bits per axis; one radix sort of all keys puts each
// cloud's points together in Morton order, and one Karras tree over the
// whole key array is a forest whose node covering a cloud's key range is
// that cloud's LBVH (keys sharing the cloud prefix form a subtree of a
// binary radix tree).  Search: one persistent launch.  Work items of <= 32
// Morton-ordered queries of one cloud, each carrying its k class, are taken
// from one device counter by every warp of the grid; an item runs the
// thread-per-query register list (k <= 16), the warp-per-query striped
// register list (k <= 256) or the warp-per-query memory list (any larger k)
// of knn_traverse.cuh against its cloud's root.  Items are queued heaviest
// class first, so the long warp-per-query items start early and the short
// ones fill the tail.  The whole pass is launch-only (no host
// synchronisation), so it can be captured as one CUDA graph and replayed.
#include <new>
#include <vector>

#include "knn_traverse.cuh"

struct rtd_batch;

namespace rtd {
namespace {

constexpr int BLOCK = 256;
constexpr int SWARPS = 4;   // warps per block of the search kernel

struct CloudDesc {
    uint32_t pt_begin, n_pts, q_begin, n_q;
    uint32_t k, root, root_count, box[6];
    float r0sq;
    uint64_t out_off;
};

struct WorkItem {
    uint32_t cloud, start, count, cls;   // cls: k class (k_class), the search it runs
};

__global__ void batch_reset_kernel(CloudDesc *cd, uint32_t n_clouds) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_clouds; c += gridDim.x * blockDim.x) {
        for (int a = 0; a < 3; ++a) {
            cd[c].box[a] = 0xFFFFFFFFu;
            cd[c].box[3 + a] = 0u;
        }
        cd[c].root = cd[c].n_pts == 0 ? CHILD_NONE : (CHILD_LEAF | cd[c].pt_begin);
        cd[c].root_count = cd[c].n_pts;
    }
}

// Cloud id of every point and every query (one block per cloud).
__global__ void batch_cloud_of_kernel(const CloudDesc *__restrict__ cd, uint32_t *__restrict__ pcloud,
                                      uint32_t *__restrict__ qcloud) {
    const uint32_t c = blockIdx.x;
    const CloudDesc d = cd[c];
    for (uint32_t i = threadIdx.x; i < d.n_pts; i += blockDim.x) pcloud[d.pt_begin + i] = c;
    for (uint32_t i = threadIdx.x; i < d.n_q; i += blockDim.x) qcloud[d.q_begin + i] = c;
}

// Per-cloud bounding boxes (NaN-ignoring); a warp whose points share one
// cloud reduces first and issues one atomic per bound.
__global__ void __launch_bounds__(BLOCK) batch_bbox_kernel(const float *__restrict__ xyz, uint64_t n,
                                                           const uint32_t *__restrict__ pcloud,
                                                           CloudDesc *cd) {
    const int lane = threadIdx.x & 31;
    for (uint64_t base = ((uint64_t)blockIdx.x * BLOCK + threadIdx.x) & ~31ull; base < n;
         base += (uint64_t)gridDim.x * BLOCK) {
        const uint64_t i = base + lane;
        const bool ok = i < n;
        const uint32_t c = ok ? pcloud[i] : 0xFFFFFFFFu;
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            float v = ok ? xyz[3 * i + a] : NAN;
            lo[a] = v;
            hi[a] = v;
        }
        const uint32_t c0 = __shfl_sync(0xffffffffu, c, 0);
        if (__all_sync(0xffffffffu, c == c0 || !ok)) {
            for (int a = 0; a < 3; ++a)
                for (int o = 16; o > 0; o >>= 1) {
                    lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
                    hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
                }
            if (lane == 0 && c0 != 0xFFFFFFFFu)
                for (int a = 0; a < 3; ++a) {
                    if (!isnan(lo[a])) atomicMin(&cd[c0].box[a], float_flip(lo[a]));
                    if (!isnan(hi[a])) atomicMax(&cd[c0].box[3 + a], float_flip(hi[a]));
                }
        } else if (ok) {
            for (int a = 0; a < 3; ++a)
                if (!isnan(lo[a])) {
                    atomicMin(&cd[c].box[a], float_flip(lo[a]));
                    atomicMax(&cd[c].box[3 + a], float_flip(hi[a]));
                }
        }
    }
}

// Initial radius of a cloud: `fixed` when > 0, else `mult` x the radius of
// a ball expected to hold k points at the cloud's mean density,
// (3 k V / 4 pi n)^(1/3).  Box extents are clamped to >= max extent /
// sqrt(n), which makes the estimate the mean spacing of a flat (2-D) cloud;
// an estimate that is too large only costs pruning, one that is too small
// costs extra rounds.
__global__ void batch_seed_kernel(CloudDesc *cd, uint32_t n_clouds, float fixed, float mult) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_clouds; c += gridDim.x * blockDim.x) {
        float r = fixed;
        if (!(r > 0.0f)) {
            const float n = (float)(cd[c].n_pts > 0 ? cd[c].n_pts : 1);
            float e[3], emax = 0.0f;
            for (int a = 0; a < 3; ++a) {
                const float lo = float_unflip(cd[c].box[a]), hi = float_unflip(cd[c].box[3 + a]);
                e[a] = hi - lo;
                if (!isfinite(e[a]) || !(e[a] > 0.0f)) e[a] = 0.0f;
                emax = fmaxf(emax, e[a]);
            }
            const float emin = fmaxf(emax / sqrtf(n), 1e-20f);
            const float v = fmaxf(e[0], emin) * fmaxf(e[1], emin) * fmaxf(e[2], emin);
            r = mult * cbrtf(3.0f * (float)cd[c].k * v / (4.0f * 3.14159265f * n));
        }
        if (!(r > 0.0f) || !(r < INFINITY)) r = 1.0f;
        cd[c].r0sq = r * r;
    }
}

__global__ void __launch_bounds__(BLOCK) batch_keys_kernel(const float *__restrict__ xyz, uint64_t n,
                                                           const uint32_t *__restrict__ cloud_of,
                                                           const CloudDesc *__restrict__ cd,
                                                           int bpa, uint64_t *__restrict__ keys) {
    const float scale = (float)((1u << bpa) - 1u);
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK) {
        const uint32_t c = cloud_of[i];
        // one cubic extent per cloud (the largest axis), as for single indexes
        float lo[3], ext = 1e-6f;
        for (int a = 0; a < 3; ++a) {
            const float hi = float_unflip(cd[c].box[3 + a]);
            lo[a] = float_unflip(cd[c].box[a]);
            ext = fmaxf(ext, __fsub_rn(hi, lo[a]));
        }
        uint32_t u[3];
        for (int a = 0; a < 3; ++a) u[a] = quantize(xyz[3 * i + a], lo[a], ext, scale);
        keys[i] = ((uint64_t)c << (3 * bpa)) | morton63(u[0], u[1], u[2]);
    }
}

__global__ void __launch_bounds__(BLOCK) batch_gather_kernel(const float *__restrict__ xyz,
                                                             const uint32_t *__restrict__ perm,
                                                             const uint32_t *__restrict__ pcloud,
                                                             const CloudDesc *__restrict__ cd,
                                                             uint64_t n, float4 *__restrict__ pts) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * BLOCK) {
        const uint32_t o = perm[i];
        const uint32_t local = o - cd[pcloud[o]].pt_begin;
        pts[i] = make_float4(xyz[3 * (uint64_t)o], xyz[3 * (uint64_t)o + 1],
                             xyz[3 * (uint64_t)o + 2], __uint_as_float(local));
    }
}

// The kept forest node whose range is exactly a cloud's points is that
// cloud's root.
__global__ void __launch_bounds__(BLOCK) batch_roots_kernel(
    const uint64_t *__restrict__ skeys, uint64_t n, int shift, const uint32_t *__restrict__ kfirst,
    const uint32_t *__restrict__ klast, const uint32_t *__restrict__ flags,
    const uint32_t *__restrict__ cidx, CloudDesc *cd) {
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i + 1 < n;
         i += (uint64_t)gridDim.x * BLOCK) {
        // only kept nodes carry their range; a cloud of <= leaf_size points
        // keeps the leaf root batch_reset_kernel gave it
        if (!flags[i]) continue;
        const uint32_t f = kfirst[i], l = klast[i];
        const uint32_t c = (uint32_t)(skeys[f] >> shift);
        const CloudDesc d = cd[c];
        if (f == d.pt_begin && l + 1 == d.pt_begin + d.n_pts) {
            cd[c].root = cidx[i];
            cd[c].root_count = d.n_pts;
        }
    }
}

struct BatchArgs {
    const float4 *pts;
    const BvhNode *nodes;
    const IndexHeader *hdr;
    const CloudDesc *cd;
    const WorkItem *items;
    uint32_t n_items;
    uint32_t *counter;
    const uint32_t *qperm;
    const float *q;
    uint32_t *ids;
    float *d2;
    float mult2;
    uint32_t max_rounds;
    uint32_t partial;   // the reference's round cap (rtd_schedule.partial_results)
    uint32_t *err;
    uint2 *wide;        // per-warp list slabs of the k > 256 class
    uint32_t wide_kk;   // entries per slab: the largest min(k, points) of that class
};

template <int KC>
__device__ __forceinline__ void item_thread(const BatchArgs &a, const TreeRef &t,
                                            const RoundSpec &rs, const CloudDesc &c,
                                            const WorkItem &w, uint2 *s_col, uint2 *l_stack) {
    const int lane = threadIdx.x & 31;
    if ((uint32_t)lane >= w.count) return;
    const uint32_t qi = a.qperm[w.start + lane];
    const float qx = a.q[3 * (uint64_t)qi], qy = a.q[3 * (uint64_t)qi + 1], qz = a.q[3 * (uint64_t)qi + 2];
    const int kk = (int)c.k;
    float bk[KC];
    uint32_t bi[KC];
    knn_query_thread<KC>(t, rs, qx, qy, qz, kk, s_col, 32, l_stack, a.err, bk, bi);
    const uint64_t ob = c.out_off + (uint64_t)(qi - c.q_begin) * kk;
#pragma unroll
    for (int j = 0; j < KC; ++j)
        if (j >= KC - kk) {
            a.ids[ob + j - (KC - kk)] = bi[j];
            if (a.d2) a.d2[ob + j - (KC - kk)] = bk[j];
        }
}

template <int S>
__device__ __forceinline__ void item_warp(const BatchArgs &a, const TreeRef &t, const RoundSpec &rs,
                                          const CloudDesc &c, const WorkItem &w, uint2 *stk,
                                          uint2 *ls) {
    const int lane = threadIdx.x & 31;
    for (uint32_t j = 0; j < w.count; ++j) {
        const uint32_t qi = a.qperm[w.start + j];
        const float qx = a.q[3 * (uint64_t)qi], qy = a.q[3 * (uint64_t)qi + 1], qz = a.q[3 * (uint64_t)qi + 2];
        float lk[S];
        uint32_t li[S];
        knn_query_warp<S>(t, rs, qx, qy, qz, c.k, stk, ls, a.err, lk, li);
        const uint64_t ob = c.out_off + (uint64_t)(qi - c.q_begin) * c.k;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const uint32_t slot = (uint32_t)(s * 32 + lane);
            if (slot < c.k) {
                a.ids[ob + slot] = li[s];
                if (a.d2) a.d2[ob + slot] = lk[s];
            }
        }
    }
}

__device__ __forceinline__ void item_wide(const BatchArgs &a, const TreeRef &t, const RoundSpec &rs,
                                          const CloudDesc &c, const WorkItem &w, uint2 *stk,
                                          uint32_t *s_r, uint2 *slab) {
    WideList list;
    list.L = slab;
    list.s_r = s_r;
    list.kk = c.k < c.n_pts ? c.k : (c.n_pts ? c.n_pts : 1u);
    for (uint32_t j = 0; j < w.count; ++j) {
        const uint32_t qi = a.qperm[w.start + j];
        const float qx = a.q[3 * (uint64_t)qi], qy = a.q[3 * (uint64_t)qi + 1], qz = a.q[3 * (uint64_t)qi + 2];
        knn_query_warp_list(t, rs, qx, qy, qz, stk, a.err, list);
        const uint64_t ob = c.out_off + (uint64_t)(qi - c.q_begin) * c.k;
        wide_list_store(list, c.k, a.ids + ob, a.d2 ? a.d2 + ob : nullptr);
        __syncwarp();
    }
}

// k classes of the search: register list of 8 or 16 slots (thread per
// query), warp list of 32, 64 or 256 slots (warp per query), memory list
// (warp per query, k > 256).
constexpr int N_CLASSES = 6;
__host__ __device__ constexpr int k_class(uint32_t k) {
    return k <= 8 ? 0 : k <= 16 ? 1 : k <= 32 ? 2 : k <= 64 ? 3 : k <= 256 ? 4 : 5;
}

// Shared memory of one warp, reused by whichever class its current item
// has: the thread classes' short stacks (SHORT_STACK x 32 entries, one
// column per lane) or the warp classes' stack, list scratch and rank words.
constexpr int WARP_SMEM = SHORT_STACK * 32;   // uint2 entries (3 KB)
static_assert(STACK_MAX + 256 + 16 <= WARP_SMEM, "warp classes fit the thread stacks' space");

__global__ void __launch_bounds__(SWARPS * 32) batch_knn_kernel(const BatchArgs a) {
    __shared__ uint2 s_warp[SWARPS][WARP_SMEM];
    uint2 l_stack[STACK_MAX - SHORT_STACK];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint2 *const sw = s_warp[warp];
    uint2 *const stk = sw;                       // warp classes: STACK_MAX entries
    uint2 *const ls = sw + STACK_MAX;            // list scratch (256 entries)
    uint32_t *const s_r = reinterpret_cast<uint32_t *>(sw + STACK_MAX + 256);   // 32 words
    uint2 *const slab = a.wide ? a.wide + ((size_t)blockIdx.x * SWARPS + warp) * a.wide_kk : nullptr;
    const uint32_t visit_cap = 2u * a.hdr->n_internal + 4u;
    while (true) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(a.counter, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= a.n_items) break;
        const WorkItem w = a.items[it];
        const CloudDesc c = a.cd[w.cloud];
        const TreeRef t{a.pts, a.nodes, nullptr, c.root, c.root_count, visit_cap};
        const RoundSpec rs{c.r0sq, a.mult2, a.max_rounds, a.partial};
        switch (w.cls) {
        case 0: item_thread<8>(a, t, rs, c, w, sw + lane, l_stack); break;
        case 1: item_thread<16>(a, t, rs, c, w, sw + lane, l_stack); break;
        case 2: item_warp<1>(a, t, rs, c, w, stk, ls); break;
        case 3: item_warp<2>(a, t, rs, c, w, stk, ls); break;
        case 4: item_warp<8>(a, t, rs, c, w, stk, ls); break;
        default: item_wide(a, t, rs, c, w, stk, s_r, slab); break;
        }
        __syncwarp();
    }
}

__global__ void batch_backward_kernel(const float *__restrict__ q, uint64_t nq,
                                      const float *__restrict__ pts,
                                      const uint32_t *__restrict__ qcloud,
                                      const CloudDesc *__restrict__ cd,
                                      const uint32_t *__restrict__ ids, const float *__restrict__ g,
                                      float *__restrict__ gq, float *__restrict__ gp) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const CloudDesc c = cd[qcloud[i]];
        const uint64_t ob = c.out_off + (uint64_t)(i - c.q_begin) * c.k;
        const float qx = q[3 * i], qy = q[3 * i + 1], qz = q[3 * i + 2];
        float ax = 0.f, ay = 0.f, az = 0.f;
        for (uint32_t j = 0; j < c.k; ++j) {
            const uint32_t id = ids[ob + j];
            if (id == EMPTY_ID || id >= c.n_pts) continue;
            const uint64_t p = (uint64_t)c.pt_begin + id;
            const float w = 2.0f * g[ob + j];
            const float dx = qx - pts[3 * p], dy = qy - pts[3 * p + 1], dz = qz - pts[3 * p + 2];
            ax += w * dx; ay += w * dy; az += w * dz;
            if (gp) {
                atomicAdd(&gp[3 * p], -w * dx);
                atomicAdd(&gp[3 * p + 1], -w * dy);
                atomicAdd(&gp[3 * p + 2], -w * dz);
            }
        }
        if (gq) { gq[3 * i] = ax; gq[3 * i + 1] = ay; gq[3 * i + 2] = az; }
    }
}

}  // namespace
}  // namespace rtd

using namespace rtd;

struct rtd_batch {
    std::vector<rtd_cloud> clouds;
    uint32_t n_clouds = 0, n_items = 0;
    int blocks = 0;             // grid of the persistent search
    uint32_t wide_kk = 0;       // list slab entries per warp (0: no k > 256 cloud)
    uint64_t n_points = 0, n_queries = 0;
    int cbits = 0, bpa = 21;
    rtd_schedule sched;
    rtd_index forest;
    DevBuf cd, items, pcloud, qcloud, qkeys, qkeys_alt, qvals, qvals_alt, counter, wide;
    // captured graph and the pointers it was captured with
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void *g_pts = nullptr, *g_q = nullptr;
    void *g_ids = nullptr, *g_d2 = nullptr;
    cudaStream_t g_stream = nullptr;
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~rtd_batch() { drop_graph(); }
};

namespace rtd {

rtd_status check_index_errors(rtd_index *idx, cudaStream_t st);

static rtd_status batch_pass(rtd_batch *b, const float *d_pts, const float *d_q, uint32_t *d_ids,
                             float *d_d2, cudaStream_t st) {
    rtd_index &f = b->forest;
    const uint64_t n = b->n_points, nq = b->n_queries;
    CloudDesc *cd = b->cd.as<CloudDesc>();
    IndexHeader *h = f.hdr.as<IndexHeader>();
    RTD_CUDA(cudaMemsetAsync(h, 0, sizeof(IndexHeader), st));
    RTD_CUDA(cudaMemsetAsync(b->counter.ptr, 0, sizeof(uint32_t), st));
    batch_reset_kernel<<<grid_for(b->n_clouds, 128, 1024), 128, 0, st>>>(cd, b->n_clouds);
    RTD_LAUNCH_CHECK();
    batch_cloud_of_kernel<<<b->n_clouds, 256, 0, st>>>(cd, b->pcloud.as<uint32_t>(),
                                                        b->qcloud.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    const int g = grid_for(n, BLOCK, 148 * 8);
    if (n) {
        batch_bbox_kernel<<<grid_for(n, BLOCK, 148 * 4), BLOCK, 0, st>>>(d_pts, n, b->pcloud.as<uint32_t>(), cd);
        RTD_LAUNCH_CHECK();
    }
    batch_seed_kernel<<<grid_for(b->n_clouds, 128, 1024), 128, 0, st>>>(
        cd, b->n_clouds, b->sched.radius_heuristic == RTD_RADIUS_FIXED ? b->sched.radius_param : 0.0f,
        b->sched.radius_param);
    RTD_LAUNCH_CHECK();
    const int kbits = 3 * b->bpa + b->cbits;
    if (n) {
        batch_keys_kernel<<<g, BLOCK, 0, st>>>(d_pts, n, b->pcloud.as<uint32_t>(), cd, b->bpa,
                                              f.keys.as<uint64_t>());
        RTD_LAUNCH_CHECK();
        bool alt = false;
        RTD_TRY(radix_sort_pairs<uint64_t>(f.keys.as<uint64_t>(), f.keys_alt.as<uint64_t>(),
                                           f.vals.as<uint32_t>(), f.vals_alt.as<uint32_t>(), true, n,
                                           0, kbits, f.sort, &h->err, st, &alt));
        const uint64_t *sk = alt ? f.keys_alt.as<uint64_t>() : f.keys.as<uint64_t>();
        const uint32_t *perm = alt ? f.vals_alt.as<uint32_t>() : f.vals.as<uint32_t>();
        batch_gather_kernel<<<g, BLOCK, 0, st>>>(d_pts, perm, b->pcloud.as<uint32_t>(), cd, n,
                                                 f.pts.as<float4>());
        RTD_LAUNCH_CHECK();
        RTD_TRY(build_tree_sorted<uint64_t>(&f, sk, n, st, true));
        if (n >= 2 && n > f.leaf_size) {
            batch_roots_kernel<<<grid_for(n, BLOCK, 148 * 8), BLOCK, 0, st>>>(
                sk, n, 3 * b->bpa, f.kfirst.as<uint32_t>(), f.klast.as<uint32_t>(),
                f.flags.as<uint32_t>(), f.cidx.as<uint32_t>(), cd);
            RTD_LAUNCH_CHECK();
        }
    }
    if (nq) {
        batch_keys_kernel<<<grid_for(nq, BLOCK, 148 * 8), BLOCK, 0, st>>>(
            d_q, nq, b->qcloud.as<uint32_t>(), cd, b->bpa, b->qkeys.as<uint64_t>());
        RTD_LAUNCH_CHECK();
        bool alt = false;
        RTD_TRY(radix_sort_pairs<uint64_t>(b->qkeys.as<uint64_t>(), b->qkeys_alt.as<uint64_t>(),
                                           b->qvals.as<uint32_t>(), b->qvals_alt.as<uint32_t>(),
                                           true, nq, 0, kbits, f.sort, &h->err, st, &alt));
        BatchArgs a;
        a.pts = f.pts.as<float4>();
        a.nodes = f.nodes.as<BvhNode>();
        a.hdr = h;
        a.cd = cd;
        a.items = nullptr;
        a.n_items = 0;
        a.counter = nullptr;
        a.qperm = alt ? b->qvals_alt.as<uint32_t>() : b->qvals.as<uint32_t>();
        a.q = d_q;
        a.ids = d_ids;
        a.d2 = d_d2;
        const float m = b->sched.radius_increment_mult;
        a.mult2 = m * m;
        a.max_rounds = b->sched.max_rounds;
        a.partial = b->sched.partial_results ? 1u : 0u;
        a.err = &h->err;
        a.items = b->items.as<WorkItem>();
        a.n_items = b->n_items;
        a.counter = b->counter.as<uint32_t>();
        a.wide = b->wide_kk ? b->wide.as<uint2>() : nullptr;
        a.wide_kk = b->wide_kk;
        if (b->n_items) {
            batch_knn_kernel<<<b->blocks, SWARPS * 32, 0, st>>>(a);
            RTD_LAUNCH_CHECK();
        }
    }
    return RTD_OK;
}

}  // namespace rtd

extern "C" {

void rtd_batch_schedule_default(rtd_schedule *s) {
    if (!s) return;
    rtd_schedule_default(s);
    s->radius_param = 1.0f;
}

rtd_status rtd_batch_create(rtd_batch **out) {
    if (!out) return fail(RTD_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = new (std::nothrow) rtd_batch();
    if (!*out) return fail(RTD_ERR_OUT_OF_MEMORY, "host allocation failed");
    rtd_batch_schedule_default(&(*out)->sched);
    return RTD_OK;
}

rtd_status rtd_batch_destroy(rtd_batch *b) {
    delete b;
    return RTD_OK;
}

rtd_status rtd_batch_plan(rtd_batch *b, const rtd_cloud *clouds, uint32_t n_clouds,
                          const rtd_schedule *sched) {
    if (!b || (n_clouds && !clouds)) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL argument");
    rtd_schedule s;
    rtd_batch_schedule_default(&s);
    if (sched) s = *sched;
    if (!(s.radius_increment_mult > 1.0f)) return fail(RTD_ERR_INVALID_ARGUMENT, "radius_increment_mult must be > 1");
    if (s.max_rounds < 1) return fail(RTD_ERR_INVALID_ARGUMENT, "max_rounds must be >= 1");
    if (s.leaf_size < 1 || s.leaf_size > 64) return fail(RTD_ERR_INVALID_ARGUMENT, "leaf_size must be in [1, 64]");
    uint64_t np = 0, nq = 0;
    uint32_t wide_kk = 0;
    std::vector<CloudDesc> cd(n_clouds);
    std::vector<WorkItem> cls_items[N_CLASSES];
    for (uint32_t c = 0; c < n_clouds; ++c) {
        const rtd_cloud &x = clouds[c];
        if (x.point_offset != np || x.query_offset != nq)
            return fail(RTD_ERR_INVALID_ARGUMENT, "clouds must be packed in order");
        if (x.k < 1) return fail(RTD_ERR_INVALID_ARGUMENT, "k must be >= 1");
        cd[c] = CloudDesc{(uint32_t)np, x.n_points, (uint32_t)nq, x.n_queries, x.k, 0u, 0u, {}, 0.f,
                          x.out_offset};
        const int cls = s.lanes_per_query == 32 && x.k <= 32 ? 2 : k_class(x.k);
        if (cls == 5 && x.n_queries) {
            const uint32_t kk = x.k < x.n_points ? x.k : (x.n_points ? x.n_points : 1u);
            if (kk > wide_kk) wide_kk = kk;
        }
        for (uint32_t s0 = 0; s0 < x.n_queries; s0 += 32)
            cls_items[cls].push_back(WorkItem{c, (uint32_t)nq + s0,
                                              x.n_queries - s0 < 32u ? x.n_queries - s0 : 32u,
                                              (uint32_t)cls});
        np += x.n_points;
        nq += x.n_queries;
    }
    if (np >= (1ull << 30) - 1 || nq >= (1ull << 30)) return fail(RTD_ERR_INVALID_ARGUMENT, "batch too large");
    // one queue, heaviest class first
    std::vector<WorkItem> items;
    for (int c = N_CLASSES - 1; c >= 0; --c) items.insert(items.end(), cls_items[c].begin(), cls_items[c].end());
    b->drop_graph();
    b->clouds.assign(clouds, clouds + n_clouds);
    b->n_clouds = n_clouds;
    b->n_points = np;
    b->n_queries = nq;
    b->n_items = (uint32_t)items.size();
    b->wide_kk = wide_kk;
    b->sched = s;
    int cb = 0;
    while (cb < 32 && (1ull << cb) < n_clouds) ++cb;
    b->cbits = cb;
    // bits per axis: the schedule's key width (auto 48 = 16 per axis), within what the
    // 63-bit key leaves beside the cloud id
    const int want = s.morton_bits ? (int)s.morton_bits / 3 : 16;
    b->bpa = (63 - cb) / 3 < want ? (63 - cb) / 3 : want;
    if (b->bpa < 8) return fail(RTD_ERR_INVALID_ARGUMENT, "too many clouds");
    rtd_index &f = b->forest;
    f.n = np;
    f.leaf_size = s.leaf_size;
    f.morton_bits = 63;
    RTD_CUDA(cudaGetDevice(&f.device));
    RTD_TRY(f.hdr.reserve(sizeof(IndexHeader)));
    RTD_TRY(f.pts.reserve((np ? np : 1) * sizeof(float4)));
    RTD_TRY(f.nodes.reserve((np > 1 ? np - 1 : 1) * sizeof(BvhNode)));
    RTD_TRY(f.keys.reserve(np * 8 + 8));
    RTD_TRY(f.keys_alt.reserve(np * 8 + 8));
    RTD_TRY(f.vals.reserve(np * 4 + 4));
    RTD_TRY(f.vals_alt.reserve(np * 4 + 4));
    RTD_TRY(b->cd.reserve(n_clouds * sizeof(CloudDesc) + 8));
    RTD_TRY(b->items.reserve(items.size() * sizeof(WorkItem) + 8));
    RTD_TRY(b->pcloud.reserve(np * 4 + 4));
    RTD_TRY(b->qcloud.reserve(nq * 4 + 4));
    RTD_TRY(b->qkeys.reserve(nq * 8 + 8));
    RTD_TRY(b->qkeys_alt.reserve(nq * 8 + 8));
    RTD_TRY(b->qvals.reserve(nq * 4 + 4));
    RTD_TRY(b->qvals_alt.reserve(nq * 4 + 4));
    RTD_TRY(b->counter.reserve(sizeof(uint32_t)));
    if (n_clouds)
        RTD_CUDA(cudaMemcpy(b->cd.ptr, cd.data(), n_clouds * sizeof(CloudDesc), cudaMemcpyHostToDevice));
    if (!items.empty())
        RTD_CUDA(cudaMemcpy(b->items.ptr, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice));
    int sms = 148;
    RTD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, f.device));
    // persistent grid: every resident warp, no more blocks than items need,
    // and (with k > 256 clouds) at most 1 GiB of list slabs
    int per_sm = 1;
    RTD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_knn_kernel, SWARPS * 32, 0));
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = (uint64_t)sms * per_sm;
    const uint64_t need = ((uint64_t)items.size() + SWARPS - 1) / SWARPS;
    if (blocks > need) blocks = need ? need : 1;
    if (wide_kk) {
        const uint64_t per_block = (uint64_t)SWARPS * wide_kk * sizeof(uint2);
        const uint64_t cap = (1ull << 30) / per_block;
        if (blocks > cap) blocks = cap ? cap : 1;
        RTD_TRY(b->wide.reserve(blocks * per_block));
    }
    b->blocks = (int)blocks;
    return RTD_OK;
}

rtd_status rtd_knn_batched(rtd_batch *b, const float *d_points, const float *d_queries,
                           uint32_t *d_ids, float *d_d2, int use_graph, rtd_stream stream) {
    if (!b) return fail(RTD_ERR_INVALID_ARGUMENT, "batch is NULL");
    if ((b->n_points && !d_points) || (b->n_queries && (!d_queries || !d_ids)))
        return fail(RTD_ERR_INVALID_ARGUMENT, "NULL device buffer");
    cudaStream_t st = (cudaStream_t)stream;
    if (!use_graph || st == nullptr) {
        RTD_TRY(batch_pass(b, d_points, d_queries, d_ids, d_d2, st));
        return check_index_errors(&b->forest, st);
    }
    const bool same = b->exec && b->g_pts == d_points && b->g_q == d_queries && b->g_ids == d_ids &&
                      b->g_d2 == d_d2 && b->g_stream == st;
    if (!same) {
        b->drop_graph();
        // an eager pass first sizes every scratch buffer (no allocation may
        // happen while capturing)
        RTD_TRY(batch_pass(b, d_points, d_queries, d_ids, d_d2, st));
        RTD_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        rtd_status s = batch_pass(b, d_points, d_queries, d_ids, d_d2, st);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (s != RTD_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        b->graph = g;
        e = cudaGraphInstantiate(&b->exec, g, 0);
        if (e != cudaSuccess) {
            b->drop_graph();
            return cuda_fail(e, "cudaGraphInstantiate");
        }
        b->g_pts = d_points;
        b->g_q = d_queries;
        b->g_ids = d_ids;
        b->g_d2 = d_d2;
        b->g_stream = st;
        return RTD_OK;   // the captured pass ran eagerly just before
    }
    RTD_CUDA(cudaGraphLaunch(b->exec, st));
    note_launch();
    return RTD_OK;
}

rtd_status rtd_knn_batched_backward(rtd_batch *b, const float *d_points, const float *d_queries,
                                    const uint32_t *d_ids, const float *d_grad_d2,
                                    float *d_grad_q, float *d_grad_p, rtd_stream stream) {
    if (!b) return fail(RTD_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (b->n_queries == 0) return RTD_OK;
    if (!d_points || !d_queries || !d_ids || !d_grad_d2)
        return fail(RTD_ERR_INVALID_ARGUMENT, "NULL device buffer");
    cudaStream_t st = (cudaStream_t)stream;
    batch_backward_kernel<<<grid_for(b->n_queries, 256, 148 * 16), 256, 0, st>>>(
        d_queries, b->n_queries, d_points, b->qcloud.as<uint32_t>(), b->cd.as<CloudDesc>(), d_ids,
        d_grad_d2, d_grad_q, d_grad_p);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

}  // extern "C"
