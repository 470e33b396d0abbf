// knn.cu -- exact unbounded k-NN with the search radius grown inside the
// kernel.  Replaces the k_nn! round loop (gprt-macros/src/lib.rs:462-595)
// and its OptiX register-heap programs (lib.rs:305-377): where the
// reference relaunches per round, copies a Q x 2k slab back to the host and
// filters there, every query here runs all its rounds inside one launch
// (knn_traverse.cuh).
#include <atomic>

#include "knn_traverse.cuh"

namespace rtd {
namespace {

struct KnnArgs {
    IndexView ix;
    const float *q;
    uint64_t nq;
    const uint32_t *perm;
    uint32_t k;
    float mult2;
    uint32_t max_rounds;
    uint32_t partial;       // the reference's round cap (rtd_schedule.partial_results)
    uint32_t *ids;
    float *d2;
    uint32_t *err;
    // Morton-window seed (RTD_RADIUS_MORTON_WINDOW): the points' sorted keys
    // (u64 when key64, else u32) and the quantisation scale of the build
    const void *skeys;
    int key64;
    float scale;
    const uint32_t *wpos;   // optional: each query's position, by processing order
};

// Position of a query among the points' sorted Morton keys (lower bound),
// with the build's quantisation.
__device__ __forceinline__ uint32_t morton_position(const IndexHeader *h, const void *skeys,
                                                    uint32_t n, int key64, float scale, float qx,
                                                    float qy, float qz) {
    uint32_t lo = 0, hi = n;
    if (key64) {
        const SceneNorm s = scene_norm_cubic(h);
        const uint64_t key = morton63(quantize(qx, s.lo[0], s.ext[0], scale),
                                      quantize(qy, s.lo[1], s.ext[1], scale),
                                      quantize(qz, s.lo[2], s.ext[2], scale));
        const uint64_t *sk = static_cast<const uint64_t *>(skeys);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(&sk[mid]) < key) lo = mid + 1;
            else hi = mid;
        }
    } else {
        const SceneNorm s = scene_norm(h);
        const uint32_t key = morton30(quantize(qx, s.lo[0], s.ext[0], 1023.0f),
                                      quantize(qy, s.lo[1], s.ext[1], 1023.0f),
                                      quantize(qz, s.lo[2], s.ext[2], 1023.0f));
        const uint32_t *sk = static_cast<const uint32_t *>(skeys);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(&sk[mid]) < key) lo = mid + 1;
            else hi = mid;
        }
    }
    return lo;
}

// Every query's position, in processing order, ahead of the search (so the
// search's dependent loads do not include the binary search).
__global__ void __launch_bounds__(256) window_pos_kernel(IndexHeader *h, const void *skeys,
                                                         uint32_t n, int key64, float scale,
                                                         const float *__restrict__ q,
                                                         const uint32_t *__restrict__ perm,
                                                         uint64_t nq, uint32_t *__restrict__ pos,
                                                         IndexHeader *qh) {
    // the query ordering's error flags move into the index's here
    if (qh && blockIdx.x == 0 && threadIdx.x == 0 && qh->err) {
        atomicOr(&h->err, qh->err);
        qh->err = 0;
    }
    for (uint64_t t = (uint64_t)blockIdx.x * 256 + threadIdx.x; t < nq;
         t += (uint64_t)gridDim.x * 256) {
        const uint64_t qi = perm ? perm[t] : t;
        pos[t] = morton_position(h, skeys, n, key64, scale, q[3 * qi], q[3 * qi + 1], q[3 * qi + 2]);
    }
}

// Seeds a query's list with the 4k points around its position in the
// points' Morton order (given in wpos, else found by binary search over the
// sorted keys); returns that window [w0, w1) of sorted indices.
template <int KC>
__device__ __forceinline__ void morton_window_seed(const KnnArgs &p, uint64_t t, float qx, float qy,
                                                   float qz, int kk, float (&bk)[KC],
                                                   uint32_t (&bi)[KC], uint32_t &w0, uint32_t &w1) {
    const uint32_t n = (uint32_t)p.ix.n;
    const uint32_t lo = p.wpos ? p.wpos[t]
                               : morton_position(p.ix.hdr, p.skeys, n, p.key64, p.scale, qx, qy, qz);
    const uint32_t w = 4u * (uint32_t)kk < n ? 4u * (uint32_t)kk : n;
    w0 = lo > w / 2u ? lo - w / 2u : 0u;
    if (w0 + w > n) w0 = n - w;
    w1 = w0 + w;
    for (uint32_t j = w0; j < w1; ++j) {
        const float4 pt = __ldg(&p.ix.pts[j]);
        const float key = exact_key(qx, qy, qz, pt.x, pt.y, pt.z);
        const uint32_t id = __float_as_uint(pt.w);
        if (key_less(key, id, bk[KC - 1], bi[KC - 1])) list_insert<KC>(bk, bi, key, id);
    }
}

// One thread per query.  Lists of up to 5 slots keep 40 warps resident per
// SM (48 registers a thread); longer lists take the registers they need.
template <int KC, int BLOCK>
__global__ void __launch_bounds__(BLOCK, KC <= 5 ? 1280 / BLOCK : 0) knn_thread_kernel(const KnnArgs p) {
    chain_wait();
    __shared__ BvhNode s_top[TOP_MAX];
    __shared__ uint2 s_stack[SHORT_STACK][BLOCK];
    const IndexHeader *h = p.ix.hdr;
    const uint32_t ntop = h->n_top;
    for (uint32_t i = threadIdx.x; i < ntop; i += BLOCK) s_top[i] = p.ix.top[i];
    __syncthreads();
    // a round visits each internal node at most once; more means a broken tree
    const TreeRef tree{p.ix.pts, p.ix.nodes, s_top, h->root, h->root_count,
                       2u * h->n_internal + 4u};
    const RoundSpec rs{h->r0sq, p.mult2, p.max_rounds, p.partial};
    const int kk = (int)p.k;
    uint2 l_stack[STACK_MAX - SHORT_STACK];

    for (uint64_t t = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; t < p.nq;
         t += (uint64_t)gridDim.x * BLOCK) {
        const uint64_t qi = p.perm ? p.perm[t] : t;
        const float qx = p.q[3 * qi], qy = p.q[3 * qi + 1], qz = p.q[3 * qi + 2];
        float bk[KC];
        uint32_t bi[KC];
        if (p.skeys) {
            // one unbounded round from a list seeded with the query's
            // Morton neighbours
            list_init<KC>(bk, bi, kk);
            uint32_t w0 = 0, w1 = 0;
            if (h->root != CHILD_NONE) morton_window_seed<KC>(p, t, qx, qy, qz, kk, bk, bi, w0, w1);
            const RoundSpec one{rs.r0sq, rs.mult2, 1u, 0u};
            knn_query_thread<KC, true>(tree, one, qx, qy, qz, kk, &s_stack[0][threadIdx.x], BLOCK,
                                       l_stack, p.err, bk, bi, w0, w1);
        } else {
            knn_query_thread<KC>(tree, rs, qx, qy, qz, kk, &s_stack[0][threadIdx.x], BLOCK,
                                 l_stack, p.err, bk, bi);
        }
        const uint64_t ob = qi * (uint64_t)kk;
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            if (j >= KC - kk) {
                p.ids[ob + j - (KC - kk)] = bi[j];
                if (p.d2) p.d2[ob + j - (KC - kk)] = bk[j];
            }
        }
    }
}

// One warp per query (knn_query_warp).
template <int S, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) knn_warp_kernel(const KnnArgs p) {
    __shared__ BvhNode s_top[TOP_MAX];
    __shared__ uint2 s_stack[WARPS][STACK_MAX];
    __shared__ uint2 s_list[WARPS][S * 32];
    const IndexHeader *h = p.ix.hdr;
    const uint32_t ntop = h->n_top;
    for (uint32_t i = threadIdx.x; i < ntop; i += WARPS * 32) s_top[i] = p.ix.top[i];
    __syncthreads();
    const TreeRef tree{p.ix.pts, p.ix.nodes, s_top, h->root, h->root_count,
                       2u * h->n_internal + 4u};
    const RoundSpec rs{h->r0sq, p.mult2, p.max_rounds, p.partial};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t kk = p.k;
    uint2 *stk = s_stack[warp];

    for (uint64_t t = (uint64_t)blockIdx.x * WARPS + warp; t < p.nq;
         t += (uint64_t)gridDim.x * WARPS) {
        const uint64_t qi = p.perm ? p.perm[t] : t;
        const float qx = p.q[3 * qi], qy = p.q[3 * qi + 1], qz = p.q[3 * qi + 2];
        float lk[S];
        uint32_t li[S];
        knn_query_warp<S>(tree, rs, qx, qy, qz, kk, stk, s_list[warp], p.err, lk, li);
        const uint64_t ob = qi * (uint64_t)kk;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            uint32_t j = (uint32_t)(s * 32 + lane);
            if (j < kk) {
                p.ids[ob + j] = li[s];
                if (p.d2) p.d2[ob + j] = lk[s];
            }
        }
    }
}

// One warp per query for k above the register lists (k > 256): the sorted
// list (WideList) lives in dynamic shared memory (kk entries per warp) when
// smem_list, else in the warp's own slab of `slab` (kk entries per warp of
// the grid; the grid then covers the queries with a grid-stride loop).  kk
// = min(k, points): no list ever holds more entries than the index has
// points.
constexpr int WIDE_WARPS = 4;
constexpr uint32_t WIDE_SMEM_MAX_K = 2048;   // 4 warps x 2048 x 8 B = 64 KB per block

__global__ void __launch_bounds__(WIDE_WARPS * 32) knn_wide_kernel(const KnnArgs p, uint2 *slab,
                                                                   uint32_t kk, int smem_list) {
    extern __shared__ uint2 s_dyn[];
    __shared__ BvhNode s_top[TOP_MAX];
    __shared__ uint2 s_stack[WIDE_WARPS][STACK_MAX];
    __shared__ uint32_t s_rank[WIDE_WARPS][32];
    const IndexHeader *h = p.ix.hdr;
    const uint32_t ntop = h->n_top;
    for (uint32_t i = threadIdx.x; i < ntop; i += WIDE_WARPS * 32) s_top[i] = p.ix.top[i];
    __syncthreads();
    const TreeRef tree{p.ix.pts, p.ix.nodes, s_top, h->root, h->root_count,
                       2u * h->n_internal + 4u};
    const RoundSpec rs{h->r0sq, p.mult2, p.max_rounds, p.partial};
    const int warp = threadIdx.x >> 5;
    WideList list;
    list.L = smem_list ? s_dyn + (size_t)warp * kk
                       : slab + ((size_t)blockIdx.x * WIDE_WARPS + warp) * kk;
    list.s_r = s_rank[warp];
    list.kk = kk;
    for (uint64_t t = (uint64_t)blockIdx.x * WIDE_WARPS + warp; t < p.nq;
         t += (uint64_t)gridDim.x * WIDE_WARPS) {
        const uint64_t qi = p.perm ? p.perm[t] : t;
        const float qx = p.q[3 * qi], qy = p.q[3 * qi + 1], qz = p.q[3 * qi + 2];
        knn_query_warp_list(tree, rs, qx, qy, qz, s_stack[warp], p.err, list);
        const uint64_t ob = qi * (uint64_t)p.k;
        wide_list_store(list, p.k, p.ids + ob, p.d2 ? p.d2 + ob : nullptr);
        __syncwarp();
    }
}

// ------------------------------------------------------- radius seeds
// k_nn! sampled percentile (gprt-macros/src/lib.rs:425-451): <= 100
// queries at stride max(nq/100,1) against the <= 1000-point stride sample;
// per query the k-th smallest key above 1e-10; radius = sorted sqrt values
// at index min(int(len*p), len-1), times 1.1.  k above 64 is capped at 64.
constexpr int SEED_K_MAX = 64;
__global__ void __launch_bounds__(128) seed_pct_kernel(const float *__restrict__ q, uint64_t nq,
                                                       uint32_t k, float pct,
                                                       const float4 *__restrict__ sample,
                                                       IndexHeader *h) {
    __shared__ float s[128];
    const uint32_t ns = h->n_sample;
    uint64_t qstep = nq / SEED_PCT_QUERIES > 1 ? nq / SEED_PCT_QUERIES : 1;
    uint64_t nsq = (nq + qstep - 1) / qstep;
    if (nsq > SEED_PCT_QUERIES) nsq = SEED_PCT_QUERIES;
    const uint32_t kk = k < SEED_K_MAX ? k : SEED_K_MAX;
    float val = INFINITY;
    bool ok = false;
    if (threadIdx.x < nsq && kk > 0) {
        uint64_t qi = threadIdx.x * qstep;
        float qx = q[3 * qi], qy = q[3 * qi + 1], qz = q[3 * qi + 2];
        float knn[SEED_K_MAX];
        for (uint32_t j = 0; j < kk; ++j) knn[j] = 3.402823466e38f;
        for (uint32_t j = 0; j < ns; ++j) {
            float4 pt = sample[j];
            float d2 = exact_key(qx, qy, qz, pt.x, pt.y, pt.z);
            if (d2 > 1e-10f && d2 < knn[kk - 1]) {
                int m = (int)kk - 1;
                while (m > 0 && knn[m - 1] > d2) { knn[m] = knn[m - 1]; --m; }
                knn[m] = d2;
            }
        }
        if (knn[kk - 1] != 3.402823466e38f) { val = __fsqrt_rn(knn[kk - 1]); ok = true; }
    }
    const int cnt = __syncthreads_count(ok);
    s[threadIdx.x] = val;
    __syncthreads();
    for (uint32_t kb = 2; kb <= 128; kb <<= 1)
        for (uint32_t j = kb >> 1; j > 0; j >>= 1) {
            uint32_t i = threadIdx.x, ixj = i ^ j;
            float x = s[i], y = s[ixj];
            __syncthreads();
            if (ixj > i) {
                bool up = (i & kb) == 0;
                if (up ? (x > y) : (x < y)) { s[i] = y; s[ixj] = x; }
            }
            __syncthreads();
        }
    if (threadIdx.x == 0) {
        float r = 1.0f;
        if (cnt > 0) {
            int idx = (int)((float)cnt * pct);
            if (idx > cnt - 1) idx = cnt - 1;
            if (idx < 0) idx = 0;
            r = __fmul_rn(s[idx], 1.1f);
        }
        h->r0sq = __fmul_rn(r, r);
    }
}

// Sampled-NN seed (param x p95 1-NN distance) or a fixed radius.
__global__ void seed_set_kernel(IndexHeader *h, int mode, float param) {
    float r;
    if (mode == RTD_RADIUS_FIXED) {
        r = param;
    } else {
        float key = h->nn95_key;
        r = key < 0.0f ? 1.0f : __fmul_rn(__fsqrt_rn(key), param);
        if (!(r > 0.0f) || !(r < INFINITY)) r = 1.0f;
    }
    h->r0sq = __fmul_rn(r, r);
}

template <int KC>
rtd_status launch_thread(const KnnArgs &a, uint32_t block, cudaStream_t st) {
    if (block == 256) {
        RTD_LAUNCH_CHAINED((knn_thread_kernel<KC, 256>), dim3(grid_for(a.nq, 256, 1 << 20)), dim3(256),
                           0, st, a);
    } else if (block == 64) {
        RTD_LAUNCH_CHAINED((knn_thread_kernel<KC, 64>), dim3(grid_for(a.nq, 64, 1 << 20)), dim3(64),
                           0, st, a);
    } else {
        RTD_LAUNCH_CHAINED((knn_thread_kernel<KC, 128>), dim3(grid_for(a.nq, 128, 1 << 20)), dim3(128),
                           0, st, a);
    }
    return RTD_OK;
}

template <int S>
rtd_status launch_warp(const KnnArgs &a, uint32_t block, cudaStream_t st) {
    uint64_t warps = a.nq;
    if (block == 256) {
        knn_warp_kernel<S, 8><<<grid_for(warps, 8, 1 << 20), 256, 0, st>>>(a);
    } else {
        knn_warp_kernel<S, 4><<<grid_for(warps, 4, 1 << 20), 128, 0, st>>>(a);
    }
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

// k > 256: the wide-list kernel, lists in shared memory up to
// WIDE_SMEM_MAX_K entries, else in a global slab on the index (one list per
// warp of a grid of at most 148 x 8 blocks, and at most 1 GiB of slab).
rtd_status launch_wide(rtd_index *idx, const KnnArgs &a, cudaStream_t st) {
    const uint64_t kk64 = a.k < a.ix.n ? a.k : a.ix.n;
    const uint32_t kk = kk64 ? (uint32_t)kk64 : 1u;
    const uint64_t warps = a.nq;
    if (kk <= WIDE_SMEM_MAX_K) {
        const size_t smem = (size_t)WIDE_WARPS * kk * sizeof(uint2);
        // the opt-in above 48 KB is per device, set once on each (an eager
        // search always comes before a captured one)
        static std::atomic<uint64_t> opted{0};
        if (smem > 48 * 1024 && (idx->device >= 64 || !(opted.load() >> idx->device & 1u))) {
            RTD_CUDA(cudaFuncSetAttribute(knn_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)(WIDE_WARPS * WIDE_SMEM_MAX_K * sizeof(uint2))));
            if (idx->device < 64) opted.fetch_or(1ull << idx->device);
        }
        knn_wide_kernel<<<grid_for(warps, WIDE_WARPS, 1 << 20), WIDE_WARPS * 32, smem, st>>>(
            a, nullptr, kk, 1);
    } else {
        uint64_t blocks = (warps + WIDE_WARPS - 1) / WIDE_WARPS;
        if (blocks > 148u * 8u) blocks = 148u * 8u;
        const uint64_t per_block = (uint64_t)WIDE_WARPS * kk * sizeof(uint2);
        const uint64_t cap = (1ull << 30) / per_block;
        if (blocks > cap) blocks = cap > 0 ? cap : 1;
        RTD_TRY(idx->wide.reserve(blocks * per_block));
        knn_wide_kernel<<<(unsigned)blocks, WIDE_WARPS * 32, 0, st>>>(a, idx->wide.as<uint2>(), kk, 0);
    }
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

// Moves the query-ordering error flags into the index's.
__global__ void fold_errors_kernel(IndexHeader *into, IndexHeader *from) {
    if (from->err) {
        atomicOr(&into->err, from->err);
        from->err = 0;
    }
}

}  // namespace

rtd_status seed_radius(rtd_index *idx, const float *d_q, uint64_t nq, uint32_t k,
                       const rtd_schedule &s, cudaStream_t st) {
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    switch (s.radius_heuristic) {
    case RTD_RADIUS_SAMPLED_PERCENTILE:
    case RTD_RADIUS_SAMPLED_MAX:
        seed_pct_kernel<<<1, 128, 0, st>>>(
            d_q, nq, k, s.radius_heuristic == RTD_RADIUS_SAMPLED_MAX ? 1.0f : s.radius_param,
            idx->sample.as<float4>(), h);
        break;
    case RTD_RADIUS_SAMPLED_NN:
    case RTD_RADIUS_MORTON_WINDOW:
        RTD_TRY(ensure_nn_seed(idx, st));
        [[fallthrough]];
    case RTD_RADIUS_FIXED:
        seed_set_kernel<<<1, 1, 0, st>>>(
            h, s.radius_heuristic == RTD_RADIUS_FIXED ? RTD_RADIUS_FIXED : RTD_RADIUS_SAMPLED_NN,
            s.radius_param);
        break;
    default:
        return fail(RTD_ERR_INVALID_ARGUMENT, "unknown radius heuristic");
    }
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

rtd_status knn_search(rtd_index *idx, const float *d_q, uint64_t nq, uint32_t k,
                      const rtd_schedule *sched, uint32_t *d_ids, float *d_d2, cudaStream_t st) {
    return knn_search_ex(idx, d_q, nq, k, sched, d_ids, d_d2, st, false, nullptr, nullptr);
}

// Whether a search with this schedule runs the Morton-window seed (the
// thread-per-query kernel with RTD_RADIUS_MORTON_WINDOW).
static bool uses_window(const rtd_index *idx, const rtd_schedule &s, uint32_t k) {
    uint32_t lanes = s.lanes_per_query;
    if (lanes == 0) lanes = k <= 16 ? 1 : 32;
    if (lanes == 1 && k > 32) lanes = 32;
    return lanes == 1 && !s.partial_results && s.radius_heuristic == RTD_RADIUS_MORTON_WINDOW &&
           idx->n > 1 && idx->skeys != nullptr;
}

// Launches the search kernel the schedule selects for the queries of a.
static rtd_status launch_search(rtd_index *idx, const rtd_schedule &s, uint32_t k, KnnArgs a,
                                cudaStream_t st) {
    uint32_t lanes = s.lanes_per_query;
    if (lanes == 0) lanes = k <= 16 ? 1 : 32;
    if (lanes == 1 && k > 32) lanes = 32;
    const uint32_t block = s.block_size;
    rtd_status r;
    if (lanes == 1) {
        // The Morton-window seed runs in the thread-per-query kernel; the
        // other launch modes treat the heuristic as RTD_RADIUS_SAMPLED_NN.
        if (uses_window(idx, s, k)) a.skeys = idx->skeys;
        else a.wpos = nullptr;
        if (k <= 1) r = launch_thread<1>(a, block, st);
        else if (k <= 2) r = launch_thread<2>(a, block, st);
        else if (k <= 4) r = launch_thread<4>(a, block, st);
        else if (k == 5) r = launch_thread<5>(a, block, st);
        else if (k <= 8) r = launch_thread<8>(a, block, st);
        else if (k <= 16) r = launch_thread<16>(a, block, st);
        else r = launch_thread<32>(a, block, st);
    } else if (k > 256) {
        r = launch_wide(idx, a, st);
    } else if (lanes == 32) {
        if (k <= 32) r = launch_warp<1>(a, block, st);
        else if (k <= 64) r = launch_warp<2>(a, block, st);
        else if (k <= 128) r = launch_warp<4>(a, block, st);
        else r = launch_warp<8>(a, block, st);
    } else {
        return fail(RTD_ERR_INVALID_ARGUMENT, "lanes_per_query must be 0, 1 or 32");
    }
    return r;
}

rtd_status knn_search_ex(rtd_index *idx, const float *d_q, uint64_t nq, uint32_t k,
                         const rtd_schedule *sched, uint32_t *d_ids, float *d_d2,
                         cudaStream_t st, bool have_perm, const uint32_t *given_perm,
                         const uint32_t *wpos, const HostChunks *hc) {
    if (!idx || !idx->hdr.ptr) return fail(RTD_ERR_INVALID_ARGUMENT, "index not built");
    if (nq == 0) return RTD_OK;
    if (!d_q || !d_ids) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL queries or ids");
    if (k == 0) return fail(RTD_ERR_INVALID_ARGUMENT, "k must be >= 1");
    rtd_schedule def;
    rtd_schedule_default(&def);
    const rtd_schedule &s = sched ? *sched : def;
    if (!(s.radius_increment_mult > 1.0f) || !(s.radius_increment_mult < INFINITY))
        return fail(RTD_ERR_INVALID_ARGUMENT, "radius_increment_mult must be > 1");
    if (s.max_rounds < 1) return fail(RTD_ERR_INVALID_ARGUMENT, "max_rounds must be >= 1");
    if (s.reserved != 0) return fail(RTD_ERR_INVALID_ARGUMENT, "schedule.reserved must be 0");
    if (s.radius_heuristic == RTD_RADIUS_FIXED && !(s.radius_param > 0.0f))
        return fail(RTD_ERR_INVALID_ARGUMENT, "fixed radius must be > 0");
    for (int e = EV_SEARCH0; e <= EV_SEARCH1; ++e) idx->ev_set[e] = false;
    idx->mark(EV_SEARCH0, st);
    // the Morton-window search runs one unbounded round: no initial radius
    if (!uses_window(idx, s, k)) RTD_TRY(seed_radius(idx, d_q, nq, k, s, st));
    idx->mark(EV_SEEDED, st);
    const uint32_t *perm = given_perm;
    if (!have_perm) RTD_TRY(order_queries(idx, d_q, nq, s.use_morton_lbv != 0, &perm, st));
    idx->mark(EV_ORDERED, st);
    KnnArgs a;
    a.ix = view_of(idx);
    a.q = d_q;
    a.nq = nq;
    a.perm = perm;
    a.k = k;
    float m = s.radius_increment_mult;
    a.mult2 = m * m;
    a.max_rounds = s.max_rounds;
    a.partial = s.partial_results ? 1u : 0u;
    a.ids = d_ids;
    a.d2 = d_d2;
    a.err = &idx->hdr.as<IndexHeader>()->err;
    a.skeys = nullptr;
    a.wpos = wpos;
    a.key64 = idx->morton_bits != 30;
    a.scale = idx->morton_bits == 30 ? 1023.0f : (float)((1u << (idx->morton_bits / 3)) - 1u);
    rtd_status r = RTD_OK;
    if (!hc || hc->chunks <= 1) {
        r = launch_search(idx, s, k, a, st);
        if (r == RTD_OK && hc) {   // one chunk: copy every row out
            RTD_CUDA(cudaMemcpyAsync(hc->h_ids, d_ids, nq * (uint64_t)k * 4, cudaMemcpyDeviceToHost, st));
            if (d_d2 && hc->h_d2)
                RTD_CUDA(cudaMemcpyAsync(hc->h_d2, d_d2, nq * (uint64_t)k * 4, cudaMemcpyDeviceToHost, st));
        }
    } else {
        // Chunk c (caller rows [b, e), processing positions [b, e)) searches
        // on its own stream and copies its rows out when it ends; the block
        // scheduler takes the chunks' blocks in launch order, so the first
        // chunks end (and copy) while the last ones still search.
        RTD_CUDA(cudaEventRecord(hc->fork, st));
        for (uint32_t c = 0; c < hc->chunks && r == RTD_OK; ++c) {
            const uint64_t b = chunk_begin(nq, hc->chunks, c), e = chunk_begin(nq, hc->chunks, c + 1);
            cudaStream_t cs = hc->streams[c];
            RTD_CUDA(cudaStreamWaitEvent(cs, hc->fork, 0));
            if (e > b) {
                KnnArgs ac = a;
                ac.nq = e - b;
                if (a.perm) {
                    ac.perm = a.perm + b;
                } else {   // caller order: the chunk's queries and rows themselves
                    ac.q = a.q + 3 * b;
                    ac.ids = a.ids + b * k;
                    if (a.d2) ac.d2 = a.d2 + b * k;
                }
                if (a.wpos) ac.wpos = a.wpos + b;
                r = launch_search(idx, s, k, ac, cs);
                if (r == RTD_OK) {
                    RTD_CUDA(cudaMemcpyAsync(hc->h_ids + b * k, d_ids + b * k, (e - b) * k * 4,
                                             cudaMemcpyDeviceToHost, cs));
                    if (d_d2 && hc->h_d2)
                        RTD_CUDA(cudaMemcpyAsync(hc->h_d2 + b * k, d_d2 + b * k, (e - b) * k * 4,
                                                 cudaMemcpyDeviceToHost, cs));
                }
            }
            RTD_CUDA(cudaEventRecord(hc->done[c], cs));
            RTD_CUDA(cudaStreamWaitEvent(st, hc->done[c], 0));
        }
    }
    idx->mark(EV_SEARCH1, st);
    return r;
}

// k_nn! on device buffers: build + search in one call.  The queries are
// Morton-ordered on the index's side stream (against their own box, with
// their own scratch) while the index builds on the caller's stream; the
// search waits for both.
rtd_status k_nn_device(rtd_index *idx, const float *d_points, uint64_t n, const float *d_q,
                       uint64_t nq, uint32_t k, const rtd_schedule *sched, uint32_t *d_ids,
                       float *d_d2, cudaStream_t st, const HostChunks *hc) {
    if (!idx) return fail(RTD_ERR_INVALID_ARGUMENT, "index is NULL");
    if (nq && (!d_q || !d_ids)) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL queries or ids");
    rtd_schedule def;
    rtd_schedule_default(&def);
    const rtd_schedule &s = sched ? *sched : def;
    const uint32_t chunks = hc ? hc->chunks : 1u;
    RTD_TRY(ensure_side_stream(idx));
    cudaStream_t side = idx->side_stream;
    RTD_CUDA(cudaEventRecord(idx->ev_fork, st));   // the queries' producers come first
    RTD_CUDA(cudaStreamWaitEvent(side, idx->ev_fork, 0));
    const uint32_t *perm = nullptr;
    rtd_status ord = RTD_OK;
    if (s.use_morton_lbv && nq >= 2 && k > 0)
        ord = order_queries_own(idx->qorder, d_q, nq, &perm, side, chunks);
    RTD_CUDA(cudaEventRecord(idx->ev_join, side));
    rtd_status r = index_build(idx, d_points, n, &s, st);
    // With the Morton-window seed, the queries' positions among the sorted
    // keys are found on the side stream as soon as the keys are sorted,
    // while the tree is built.
    const uint32_t *wpos = nullptr;
    if (r == RTD_OK && ord == RTD_OK && nq && uses_window(idx, s, k)) {
        r = idx->wpos.reserve(nq * sizeof(uint32_t));
        if (r == RTD_OK) {
            RTD_CUDA(cudaStreamWaitEvent(side, idx->ev_sorted, 0));
            window_pos_kernel<<<grid_for(nq, 256, 148 * 8), 256, 0, side>>>(
                idx->hdr.as<IndexHeader>(), idx->skeys, (uint32_t)idx->n, idx->morton_bits != 30,
                idx->morton_bits == 30 ? 1023.0f : (float)((1u << (idx->morton_bits / 3)) - 1u),
                d_q, perm, nq, idx->wpos.as<uint32_t>(),
                perm ? idx->qorder.hdr.as<IndexHeader>() : nullptr);
            RTD_LAUNCH_CHECK();
            RTD_CUDA(cudaEventRecord(idx->ev_join, side));
            wpos = idx->wpos.as<uint32_t>();
        }
    }
    RTD_CUDA(cudaStreamWaitEvent(st, idx->ev_join, 0));   // also on the error paths
    RTD_TRY(ord);
    RTD_TRY(r);
    if (perm && !wpos) {   // (window_pos_kernel has folded them otherwise)
        fold_errors_kernel<<<1, 1, 0, st>>>(idx->hdr.as<IndexHeader>(), idx->qorder.hdr.as<IndexHeader>());
        RTD_LAUNCH_CHECK();
    }
    return knn_search_ex(idx, d_q, nq, k, &s, d_ids, d_d2, st, true, perm, wpos, hc);
}

}  // namespace rtd
