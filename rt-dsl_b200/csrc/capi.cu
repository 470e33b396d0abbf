// capi.cu -- the extern "C" boundary declared in include/rtdsl.h.
// Every entry point validates its arguments, returns an rtd_status and
// records a message for rtd_last_error(); nothing calls exit() (the
// reference's CUDA_CHECK/OPTIX_CHECK do, gprt-optix/host/main.cpp:12-28).
#include <atomic>
#include <cstdio>
#include <new>

#include "bh.cuh"
#include "index.cuh"
#include "sort.cuh"

namespace rtd {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const std::string &msg) { g_last_error = msg; }

rtd_status fail(rtd_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

rtd_status cuda_fail(cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    g_last_error = m;
    if (e == cudaErrorMemoryAllocation) return RTD_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return RTD_ERR_NO_DEVICE;
    return RTD_ERR_CUDA;
}

rtd_status status_from_deverr(uint32_t f) {
    if (f == 0) return RTD_OK;
    if (f & DEVERR_TIMEOUT) return fail(RTD_ERR_TIMEOUT, "a device wait hit its iteration limit");
    if (f & DEVERR_STACK) return fail(RTD_ERR_OVERFLOW, "traversal stack overflow");
    if (f & DEVERR_OVERFLOW) return fail(RTD_ERR_OVERFLOW, "output buffer too small");
    if (f & DEVERR_NOT_CONVERGED) return fail(RTD_ERR_NOT_CONVERGED, "radius expansion did not converge");
    if (f & DEVERR_DEPTH) return fail(RTD_ERR_UNSUPPORTED, "tree deeper than the key supports");
    if (f & DEVERR_MISMATCH)
        return fail(RTD_ERR_INVALID_ARGUMENT, "range fill: hit counts differ from the count pass "
                                              "(queries changed between count and fill)");
    return fail(RTD_ERR_CUDA, "unknown device error flag");
}

rtd_status DevBuf::reserve(size_t want) {
    if (want <= bytes && ptr) return RTD_OK;
    release();
    size_t b = want < 256 ? 256 : want;
    cudaError_t e = cudaMalloc(&ptr, b);
    if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        cudaGetLastError();
        return cuda_fail(e, "cudaMalloc");
    }
    bytes = b;
    return RTD_OK;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

// Implemented in lbvh.cu / knn.cu / range.cu / knn_backward.cu.
rtd_status index_build(rtd_index *idx, const float *d_xyz, uint64_t n, const rtd_schedule *s,
                       cudaStream_t st);
rtd_status k_nn_device(rtd_index *idx, const float *d_points, uint64_t n, const float *d_q,
                       uint64_t nq, uint32_t k, const rtd_schedule *sched, uint32_t *d_ids,
                       float *d_d2, cudaStream_t st, const HostChunks *hc = nullptr);
rtd_status knn_search(rtd_index *idx, const float *d_q, uint64_t nq, uint32_t k,
                      const rtd_schedule *sched, uint32_t *d_ids, float *d_d2, cudaStream_t st);
rtd_status range_count(rtd_index *idx, const float *d_q, uint64_t nq, float r,
                       const rtd_schedule *s, uint32_t *d_counts, uint64_t *h_total,
                       cudaStream_t st);
rtd_status range_fill(rtd_index *idx, const float *d_q, uint64_t nq, float r,
                      const rtd_schedule *s, uint32_t *d_pairs, uint64_t capacity, int sort_pairs,
                      uint64_t *h_written, cudaStream_t st);
rtd_status knn_backward(const float *q, uint64_t nq, const float *pts, uint64_t n, uint32_t k,
                        const uint32_t *ids, const float *g, float *gq, float *gp, cudaStream_t st);

// Reads and clears the device error flags of an index (synchronises).
rtd_status check_index_errors(rtd_index *idx, cudaStream_t st) {
    if (!idx->hdr.ptr) return RTD_OK;
    uint32_t f = 0;
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    RTD_CUDA(cudaMemcpyAsync(&f, &h->err, sizeof(f), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    if (f) RTD_CUDA(cudaMemsetAsync(&h->err, 0, sizeof(uint32_t), st));
    return status_from_deverr(f);
}

}  // namespace rtd

using namespace rtd;

static void destroy_chunk_streams(HostChunks &hc);

// Host-buffer context: an index plus device staging buffers and a stream.
struct rtd_context {
    rtd_index index;
    DevBuf data, queries, ids, d2, pairs;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_data = nullptr;  // the points are on the device (k_nn!)
    rtd_context_bh *bh = nullptr;   // created on the first barnes_hut! call
    HostChunks chunks;              // k_nn! result chunks (streams made on first use)
    ~rtd_context() {
        delete bh;
        if (ev_data) cudaEventDestroy(ev_data);
        destroy_chunk_streams(chunks);
    }
};

static void destroy_chunk_streams(HostChunks &hc) {
    if (hc.fork) cudaEventDestroy(hc.fork);
    for (int c = 0; c < MAX_CHUNKS; ++c) {
        if (hc.done[c]) cudaEventDestroy(hc.done[c]);
        if (hc.streams[c]) cudaStreamDestroy(hc.streams[c]);
    }
    hc = HostChunks();
}

// k_nn! returns results in this many chunks of the queries once there are
// enough of them to fill the GPU several times over.
constexpr uint64_t CHUNKED_MIN_QUERIES = 65536;

static rtd_status ensure_chunk_streams(HostChunks &hc) {
    if (hc.fork) return RTD_OK;
    for (int c = 0; c < MAX_CHUNKS; ++c) {
        RTD_CUDA(cudaStreamCreateWithFlags(&hc.streams[c], cudaStreamNonBlocking));
        RTD_CUDA(cudaEventCreateWithFlags(&hc.done[c], cudaEventDisableTiming));
    }
    RTD_CUDA(cudaEventCreateWithFlags(&hc.fork, cudaEventDisableTiming));
    return RTD_OK;
}

// Host-buffer k_nn! (rtd_k_nn_host and its captured form): copies the
// points and queries in, builds, searches and copies the results out on
// stream st, in chunks of the queries once there are enough of them.  Does
// not synchronise.
static rtd_status k_nn_host_run(rtd_index *idx, DevBuf &data, DevBuf &queries, DevBuf &ids,
                                DevBuf &d2buf, cudaEvent_t ev_data, HostChunks &chunks,
                                const rtd_vec3 *h_data, uint64_t n, const rtd_vec3 *h_queries,
                                uint64_t nq, uint32_t k, const rtd_schedule *sched,
                                uint32_t *h_ids, float *h_d2, cudaStream_t st) {
    if ((n && !h_data) || (nq && (!h_queries || !h_ids)))
        return fail(RTD_ERR_INVALID_ARGUMENT, "NULL host buffer");
    RTD_TRY(ensure_side_stream(idx));
    RTD_TRY(data.reserve(n * sizeof(rtd_vec3)));
    RTD_TRY(queries.reserve(nq * sizeof(rtd_vec3)));
    RTD_TRY(ids.reserve(nq * (uint64_t)k * sizeof(uint32_t)));
    if (h_d2) RTD_TRY(d2buf.reserve(nq * (uint64_t)k * sizeof(float)));
    // The points go first at full copy bandwidth; the queries follow on the
    // index's side stream, where k_nn_device then orders them (and finds
    // their Morton-window positions) while the index is built.
    if (n) RTD_CUDA(cudaMemcpyAsync(data.ptr, h_data, n * sizeof(rtd_vec3), cudaMemcpyHostToDevice, st));
    RTD_CUDA(cudaEventRecord(ev_data, st));
    RTD_CUDA(cudaStreamWaitEvent(idx->side_stream, ev_data, 0));
    if (nq)
        RTD_CUDA(cudaMemcpyAsync(queries.ptr, h_queries, nq * sizeof(rtd_vec3),
                                 cudaMemcpyHostToDevice, idx->side_stream));
    // The results come back in chunks of the queries: each chunk's rows are
    // copied to the host while the later chunks still search.
    RTD_TRY(ensure_chunk_streams(chunks));
    HostChunks hc = chunks;
    hc.chunks = nq >= CHUNKED_MIN_QUERIES ? (uint32_t)MAX_CHUNKS : 1u;
    hc.h_ids = h_ids;
    hc.h_d2 = h_d2;
    return k_nn_device(idx, data.as<float>(), n, queries.as<float>(), nq, k, sched,
                       ids.as<uint32_t>(), h_d2 ? d2buf.as<float>() : nullptr, st,
                       nq ? &hc : nullptr);
}



rtd_context_bh *context_bh(rtd_context *ctx) {
    if (!ctx->bh) ctx->bh = new (std::nothrow) rtd_context_bh();
    return ctx->bh;
}

cudaStream_t context_stream(rtd_context *ctx) { return ctx->stream; }

namespace {
// The bounded wait helper (spin_more) on one flag: waits for
// *flag != 0; when `limit` retries run out it sets DEVERR_TIMEOUT in *err
// and returns.
__global__ void wait_flag_kernel(const volatile uint32_t *flag, uint32_t limit, uint32_t *err) {
    uint32_t spins = 0;
    while (*flag == 0) {
        if (!spin_more(spins, limit)) {
            atomicOr(err, DEVERR_TIMEOUT);
            return;
        }
    }
}

std::atomic<uint32_t> g_bh_stack_entries{BH_STACK_CAP_MAX};
}  // namespace

uint32_t rtd::bh_stack_entries() { return g_bh_stack_entries.load(std::memory_order_relaxed); }

extern "C" {

rtd_status rtd_wait_selftest(uint32_t spin_limit, int flag_set, rtd_stream stream) {
    cudaStream_t st = (cudaStream_t)stream;
    DevBuf words;   // flag, err
    RTD_TRY(words.reserve(2 * sizeof(uint32_t)));
    uint32_t *w = words.as<uint32_t>();
    RTD_CUDA(cudaMemsetAsync(w, 0, 2 * sizeof(uint32_t), st));
    if (flag_set) RTD_CUDA(cudaMemsetAsync(w, 0xFF, sizeof(uint32_t), st));
    wait_flag_kernel<<<1, 1, 0, st>>>(w, spin_limit, w + 1);
    RTD_LAUNCH_CHECK();
    uint32_t err = 0;
    RTD_CUDA(cudaMemcpyAsync(&err, w + 1, sizeof(err), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    return status_from_deverr(err);
}

rtd_status rtd_radix_sort_pairs(void *d_keys, uint32_t key_bytes, uint32_t *d_vals, uint64_t n,
                                uint32_t end_bit, rtd_stream stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (key_bytes != 4 && key_bytes != 8) return fail(RTD_ERR_INVALID_ARGUMENT, "key_bytes must be 4 or 8");
    if (end_bit < 1 || end_bit > 8 * key_bytes) return fail(RTD_ERR_INVALID_ARGUMENT, "bad end_bit");
    if (n == 0) return RTD_OK;
    if (!d_keys || !d_vals) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL keys or values");
    DevBuf kalt, valt, err;
    SortScratch scr;
    RTD_TRY(kalt.reserve(n * key_bytes));
    RTD_TRY(valt.reserve(n * sizeof(uint32_t)));
    RTD_TRY(err.reserve(sizeof(uint32_t)));
    RTD_CUDA(cudaMemsetAsync(err.ptr, 0, sizeof(uint32_t), st));
    bool in_alt = false;
    if (key_bytes == 8 && end_bit > 32 && end_bit <= 48) {
        // the split sort the index build runs on keys of this width
        DevBuf k32;
        RTD_TRY(k32.reserve(2 * n * sizeof(uint32_t)));
        uint32_t *sv = nullptr;
        RTD_TRY(radix_sort_split64(static_cast<const uint64_t *>(d_keys), kalt.as<uint64_t>(),
                                   k32.as<uint32_t>(), k32.as<uint32_t>() + n, d_vals,
                                   valt.as<uint32_t>(), n, (int)end_bit, scr, st, nullptr, nullptr,
                                   kalt.as<uint64_t>(), &sv));
        RTD_CUDA(cudaMemcpyAsync(d_keys, kalt.ptr, n * key_bytes, cudaMemcpyDeviceToDevice, st));
        if (sv != d_vals)
            RTD_CUDA(cudaMemcpyAsync(d_vals, sv, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        RTD_CUDA(cudaStreamSynchronize(st));   // k32 is freed on return
    } else if (key_bytes == 4)
        RTD_TRY(radix_sort_pairs<uint32_t>(static_cast<uint32_t *>(d_keys), kalt.as<uint32_t>(),
                                           d_vals, valt.as<uint32_t>(), true, n, 0, (int)end_bit,
                                           scr, err.as<uint32_t>(), st, &in_alt));
    else
        RTD_TRY(radix_sort_pairs<uint64_t>(static_cast<uint64_t *>(d_keys), kalt.as<uint64_t>(),
                                           d_vals, valt.as<uint32_t>(), true, n, 0, (int)end_bit,
                                           scr, err.as<uint32_t>(), st, &in_alt));
    if (in_alt) {
        RTD_CUDA(cudaMemcpyAsync(d_keys, kalt.ptr, n * key_bytes, cudaMemcpyDeviceToDevice, st));
        RTD_CUDA(cudaMemcpyAsync(d_vals, valt.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    }
    uint32_t e = 0;
    RTD_CUDA(cudaMemcpyAsync(&e, err.ptr, sizeof(e), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    return status_from_deverr(e);
}

rtd_status rtd_exclusive_scan(const uint32_t *d_in, uint32_t *d_out, uint32_t *d_select, uint64_t n,
                              uint32_t *h_total, rtd_stream stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (n > 0 && (!d_in || !d_out)) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL input or output");
    DevBuf words;   // total, err
    ScanScratch scr;
    RTD_TRY(words.reserve(2 * sizeof(uint32_t)));
    uint32_t *w = words.as<uint32_t>();
    RTD_CUDA(cudaMemsetAsync(w, 0, 2 * sizeof(uint32_t), st));
    if (d_select)
        RTD_TRY(exclusive_scan_select_u32(d_in, d_out, d_select, n, w, scr, w + 1, st));
    else
        RTD_TRY(exclusive_scan_u32_32(d_in, d_out, n, w, scr, w + 1, st));
    uint32_t hw[2] = {0, 0};
    RTD_CUDA(cudaMemcpyAsync(hw, w, sizeof(hw), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    if (h_total) *h_total = hw[0];
    return status_from_deverr(hw[1]);
}

rtd_status rtd_limits_set(const rtd_limits *l) {
    if (!l) return fail(RTD_ERR_INVALID_ARGUMENT, "limits is NULL");
    const uint32_t e = l->bh_stack_entries ? l->bh_stack_entries : BH_STACK_CAP_MAX;
    if (e < 8 || e > BH_STACK_CAP_MAX)
        return fail(RTD_ERR_INVALID_ARGUMENT, "bh_stack_entries must be 0 or in [8, 8192]");
    g_bh_stack_entries.store(e, std::memory_order_relaxed);
    return RTD_OK;
}

void rtd_limits_get(rtd_limits *l) {
    if (!l) return;
    memset(l, 0, sizeof(*l));
    l->bh_stack_entries = bh_stack_entries();
}

void rtd_schedule_default(rtd_schedule *s) {
    if (!s) return;
    s->radius_increment_mult = 2.0f;
    s->max_rounds = 32;
    s->radius_heuristic = RTD_RADIUS_SAMPLED_NN;
    s->radius_param = 0.0625f;   // 2^-4 x p95 1-NN distance of a 4096-point sample
    s->use_morton_lbv = 1;
    s->leaf_size = 4;
    s->block_size = 0;
    s->lanes_per_query = 0;
    s->morton_bits = 0;
    s->partial_results = 0;
    s->reserved = 0;
}

const char *rtd_status_string(rtd_status s) {
    switch (s) {
    case RTD_OK: return "RTD_OK";
    case RTD_ERR_INVALID_ARGUMENT: return "RTD_ERR_INVALID_ARGUMENT";
    case RTD_ERR_CUDA: return "RTD_ERR_CUDA";
    case RTD_ERR_OUT_OF_MEMORY: return "RTD_ERR_OUT_OF_MEMORY";
    case RTD_ERR_OVERFLOW: return "RTD_ERR_OVERFLOW";
    case RTD_ERR_NOT_CONVERGED: return "RTD_ERR_NOT_CONVERGED";
    case RTD_ERR_TIMEOUT: return "RTD_ERR_TIMEOUT";
    case RTD_ERR_UNSUPPORTED: return "RTD_ERR_UNSUPPORTED";
    case RTD_ERR_NO_DEVICE: return "RTD_ERR_NO_DEVICE";
    }
    return "RTD_ERR_UNKNOWN";
}

const char *rtd_last_error(void) { return g_last_error.c_str(); }

int rtd_version(void) { return RTDSL_VERSION; }

rtd_status rtd_index_create(rtd_index **out) {
    if (!out) return fail(RTD_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = new (std::nothrow) rtd_index();
    if (!*out) return fail(RTD_ERR_OUT_OF_MEMORY, "host allocation failed");
    return RTD_OK;
}

rtd_status rtd_index_destroy(rtd_index *idx) {
    delete idx;
    return RTD_OK;
}

rtd_status rtd_index_build(rtd_index *idx, const float *d_xyz, uint64_t n,
                           const rtd_schedule *sched, rtd_stream stream) {
    return index_build(idx, d_xyz, n, sched, (cudaStream_t)stream);
}

rtd_status rtd_index_info_get(rtd_index *idx, rtd_index_info *info, rtd_stream stream) {
    if (!idx || !info) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL argument");
    memset(info, 0, sizeof(*info));
    info->n_points = idx->n;
    info->leaf_size = idx->leaf_size;
    info->morton_bits = (uint32_t)idx->morton_bits;
    if (!idx->hdr.ptr) return RTD_OK;
    IndexHeader h;
    cudaStream_t st = (cudaStream_t)stream;
    RTD_CUDA(cudaMemcpyAsync(&h, idx->hdr.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    info->n_internal = h.n_internal;
    for (int a = 0; a < 3; ++a) {
        info->lo[a] = float_unflip(h.box[a]);
        info->hi[a] = float_unflip(h.box[3 + a]);
    }
    return check_index_errors(idx, st);
}

rtd_status rtd_index_profile_enable(rtd_index *idx, int enable) {
    if (!idx) return fail(RTD_ERR_INVALID_ARGUMENT, "index is NULL");
    idx->prof = enable != 0;
    return RTD_OK;
}

static float ev_ms(rtd_index *idx, int a, int b) {
    if (!idx->ev_set[a] || !idx->ev_set[b]) return 0.0f;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, idx->ev[a], idx->ev[b]) != cudaSuccess) {
        cudaGetLastError();
        return 0.0f;
    }
    return ms;
}

rtd_status rtd_index_profile_get(rtd_index *idx, rtd_profile *out) {
    if (!idx || !out) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL argument");
    memset(out, 0, sizeof(*out));
    for (int i = 0; i < 8; ++i)
        if (idx->ev_set[i]) RTD_CUDA(cudaEventSynchronize(idx->ev[i]));
    out->build_sort_ms = ev_ms(idx, EV_BUILD0, EV_BUILD_SORTED);
    out->build_tree_ms = ev_ms(idx, EV_BUILD_SORTED, EV_BUILD1);
    out->seed_ms = ev_ms(idx, EV_SEARCH0, EV_SEEDED);
    out->order_ms = ev_ms(idx, EV_SEEDED, EV_ORDERED);
    out->search_ms = ev_ms(idx, EV_ORDERED, EV_SEARCH1);
    return RTD_OK;
}

uint64_t rtd_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

rtd_status rtd_knn(rtd_index *idx, const float *d_queries, uint64_t nq, uint32_t k,
                   const rtd_schedule *sched, uint32_t *d_ids, float *d_d2, rtd_stream stream) {
    return knn_search(idx, d_queries, nq, k, sched, d_ids, d_d2, (cudaStream_t)stream);
}

rtd_status rtd_k_nn(rtd_index *idx, const float *d_points, uint64_t n, const float *d_queries,
                    uint64_t nq, uint32_t k, const rtd_schedule *sched, uint32_t *d_ids,
                    float *d_d2, rtd_stream stream) {
    return k_nn_device(idx, d_points, n, d_queries, nq, k, sched, d_ids, d_d2, (cudaStream_t)stream);
}

}  // extern "C"

struct rtd_knn_graph {
    rtd_index index;
    cudaStream_t cap = nullptr;   // capture stream (the NULL stream cannot capture)
    cudaEvent_t ev = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;         // kernel launches recorded in the graph
    // host-buffer form: device staging and the result-chunk streams
    DevBuf data, queries, ids, d2;
    cudaEvent_t ev_data = nullptr;
    HostChunks chunks;
    ~rtd_knn_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ev) cudaEventDestroy(ev);
        if (ev_data) cudaEventDestroy(ev_data);
        destroy_chunk_streams(chunks);
        if (cap) cudaStreamDestroy(cap);
    }
};

// Records `run` on the graph's capture stream after an eager run of it
// (which sizes every buffer: nothing may be allocated while capturing).
template <typename Run>
static rtd_status knn_graph_capture(rtd_knn_graph *g, Run run) {
    RTD_TRY(run());
    RTD_TRY(check_index_errors(&g->index, g->cap));   // synchronises
    RTD_CUDA(cudaStreamBeginCapture(g->cap, cudaStreamCaptureModeRelaxed));
    const uint64_t before = g_launches.load(std::memory_order_relaxed);
    const rtd_status r = run();
    // recorded, not run: each launch of the graph counts them instead
    g->kernels = g_launches.load(std::memory_order_relaxed) - before;
    g_launches.fetch_sub(g->kernels, std::memory_order_relaxed);
    const cudaError_t e = cudaStreamEndCapture(g->cap, &g->graph);
    RTD_TRY(r);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    RTD_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
    return RTD_OK;
}

static rtd_status knn_graph_build(rtd_knn_graph *g, const float *d_points, uint64_t n,
                                  const float *d_queries, uint64_t nq, uint32_t k,
                                  const rtd_schedule *sched, uint32_t *d_ids, float *d_d2,
                                  cudaStream_t st) {
    RTD_CUDA(cudaStreamCreateWithFlags(&g->cap, cudaStreamNonBlocking));
    RTD_CUDA(cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming));
    // after the caller's work on its stream; an eager run sizes every
    // buffer (nothing may be allocated while capturing) and checks the inputs
    RTD_CUDA(cudaEventRecord(g->ev, st));
    RTD_CUDA(cudaStreamWaitEvent(g->cap, g->ev, 0));
    return knn_graph_capture(g, [&] {
        return k_nn_device(&g->index, d_points, n, d_queries, nq, k, sched, d_ids, d_d2, g->cap);
    });
}

// Page-locked host memory (or NULL): what a captured copy may use.
static bool host_pinned(const void *p) {
    if (!p) return true;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static rtd_status knn_graph_build_host(rtd_knn_graph *g, const rtd_vec3 *h_points, uint64_t n,
                                       const rtd_vec3 *h_queries, uint64_t nq, uint32_t k,
                                       const rtd_schedule *sched, uint32_t *h_ids, float *h_d2) {
    if (!host_pinned(h_points) || !host_pinned(h_queries) || !host_pinned(h_ids) ||
        !host_pinned(h_d2))
        return fail(RTD_ERR_INVALID_ARGUMENT, "host buffers of a captured pipeline must be page-locked");
    RTD_CUDA(cudaStreamCreateWithFlags(&g->cap, cudaStreamNonBlocking));
    RTD_CUDA(cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming));
    RTD_CUDA(cudaEventCreateWithFlags(&g->ev_data, cudaEventDisableTiming));
    return knn_graph_capture(g, [&] {
        return k_nn_host_run(&g->index, g->data, g->queries, g->ids, g->d2, g->ev_data, g->chunks,
                             h_points, n, h_queries, nq, k, sched, h_ids, h_d2, g->cap);
    });
}

extern "C" {

rtd_status rtd_knn_graph_create(const float *d_points, uint64_t n, const float *d_queries,
                                uint64_t nq, uint32_t k, const rtd_schedule *sched,
                                uint32_t *d_ids, float *d_d2, rtd_stream stream,
                                rtd_knn_graph **out) {
    if (!out) return fail(RTD_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    rtd_knn_graph *g = new (std::nothrow) rtd_knn_graph();
    if (!g) return fail(RTD_ERR_OUT_OF_MEMORY, "graph handle");
    const rtd_status r = knn_graph_build(g, d_points, n, d_queries, nq, k, sched, d_ids, d_d2,
                                         (cudaStream_t)stream);
    if (r != RTD_OK) {
        delete g;
        return r;
    }
    *out = g;
    return RTD_OK;
}

rtd_status rtd_knn_graph_create_host(const rtd_vec3 *h_points, uint64_t n,
                                     const rtd_vec3 *h_queries, uint64_t nq, uint32_t k,
                                     const rtd_schedule *sched, uint32_t *h_ids, float *h_d2,
                                     rtd_knn_graph **out) {
    if (!out) return fail(RTD_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    rtd_knn_graph *g = new (std::nothrow) rtd_knn_graph();
    if (!g) return fail(RTD_ERR_OUT_OF_MEMORY, "graph handle");
    const rtd_status r = knn_graph_build_host(g, h_points, n, h_queries, nq, k, sched, h_ids, h_d2);
    if (r != RTD_OK) {
        delete g;
        return r;
    }
    *out = g;
    return RTD_OK;
}

rtd_status rtd_knn_graph_launch(rtd_knn_graph *g, rtd_stream stream) {
    if (!g || !g->exec) return fail(RTD_ERR_INVALID_ARGUMENT, "graph is NULL");
    RTD_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    g_launches.fetch_add(g->kernels, std::memory_order_relaxed);
    return RTD_OK;
}

rtd_status rtd_knn_graph_errors(rtd_knn_graph *g, rtd_stream stream) {
    if (!g) return fail(RTD_ERR_INVALID_ARGUMENT, "graph is NULL");
    return check_index_errors(&g->index, (cudaStream_t)stream);
}

rtd_status rtd_knn_graph_destroy(rtd_knn_graph *g) {
    if (g) {
        cudaDeviceSynchronize();   // no launch may still use its buffers
        delete g;
    }
    return RTD_OK;
}

rtd_status rtd_context_create(rtd_context **out) {
    if (!out) return fail(RTD_ERR_INVALID_ARGUMENT, "out is NULL");
    rtd_context *c = new (std::nothrow) rtd_context();
    if (!c) return fail(RTD_ERR_OUT_OF_MEMORY, "host allocation failed");
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_data, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    *out = c;
    return RTD_OK;
}

rtd_status rtd_context_destroy(rtd_context *ctx) {
    if (!ctx) return RTD_OK;
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return RTD_OK;
}

rtd_status rtd_k_nn_host(rtd_context *ctx, const rtd_vec3 *data, uint64_t n,
                         const rtd_vec3 *queries, uint64_t nq, uint32_t k,
                         const rtd_schedule *sched, uint32_t *ids, float *d2) {
    if (!ctx) return fail(RTD_ERR_INVALID_ARGUMENT, "context is NULL");
    RTD_TRY(k_nn_host_run(&ctx->index, ctx->data, ctx->queries, ctx->ids, ctx->d2, ctx->ev_data,
                          ctx->chunks, data, n, queries, nq, k, sched, ids, d2, ctx->stream));
    return check_index_errors(&ctx->index, ctx->stream);   // synchronises
}

rtd_status rtd_range_count(rtd_index *idx, const float *d_queries, uint64_t nq, float radius,
                           const rtd_schedule *sched, uint32_t *d_counts, uint64_t *h_total,
                           rtd_stream stream) {
    return range_count(idx, d_queries, nq, radius, sched, d_counts, h_total, (cudaStream_t)stream);
}

rtd_status rtd_range_fill(rtd_index *idx, const float *d_queries, uint64_t nq, float radius,
                          const rtd_schedule *sched, uint32_t *d_pairs, uint64_t capacity,
                          int sort_pairs, uint64_t *h_written, rtd_stream stream) {
    return range_fill(idx, d_queries, nq, radius, sched, d_pairs, capacity, sort_pairs, h_written,
                      (cudaStream_t)stream);
}

rtd_status rtd_range_query_host(rtd_context *ctx, const rtd_vec3 *data, uint64_t n,
                                const rtd_vec3 *queries, uint64_t nq, float radius,
                                uint32_t *pairs, uint64_t capacity, uint64_t *n_pairs) {
    if (!ctx || !n_pairs) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL argument");
    if ((n && !data) || (nq && !queries) || (capacity && !pairs))
        return fail(RTD_ERR_INVALID_ARGUMENT, "NULL host buffer");
    cudaStream_t st = ctx->stream;
    RTD_TRY(ctx->data.reserve(n * sizeof(rtd_vec3)));
    RTD_TRY(ctx->queries.reserve(nq * sizeof(rtd_vec3)));
    RTD_TRY(ctx->ids.reserve(nq * sizeof(uint32_t)));
    if (n) RTD_CUDA(cudaMemcpyAsync(ctx->data.ptr, data, n * sizeof(rtd_vec3), cudaMemcpyHostToDevice, st));
    if (nq) RTD_CUDA(cudaMemcpyAsync(ctx->queries.ptr, queries, nq * sizeof(rtd_vec3), cudaMemcpyHostToDevice, st));
    RTD_TRY(index_build(&ctx->index, ctx->data.as<float>(), n, nullptr, st));
    uint64_t total = 0;
    RTD_TRY(range_count(&ctx->index, ctx->queries.as<float>(), nq, radius, nullptr,
                        ctx->ids.as<uint32_t>(), &total, st));
    *n_pairs = total;
    if (total > capacity) return fail(RTD_ERR_OVERFLOW, "pair buffer smaller than the pair count");
    RTD_TRY(ctx->pairs.reserve(total * 2 * sizeof(uint32_t)));
    uint64_t written = 0;
    RTD_TRY(range_fill(&ctx->index, ctx->queries.as<float>(), nq, radius, nullptr,
                       ctx->pairs.as<uint32_t>(), total, 1, &written, st));
    if (total) RTD_CUDA(cudaMemcpyAsync(pairs, ctx->pairs.ptr, total * 8, cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    return check_index_errors(&ctx->index, st);
}

rtd_status rtd_knn_backward(const float *d_queries, uint64_t nq, const float *d_points,
                            uint64_t n, uint32_t k, const uint32_t *d_ids,
                            const float *d_grad_d2, float *d_grad_q, float *d_grad_p,
                            rtd_stream stream) {
    return knn_backward(d_queries, nq, d_points, n, k, d_ids, d_grad_d2, d_grad_q, d_grad_p,
                        (cudaStream_t)stream);
}

}  // extern "C"
