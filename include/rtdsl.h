/*
 * rtdsl.h -- C ABI of the B200-native spatial-search path of rt-dsl:
 * exact unbounded k-NN by in-kernel radius expansion, fixed-radius range
 * query with push-to-buffer output, Barnes-Hut gravity, their backward
 * passes, and batched many-cloud k-NN.
 *
 * This header replaces the reference's C ABI, declared on the Rust side at
 * gprt-optix/src/lib.rs:13-31 and implemented in C++ at
 * gprt-optix/host/main.cpp:99-417 (OptiX pipeline / SBT / BVH / named
 * device arrays).  Each entry point below cites the reference function it
 * stands in for.  Differences from the reference boundary:
 *   - every call returns an rtd_status instead of calling exit()
 *     (main.cpp:12-28);
 *   - device-pointer entry points take a cudaStream_t and never synchronise;
 *     the *_host convenience entry points copy host buffers in and out,
 *     like the reference's gprt_execute / gprt_retrieve_* pair;
 *   - handles are not thread-safe: one handle per host thread / stream, as
 *     the reference's CGprtPipeline (main.cpp:40-61) is used.
 * No PyTorch or CUDA C++ types appear in the signatures: pointers, sizes and
 * an opaque stream handle only.
 */
#ifndef RTDSL_H
#define RTDSL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTDSL_VERSION 100

/* cudaStream_t without including cuda_runtime.h; NULL = legacy stream. */
typedef struct CUstream_st *rtd_stream;

typedef enum rtd_status {
    RTD_OK = 0,
    RTD_ERR_INVALID_ARGUMENT = 1,
    RTD_ERR_CUDA = 2,            /* a CUDA runtime call failed */
    RTD_ERR_OUT_OF_MEMORY = 3,
    RTD_ERR_OVERFLOW = 4,        /* output buffer too small; required size reported */
    RTD_ERR_NOT_CONVERGED = 5,   /* a bounded in-kernel loop ran out of rounds */
    RTD_ERR_TIMEOUT = 6,         /* a bounded device spin-wait gave up */
    RTD_ERR_UNSUPPORTED = 7,
    RTD_ERR_NO_DEVICE = 8
} rtd_status;

/* gprt-core Vec3 (#[repr(C)] f32 x,y,z), gprt-core/src/lib.rs:8-10. */
typedef struct rtd_vec3 { float x, y, z; } rtd_vec3;

/* gprt-core Body {pos, mass, velocity} (28 B), gprt-core/src/lib.rs:311-317. */
typedef struct rtd_body { rtd_vec3 pos; float mass; rtd_vec3 velocity; } rtd_body;

/* Initial-radius heuristic, gprt-ir RadiusHeuristic (gprt-ir/src/lib.rs:33-37)
 * plus the sampled nearest-neighbour seed used by the plain-kNN workload. */
typedef enum rtd_radius_heuristic {
    RTD_RADIUS_SAMPLED_NN = 0,          /* param x p95 1-NN distance of a 4096-point sample */
    RTD_RADIUS_SAMPLED_PERCENTILE = 1,  /* k_nn! default: param = percentile P, x1.1 */
    RTD_RADIUS_FIXED = 2,               /* param = radius */
    RTD_RADIUS_SAMPLED_MAX = 3,         /* percentile 1.0 */
    RTD_RADIUS_MORTON_WINDOW = 4        /* no radius rounds: each query's list starts with the
                                           4k points around it in the index's Morton order and
                                           one unbounded round follows (thread-per-query search;
                                           elsewhere as RTD_RADIUS_SAMPLED_NN with param) */
} rtd_radius_heuristic;

/* gprt-ir Schedule (gprt-ir/src/lib.rs:58-89) re-expressed for the kernels
 * here.  radius_increment_mult, radius_heuristic and use_morton_lbv keep
 * their meaning; max_hits_per_query / memory_strategy have no counterpart
 * (no per-query hit slab exists); the rest are launch knobs the autotuner
 * picks. */
typedef struct rtd_schedule {
    float radius_increment_mult;  /* M > 1: radius *= M per round (k_nn! lib.rs:592) */
    uint32_t max_rounds;          /* the last round is unbounded, so results stay exact
                                     (unless partial_results) */
    int32_t radius_heuristic;     /* rtd_radius_heuristic */
    float radius_param;           /* see rtd_radius_heuristic */
    uint32_t use_morton_lbv;      /* process queries in Morton order (k_nn! lib.rs:456-460) */
    uint32_t leaf_size;           /* LBVH leaf size: subtrees of <= leaf_size points collapse */
    uint32_t block_size;          /* threads per block of the search kernel (0 = auto) */
    uint32_t lanes_per_query;     /* 1 = thread per query, 32 = warp per query (0 = auto) */
    uint32_t morton_bits;         /* 30 (u32 keys, the reference layout) or 33..63 in steps
                                     of 3 (u64 keys, bits/3 per axis); 0 = auto */
    uint32_t partial_results;     /* 0 (default): exact; the last allowed round is unbounded.
                                     1: the reference's round cap (k_nn! gprt-macros/src/lib.rs:
                                     466, 528-530): every round stays bounded, a query short of
                                     k hits after max_rounds keeps the hits it has (remaining
                                     slots 0xFFFFFFFF / +inf) and the call's device flags report
                                     RTD_ERR_NOT_CONVERGED */
    uint32_t reserved;            /* must be 0 */
} rtd_schedule;

/* Defaults: M = 2, 32 rounds, sampled-NN seed x 2^-4, Morton query order,
 * leaf 4, auto launch shape, auto key width. */
void rtd_schedule_default(rtd_schedule *s);

const char *rtd_status_string(rtd_status s);
/* Message of the last failing call on this host thread ("" if none). */
const char *rtd_last_error(void);
int rtd_version(void);

/* ---------------------------------------------------------------------
 * LBVH index over one point cloud.  Replaces gprt_bvh_build /
 * gprt_bvh_refit / gprt_bvh_destroy (main.cpp:200-292; Rust decls
 * gprt-optix/src/lib.rs:16-19).  The tree is radius-independent, so the
 * reference's per-round refit (K1 kernels.cu:3-16 + OPTIX_BUILD_OPERATION_
 * UPDATE) has no counterpart: the radius grows inside the search kernel.
 * ------------------------------------------------------------------- */
typedef struct rtd_index rtd_index;

rtd_status rtd_index_create(rtd_index **out);
rtd_status rtd_index_destroy(rtd_index *idx);
/* d_xyz: n points, x,y,z float triples (Vec3 layout) in device memory.
 * Morton codes -> LSD radix sort -> Karras radix tree; subtrees of
 * <= leaf_size points become leaves, and every child box is taken from a
 * pyramid of boxes over runs of 8, 64, 512 ... sorted points (no bottom-up
 * refit pass). */
rtd_status rtd_index_build(rtd_index *idx, const float *d_xyz, uint64_t n,
                           const rtd_schedule *sched, rtd_stream stream);
typedef struct rtd_index_info {
    uint64_t n_points;
    uint64_t n_internal;   /* internal nodes after leaf collapse */
    uint32_t leaf_size;
    uint32_t morton_bits;
    float lo[3], hi[3];    /* scene bounding box */
} rtd_index_info;
/* Synchronises the stream, then reports sizes and device error flags. */
rtd_status rtd_index_info_get(rtd_index *idx, rtd_index_info *info, rtd_stream stream);

/* Phase timers, the counterpart of the reference's [CUDA_EVENTS] prints
 * (bvh_build / bvh_refit / kernel, gprt-optix/host/main.cpp:201-246,
 * 314-340): when enabled, the index records CUDA events around its phases
 * on the caller's stream; rtd_index_profile_get waits for them. */
typedef struct rtd_profile {
    float build_sort_ms;   /* scene box + Morton codes + radix sort + point gather */
    float build_tree_ms;   /* Karras tree + leaf collapse + child boxes + top staging */
    float seed_ms;         /* initial-radius seed */
    float order_ms;        /* query Morton ordering */
    float search_ms;       /* the search kernel (kNN or range count + fill) */
} rtd_profile;
rtd_status rtd_index_profile_enable(rtd_index *idx, int enable);
rtd_status rtd_index_profile_get(rtd_index *idx, rtd_profile *out);
/* Kernels this library has launched in this process (all handles). */
uint64_t rtd_launch_count(void);

/* Diagnostic of the bounded device wait (no reference counterpart: the
 * reference exits on any error).  No kernel of this library waits on
 * another block's progress (the radix sort and the scans run each pass as a
 * count kernel and a scatter kernel); the bounded wait helper that any such
 * wait must use gives up after a retry limit and reports RTD_ERR_TIMEOUT
 * instead of hanging the GPU.  This call runs it on a device flag: never
 * set (flag_set = 0), the wait gives up after spin_limit retries and the
 * call returns RTD_ERR_TIMEOUT with the context still usable; set
 * (flag_set = 1), it returns RTD_OK.  Synchronises. */
rtd_status rtd_wait_selftest(uint32_t spin_limit, int flag_set, rtd_stream stream);

/* Diagnostics of the two device primitives the index build runs (no
 * reference counterpart), exposed so that their results can be checked
 * against a CPU sort and scan.  rtd_radix_sort_pairs sorts n keys of
 * key_bytes (4 or 8) bytes in place by their bits [0, end_bit) with the
 * LSD radix sort (8-bit digits; 8-byte keys with 32 < end_bit <= 48 as the
 * index build sorts its Morton codes: the low end_bit - 32 bits as 8-byte
 * keys, then the top 32 bits as 4-byte keys), stably, and writes to d_vals
 * each key's index in the
 * input (d_vals is also scratch: its input is ignored).  rtd_exclusive_scan
 * writes d_out[i] = sum(d_in[0..i)) (32-bit; the caller guarantees the sum
 * fits), *h_total = sum(d_in) and, when d_select != NULL and every d_in[i] is
 * 0 or 1, d_select[d_out[i]] = i for every i with d_in[i] = 1.  Both
 * synchronise the stream. */
rtd_status rtd_radix_sort_pairs(void *d_keys, uint32_t key_bytes, uint32_t *d_vals, uint64_t n,
                                uint32_t end_bit, rtd_stream stream);
rtd_status rtd_exclusive_scan(const uint32_t *d_in, uint32_t *d_out, uint32_t *d_select,
                              uint64_t n, uint32_t *h_total, rtd_stream stream);

/* Process-wide bounds of bounded device loops.  0 keeps a field's default.
 * bh_stack_entries: traversal stack entries each warp of the Plummer-law
 * Barnes-Hut walks may use (default and maximum 8192, minimum 8); a walk
 * that needs more refuses the push and its tree reports RTD_ERR_OVERFLOW,
 * so lowering it exercises that failure path.  Takes effect at the next
 * launch. */
typedef struct rtd_limits {
    uint32_t bh_stack_entries;
    uint32_t reserved[7];
} rtd_limits;
rtd_status rtd_limits_set(const rtd_limits *l);
void rtd_limits_get(rtd_limits *l);

/* ---------------------------------------------------------------------
 * Exact k-NN.  Replaces the k_nn! round loop (gprt-macros/src/lib.rs:
 * 408-604) and its per-round gprt_execute + gprt_retrieve_array_* calls
 * (main.cpp:313-365): all rounds run inside one kernel launch.
 * Output per query: the k smallest (FP32 squared distance, point id)
 * pairs, ascending, ties to the lower id; ids[q*k+j] (and d2[q*k+j] when
 * d2 != NULL).  Slots beyond the number of points hold 0xFFFFFFFF / +inf.
 * Any k >= 1, as the reference's 2K-slot per-query slab
 * (gprt-macros/src/lib.rs:300-310): k <= 16 keeps a thread's list in
 * registers, k <= 256 a warp's list striped over its registers, and larger
 * k a warp's sorted list in shared memory (min(k, n) <= 2048) or in a
 * device slab the index keeps (grown on demand, at most 1 GiB).
 * ------------------------------------------------------------------- */
rtd_status rtd_knn(rtd_index *idx, const float *d_queries, uint64_t nq, uint32_t k,
                   const rtd_schedule *sched, uint32_t *d_ids, float *d_d2, rtd_stream stream);

/* k_nn!(data, queries, k, out[, schedule]) on device buffers: builds the
 * index over d_points (as rtd_index_build) and searches d_queries (as
 * rtd_knn) in one call, the whole k_nn! macro of gprt-macros/src/lib.rs:
 * 408-604.  The queries are Morton-ordered on a second stream owned by the
 * index while the index builds on `stream`; the call does not synchronise. */
rtd_status rtd_k_nn(rtd_index *idx, const float *d_points, uint64_t n, const float *d_queries,
                    uint64_t nq, uint32_t k, const rtd_schedule *sched, uint32_t *d_ids,
                    float *d_d2, rtd_stream stream);

/* A captured k_nn! pipeline: rtd_k_nn over fixed device buffers, recorded
 * once as a CUDA graph over an index of its own, then replayed -- the
 * per-frame pattern of repeated builds and searches of same-sized inputs,
 * without the per-kernel launch cost.  Every launch rebuilds the index from
 * the points' current contents and searches the queries' current contents;
 * nothing is cached between launches.  create runs the pipeline once
 * (results valid on return) and synchronises; the buffers must stay
 * allocated with their sizes until destroy.  launch does not synchronise;
 * errors reports the device error flags of the last launch (synchronises). */
typedef struct rtd_knn_graph rtd_knn_graph;
rtd_status rtd_knn_graph_create(const float *d_points, uint64_t n, const float *d_queries,
                                uint64_t nq, uint32_t k, const rtd_schedule *sched,
                                uint32_t *d_ids, float *d_d2, rtd_stream stream,
                                rtd_knn_graph **out);
/* The host-buffer form (k_nn! with host buffers, as rtd_k_nn_host):
 * copies the points and queries in, builds, searches and copies ids (and d2
 * if non-NULL) out, results in chunks as rtd_k_nn_host does.  Every host
 * buffer must be page-locked (cudaHostAlloc / cudaHostRegister); a launch
 * followed by rtd_knn_graph_errors leaves the results in h_ids / h_d2. */
rtd_status rtd_knn_graph_create_host(const rtd_vec3 *h_points, uint64_t n,
                                     const rtd_vec3 *h_queries, uint64_t nq, uint32_t k,
                                     const rtd_schedule *sched, uint32_t *h_ids, float *h_d2,
                                     rtd_knn_graph **out);
rtd_status rtd_knn_graph_launch(rtd_knn_graph *g, rtd_stream stream);
rtd_status rtd_knn_graph_errors(rtd_knn_graph *g, rtd_stream stream);
rtd_status rtd_knn_graph_destroy(rtd_knn_graph *g);

/* Host-buffer k_nn!(data, queries, k, out[, schedule]): copies in, builds
 * the index, searches, copies ids (and d2 if non-NULL) out, synchronises.
 * The context caches device buffers and streams across calls.  With 65,536
 * queries or more the search runs in eight chunks of the caller's query
 * order on the context's streams, each chunk's rows copied out while the
 * later chunks search; results are the same. */
typedef struct rtd_context rtd_context;
rtd_status rtd_context_create(rtd_context **out);
rtd_status rtd_context_destroy(rtd_context *ctx);
rtd_status rtd_k_nn_host(rtd_context *ctx, const rtd_vec3 *data, uint64_t n,
                         const rtd_vec3 *queries, uint64_t nq, uint32_t k,
                         const rtd_schedule *sched, uint32_t *ids, float *d2);

/* ---------------------------------------------------------------------
 * Fixed-radius range query with push-to-buffer output.  Replaces the
 * global-push programs (gprt-macros/src/lib.rs:276-295: atomicAdd on a
 * per-query length, store while below cap) and r_nn!/gprt_trace!
 * (lib.rs:625-672, 729-750).  Membership: FP32 key <= RN(r*r).
 * Count pass: d_counts[q] hits per query, *h_total the sum (this call
 * synchronises to return it).  Fill pass: (query, id) uint32 pairs into
 * d_pairs (2 u32 per pair).  When the last count on this index was over the
 * same d_queries / nq / radius (and no build, k-NN search or other count
 * came between) and capacity >= its total, every query's pairs go into its
 * own segment at the count's offsets: grouped by query in the caller's
 * order (order within a query unspecified), and RTD_ERR_INVALID_ARGUMENT if
 * the hit counts no longer match (queries changed in place).  Once an
 * earlier count has sized them, the index keeps buffers for the count's own
 * pairs (grown only, at most 2^28 pairs, 2 GiB) and for records of the
 * subtrees that lie inside a query's ball: such a count pushes its hits and
 * records while counting, and the fill of the same queries only scatters
 * and expands them into the segments (the queries are fingerprinted at both
 * calls; changed queries make the fill traverse again).  Otherwise the fill
 * pushes by warp-aggregated atomics in unspecified order.  sort_pairs != 0
 * sorts by (query, id).  If capacity < total, nothing past capacity is
 * written, *h_written = total and RTD_ERR_OVERFLOW is returned.
 * ------------------------------------------------------------------- */
rtd_status rtd_range_count(rtd_index *idx, const float *d_queries, uint64_t nq, float radius,
                           const rtd_schedule *sched, uint32_t *d_counts, uint64_t *h_total,
                           rtd_stream stream);
rtd_status rtd_range_fill(rtd_index *idx, const float *d_queries, uint64_t nq, float radius,
                          const rtd_schedule *sched, uint32_t *d_pairs, uint64_t capacity,
                          int sort_pairs, uint64_t *h_written, rtd_stream stream);
/* Host-buffer range_query!(data, queries, r, out): returns the pair count in
 * *n_pairs; pairs (2*capacity u32) receives them sorted by (query, id). */
rtd_status rtd_range_query_host(rtd_context *ctx, const rtd_vec3 *data, uint64_t n,
                                const rtd_vec3 *queries, uint64_t nq, float radius,
                                uint32_t *pairs, uint64_t capacity, uint64_t *n_pairs);

/* The reference's point files (load_points_fast, gprt-sandbox/src/io.rs:
 * 8-30): "x,y,z" lines, empty lines and lines whose first three fields do
 * not parse as f32 skipped, extra fields ignored, line order kept.  Writes
 * up to `capacity` points (3 floats each) to the host buffer `out` and the
 * file's point count to *n_points; RTD_ERR_OVERFLOW when it exceeds
 * capacity (call with capacity 0 to size the buffer). */
rtd_status rtd_load_points_csv(const char *path, float *out, uint64_t capacity,
                               uint64_t *n_points);

/* DBSCAN over the range query: the reference advertises DBSCAN on its
 * push-to-buffer range search (README.md:13) but ships no implementation.
 * idx must be built over d_points (n points); membership is the range
 * query's (FP32 key <= RN(eps*eps), the point itself included).  Core
 * points have >= min_pts neighbours; clusters are numbered 0.. in the order
 * of their smallest core point; a non-core neighbour of core points takes
 * the smallest of their cluster numbers; all other points get -1.  These
 * are the labels of the sequential algorithm expanding clusters from core
 * points in index order.  Writes d_labels (n int32) and *h_n_clusters;
 * synchronises.  Holds every neighbour pair in device memory meanwhile. */
rtd_status rtd_dbscan(rtd_index *idx, const float *d_points, uint64_t n, float eps,
                      uint32_t min_pts, int32_t *d_labels, uint64_t *h_n_clusters,
                      rtd_stream stream);

/* ---------------------------------------------------------------------
 * k-NN distance backward (no reference counterpart: the reference has no
 * gradients).  Loss gradient g[q*k+j] = dL/d(d2_qj) with ids held fixed;
 * d2_qj = |q - p_id|^2.  grad_q (nq*3) is overwritten; grad_p (n*3) is
 * accumulated with atomics (zero it first).  Slots with id 0xFFFFFFFF are
 * skipped.
 * ------------------------------------------------------------------- */
rtd_status rtd_knn_backward(const float *d_queries, uint64_t nq, const float *d_points,
                            uint64_t n, uint32_t k, const uint32_t *d_ids,
                            const float *d_grad_d2, float *d_grad_q, float *d_grad_p,
                            rtd_stream stream);

/* ---------------------------------------------------------------------
 * Batched k-NN over many independent point clouds, each with its own
 * queries and k (no reference counterpart: the reference searches one scene
 * per k_nn! call).  One pass builds every cloud's LBVH as one forest (a
 * single sort over (cloud, Morton) keys) and searches every query of every
 * cloud, whatever its k, in one persistent launch fed from one device work
 * queue; with use_graph the pass is captured once as a CUDA graph and
 * replayed.
 * ------------------------------------------------------------------- */
typedef struct rtd_cloud {
    uint64_t point_offset;  /* first point of the cloud in the packed point array */
    uint64_t query_offset;  /* first query of the cloud in the packed query array */
    uint64_t out_offset;    /* results of the cloud's query j at out_offset + j*k */
    uint32_t n_points;
    uint32_t n_queries;
    uint32_t k;             /* >= 1, any size (k above 256 keeps its list in a device slab) */
    uint32_t pad;
} rtd_cloud;

typedef struct rtd_batch rtd_batch;
rtd_status rtd_batch_create(rtd_batch **out);
rtd_status rtd_batch_destroy(rtd_batch *b);
/* Clouds must be packed in order: point_offset and query_offset of cloud c
 * are the sums of n_points / n_queries of clouds 0..c-1.  The initial radius
 * of a cloud is radius_param when radius_heuristic is RTD_RADIUS_FIXED, else
 * radius_param x the radius of a ball expected to hold k points at the
 * cloud's mean density (box volume / n_points, box extents clamped to >= max
 * extent / sqrt(n)).  leaf_size, radius_increment_mult and max_rounds apply
 * as for rtd_knn; lanes_per_query = 32 sends clouds with k <= 32 to the
 * warp-per-query search (else thread per query for k <= 16).  sched = NULL
 * means rtd_batch_schedule_default. */
rtd_status rtd_batch_plan(rtd_batch *b, const rtd_cloud *clouds, uint32_t n_clouds,
                          const rtd_schedule *sched);
/* rtd_schedule_default with radius_param = 1 (one expected k-ball). */
void rtd_batch_schedule_default(rtd_schedule *s);
/* Ids are cloud-local point indices; d_d2 may be NULL. */
rtd_status rtd_knn_batched(rtd_batch *b, const float *d_points, const float *d_queries,
                           uint32_t *d_ids, float *d_d2, int use_graph, rtd_stream stream);
/* Backward of a loss on the batched squared distances with ids fixed:
 * grad_q (all queries * 3) overwritten, grad_p (all points * 3) accumulated. */
rtd_status rtd_knn_batched_backward(rtd_batch *b, const float *d_points, const float *d_queries,
                                    const uint32_t *d_ids, const float *d_grad_d2,
                                    float *d_grad_q, float *d_grad_p, rtd_stream stream);

/* ---------------------------------------------------------------------
 * Barnes-Hut gravity.  Replaces barnes_hut! (gprt-macros/src/lib.rs:
 * 752-834): the CPU BarnesHutTree::build (gprt-core/src/lib.rs:427-539)
 * becomes a GPU build of the same tree, and gprt_execute_autorope_soa_ffi
 * (gprt-optix/host/main.cpp:371-415) becomes the walk kernels.
 * ------------------------------------------------------------------- */
typedef enum rtd_bh_law {
    /* The reference law and MAC (gprt-macros/src/lib.rs:760-806): per-body
     * stackless walk, a node is accepted when width < max(1e-6, theta*d) +
     * 1e-5; leaves are summed directly, accepted cells as monopoles; force
     * G*mi*mj*delta/(r2*sqrt(r2+1e-6)), skipped when r2 <= 1e-10.  Output:
     * forces (n*3). */
    RTD_BH_LAW_REFERENCE = 0,
    /* Plummer-softened gravity: phi_i = -G sum_j m_j/sqrt(r2+eps^2),
     * a_i = -grad phi_i; monopole + traceless quadrupole about the COM;
     * warp-coherent walk of 32 consecutive bodies with the group MAC
     * width^2 < theta^2 * dist^2(com, group box).  Output: accelerations
     * (n*3) and potentials (n). */
    RTD_BH_LAW_PLUMMER = 1
} rtd_bh_law;

typedef struct rtd_bh_params {
    float theta;
    float G;
    float eps;            /* Plummer softening length */
    int32_t law;          /* rtd_bh_law */
    int32_t quadrupole;   /* Plummer law: 1 = monopole + quadrupole, 0 = monopole */
    uint32_t bucket;      /* leaf bucket size; reference BUCKET_SIZE = 128 (lib.rs:275) */
    float min_width;      /* reference MIN_SPLIT_SIZE = 1e-5 (lib.rs:276) */
} rtd_bh_params;

/* theta 0.5, G 6.674e-11, eps 1e-3, reference law, quadrupole on,
 * bucket 128, min_width 1e-5. */
void rtd_bh_params_default(rtd_bh_params *p);

typedef struct rtd_bh rtd_bh;
rtd_status rtd_bh_create(rtd_bh **out);
rtd_status rtd_bh_destroy(rtd_bh *b);
/* Builds the octree over n bodies (d_pos n*3, d_mass n, device).  The tree
 * holds its own copy of the bodies in flat (leaf) order. */
rtd_status rtd_bh_build(rtd_bh *b, const float *d_pos, const float *d_mass, uint64_t n,
                        const rtd_bh_params *p, rtd_stream stream);
/* Frees the tree and every device buffer the handle holds (build scratch,
 * walk structures and stacks, adjoint scratch), except its 256-byte header;
 * the handle stays valid and the next walk or backward needs a new build. */
rtd_status rtd_bh_release(rtd_bh *b);
/* Walk over the built tree.  Reference law: d_out = forces, d_phi unused.
 * Plummer law: d_out = accelerations, d_phi = potentials (may be NULL).
 * Outputs are in the caller's body order. */
rtd_status rtd_bh_forward(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                          rtd_stream stream);
/* rtd_bh_forward for the Plummer law that allocates no device memory; no
 * counterpart in the reference.  For callers that cannot let a library call
 * cudaMalloc once their tree is built: hosts whose own memory manager owns
 * the device memory, and step loops that must not stall on the device-wide
 * synchronisation cudaMalloc / cudaFree can cause.  The walk's per-warp
 * traversal stack, which rtd_bh_forward reserves on first use, comes here
 * from a fixed 37 MiB array (592 warp stacks).  The CUDA module loader
 * places that array on a device the first time a call runs there (in that
 * context), and it stays until the process exits: make the first call
 * during set-up, while the device still has 37 MiB free, and before any
 * stream capture.  Later calls take no device memory.  Each call looks up
 * the array's address in the current context, so a call after
 * cudaDeviceReset or under another context finds the array there.  The
 * array limits how many warps walk at once, not the number of bodies, so no
 * tree is refused for its size; a traversal deeper than a warp's stack is
 * reported as RTD_ERR_OVERFLOW like rtd_bh_forward.  Every call shares the
 * array: calls that overlap on the GPU (other streams, other threads) race
 * and must be serialised by the caller.  Results equal rtd_bh_forward's bit
 * for bit.  RTD_BH_LAW_REFERENCE is refused with RTD_ERR_UNSUPPORTED. */
rtd_status rtd_bh_forward_noalloc(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                                  rtd_stream stream);
/* Adjoint of the Plummer-law walk (same tree, same decisions): given
 * dL/da (n*3) and dL/dphi (n, may be NULL = 0), writes dL/dpos (n*3) and
 * dL/dmass (n).  No reference counterpart (the reference has no gradients).
 * Once a backward has run on a handle, each later rtd_bh_forward also
 * records its interaction tiles (which cells and bodies each warp group
 * evaluated, about 1.5 GB at 1M bodies, theta 0.5) in a pool the handle
 * keeps, sized from the previous forward's need; a backward on the same
 * tree with the same theta and quadrupole setting then replays them
 * instead of walking the tree again (same decisions, same results).  A
 * build or rtd_bh_release drops the log. */
rtd_status rtd_bh_backward(rtd_bh *b, const rtd_bh_params *p, const float *d_g_acc,
                           const float *d_g_phi, float *d_g_pos, float *d_g_mass,
                           rtd_stream stream);
/* Time integration with the Plummer law: `steps` kick-drift-kick leapfrog
 * steps of size dt on d_pos / d_vel (n*3 each, caller order; the reference's
 * Body.velocity, gprt-core/src/lib.rs:311-317, which the reference never
 * advances), rebuilding the tree every step.  d_acc (n*3) holds a(x) of the
 * positions passed in when acc_valid != 0 (else it is computed first) and
 * a(x) of the final positions on return, so consecutive calls chain.
 * G, eps, theta, quadrupole and bucket come from p. */
rtd_status rtd_bh_leapfrog(rtd_bh *b, const rtd_bh_params *p, float *d_pos, float *d_vel,
                           const float *d_mass, uint64_t n, float dt, uint32_t steps,
                           float *d_acc, int acc_valid, rtd_stream stream);
typedef struct rtd_bh_info {
    uint64_t n_bodies, n_nodes, n_leaves;
    uint32_t depth;          /* deepest level (root = 0) */
    float root_min[3], root_max[3];
    uint32_t max_stack;      /* deepest per-warp traversal stack of the Plummer walks on
                                this tree since its build */
    uint32_t log_pages;      /* interaction-log pages (16 tiles of up to 32 interactions)
                                the last Plummer forward recorded for the adjoint; 0 = none */
} rtd_bh_info;
rtd_status rtd_bh_info_get(rtd_bh *b, rtd_bh_info *info, rtd_stream stream);
/* Interaction counts of the Plummer-law walk at opening angle theta, for
 * every stride-th body in tree order: *cells = accepted cells, *bodies =
 * bodies of opened leaves, summed over the *sampled bodies.  Measurement aid
 * (bytes and flops the walk streams per body); no reference counterpart.
 * Synchronises. */
rtd_status rtd_bh_interaction_counts(rtd_bh *b, float theta, uint64_t stride, uint64_t *cells,
                                     uint64_t *bodies, uint64_t *sampled, rtd_stream stream);
/* Host copies of the tree in the reference's FlatNode layout
 * (gprt-core/src/lib.rs:299-308, 40 B per node) and the flat body order
 * (order[i] = caller index of the i-th flat body).  Synchronises. */
rtd_status rtd_bh_export(rtd_bh *b, void *h_flat_nodes, uint32_t *h_order, rtd_stream stream);
/* Host-buffer barnes_hut!(bodies, theta, G, out) with the reference law;
 * bodies with mass <= 0 are kept (the CLI loader drops them). */
rtd_status rtd_barnes_hut_host(rtd_context *ctx, const rtd_body *bodies, uint64_t n, float theta,
                               float G, rtd_vec3 *out_forces);

#ifdef __cplusplus
}
#endif
#endif /* RTDSL_H */
