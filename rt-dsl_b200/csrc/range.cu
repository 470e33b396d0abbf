// range.cu -- fixed-radius range query: a count pass sizes the output, a
// fill pass writes (query, id) pairs into it.  Replaces the reference's
// global-push programs (gprt-macros/src/lib.rs:276-295), where every
// any-hit does atomicAdd(&lens[q], 1) into a capped per-query slab that the
// host then copies back and filters (lib.rs:538-583).  Here the buffer is
// exactly sized by the count pass.  A fill that follows the count of the
// same queries writes every query's hits into its own segment of the
// buffer, at the offsets the count's exclusive scan left on the index (no
// atomics; pairs come out grouped by query in the caller's order).  Any
// other fill stages hits per warp in shared memory and pushes them with one
// global atomicAdd per flush (warp-aggregated compaction).  Membership:
// exact FP32 key <= RN(r*r), as the intersection program tests
// dist_sq <= r_val*r_val (lib.rs:283, 341).
#include "index.cuh"

namespace rtd {
namespace {

constexpr int RBLOCK = 128;
constexpr int RWARPS = RBLOCK / 32;
constexpr int SHORT_DEPTH = 12;  // stack entries per thread in shared memory
constexpr int STACK_DEPTH = 104; // >= maximal tree depth
constexpr int WBUF = 256;        // staged pairs per warp (2 KB)
constexpr uint32_t BIG_SUB = 32;  // contained subtrees of this size or more: copied by the warp

// Kernel modes: count hits, push pairs through warp staging and a global
// cursor, write pairs into per-query segments at known offsets, or count
// hits and push them at once (a count whose pairs the next fill scatters).
enum : int { MODE_COUNT = 0, MODE_PUSH = 1, MODE_SEG = 2, MODE_CPUSH = 3 };

struct RangeArgs {
    IndexView ix;
    const float *q;
    uint64_t nq;
    const uint32_t *perm;
    float r2;
    uint32_t *counts;
    uint2 *pairs;
    uint64_t capacity;
    unsigned long long *cursor;
    const uint64_t *offsets;   // MODE_SEG: exclusive offsets of the count pass
    uint64_t total;            // MODE_SEG: end of the last segment
    int skip_if_same;          // MODE_SEG: do nothing when the header's two query
                               // fingerprints agree (the scatter fills instead)
    // MODE_CPUSH: every contained subtree becomes a record (query, first
    // sorted point, points) that the fill's expansion writes out;
    // cursor[1] counts records, cursor[2] the points they cover
    uint4 *recs;
    uint64_t rec_cap;
    uint32_t *err;
};

__device__ __forceinline__ void load_node_r(const BvhNode *__restrict__ s_top,
                                            const BvhNode *__restrict__ g, uint32_t w, float4 &a,
                                            float4 &b, float4 &c, uint4 &d) {
    if (w & CHILD_TOP) {
        const BvhNode &n = s_top[w & CHILD_INDEX];
        a = n.a; b = n.b; c = n.c; d = n.d;
    } else {
        const BvhNode *n = g + (w & CHILD_INDEX);
        a = __ldg(&n->a); b = __ldg(&n->b); c = __ldg(&n->c); d = __ldg(&n->d);
    }
}

// One traversal step state per thread.
struct Walk {
    uint32_t node;
    int sp;
};

// Fields of the per-lane work a traversal step stages for the warp (one
// 32-word row per field, so lanes reading different owners hit different
// banks).
enum : int { F_QX = 0, F_QY, F_QZ, F_F0, F_C0, F_F1, F_T, F_DONE,   // count needs these
             F_QI, F_G0, F_N0, F_G1, F_WLEN, F_WBLO, F_WBHI, F_COUNT_ALL };
constexpr int F_COUNT_ONLY = F_DONE + 1;

// MODE_COUNT: count hits per query.  MODE_PUSH / MODE_SEG: write pairs.
// Threads of a warp advance their own traversals one node per iteration of
// a warp-converged loop; a stack entry carries the node and the first
// sorted point below it.  A child whose whole box lies inside the ball
// (farthest-corner key <= r^2, a bound on every point's key) contributes
// all its points without a test: its count in the count pass, its
// contiguous ids in the fills (by the whole warp, one pair per lane, for
// subtrees of BIG_SUB points or more).  After each step the lanes' other
// work -- points of the leaves that straddle the sphere, to test, and
// (fills) points of small contained subtrees, to take -- is flattened over the warp by a prefix sum
// and processed 32 candidates at a time with every lane busy: a lane finds
// its candidate's owner by a binary search over the prefix (shuffles) and
// reads the owner's query and ranges from shared memory.  One ballot per
// batch gives every hit its rank among its owner's hits in the batch.
// MODE_COUNT adds each owner's hits; MODE_SEG writes them at the owner's
// next slots of its segment and checks that the query fills it exactly;
// MODE_PUSH compacts them into the warp's staging buffer, which the warp
// pushes with one global atomic per flush.
template <int MODE>
__global__ void __launch_bounds__(RBLOCK, MODE == MODE_COUNT ? 10 : 8) range_kernel(const RangeArgs p) {
    constexpr bool PUSH = MODE == MODE_PUSH || MODE == MODE_CPUSH;   // through warp staging
    constexpr bool SEG = MODE == MODE_SEG;
    constexpr bool FILL = PUSH || SEG;
    constexpr bool COUNTS = MODE == MODE_COUNT || MODE == MODE_CPUSH;
    constexpr int NF = FILL ? F_COUNT_ALL : F_COUNT_ONLY;
    if (SEG && p.skip_if_same && p.ix.hdr->qfp[0] == p.ix.hdr->qfp[1]) return;
    __shared__ BvhNode s_top[TOP_MAX];
    __shared__ uint2 s_stack[SHORT_DEPTH][RBLOCK];
    __shared__ uint2 s_buf[PUSH ? RWARPS : 1][PUSH ? WBUF : 1];
    __shared__ uint32_t s_work[RWARPS][NF][32];
    const IndexHeader *h = p.ix.hdr;
    const uint32_t ntop = h->n_top;
    for (uint32_t i = threadIdx.x; i < ntop; i += RBLOCK) s_top[i] = p.ix.top[i];
    __syncthreads();
    const uint32_t root = h->root, root_count = h->root_count;
    const float4 *__restrict__ pts = p.ix.pts;
    const BvhNode *__restrict__ gn = p.ix.nodes;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    const float r2 = p.r2;
    const uint32_t visit_cap = 2u * h->n_internal + 4u;
    uint2 l_stack[STACK_DEPTH - SHORT_DEPTH];
    uint2 *buf = s_buf[PUSH ? warp : 0];
    uint32_t (*W)[32] = s_work[warp];
    uint32_t fill = 0;   // staged pairs of this warp (warp-uniform)

    // pushes the staged pairs with one reservation on the global cursor
    auto flush = [&]() {
        if (!PUSH || fill == 0) return;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(p.cursor, (unsigned long long)fill);
        base = __shfl_sync(0xffffffffu, base, 0);
        __syncwarp();
        for (uint32_t j = lane; j < fill; j += 32) {
            const uint64_t dst = base + j;
            if (dst < p.capacity) p.pairs[dst] = buf[j];
        }
        // (the count's own pushes are speculative: a short buffer only
        // means the fill runs its own traversal)
        if (MODE == MODE_PUSH && lane == 0 && base + fill > p.capacity)
            atomicOr(p.err, DEVERR_OVERFLOW);
        __syncwarp();
        fill = 0;
    };

    const uint64_t stride = (uint64_t)gridDim.x * RBLOCK;
    const uint64_t t0 = (uint64_t)blockIdx.x * RBLOCK + warp * 32;
    // warp-uniform loop over query batches
    for (uint64_t tb = t0; tb < p.nq; tb += stride) {
        const uint64_t t = tb + lane;
        const bool have = t < p.nq;
        uint64_t qi = 0;
        float qx = 0.f, qy = 0.f, qz = 0.f;
        if (have) {
            qi = p.perm ? p.perm[t] : t;
            qx = p.q[3 * qi]; qy = p.q[3 * qi + 1]; qz = p.q[3 * qi + 2];
        }
        __syncwarp();   // the previous batch's readers of W are done
        W[F_QX][lane] = __float_as_uint(qx);
        W[F_QY][lane] = __float_as_uint(qy);
        W[F_QZ][lane] = __float_as_uint(qz);
        W[F_DONE][lane] = 0;
        uint64_t wend = 0;
        if (FILL) W[F_QI][lane] = (uint32_t)qi;
        if (SEG) {   // this query's segment of the pair buffer
            uint64_t wb = 0;
            if (have) {
                wb = p.offsets[qi];
                wend = qi + 1 < p.nq ? p.offsets[qi + 1] : p.total;
            }
            W[F_WLEN][lane] = (uint32_t)(wend - wb);
            W[F_WBLO][lane] = (uint32_t)wb;
            W[F_WBHI][lane] = (uint32_t)(wb >> 32);
        }
        // a query with a NaN coordinate has no neighbours (its keys are NaN)
        const bool live = have && !isnan(qx) && !isnan(qy) && !isnan(qz);
        uint32_t node = (live && root != CHILD_NONE) ? root : CHILD_NONE;
        uint32_t first = 0;   // first sorted point below `node`
        int sp = 0;
        uint32_t cnt = 0;     // points of contained subtrees (count pass)
        uint32_t visits = 0;
        bool seg_bad = false;
        while (__any_sync(0xffffffffu, node != CHILD_NONE)) {
            if (node != CHILD_NONE && ++visits > visit_cap) {   // broken tree: give up
                atomicOr(p.err, DEVERR_STACK);
                node = CHILD_NONE;
                sp = 0;
            }
            uint32_t f0 = 0, c0 = 0, f1 = 0, c1 = 0;   // leaves to test
            uint32_t g0 = 0, n0 = 0, g1 = 0, n1 = 0;   // subtrees inside the ball
            if (node != CHILD_NONE) {
                uint32_t next = CHILD_NONE, next_first = 0;
                if (node & CHILD_LEAF) {
                    f0 = node & CHILD_INDEX;
                    c0 = root_count;
                } else {
                    float4 a, b, c;
                    uint4 d;
                    load_node_r(s_top, gn, node, a, b, c, d);
                    const uint32_t fl = first, fr = first + d.z;
                    bool v0 = !(box_min_key(qx, qy, qz, a.x, a.y, a.z, a.w, b.x, b.y) > r2);
                    bool v1 = !(box_min_key(qx, qy, qz, b.z, b.w, c.x, c.y, c.z, c.w) > r2);
                    if (v0 && !(box_max_key(qx, qy, qz, a.x, a.y, a.z, a.w, b.x, b.y) > r2)) {
                        g0 = fl; n0 = d.z; v0 = false;
                    }
                    if (v1 && !(box_max_key(qx, qy, qz, b.z, b.w, c.x, c.y, c.z, c.w) > r2)) {
                        g1 = fr; n1 = d.w; v1 = false;
                    }
                    if (v0 && (d.x & CHILD_LEAF)) { f0 = fl; c0 = d.z; v0 = false; }
                    if (v1 && (d.y & CHILD_LEAF)) {
                        if (c0) { f1 = fr; c1 = d.w; }
                        else { f0 = fr; c0 = d.w; }
                        v1 = false;
                    }
                    if (v0 && v1) {
                        next = d.x;
                        next_first = fl;
                        const uint2 e = make_uint2(d.y, fr);
                        if (sp < SHORT_DEPTH) s_stack[sp++][threadIdx.x] = e;
                        else if (sp < STACK_DEPTH) { l_stack[sp - SHORT_DEPTH] = e; ++sp; }
                        else atomicOr(p.err, DEVERR_STACK);
                    } else if (v0) {
                        next = d.x;
                        next_first = fl;
                    } else if (v1) {
                        next = d.y;
                        next_first = fr;
                    }
                }
                if (next == CHILD_NONE && sp > 0) {
                    --sp;
                    const uint2 e = sp < SHORT_DEPTH ? s_stack[sp][threadIdx.x] : l_stack[sp - SHORT_DEPTH];
                    next = e.x;
                    next_first = e.y;
                }
                node = next;
                first = next_first;
            }
            if (!FILL) cnt += n0 + n1;
            if (FILL) {
                // contained subtrees of BIG_SUB points or more: the whole
                // warp copies each one's contiguous ids, one pair per lane
                // (the pushing count records every contained subtree)
                constexpr uint32_t BIG = MODE == MODE_CPUSH ? 1u : BIG_SUB;
                const uint32_t b0 = n0 >= BIG ? n0 : 0u, b1 = n1 >= BIG ? n1 : 0u;
                if (MODE == MODE_CPUSH) cnt += b0 + b1;
                if (b0) n0 = 0;
                if (b1) n1 = 0;
                if (MODE == MODE_CPUSH) {
                    // records, not copies: a query inside a dense cluster
                    // would keep its warp copying for thousands of steps,
                    // while the scatter expands records with every warp
                    const uint32_t rm0 = __ballot_sync(0xffffffffu, b0 != 0);
                    const uint32_t rm1 = __ballot_sync(0xffffffffu, b1 != 0);
                    const uint32_t nr = __popc(rm0) + __popc(rm1);
                    if (nr) {
                        uint32_t covered = b0 + b1;
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) covered += __shfl_xor_sync(0xffffffffu, covered, o);
                        unsigned long long base = 0;
                        if (lane == 0) {
                            base = atomicAdd(&p.cursor[1], (unsigned long long)nr);
                            atomicAdd(&p.cursor[2], (unsigned long long)covered);
                        }
                        base = __shfl_sync(0xffffffffu, base, 0);
                        // slots: the lanes' first records in lane order, then their second ones
                        uint64_t r = base + __popc(rm0 & lt);
                        if (b0 && r < p.rec_cap) p.recs[r] = make_uint4((uint32_t)qi, g0, b0, 0u);
                        r = base + __popc(rm0) + __popc(rm1 & lt);
                        if (b1 && r < p.rec_cap) p.recs[r] = make_uint4((uint32_t)qi, g1, b1, 0u);
                    }
                }
                uint32_t m = MODE == MODE_CPUSH ? 0u : __ballot_sync(0xffffffffu, (b0 | b1) != 0);
                while (m) {
                    const int src = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t sq = (uint32_t)__shfl_sync(0xffffffffu, (uint32_t)qi, src);
                    for (int r = 0; r < 2; ++r) {
                        const uint32_t gs = __shfl_sync(0xffffffffu, r ? g1 : g0, src);
                        const uint32_t ns = __shfl_sync(0xffffffffu, r ? b1 : b0, src);
                        if (ns == 0) continue;
                        if (SEG) {
                            const uint32_t done = W[F_DONE][src];
                            if ((uint64_t)done + ns <= W[F_WLEN][src]) {
                                const uint64_t dst =
                                    (((uint64_t)W[F_WBHI][src] << 32) | W[F_WBLO][src]) + done;
                                for (uint32_t k = lane; k < ns; k += 32)
                                    p.pairs[dst + k] = make_uint2(sq, __float_as_uint(__ldg(&pts[gs + k].w)));
                            } else {
                                seg_bad = true;
                            }
                            __syncwarp();
                            if (lane == src) W[F_DONE][src] = done + ns;
                            __syncwarp();
                        } else {
                            for (uint32_t base = 0; base < ns; base += 32) {
                                const uint32_t take = ns - base < 32u ? ns - base : 32u;
                                if ((uint32_t)lane < take)
                                    buf[fill + lane] = make_uint2(sq, __float_as_uint(__ldg(&pts[gs + base + lane].w)));
                                fill += take;
                                if (fill > WBUF - 32) flush();
                            }
                        }
                    }
                }
            }
            // flatten this step's remaining candidates over the warp
            const uint32_t tl = c0 + c1;
            const uint32_t items = tl + (FILL ? n0 + n1 : 0u);
            uint32_t incl = items;
#pragma unroll
            for (int dlt = 1; dlt < 32; dlt <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, dlt);
                if (lane >= dlt) incl += v;
            }
            const uint32_t excl = incl - items;
            const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
            if (total == 0) continue;
            W[F_F0][lane] = f0;
            W[F_C0][lane] = c0;
            W[F_F1][lane] = f1;
            W[F_T][lane] = tl;
            if (FILL) {
                W[F_G0][lane] = g0;
                W[F_N0][lane] = n0;
                W[F_G1][lane] = g1;
            }
            __syncwarp();
            for (uint32_t base = 0; base < total; base += 32) {
                const uint32_t ci = base + lane;
                const bool valid = ci < total;
                // owner: the last lane whose prefix is <= ci
                int o = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const uint32_t pv = __shfl_sync(0xffffffffu, excl, o + step);
                    if (pv <= ci) o += step;
                }
                const uint32_t oexcl = __shfl_sync(0xffffffffu, excl, o);
                const uint32_t oitems = __shfl_sync(0xffffffffu, items, o);
                bool hit = false;
                uint32_t id = 0;
                if (valid) {
                    const uint32_t j = ci - oexcl;
                    const uint32_t ot = W[F_T][o];
                    if (j < ot) {
                        const uint32_t oc0 = W[F_C0][o];
                        const uint32_t pi = j < oc0 ? W[F_F0][o] + j : W[F_F1][o] + (j - oc0);
                        const float4 pt = __ldg(&pts[pi]);
                        hit = exact_key(__uint_as_float(W[F_QX][o]), __uint_as_float(W[F_QY][o]),
                                        __uint_as_float(W[F_QZ][o]), pt.x, pt.y, pt.z) <= r2;
                        id = __float_as_uint(pt.w);
                    } else if (FILL) {
                        const uint32_t j2 = j - ot, on0 = W[F_N0][o];
                        const uint32_t pi = j2 < on0 ? W[F_G0][o] + j2 : W[F_G1][o] + (j2 - on0);
                        id = __float_as_uint(__ldg(&pts[pi].w));
                        hit = true;
                    }
                }
                const uint32_t hm = __ballot_sync(0xffffffffu, hit);
                // this owner's lanes in the batch: [rs, re]
                const int rs = oexcl > base ? (int)(oexcl - base) : 0;
                const uint32_t rend = oexcl + oitems - base;
                const int re = (int)(rend < 32u ? rend : 32u) - 1;
                const uint32_t below_rs = (1u << rs) - 1u;
                const uint32_t upto_re = re >= 31 ? 0xffffffffu : ((1u << (re + 1)) - 1u);
                const uint32_t run_hits = __popc(hm & upto_re & ~below_rs);
                if (SEG) {
                    const uint32_t done = W[F_DONE][o];
                    if (hit) {
                        const uint32_t dst = done + __popc(hm & lt & ~below_rs);
                        if (dst < W[F_WLEN][o]) {
                            const uint64_t wb = ((uint64_t)W[F_WBHI][o] << 32) | W[F_WBLO][o];
                            p.pairs[wb + dst] = make_uint2(W[F_QI][o], id);
                        } else {
                            seg_bad = true;
                        }
                    }
                    __syncwarp();
                    if (valid && lane == re) W[F_DONE][o] = done + run_hits;
                } else if (PUSH) {
                    if (hm) {
                        if (hit) buf[fill + __popc(hm & lt)] = make_uint2(W[F_QI][o], id);
                        fill += __popc(hm);
                        if (fill > WBUF - 32) flush();
                    }
                    if (MODE == MODE_CPUSH && valid && lane == re) W[F_DONE][o] += run_hits;
                } else {
                    if (valid && lane == re) W[F_DONE][o] += run_hits;
                }
                __syncwarp();
            }
        }
        __syncwarp();
        if (COUNTS && have) p.counts[qi] = cnt + W[F_DONE][lane];
        // a segment left short or overrun: the queries changed since the count
        if (SEG && (seg_bad || (have && W[F_DONE][lane] != W[F_WLEN][lane])))
            atomicOr(p.err, DEVERR_MISMATCH);
    }
    flush();
}

// Order-free 64-bit fingerprint of a query array (wrapping sum of mixed
// per-query words, splitmix64 finalizer), added into *out.
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

__global__ void __launch_bounds__(256) query_fingerprint_kernel(const float *__restrict__ q,
                                                                uint64_t nq,
                                                                unsigned long long *out) {
    uint64_t acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x; i < nq;
         i += (uint64_t)gridDim.x * 256) {
        const uint64_t xy = (uint64_t)__float_as_uint(q[3 * i]) |
                            ((uint64_t)__float_as_uint(q[3 * i + 1]) << 32);
        const uint64_t z = __float_as_uint(q[3 * i + 2]);
        acc += mix64(xy ^ mix64(z + (i + 1) * 0x9e3779b97f4a7c15ull));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)acc);
}

// The count's records into their queries' segments: eight lanes per record,
// its slots reserved with one atomic, each lane writing every 8th pair (the
// id read from the sorted point).  Skipped like range_scatter_kernel.
__global__ void __launch_bounds__(256) range_expand_kernel(const uint4 *__restrict__ recs,
                                                           uint64_t n_recs,
                                                           const uint64_t *__restrict__ offsets,
                                                           uint32_t *__restrict__ qcur,
                                                           const float4 *__restrict__ pts,
                                                           uint2 *__restrict__ out,
                                                           const IndexHeader *h) {
    if (h->qfp[0] != h->qfp[1]) return;
    const int lane = threadIdx.x & 31, sub = lane & 7;
    // warp-uniform loop: four records per warp and trip
    for (uint64_t wb = (((uint64_t)blockIdx.x * 256 + threadIdx.x) >> 5) * 4; wb < n_recs;
         wb += (((uint64_t)gridDim.x * 256) >> 5) * 4) {
        const uint64_t w = wb + (lane >> 3);
        const bool ok = w < n_recs;
        const uint4 rc = ok ? recs[w] : make_uint4(0u, 0u, 0u, 0u);
        uint32_t base = 0;
        if (ok && sub == 0) base = atomicAdd(&qcur[rc.x], rc.z);
        base = __shfl_sync(0xffffffffu, base, lane & 24);
        if (ok) {
            const uint64_t dst = offsets[rc.x] + base;
            for (uint32_t j = sub; j < rc.z; j += 8)
                out[dst + j] = make_uint2(rc.x, __float_as_uint(__ldg(&pts[rc.y + j].w)));
        }
    }
}

// The count's pairs into their queries' segments (order within a segment
// unspecified), unless the queries changed since the count (fingerprints
// differ), in which case the segment fill that follows runs instead.  A
// query's pairs were pushed together, so the lanes of a warp mostly share
// queries: one atomic per query and warp reserves their slots.
__global__ void __launch_bounds__(256) range_scatter_kernel(const uint2 *__restrict__ spec,
                                                            uint64_t n_pairs,
                                                            const uint64_t *__restrict__ offsets,
                                                            uint32_t *__restrict__ qcur,
                                                            uint2 *__restrict__ out,
                                                            const IndexHeader *h) {
    if (h->qfp[0] != h->qfp[1]) return;
    const int lane = threadIdx.x & 31;
    uint32_t lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    for (uint64_t w = (uint64_t)blockIdx.x * 256 + (threadIdx.x & ~31u); w < n_pairs;
         w += (uint64_t)gridDim.x * 256) {
        const uint64_t t = w + lane;
        const bool ok = t < n_pairs;
        const uint2 pr = ok ? spec[t] : make_uint2(0xFFFFFFFFu, 0u);
        const uint32_t peers = __match_any_sync(0xffffffffu, pr.x);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (ok && lane == leader) base = atomicAdd(&qcur[pr.x], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (ok) out[offsets[pr.x] + base + __popc(peers & lt)] = pr;
    }
}

__global__ void pairs_from_keys_kernel(const uint64_t *__restrict__ keys, uint64_t n,
                                       uint2 *__restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
        out[i] = make_uint2((uint32_t)(k >> 32), (uint32_t)k);
    }
}

__global__ void keys_from_pairs_kernel(const uint2 *__restrict__ pairs, uint64_t n,
                                       uint64_t *__restrict__ keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint2 p = pairs[i];
        keys[i] = ((uint64_t)p.x << 32) | p.y;
    }
}

rtd_status range_args(rtd_index *idx, const float *d_q, uint64_t nq, float r,
                      const rtd_schedule *sched, RangeArgs &a, cudaStream_t st) {
    if (!idx || !idx->hdr.ptr) return fail(RTD_ERR_INVALID_ARGUMENT, "index not built");
    if (nq && !d_q) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL queries");
    if (!(r >= 0.0f)) return fail(RTD_ERR_INVALID_ARGUMENT, "radius must be >= 0");
    if (idx->leaf_size > 64) return fail(RTD_ERR_UNSUPPORTED, "leaf_size > 64");
    rtd_schedule def;
    rtd_schedule_default(&def);
    const rtd_schedule &s = sched ? *sched : def;
    const uint32_t *perm = nullptr;
    for (int e = EV_SEARCH0; e <= EV_SEARCH1; ++e) idx->ev_set[e] = false;
    idx->mark(EV_SEARCH0, st);
    idx->mark(EV_SEEDED, st);
    RTD_TRY(order_queries(idx, d_q, nq, s.use_morton_lbv != 0, &perm, st));
    idx->mark(EV_ORDERED, st);
    a.ix = view_of(idx);
    a.q = d_q;
    a.nq = nq;
    a.perm = perm;
    a.r2 = r * r;
    a.counts = nullptr;
    a.pairs = nullptr;
    a.capacity = 0;
    a.cursor = nullptr;
    a.offsets = nullptr;
    a.total = 0;
    a.skip_if_same = 0;
    a.recs = nullptr;
    a.rec_cap = 0;
    a.err = &idx->hdr.as<IndexHeader>()->err;
    return RTD_OK;
}

// Largest buffer kept for the count's own pairs (2^28 pairs, 2 GiB).
constexpr uint64_t RSPEC_MAX = 1ull << 28;

rtd_status query_fingerprint(const float *d_q, uint64_t nq, unsigned long long *out,
                             cudaStream_t st) {
    RTD_CUDA(cudaMemsetAsync(out, 0, sizeof(unsigned long long), st));
    query_fingerprint_kernel<<<grid_for(nq, 256, 148 * 4), 256, 0, st>>>(d_q, nq, out);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

template <int MODE>
rtd_status launch_range(RangeArgs &a, cudaStream_t st) {
    range_kernel<MODE><<<grid_for(a.nq, RBLOCK, 1 << 20), RBLOCK, 0, st>>>(a);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

}  // namespace

rtd_status check_index_errors(rtd_index *idx, cudaStream_t st);

rtd_status range_count(rtd_index *idx, const float *d_q, uint64_t nq, float r,
                       const rtd_schedule *s, uint32_t *d_counts, uint64_t *h_total,
                       cudaStream_t st) {
    if (!d_counts && nq) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL counts");
    RangeArgs a;
    RTD_TRY(range_args(idx, d_q, nq, r, s, a, st));
    a.counts = d_counts;
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    // With a buffer left by an earlier count, this count also pushes its
    // pairs there (and fingerprints the queries), so that a fill of the same
    // queries only scatters them into their segments.
    const bool spec = nq > 0 && idx->rspec_cap > 0;
    if (nq) {
        if (spec) {
            RTD_TRY(idx->rcursor.reserve(3 * sizeof(unsigned long long)));
            RTD_CUDA(cudaMemsetAsync(idx->rcursor.ptr, 0, 3 * sizeof(unsigned long long), st));
            a.pairs = idx->rspec.as<uint2>();
            a.capacity = idx->rspec_cap;
            a.cursor = idx->rcursor.as<unsigned long long>();
            a.recs = idx->rrec.as<uint4>();
            a.rec_cap = idx->rrec_cap;
            RTD_TRY(query_fingerprint(d_q, nq, &h->qfp[0], st));
            RTD_TRY(launch_range<MODE_CPUSH>(a, st));
        } else {
            RTD_TRY(launch_range<MODE_COUNT>(a, st));
        }
        idx->mark(EV_SEARCH1, st);
        RTD_TRY(idx->roffsets.reserve(nq * sizeof(uint64_t)));
        RTD_TRY(exclusive_scan_u32(d_counts, idx->roffsets.as<uint64_t>(), nq, &h->total,
                                   idx->scan, &h->err, st));
    } else {
        RTD_CUDA(cudaMemsetAsync(&h->total, 0, sizeof(uint64_t), st));
    }
    uint64_t total = 0;
    unsigned long long cur[3] = {0, 0, 0};   // pairs pushed, records, points the records cover
    RTD_CUDA(cudaMemcpyAsync(&total, &h->total, sizeof(total), cudaMemcpyDeviceToHost, st));
    if (spec)
        RTD_CUDA(cudaMemcpyAsync(cur, idx->rcursor.ptr, sizeof(cur), cudaMemcpyDeviceToHost, st));
    RTD_TRY(check_index_errors(idx, st));   // synchronises
    if (h_total) *h_total = total;
    const bool spec_ok = spec && cur[0] + cur[2] == total && cur[0] <= idx->rspec_cap &&
                         cur[1] <= idx->rrec_cap;
    if (!spec_ok && total > 0 && total < RSPEC_MAX) {
        // room for the next count's pairs and records (grown only; a
        // record covers at least one pair)
        uint64_t want = total + total / 8 + 4096;
        if (want > RSPEC_MAX) want = RSPEC_MAX;
        if (want > idx->rspec_cap) {
            RTD_TRY(idx->rspec.reserve(want * sizeof(uint2)));
            idx->rspec_cap = want;
        }
        const uint64_t want_r = (spec ? cur[1] + cur[1] / 8 : want / 4) + 4096;
        if (want_r > idx->rrec_cap) {
            RTD_TRY(idx->rrec.reserve(want_r * sizeof(uint4)));
            idx->rrec_cap = want_r;
        }
    }
    // a fill of the same queries can write straight into per-query segments
    idx->rtoken.valid = true;
    idx->rtoken.q = d_q;
    idx->rtoken.nq = nq;
    idx->rtoken.radius = r;
    idx->rtoken.total = total;
    idx->rtoken.perm = a.perm;
    idx->rtoken.spec = spec_ok;
    idx->rtoken.spec_pairs = spec_ok ? cur[0] : 0;
    idx->rtoken.spec_recs = spec_ok ? cur[1] : 0;
    return RTD_OK;
}

rtd_status range_fill(rtd_index *idx, const float *d_q, uint64_t nq, float r,
                      const rtd_schedule *s, uint32_t *d_pairs, uint64_t capacity, int sort_pairs,
                      uint64_t *h_written, cudaStream_t st) {
    if (capacity && !d_pairs) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL pairs");
    // Segment mode: the last count pass on this index was over these queries
    // at this radius, its offsets and query order are still on the index,
    // and the buffer holds every pair.
    const auto &tk = idx->rtoken;
    const bool seg = tk.valid && tk.q == d_q && tk.nq == nq && tk.radius == r && nq > 0 &&
                     capacity >= tk.total;
    RangeArgs a;
    if (seg) {
        if (!idx->hdr.ptr) return fail(RTD_ERR_INVALID_ARGUMENT, "index not built");
        for (int e = EV_SEARCH0; e <= EV_SEARCH1; ++e) idx->ev_set[e] = false;
        idx->mark(EV_SEARCH0, st);
        idx->mark(EV_SEEDED, st);
        idx->mark(EV_ORDERED, st);
        a.ix = view_of(idx);
        a.q = d_q;
        a.nq = nq;
        a.perm = tk.perm;
        a.r2 = r * r;
        a.counts = nullptr;
        a.cursor = nullptr;
        a.offsets = idx->roffsets.as<uint64_t>();
        a.total = tk.total;
        a.skip_if_same = 0;
        a.err = &idx->hdr.as<IndexHeader>()->err;
    } else {
        RTD_TRY(range_args(idx, d_q, nq, r, s, a, st));
        RTD_TRY(idx->rcursor.reserve(sizeof(unsigned long long)));
        RTD_CUDA(cudaMemsetAsync(idx->rcursor.ptr, 0, sizeof(unsigned long long), st));
        a.cursor = idx->rcursor.as<unsigned long long>();
    }
    a.pairs = reinterpret_cast<uint2 *>(d_pairs);
    a.capacity = capacity;
    if (seg && tk.spec) {
        // the count's own pairs, scattered into the segments; the segment
        // fill runs only if the queries changed since the count
        IndexHeader *h = idx->hdr.as<IndexHeader>();
        RTD_TRY(query_fingerprint(d_q, nq, &h->qfp[1], st));
        RTD_TRY(idx->rqcur.reserve(nq * sizeof(uint32_t)));
        RTD_CUDA(cudaMemsetAsync(idx->rqcur.ptr, 0, nq * sizeof(uint32_t), st));
        if (tk.spec_pairs) {
            range_scatter_kernel<<<grid_for(tk.spec_pairs, 256, 148 * 16), 256, 0, st>>>(
                idx->rspec.as<uint2>(), tk.spec_pairs, a.offsets, idx->rqcur.as<uint32_t>(), a.pairs, h);
            RTD_LAUNCH_CHECK();
        }
        if (tk.spec_recs) {
            range_expand_kernel<<<grid_for((tk.spec_recs + 3) / 4 * 32, 256, 148 * 16), 256, 0, st>>>(
                idx->rrec.as<uint4>(), tk.spec_recs, a.offsets, idx->rqcur.as<uint32_t>(),
                a.ix.pts, a.pairs, h);
            RTD_LAUNCH_CHECK();
        }
        a.skip_if_same = 1;
        RTD_TRY(launch_range<MODE_SEG>(a, st));
        idx->mark(EV_SEARCH1, st);
    } else if (seg) {
        RTD_TRY(launch_range<MODE_SEG>(a, st));
        idx->mark(EV_SEARCH1, st);
    } else if (nq) {
        RTD_TRY(launch_range<MODE_PUSH>(a, st));
        idx->mark(EV_SEARCH1, st);
    }
    unsigned long long total = 0;
    if (seg) {
        total = tk.total;
    } else {
        RTD_CUDA(cudaMemcpyAsync(&total, idx->rcursor.ptr, sizeof(total), cudaMemcpyDeviceToHost, st));
        RTD_CUDA(cudaStreamSynchronize(st));
    }
    if (h_written) *h_written = total;
    if (total > capacity) {
        IndexHeader *h = idx->hdr.as<IndexHeader>();
        RTD_CUDA(cudaMemsetAsync(&h->err, 0, sizeof(uint32_t), st));
        return fail(RTD_ERR_OVERFLOW, "pair buffer smaller than the pair count");
    }
    if (sort_pairs && total > 1) {
        if (total >= (1ull << 30)) return fail(RTD_ERR_UNSUPPORTED, "sorting >= 2^30 pairs");
        RTD_TRY(idx->rkeys.reserve(total * 8));
        RTD_TRY(idx->rkeys_alt.reserve(total * 8));
        RTD_TRY(idx->rpairs_alt.reserve(total * 8));   // dummy values, ping-pong halves
        uint32_t *v0 = idx->rpairs_alt.as<uint32_t>();
        uint32_t *v1 = v0 + total;
        const int g = grid_for(total, 256, 148 * 8);
        keys_from_pairs_kernel<<<g, 256, 0, st>>>(a.pairs, total, idx->rkeys.as<uint64_t>());
        RTD_LAUNCH_CHECK();
        int qbits = 1;
        while (qbits < 32 && (1ull << qbits) < nq) ++qbits;
        bool in_alt = false;
        IndexHeader *h = idx->hdr.as<IndexHeader>();
        RTD_TRY(radix_sort_pairs<uint64_t>(idx->rkeys.as<uint64_t>(), idx->rkeys_alt.as<uint64_t>(),
                                           v0, v1, true, total, 0, 32 + qbits, idx->sort, &h->err,
                                           st, &in_alt));
        const uint64_t *sk = in_alt ? idx->rkeys_alt.as<uint64_t>() : idx->rkeys.as<uint64_t>();
        pairs_from_keys_kernel<<<g, 256, 0, st>>>(sk, total, a.pairs);
        RTD_LAUNCH_CHECK();
    }
    return check_index_errors(idx, st);
}

// ------------------------------------------------------- kNN backward
namespace {
__global__ void knn_backward_kernel(const float *__restrict__ q, uint64_t nq,
                                    const float *__restrict__ pts, uint64_t n, uint32_t k,
                                    const uint32_t *__restrict__ ids, const float *__restrict__ g,
                                    float *__restrict__ gq, float *__restrict__ gp) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq;
         i += (uint64_t)gridDim.x * blockDim.x) {
        float qx = q[3 * i], qy = q[3 * i + 1], qz = q[3 * i + 2];
        float ax = 0.f, ay = 0.f, az = 0.f;
        for (uint32_t j = 0; j < k; ++j) {
            uint32_t id = ids[i * k + j];
            if (id == EMPTY_ID || id >= n) continue;
            float w = 2.0f * g[i * k + j];
            float dx = qx - pts[3 * (uint64_t)id], dy = qy - pts[3 * (uint64_t)id + 1],
                  dz = qz - pts[3 * (uint64_t)id + 2];
            ax += w * dx; ay += w * dy; az += w * dz;
            if (gp) {
                atomicAdd(&gp[3 * (uint64_t)id], -w * dx);
                atomicAdd(&gp[3 * (uint64_t)id + 1], -w * dy);
                atomicAdd(&gp[3 * (uint64_t)id + 2], -w * dz);
            }
        }
        if (gq) { gq[3 * i] = ax; gq[3 * i + 1] = ay; gq[3 * i + 2] = az; }
    }
}
}  // namespace

rtd_status knn_backward(const float *q, uint64_t nq, const float *pts, uint64_t n, uint32_t k,
                        const uint32_t *ids, const float *g, float *gq, float *gp, cudaStream_t st) {
    if (nq == 0 || k == 0) return RTD_OK;
    if (!q || !pts || !ids || !g) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL input");
    knn_backward_kernel<<<grid_for(nq, 256, 148 * 16), 256, 0, st>>>(q, nq, pts, n, k, ids, g, gq, gp);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

}  // namespace rtd
