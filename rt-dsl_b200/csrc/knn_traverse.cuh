// knn_traverse.cuh -- one query's exact k-NN by in-kernel radius expansion,
// shared by the single-cloud kernels (knn.cu) and the batched many-cloud
// kernel (batch.cu).
//
// Round i accepts points with prev < key <= bound_i (bound_{i+1} = bound_i *
// M^2, prev = bound_{i-1}); a query stops once it holds k points (they are
// then its exact k nearest) and the last allowed round is unbounded, so the
// result is exact for every input.  Nodes whose box lies inside the
// previous radius are skipped (their points were all collected), nodes
// whose nearest box key exceeds min(bound, current k-th key) are pruned,
// and children are visited near-first.  Keys are the exact FP32 keys of
// the reference intersection program; ties go to the lower point id.
#pragma once

#include "index.cuh"

namespace rtd {

constexpr int SHORT_STACK = 12;   // per-thread stack entries kept in shared memory
constexpr int STACK_MAX = 104;    // >= maximal tree depth (63 key bits + 32 index bits)

// One tree to search: a whole index, or one cloud's subtree of a forest.
struct TreeRef {
    const float4 *pts;
    const BvhNode *nodes;
    const BvhNode *s_top;    // staged top levels (nullptr: no CHILD_TOP words)
    uint32_t root;           // child word of the root
    uint32_t root_count;     // points when the root is a leaf
    uint32_t visit_cap;      // more node visits than this per round = broken tree
};

struct RoundSpec {
    float r0sq;              // squared radius of round 0
    float mult2;             // growth of the squared radius per round
    uint32_t max_rounds;     // the last round is unbounded, unless partial
    uint32_t partial;        // the reference's round cap: every round bounded; a query
                             // short of k hits after max_rounds keeps its partial list
                             // and raises DEVERR_NOT_CONVERGED
};

__device__ __forceinline__ void load_node(const BvhNode *__restrict__ s_top,
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

// Sorted (key, id) list of KC slots in registers; slot KC-1 is the k-th best.
// For k < KC the first KC-k slots hold -inf and never move.
template <int KC>
__device__ __forceinline__ void list_insert(float (&bk)[KC], uint32_t (&bi)[KC], float key,
                                            uint32_t id) {
#pragma unroll
    for (int j = KC - 1; j > 0; --j) {
        bool bp = key_less(key, id, bk[j - 1], bi[j - 1]);
        bool bc = key_less(key, id, bk[j], bi[j]);
        float nk = bp ? bk[j - 1] : (bc ? key : bk[j]);
        uint32_t ni = bp ? bi[j - 1] : (bc ? id : bi[j]);
        bk[j] = nk;
        bi[j] = ni;
    }
    if (key_less(key, id, bk[0], bi[0])) { bk[0] = key; bi[0] = id; }
}

// Empty register list for k <= KC: slots before KC-k hold -inf and never
// move; slot KC-1 is the k-th best.
template <int KC>
__device__ __forceinline__ void list_init(float (&bk)[KC], uint32_t (&bi)[KC], int kk) {
#pragma unroll
    for (int j = 0; j < KC; ++j) {
        bool pad = j < KC - kk;
        bk[j] = pad ? -INFINITY : INFINITY;
        bi[j] = pad ? 0u : EMPTY_ID;
    }
}

// Thread per query: the register list ends holding the k best (key, id)
// pairs in slots KC-k .. KC-1.  The stack keeps SHORT_STACK entries in this
// thread's shared-memory column (s_col[sp * s_stride]) and the rest in
// l_stack (local memory).  SEEDED: the caller has already put the points
// with sorted indices [skip_lo, skip_hi) through the list, so leaves skip
// them; otherwise the list starts empty.
template <int KC, bool SEEDED = false>
__device__ __forceinline__ void knn_query_thread(const TreeRef &t, const RoundSpec &rs, float qx,
                                                 float qy, float qz, int kk, uint2 *s_col,
                                                 int s_stride, uint2 *l_stack, uint32_t *err,
                                                 float (&bk)[KC], uint32_t (&bi)[KC],
                                                 uint32_t skip_lo = 0, uint32_t skip_hi = 0) {
    if (!SEEDED) list_init<KC>(bk, bi, kk);
    const bool valid = t.root != CHILD_NONE && !isnan(qx) && !isnan(qy) && !isnan(qz);
    float bound = rs.r0sq > 0.0f ? rs.r0sq : 1e-30f, prev = -1.0f;
    for (uint32_t round = 0; valid; ++round) {
        const bool last = round + 1 >= rs.max_rounds || !(bound < INFINITY);
        if (last && !rs.partial) bound = INFINITY;
        float lim = fminf(bound, bk[KC - 1]);
        uint32_t node = t.root;
        int sp = 0;
        uint32_t visits = 0;
        while (true) {
            // up to two leaf ranges to test, [fa, fa + ca) then [fb, fb + cb)
            // (named scalars: an array indexed by a leaf count would live in
            // local memory)
            uint32_t fa = 0, ca = 0, fb = 0, cb = 0;
            uint32_t next = CHILD_NONE;
            if (++visits > t.visit_cap) {
                atomicOr(err, DEVERR_STACK);
                break;
            }
            float k0 = 0.f, k1 = 0.f;
            bool v0 = false, v1 = false;
            uint4 d = make_uint4(0, 0, 0, 0);
            if (node & CHILD_LEAF) {
                fa = node & CHILD_INDEX;
                ca = t.root_count;
            } else {
                float4 a, b, c;
                load_node(t.s_top, t.nodes, node, a, b, c, d);
                k0 = box_min_key(qx, qy, qz, a.x, a.y, a.z, a.w, b.x, b.y);
                k1 = box_min_key(qx, qy, qz, b.z, b.w, c.x, c.y, c.z, c.w);
                v0 = !(k0 > lim);
                v1 = !(k1 > lim);
                if (prev >= 0.0f) {
                    if (v0) v0 = !(box_max_key(qx, qy, qz, a.x, a.y, a.z, a.w, b.x, b.y) <= prev);
                    if (v1) v1 = !(box_max_key(qx, qy, qz, b.z, b.w, c.x, c.y, c.z, c.w) <= prev);
                }
                if (v0 && (d.x & CHILD_LEAF)) { fa = d.x & CHILD_INDEX; ca = d.z; v0 = false; }
                if (v1 && (d.y & CHILD_LEAF)) { fb = d.y & CHILD_INDEX; cb = d.w; v1 = false; }
            }
            const uint32_t tot = ca + cb;
            for (uint32_t j = 0; j < tot; ++j) {
                const uint32_t pi = j < ca ? fa + j : fb + (j - ca);
                if (SEEDED && pi - skip_lo < skip_hi - skip_lo) continue;
                float4 pt = __ldg(&t.pts[pi]);
                float key = exact_key(qx, qy, qz, pt.x, pt.y, pt.z);
                uint32_t id = __float_as_uint(pt.w);
                if (key <= bound && key > prev && key_less(key, id, bk[KC - 1], bi[KC - 1]))
                    list_insert<KC>(bk, bi, key, id);
            }
            if (tot) lim = fminf(bound, bk[KC - 1]);
            if (!(node & CHILD_LEAF)) {
                v0 = v0 && !(k0 > lim);
                v1 = v1 && !(k1 > lim);
                if (v0 && v1) {
                    bool near0 = k0 <= k1;
                    uint2 far = near0 ? make_uint2(d.y, __float_as_uint(k1))
                                      : make_uint2(d.x, __float_as_uint(k0));
                    next = near0 ? d.x : d.y;
                    if (sp < SHORT_STACK) s_col[sp * s_stride] = far;
                    else if (sp < STACK_MAX) l_stack[sp - SHORT_STACK] = far;
                    else atomicOr(err, DEVERR_STACK);
                    if (sp < STACK_MAX) ++sp;
                } else if (v0) {
                    next = d.x;
                } else if (v1) {
                    next = d.y;
                }
            }
            if (next == CHILD_NONE) {
                while (sp > 0) {
                    --sp;
                    uint2 e = sp < SHORT_STACK ? s_col[sp * s_stride] : l_stack[sp - SHORT_STACK];
                    if (!(__uint_as_float(e.y) > lim)) { next = e.x; break; }
                }
                if (next == CHILD_NONE) break;
            }
            node = next;
        }
        if (bi[KC - 1] != EMPTY_ID) break;
        if (last) {
            if (rs.partial) atomicOr(err, DEVERR_NOT_CONVERGED);
            break;
        }
        prev = bound;
        bound = __fmul_rn(bound, rs.mult2);
    }
}

// Merges the candidates of one batch (lane i holds (key, id) when acc) into
// a sorted list of kk <= S*32 slots striped over the warp (slot j in lane
// j % 32, register j / 32; slots >= kk stay empty).  For every accepted
// candidate, broadcast in turn, a ballot per register counts the list
// entries before it and each lane counts how many candidates precede its
// own entries and its own candidate; every item then lands at its merged
// position through the warp's shared scratch ls (S*32 entries), and items
// past kk drop out.  (key, id) pairs are distinct, so the order is strict.
template <int S>
__device__ __forceinline__ void warp_list_merge(float (&lk)[S], uint32_t (&li)[S], uint32_t kk,
                                                bool acc, float key, uint32_t id, uint2 *ls,
                                                float &wk, uint32_t &wi) {
    const int lane = threadIdx.x & 31;
    uint32_t m = __ballot_sync(0xffffffffu, acc);
    if (!m) return;
    int before[S];                 // candidates ordered before each of my entries
#pragma unroll
    for (int s = 0; s < S; ++s) before[s] = 0;
    int r_list = 0, r_cand = 0;    // for my candidate: entries / candidates before it
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        const float ck = __shfl_sync(0xffffffffu, key, src);
        const uint32_t ci = __shfl_sync(0xffffffffu, id, src);
        int n_before = 0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const bool in_list = (uint32_t)(s * 32 + lane) < kk;
            const bool e_lt = in_list && key_less(lk[s], li[s], ck, ci);
            n_before += __popc(__ballot_sync(0xffffffffu, e_lt));
            before[s] += (in_list && !e_lt) ? 1 : 0;
        }
        if (lane == src) r_list = n_before;
        if (acc && key_less(ck, ci, key, id)) ++r_cand;
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const uint32_t j = (uint32_t)(s * 32 + lane);
        const uint32_t pos = j + (uint32_t)before[s];
        if (j < kk && pos < kk) ls[pos] = make_uint2(__float_as_uint(lk[s]), li[s]);
    }
    if (acc) {
        const uint32_t pos = (uint32_t)(r_list + r_cand);
        if (pos < kk) ls[pos] = make_uint2(__float_as_uint(key), id);
    }
    __syncwarp();
    const int wslot = (int)((kk - 1) >> 5), wlane = (int)((kk - 1) & 31);
    float nk = 0.f;
    uint32_t ni = 0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const uint32_t j = (uint32_t)(s * 32 + lane);
        if (j < kk) {
            const uint2 e = ls[j];
            lk[s] = __uint_as_float(e.x);
            li[s] = e.y;
        }
        if (s == wslot) { nk = lk[s]; ni = li[s]; }
    }
    __syncwarp();
    wk = __shfl_sync(0xffffffffu, nk, wlane);
    wi = __shfl_sync(0xffffffffu, ni, wlane);
}

// The warp-striped register list of S*32 slots (k <= S*32) as a list type
// of knn_query_warp_list: slot j in lane j % 32, register j / 32; ls is the
// warp's shared merge scratch (S*32 entries).  wk / wi: the k-th entry.
template <int S>
struct RegList {
    float lk[S];
    uint32_t li[S];
    uint2 *ls;
    uint32_t kk;
    float wk;
    uint32_t wi;
    __device__ __forceinline__ void reset() {
#pragma unroll
        for (int s = 0; s < S; ++s) { lk[s] = INFINITY; li[s] = EMPTY_ID; }
        wk = INFINITY;
        wi = EMPTY_ID;
    }
    __device__ __forceinline__ void merge(bool acc, float key, uint32_t id) {
        warp_list_merge<S>(lk, li, kk, acc, key, id, ls, wk, wi);
    }
};

// A sorted list of kk (key, id) entries in memory, owned by one warp, for k
// above what registers hold: L[0 .. cnt) ascending, in shared memory or in
// a global-memory slab of the warp's own.  s_r is 32 words of the warp's
// shared scratch.  A merge of up to 32 candidates (one per lane) works in
// place, top down:
//   - each candidate c finds r_c = #entries before it (binary search) and
//     its rank j_c among the candidates; it lands at r_c + j_c;
//   - entry t moves up by s(t) = #candidates with r_c <= t, the candidates'
//     ranks sorted in s_r and counted by binary search;
//   - entries move in chunks of 32 from the top, each chunk read before it
//     is written; a destination is never below its source, so no chunk
//     overwrites an entry that a later (lower) chunk still has to read;
//   - destinations at or past kk drop out.
// (key, id) pairs are distinct, so every position is unique.
struct WideList {
    uint2 *L;
    uint32_t *s_r;
    uint32_t kk;
    uint32_t cnt;
    float wk;
    uint32_t wi;
    __device__ __forceinline__ void reset() {
        cnt = 0;
        wk = INFINITY;
        wi = EMPTY_ID;
    }
    __device__ __forceinline__ void merge(bool acc, float key, uint32_t id) {
        const int lane = threadIdx.x & 31;
        const uint32_t m = __ballot_sync(0xffffffffu, acc);
        if (!m) return;
        const uint32_t nc = __popc(m);
        // rank among the candidates
        uint32_t jc = 0;
        for (uint32_t mm = m; mm;) {
            const int src = __ffs(mm) - 1;
            mm &= mm - 1;
            const float ck = __shfl_sync(0xffffffffu, key, src);
            const uint32_t ci = __shfl_sync(0xffffffffu, id, src);
            if (acc && key_less(ck, ci, key, id)) ++jc;
        }
        // entries before the candidate (lower bound over L[0 .. cnt))
        uint32_t rc = 0;
        if (acc) {
            uint32_t lo = 0, hi = cnt;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                const uint2 e = L[mid];
                if (key_less(__uint_as_float(e.x), e.y, key, id)) lo = mid + 1;
                else hi = mid;
            }
            rc = lo;
            s_r[jc] = rc;   // ranks in candidate order are non-decreasing
        }
        uint32_t rmin = acc ? rc : 0xFFFFFFFFu;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
        __syncwarp();
        // move entries [rmin, cnt) up, top chunk first
        const uint32_t top = cnt < kk ? cnt : kk;
        for (int64_t hi = (int64_t)top - 1; hi >= (int64_t)rmin; hi -= 32) {
            const int64_t t = hi - lane;
            uint2 v = make_uint2(0, 0);
            uint32_t dst = 0xFFFFFFFFu;
            if (t >= (int64_t)rmin) {
                v = L[t];
                // s(t) = #candidates with r_c <= t (s_r ascending)
                uint32_t lo = 0, hi2 = nc;
                while (lo < hi2) {
                    const uint32_t mid = (lo + hi2) >> 1;
                    if (s_r[mid] <= (uint32_t)t) lo = mid + 1;
                    else hi2 = mid;
                }
                dst = (uint32_t)t + lo;
            }
            __syncwarp();
            if (dst < kk) L[dst] = v;
            __syncwarp();
        }
        if (acc && rc + jc < kk) L[rc + jc] = make_uint2(__float_as_uint(key), id);
        cnt = cnt + nc < kk ? cnt + nc : kk;
        __syncwarp();
        if (cnt == kk) {
            const uint2 e = L[kk - 1];
            wk = __uint_as_float(e.x);
            wi = e.y;
        }
    }
};

// Warp per query over any list type (RegList, WideList): the candidates of
// a node's leaf children are tested one per lane and the accepted ones
// merged into the list in one batch.  stk is the warp's shared-memory stack
// (STACK_MAX entries).  All arguments must be warp-uniform.
template <class List>
__device__ __forceinline__ void knn_query_warp_list(const TreeRef &t, const RoundSpec &rs,
                                                    float qx, float qy, float qz, uint2 *stk,
                                                    uint32_t *err, List &list) {
    const int lane = threadIdx.x & 31;
    list.reset();
    const bool valid = t.root != CHILD_NONE && !isnan(qx) && !isnan(qy) && !isnan(qz);
    float bound = rs.r0sq > 0.0f ? rs.r0sq : 1e-30f, prev = -1.0f;
    for (uint32_t round = 0; valid; ++round) {
        const bool last = round + 1 >= rs.max_rounds || !(bound < INFINITY);
        if (last && !rs.partial) bound = INFINITY;
        float lim = fminf(bound, list.wk);
        uint32_t node = t.root;
        int sp = 0;
        uint32_t visits = 0;
        while (true) {
            uint32_t fa = 0, ca = 0, fb = 0, cb = 0;   // leaf ranges, as in knn_query_thread
            uint32_t next = CHILD_NONE;
            float k0 = 0.f, k1 = 0.f;
            uint4 d = make_uint4(0, 0, 0, 0);
            bool v0 = false, v1 = false;
            if (++visits > t.visit_cap) {   // warp-uniform
                if (lane == 0) atomicOr(err, DEVERR_STACK);
                break;
            }
            if (node & CHILD_LEAF) {
                fa = node & CHILD_INDEX;
                ca = t.root_count;
            } else {
                float4 a, b, c;
                load_node(t.s_top, t.nodes, node, a, b, c, d);
                k0 = box_min_key(qx, qy, qz, a.x, a.y, a.z, a.w, b.x, b.y);
                k1 = box_min_key(qx, qy, qz, b.z, b.w, c.x, c.y, c.z, c.w);
                v0 = !(k0 > lim);
                v1 = !(k1 > lim);
                if (prev >= 0.0f) {
                    if (v0) v0 = !(box_max_key(qx, qy, qz, a.x, a.y, a.z, a.w, b.x, b.y) <= prev);
                    if (v1) v1 = !(box_max_key(qx, qy, qz, b.z, b.w, c.x, c.y, c.z, c.w) <= prev);
                }
                if (v0 && (d.x & CHILD_LEAF)) { fa = d.x & CHILD_INDEX; ca = d.z; v0 = false; }
                if (v1 && (d.y & CHILD_LEAF)) { fb = d.y & CHILD_INDEX; cb = d.w; v1 = false; }
            }
            const uint32_t tot = ca + cb;
            if (tot) {   // both leaves' points, 32 per batch
                for (uint32_t j0 = 0; j0 < tot; j0 += 32) {
                    const uint32_t j = j0 + lane;
                    float key = INFINITY;
                    uint32_t id = EMPTY_ID;
                    bool acc = false;
                    if (j < tot) {
                        const float4 pt = __ldg(&t.pts[j < ca ? fa + j : fb + (j - ca)]);
                        key = exact_key(qx, qy, qz, pt.x, pt.y, pt.z);
                        id = __float_as_uint(pt.w);
                        acc = key <= bound && key > prev && key_less(key, id, list.wk, list.wi);
                    }
                    list.merge(acc, key, id);
                }
                lim = fminf(bound, list.wk);
            }
            if (!(node & CHILD_LEAF)) {
                v0 = v0 && !(k0 > lim);
                v1 = v1 && !(k1 > lim);
                if (v0 && v1) {
                    bool near0 = k0 <= k1;
                    uint2 far = near0 ? make_uint2(d.y, __float_as_uint(k1))
                                      : make_uint2(d.x, __float_as_uint(k0));
                    next = near0 ? d.x : d.y;
                    if (sp < STACK_MAX) {
                        if (lane == 0) stk[sp] = far;
                        ++sp;
                    } else if (lane == 0) {
                        atomicOr(err, DEVERR_STACK);
                    }
                } else if (v0) {
                    next = d.x;
                } else if (v1) {
                    next = d.y;
                }
            }
            __syncwarp();
            if (next == CHILD_NONE) {
                while (sp > 0) {
                    --sp;
                    uint2 e = stk[sp];
                    if (!(__uint_as_float(e.y) > lim)) { next = e.x; break; }
                }
                if (next == CHILD_NONE) break;
            }
            __syncwarp();
            node = next;
        }
        if (list.wi != EMPTY_ID) break;
        if (last) {
            if (rs.partial && lane == 0) atomicOr(err, DEVERR_NOT_CONVERGED);
            break;
        }
        prev = bound;
        bound = __fmul_rn(bound, rs.mult2);
    }
}

// Warp per query with the warp-striped register list (k <= S*32); ls is
// the warp's list scratch (S*32 entries).
template <int S>
__device__ __forceinline__ void knn_query_warp(const TreeRef &t, const RoundSpec &rs, float qx,
                                               float qy, float qz, uint32_t kk, uint2 *stk,
                                               uint2 *ls, uint32_t *err, float (&lk)[S],
                                               uint32_t (&li)[S]) {
    RegList<S> list;
    list.ls = ls;
    list.kk = kk;
    knn_query_warp_list(t, rs, qx, qy, qz, stk, err, list);
#pragma unroll
    for (int s = 0; s < S; ++s) { lk[s] = list.lk[s]; li[s] = list.li[s]; }
}

// Writes a WideList to the k slots of an ids / d2 row (EMPTY_ID / +inf
// past cnt; k may exceed the list's kk, which is at most the tree's points).
__device__ __forceinline__ void wide_list_store(const WideList &l, uint32_t k, uint32_t *ids,
                                                float *d2) {
    const int lane = threadIdx.x & 31;
    for (uint32_t j = lane; j < k; j += 32) {
        const uint2 e = j < l.cnt ? l.L[j] : make_uint2(__float_as_uint(INFINITY), EMPTY_ID);
        ids[j] = e.y;
        if (d2) d2[j] = __uint_as_float(e.x);
    }
}

}  // namespace rtd
