// lbvh.cu -- LBVH builder: scene box -> Morton codes -> LSD radix sort
// -> Karras radix tree -> leaf collapse with every child box taken from a
// pyramid of run boxes over the sorted points -> top-level staging.
// Replaces the OptiX GAS build/refit of
// gprt-optix/host/main.cpp:200-292 and the sphere-AABB kernel of
// gprt-optix/host/kernels.cu:3-16: the tree holds point boxes only and the
// search radius is applied inside the search kernels.
#include "index.cuh"

namespace rtd {
namespace {

constexpr int BLOCK = 256;

// Whether a device array can be read as float4.
inline int aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0 ? 1 : 0; }

__global__ void hdr_init_kernel(IndexHeader *h) {
    chain_wait();
    h->root = CHILD_NONE;
    h->root_count = 0;
    h->n_internal = 0;
    h->n_top = 0;
    for (int a = 0; a < 3; ++a) {
        h->box[a] = 0xFFFFFFFFu;   // flip(+inf) side: any atomicMin lowers it
        h->box[3 + a] = 0u;
    }
    h->err = 0;
    h->r0sq = 0.0f;
    h->total = 0;
    h->nn95_key = -1.0f;   // "no sample": the seed falls back to radius 1
    h->n_sample = 0;
}

// Points 4g .. 4g+3 of a 16-byte aligned xyz array: three float4 loads.
__device__ __forceinline__ void load_point4(const float *__restrict__ xyz, uint64_t g,
                                            float (&x)[4], float (&y)[4], float (&z)[4]) {
    const float4 *p = reinterpret_cast<const float4 *>(xyz) + 3 * g;
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    x[0] = a.x; y[0] = a.y; z[0] = a.z;
    x[1] = a.w; y[1] = b.x; z[1] = b.y;
    x[2] = b.z; y[2] = b.w; z[2] = c.x;
    x[3] = c.y; y[3] = c.z; z[3] = c.w;
}

// Scene box, NaN-ignoring (fminf/fmaxf), as order-preserving atomics.  With
// vec4 (a 16-byte aligned array) whole groups of 4 points are read as three
// float4 each; the last n % 4 points, or all of them without vec4, one
// coordinate at a time.
__global__ void __launch_bounds__(BLOCK) bbox_kernel(const float *__restrict__ xyz, uint64_t n,
                                                     IndexHeader *h, int vec4) {
    chain_wait();
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const uint64_t t0 = (uint64_t)blockIdx.x * BLOCK + threadIdx.x, stride = (uint64_t)gridDim.x * BLOCK;
    const uint64_t groups = vec4 ? n / 4 : 0;
    for (uint64_t g = t0; g < groups; g += stride) {
        float x[4], y[4], z[4];
        load_point4(xyz, g, x, y, z);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            lo[0] = fminf(lo[0], x[u]); hi[0] = fmaxf(hi[0], x[u]);
            lo[1] = fminf(lo[1], y[u]); hi[1] = fmaxf(hi[1], y[u]);
            lo[2] = fminf(lo[2], z[u]); hi[2] = fmaxf(hi[2], z[u]);
        }
    }
    for (uint64_t i = 4 * groups + t0; i < n; i += stride) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float v = xyz[3 * i + a];
            lo[a] = fminf(lo[a], v);
            hi[a] = fmaxf(hi[a], v);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    __shared__ float s[BLOCK / 32][6];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) { s[warp][a] = lo[a]; s[warp][3 + a] = hi[a]; }
    __syncthreads();
    if (threadIdx.x < 3) {
        int a = threadIdx.x;
        float l = INFINITY, u = -INFINITY;
        for (int w = 0; w < BLOCK / 32; ++w) { l = fminf(l, s[w][a]); u = fmaxf(u, s[w][3 + a]); }
        atomicMin(&h->box[a], float_flip(l));
        atomicMax(&h->box[3 + a], float_flip(u));
    }
}

// 30-bit codes follow compute_morton_codes (gprt-core/src/morton.rs:19-48),
// extent per axis; wider codes (B = bits / 3 per axis, scale = 2^B - 1,
// B <= 21, interleaved in the low 3B bits of a u64) use one cubic extent.
template <typename K>
__device__ __forceinline__ K morton_key(const SceneNorm &s, float scale, float x, float y, float z) {
    if (sizeof(K) == 4)
        return (K)morton30(quantize(x, s.lo[0], s.ext[0], 1023.0f),
                           quantize(y, s.lo[1], s.ext[1], 1023.0f),
                           quantize(z, s.lo[2], s.ext[2], 1023.0f));
    return (K)morton63(quantize(x, s.lo[0], s.ext[0], scale), quantize(y, s.lo[1], s.ext[1], scale),
                       quantize(z, s.lo[2], s.ext[2], scale));
}

// Keys of the points; with vec4 (as bbox_kernel) whole groups of 4 points
// are read as three float4 each.
template <typename K>
__global__ void __launch_bounds__(BLOCK) morton_kernel(const float *__restrict__ xyz, uint64_t n,
                                                       const IndexHeader *h, float scale,
                                                       K *__restrict__ keys, int vec4) {
    chain_wait();
    const SceneNorm s = sizeof(K) == 4 ? scene_norm(h) : scene_norm_cubic(h);
    const uint64_t t0 = (uint64_t)blockIdx.x * BLOCK + threadIdx.x, stride = (uint64_t)gridDim.x * BLOCK;
    const uint64_t groups = vec4 ? n / 4 : 0;
    for (uint64_t g = t0; g < groups; g += stride) {
        float x[4], y[4], z[4];
        load_point4(xyz, g, x, y, z);
#pragma unroll
        for (int u = 0; u < 4; ++u) keys[4 * g + u] = morton_key<K>(s, scale, x[u], y[u], z[u]);
    }
    for (uint64_t i = 4 * groups + t0; i < n; i += stride)
        keys[i] = morton_key<K>(s, scale, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}

// Common-prefix length of sorted keys i and j (ki = keys[i]), ties broken
// by index (Karras 2012, "Maximizing parallelism in the construction of
// BVHs"); -1 when j is outside [0, n).
template <typename K>
__device__ __forceinline__ int delta(const K *__restrict__ keys, int64_t n, K ki, int64_t i,
                                     int64_t j) {
    if (j < 0 || j >= n) return -1;
    const K b = keys[j];
    if (ki == b) return (int)(8 * sizeof(K)) + __clz((uint32_t)(i ^ j));
    return sizeof(K) == 8 ? __clzll((unsigned long long)(ki ^ b)) : __clz((uint32_t)(ki ^ b));
}

// Direction of Karras node i and the lower bound on its common prefix (the
// prefix shared with the neighbour away from the direction).
template <typename K>
__device__ __forceinline__ void karras_dir(const K *__restrict__ keys, int64_t n, K ki, int64_t i,
                                           int &dir, int &dmin) {
    const int dp = delta(keys, n, ki, i, i + 1), dm = delta(keys, n, ki, i, i - 1);
    dir = (dp - dm) >= 0 ? 1 : -1;
    dmin = dir > 0 ? dm : dp;
}

// Karras nodes.  Only nodes with more than leaf_size points are kept (the
// rest collapse into leaves), and a node's point count exceeds leaf_size
// exactly when the key leaf_size steps away in its direction still shares
// more than the node's lower bound on the common prefix: the prefix length
// of the (key, position) pairs, which are strictly increasing, cannot grow
// with distance.  This kernel makes that one test per node; the range and
// split searches run afterwards for the kept nodes alone, packed densely by
// the scan of these flags (node_kernel), so no warp carries idle lanes of
// collapsed nodes through them.
// A block takes FLAG_TILE consecutive nodes and first stages their keys
// with a halo of leaf_size + 1 on each side in shared memory (one
// coalesced read), so that the four keys of each test come from there.
constexpr int FLAG_TILE = 2048;
constexpr int FLAG_HALO = 65;   // leaf_size (<= 64) + 1
template <typename K>
__global__ void __launch_bounds__(BLOCK) karras_flag_kernel(const K *__restrict__ keys, int64_t n,
                                                            uint32_t leaf_size, uint32_t *flags) {
    chain_wait();
    __shared__ K s_k[FLAG_TILE + 2 * FLAG_HALO];
    const int64_t b0 = (int64_t)blockIdx.x * FLAG_TILE, base = b0 - FLAG_HALO;
    for (int t = threadIdx.x; t < FLAG_TILE + 2 * FLAG_HALO; t += BLOCK) {
        const int64_t j = base + t;
        if (j >= 0 && j < n) s_k[t] = keys[j];
    }
    __syncthreads();
    // delta on the staged keys (j within the halo whenever j is in [0, n))
    auto dl = [&](K ki, int64_t i, int64_t j) -> int {
        if (j < 0 || j >= n) return -1;
        const K b = s_k[j - base];
        if (ki == b) return (int)(8 * sizeof(K)) + __clz((uint32_t)(i ^ j));
        return sizeof(K) == 8 ? __clzll((unsigned long long)(ki ^ b)) : __clz((uint32_t)(ki ^ b));
    };
    for (int t = threadIdx.x; t < FLAG_TILE; t += BLOCK) {
        const int64_t i = b0 + t;
        if (i >= n - 1) break;
        const K ki = s_k[i - base];
        const int dir = (dl(ki, i, i + 1) - dl(ki, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = dl(ki, i, i - dir);
        flags[i] = dl(ki, i, i + (int64_t)leaf_size * dir) > dmin ? 1u : 0u;
    }
}

// Point range [first, last] and split of kept Karras node i: the children
// hold [first, split] and [split + 1, last].
template <typename K>
__device__ __forceinline__ void karras_range(const K *__restrict__ keys, int64_t n, int64_t i,
                                             uint32_t leaf_size, uint32_t &first, uint32_t &last,
                                             uint32_t &split) {
    const K ki = keys[i];
    int dir, dmin;
    karras_dir(keys, n, ki, i, dir, dmin);
    int64_t lmax = 2;
    while (lmax <= (int64_t)leaf_size) lmax <<= 1;
    while (delta(keys, n, ki, i, i + lmax * dir) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, ki, i, i + (l + t) * dir) > dmin) l += t;
    const int64_t j = i + l * dir;
    const int dnode = delta(keys, n, ki, i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(keys, n, ki, i, i + (s + t) * dir) > dnode) s += t;
    } while (t > 1);
    split = (uint32_t)(i + s * dir + (dir < 0 ? -1 : 0));
    first = (uint32_t)(i < j ? i : j);
    last = (uint32_t)(i < j ? j : i);
}

// ---------------------------------------------------- box pyramid
// Boxes of aligned runs of the sorted points: level j entry e covers points
// [e * 8^j, (e+1) * 8^j) as (lo.xyz, -) (hi.xyz, -).  A run holding a
// point with a NaN coordinate gets an unbounded box: such a point is never
// a neighbour, but no finite box holds it, so no search may treat a
// subtree containing it as lying wholly inside a ball.  Base 8 keeps the
// walk of a range short: at most 7 entries per end and level.
constexpr int PYR_SH = 3;                  // log2 of the base
constexpr uint32_t PYR_B = 1u << PYR_SH;   // 8 entries of a level per entry of the next
constexpr int PYR_MAX = 10;                // levels 1..10 cover 8^10 = 2^30 points
// Levels 1..nlev lie back to back in pyr (2 float4 per entry), level j
// holding ceil(n / 8^j) entries; nlev is the first level of <= 8 entries.
struct Pyramid {
    const float4 *pts;
    const float4 *pyr;
    uint32_t n;
    int nlev;
};

struct Box {
    float lo[3], hi[3];
};

__device__ __forceinline__ void box_empty(Box &b) {
    for (int a = 0; a < 3; ++a) { b.lo[a] = INFINITY; b.hi[a] = -INFINITY; }
}
__device__ __forceinline__ void box_add_point(Box &b, bool &nan, const float4 p) {
    b.lo[0] = fminf(b.lo[0], p.x); b.hi[0] = fmaxf(b.hi[0], p.x);
    b.lo[1] = fminf(b.lo[1], p.y); b.hi[1] = fmaxf(b.hi[1], p.y);
    b.lo[2] = fminf(b.lo[2], p.z); b.hi[2] = fmaxf(b.hi[2], p.z);
    nan |= isnan(p.x) || isnan(p.y) || isnan(p.z);
}
__device__ __forceinline__ void box_add(Box &b, const float4 lo, const float4 hi) {
    b.lo[0] = fminf(b.lo[0], lo.x); b.hi[0] = fmaxf(b.hi[0], hi.x);
    b.lo[1] = fminf(b.lo[1], lo.y); b.hi[1] = fmaxf(b.hi[1], hi.y);
    b.lo[2] = fminf(b.lo[2], lo.z); b.hi[2] = fmaxf(b.hi[2], hi.z);
}
__device__ __forceinline__ void box_unbounded(Box &b) {
    for (int a = 0; a < 3; ++a) { b.lo[a] = -INFINITY; b.hi[a] = INFINITY; }
}

// One step of a butterfly min / max over the lanes at xor distance o.
__device__ __forceinline__ void box_xor(Box &b, int o) {
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = fminf(b.lo[a], __shfl_xor_sync(0xffffffffu, b.lo[a], o));
        b.hi[a] = fmaxf(b.hi[a], __shfl_xor_sync(0xffffffffu, b.hi[a], o));
    }
}

__device__ __forceinline__ void box_store(float4 *out, uint64_t e, const Box &b) {
    out[2 * e] = make_float4(b.lo[0], b.lo[1], b.lo[2], 0.f);
    out[2 * e + 1] = make_float4(b.hi[0], b.hi[1], b.hi[2], 0.f);
}

// Three levels of the pyramid from `count` inputs (the sorted points when
// PTS, else the boxes of the level below o1): a 512-thread block per 512
// inputs, one input a thread.  Lanes fold 8 inputs into an o1 entry and a
// warp's 32 into half an o2 entry; warp 0 folds the block's 16 warp boxes
// into its 8 o2 entries and its o3 entry.  Inputs past count hold the empty
// box; a null output is a level above the top and is not written.
template <bool PTS>
__global__ void __launch_bounds__(512) pyramid_fold_kernel(const float4 *__restrict__ in,
                                                           uint64_t count, float4 *o1, float4 *o2,
                                                           float4 *o3) {
    __shared__ float4 s_lo[16], s_hi[16];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t i = (uint64_t)blockIdx.x * 512 + threadIdx.x;
    Box b;
    box_empty(b);
    if (i < count) {
        if (PTS) {
            bool nan = false;
            box_add_point(b, nan, __ldg(&in[i]));
            if (nan) box_unbounded(b);
        } else {
            box_add(b, __ldg(&in[2 * i]), __ldg(&in[2 * i + 1]));
        }
    }
    box_xor(b, 1);
    box_xor(b, 2);
    box_xor(b, 4);
    if ((lane & 7) == 0 && (i >> 3) * 8 < count) box_store(o1, i >> 3, b);
    box_xor(b, 8);
    box_xor(b, 16);
    if (lane == 0) {
        s_lo[warp] = make_float4(b.lo[0], b.lo[1], b.lo[2], 0.f);
        s_hi[warp] = make_float4(b.hi[0], b.hi[1], b.hi[2], 0.f);
    }
    __syncthreads();
    if (warp == 0 && o2) {
        Box c;
        box_empty(c);
        if (lane < 16) box_add(c, s_lo[lane], s_hi[lane]);
        box_xor(c, 1);   // lanes 2m, 2m + 1: the 64 inputs of o2 entry m
        const uint64_t e2 = (uint64_t)blockIdx.x * 8 + (lane >> 1);
        if (lane < 16 && (lane & 1) == 0 && e2 * 64 < count) box_store(o2, e2, c);
        box_xor(c, 2);
        box_xor(c, 4);
        box_xor(c, 8);   // lane 0: the block's 512 inputs
        if (lane == 0 && o3) box_store(o3, blockIdx.x, c);
    }
}

// Adds entries [a, b) of one level (the points when PTS) to a box, loading
// BATCH entries at a time so that their loads are in flight together.  The
// last batch repeats entry b - 1 in place of entries past b: a min / max
// does not change when an entry is added twice.
template <bool PTS>
__device__ __forceinline__ void add_run(Box &bx, bool &nan, const float4 *__restrict__ base,
                                        uint32_t a, uint32_t b) {
    constexpr int BATCH = PTS ? 8 : 4;
#pragma unroll 1
    for (uint32_t t = a; t < b; t += BATCH) {
        float4 lo[BATCH], hi[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            const uint32_t e = t + u < b ? t + u : b - 1;
            if (PTS) {
                lo[u] = __ldg(&base[e]);
            } else {
                lo[u] = __ldg(&base[2 * (uint64_t)e]);
                hi[u] = __ldg(&base[2 * (uint64_t)e + 1]);
            }
        }
#pragma unroll
        for (int u = 0; u < BATCH; ++u) {
            if (PTS) box_add_point(bx, nan, lo[u]);
            else box_add(bx, lo[u], hi[u]);
        }
    }
}

// Box of the sorted points [first, first + count): partial runs at both
// ends point by point, then whole runs from the pyramid level by level (at
// most 7 entries per end and level); the highest level is taken whole.
// The level offsets follow from n as the walk goes up, so the pyramid is
// passed as scalars (a struct taken by reference would be copied to local
// memory).
__device__ __noinline__ Box range_box(const float4 *__restrict__ pts,
                                      const float4 *__restrict__ pyr, uint32_t n, int nlev,
                                      uint32_t first, uint32_t count) {
    Box b;
    box_empty(b);
    bool nan = false;
    uint32_t l = first, r = first + count;   // n < 2^30: no overflow
    uint32_t size = n;                       // entries of the current level
    const float4 *lvl = pyr;                 // level j >= 1 (2 float4 per entry)
#pragma unroll 1
    for (int j = 0; j <= PYR_MAX; ++j) {
        if (l >= r) break;
        if (j == nlev) {
            if (j == 0) add_run<true>(b, nan, pts, l, r);
            else add_run<false>(b, nan, lvl, l, r);
            break;
        }
        uint32_t head = (l + PYR_B - 1) & ~(PYR_B - 1);
        if (head > r) head = r;
        uint32_t tail = r & ~(PYR_B - 1);
        if (tail < head) tail = head;
        if (j == 0) {
            add_run<true>(b, nan, pts, l, head);
            add_run<true>(b, nan, pts, tail, r);
        } else {
            add_run<false>(b, nan, lvl, l, head);
            add_run<false>(b, nan, lvl, tail, r);
            lvl += 2 * (uint64_t)size;
        }
        l = head >> PYR_SH;
        r = tail >> PYR_SH;
        size = (size + PYR_B - 1) >> PYR_SH;
    }
    if (nan) box_unbounded(b);
    return b;
}

// Compact nodes: children become leaves when their subtree has <= leaf_size
// points.  A thread per kept node (sel[c] = its Karras index) finds the
// node's range and split, then writes it.  Every child carries the number
// of points below it (a subtree's points are contiguous in sorted order,
// starting at the parent's first point for the left child and after the
// left child's points for the right one), and its box: the box of its
// contiguous points, from the pyramid.  Every node's boxes are computed
// independently, so no bottom-up pass over the tree follows.  With kfirst
// non-null the range is also stored by Karras index.
template <typename K>
__global__ void __launch_bounds__(BLOCK) node_kernel(
    const K *__restrict__ keys, uint64_t n, const IndexHeader *h, const uint32_t *__restrict__ sel,
    const uint32_t *__restrict__ cidx, uint32_t leaf_size, const Pyramid P, BvhNode *nodes,
    uint32_t *kfirst, uint32_t *klast) {
    chain_wait();
    const uint32_t n_int = h->n_internal;
    for (uint32_t c = blockIdx.x * BLOCK + threadIdx.x; c < n_int && c + 1 < n;
         c += gridDim.x * BLOCK) {
        const uint32_t i = sel[c];
        uint32_t f0, last, sp;
        karras_range<K>(keys, (int64_t)n, i, leaf_size, f0, last, sp);
        if (kfirst) {
            kfirst[i] = f0;
            klast[i] = last;
        }
        // children [first, split] and [split + 1, last]: Karras nodes split
        // and split + 1 when they keep more than leaf_size points, else leaves
        uint32_t word[2], cnt[2];
        cnt[0] = sp - f0 + 1;
        cnt[1] = last - sp;
        word[0] = cnt[0] > leaf_size ? cidx[sp] : (CHILD_LEAF | f0);
        word[1] = cnt[1] > leaf_size ? cidx[sp + 1] : (CHILD_LEAF | (sp + 1));
        const Box b0 = range_box(P.pts, P.pyr, P.n, P.nlev, f0, cnt[0]);
        const Box b1 = range_box(P.pts, P.pyr, P.n, P.nlev, f0 + cnt[0], cnt[1]);
        BvhNode nd;
        // layout: [lo.x0 lo.y0 lo.z0 hi.x0] [hi.y0 hi.z0 lo.x1 lo.y1] [lo.z1 hi.x1 hi.y1 hi.z1]
        nd.a = make_float4(b0.lo[0], b0.lo[1], b0.lo[2], b0.hi[0]);
        nd.b = make_float4(b0.hi[1], b0.hi[2], b1.lo[0], b1.lo[1]);
        nd.c = make_float4(b1.lo[2], b1.hi[0], b1.hi[1], b1.hi[2]);
        nd.d = make_uint4(word[0], word[1], cnt[0], cnt[1]);
        nodes[c] = nd;
    }
}

// Root word and the breadth-first top levels, copied into `top`.  One warp:
// each level's nodes are loaded in parallel (level TOP_LEVELS-1 has at most
// 32 nodes) and their internal children are placed by a warp prefix sum.
__global__ void __launch_bounds__(32) stage_top_kernel(IndexHeader *h,
                                                       const BvhNode *__restrict__ nodes,
                                                       BvhNode *top, uint64_t n,
                                                       uint32_t leaf_size) {
    chain_wait();
    const int lane = threadIdx.x;
    if (n == 0 || n == 1 || n <= leaf_size) {
        if (lane == 0) {
            h->root = n == 0 ? CHILD_NONE : (CHILD_LEAF | 0u);
            h->root_count = (uint32_t)n;
            h->n_top = 0;
        }
        return;
    }
    __shared__ uint32_t s_q[TOP_MAX];
    if (lane == 0) s_q[0] = 0;
    __syncwarp();
    int begin = 0, end = 1;
    for (int depth = 0; depth < TOP_LEVELS; ++depth) {
        const int i = begin + lane;
        const bool has = i < end;
        BvhNode nd;
        if (has) nd = nodes[s_q[i]];
        const bool deeper = depth + 1 < TOP_LEVELS;
        const bool c0 = has && deeper && !(nd.d.x & CHILD_LEAF);
        const bool c1 = has && deeper && !(nd.d.y & CHILD_LEAF);
        const uint32_t cnt = (uint32_t)c0 + (uint32_t)c1;
        uint32_t incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t pos = (uint32_t)end + incl - cnt;
        if (c0) s_q[pos] = nd.d.x;
        if (c1) s_q[pos + (c0 ? 1u : 0u)] = nd.d.y;
        if (has) {
            if (c0) nd.d.x = CHILD_TOP | pos;
            if (c1) nd.d.y = CHILD_TOP | (pos + (c0 ? 1u : 0u));
            top[i] = nd;
        }
        __syncwarp();
        begin = end;
        end += (int)total;
        if (total == 0) break;
    }
    if (lane == 0) {
        h->root = CHILD_TOP | 0u;
        h->n_top = (uint32_t)end;
    }
}

// ------------------------------------------------ radius-seed sample data
// Two stride samples of the points in input order, kept with the index:
// <= 1000 points (sample[0..n_sample)) for the k_nn! sampled-percentile seed
// (gprt-macros/src/lib.rs:433-434), and S = min(n, 4096) points, index
// b*n/S (sample[SEED_PCT_POINTS + b]), for the sampled 1-NN seed, which is
// computed from them on the first search that needs it (ensure_nn_seed).
__global__ void seed_sample_kernel(const float *__restrict__ xyz, uint64_t n, float4 *sample,
                                   IndexHeader *h) {
    uint64_t pstep = n / SEED_PCT_POINTS > 1 ? n / SEED_PCT_POINTS : 1;
    uint64_t cnt = (n + pstep - 1) / pstep;
    if (cnt > SEED_PCT_POINTS) cnt = SEED_PCT_POINTS;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (uint64_t t = t0; t < cnt; t += stride) {
        uint64_t i = t * pstep;
        sample[t] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0f);
    }
    const uint32_t S = n < SEED_NN_SAMPLE ? (uint32_t)n : (uint32_t)SEED_NN_SAMPLE;
    for (uint32_t b = t0; b < S; b += stride) {
        const uint64_t i = (uint64_t)b * n / S;
        sample[SEED_PCT_POINTS + b] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0f);
    }
    if (t0 == 0) h->n_sample = (uint32_t)cnt;
}

// Squared 1-NN distance of each of the S sample points p[a] among the other
// sample points.  Grid (a-tiles x b-chunks); each thread folds its chunk's
// minimum into out[a] (order-preserving u32, pre-set to 0xFFFFFFFF).  The
// minimum does not depend on the order.
constexpr int SEED_CHUNK = 256;
__global__ void __launch_bounds__(128) seed_nn_kernel(const float4 *__restrict__ p, uint32_t S,
                                                      uint32_t *__restrict__ out) {
    __shared__ float3 s_p[SEED_CHUNK];
    const uint32_t a = blockIdx.x * 128 + threadIdx.x;
    const uint32_t b0 = blockIdx.y * SEED_CHUNK;
    for (uint32_t t = threadIdx.x; t < SEED_CHUNK; t += 128) {
        uint32_t b = b0 + t;
        if (b < S) {
            const float4 v = p[b];
            s_p[t] = make_float3(v.x, v.y, v.z);
        }
    }
    __syncthreads();
    if (a >= S) return;
    const float4 va = p[a];
    const float ax = va.x, ay = va.y, az = va.z;
    const uint32_t lim = S - b0 < (uint32_t)SEED_CHUNK ? S - b0 : (uint32_t)SEED_CHUNK;
    float best = INFINITY;
    for (uint32_t j = 0; j < lim; ++j) {
        if (b0 + j == a) continue;
        float key = exact_key(ax, ay, az, s_p[j].x, s_p[j].y, s_p[j].z);
        if (key < best) best = key;
    }
    if (best < INFINITY) atomicMin(&out[a], float_flip(best));
}

// rank-th smallest of S <= 4096 order-preserving u32 values: an 8-bit
// radix select in one 1024-thread block (4 histogram passes).
__global__ void __launch_bounds__(1024) seed_nn_select_kernel(const uint32_t *__restrict__ keys,
                                                              uint32_t S, IndexHeader *h) {
    __shared__ uint32_t s_hist[256];
    __shared__ uint32_t s_sel[2];   // prefix chosen so far, remaining rank
    uint32_t v[4];
    for (int j = 0; j < 4; ++j) {
        uint32_t i = threadIdx.x + 1024u * j;
        v[j] = i < S ? keys[i] : 0xFFFFFFFFu;
    }
    uint32_t rank = (uint32_t)(0.95f * (float)S);
    if (rank > S - 1) rank = S - 1;
    uint32_t prefix = 0;
    for (int pass = 3; pass >= 0; --pass) {
        const int shift = 8 * pass;
        const uint32_t hi_mask = pass == 3 ? 0u : (0xFFFFFFFFu << (shift + 8));
        if (threadIdx.x < 256) s_hist[threadIdx.x] = 0;
        __syncthreads();
        for (int j = 0; j < 4; ++j) {
            uint32_t i = threadIdx.x + 1024u * j;
            if (i < S && (v[j] & hi_mask) == prefix) atomicAdd(&s_hist[(v[j] >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0, d = 0;
            for (; d < 255; ++d) {
                if (acc + s_hist[d] > rank) break;
                acc += s_hist[d];
            }
            s_sel[0] = prefix | (d << shift);
            s_sel[1] = rank - acc;
        }
        __syncthreads();
        prefix = s_sel[0];
        rank = s_sel[1];
        __syncthreads();
    }
    if (threadIdx.x == 0) h->nn95_key = float_unflip(prefix);
}

rtd_status build_seed(rtd_index *idx, const float *d_xyz, uint64_t n, cudaStream_t st) {
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    RTD_TRY(idx->sample.reserve((SEED_PCT_POINTS + SEED_NN_SAMPLE) * sizeof(float4)));
    RTD_TRY(idx->seed.reserve(SEED_NN_SAMPLE * sizeof(float)));
    seed_sample_kernel<<<(SEED_NN_SAMPLE + 255) / 256, 256, 0, st>>>(d_xyz, n,
                                                                    idx->sample.as<float4>(), h);
    RTD_LAUNCH_CHECK();
    idx->nn_seeded = false;
    return RTD_OK;
}

}  // namespace

rtd_status ensure_nn_seed(rtd_index *idx, cudaStream_t st) {
    if (idx->nn_seeded || idx->n < 2) return RTD_OK;
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    const uint32_t S = idx->n < SEED_NN_SAMPLE ? (uint32_t)idx->n : (uint32_t)SEED_NN_SAMPLE;
    RTD_CUDA(cudaMemsetAsync(idx->seed.ptr, 0xFF, S * sizeof(uint32_t), st));
    dim3 grid((S + 127) / 128, (S + SEED_CHUNK - 1) / SEED_CHUNK);
    seed_nn_kernel<<<grid, 128, 0, st>>>(idx->sample.as<float4>() + SEED_PCT_POINTS, S,
                                         idx->seed.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    seed_nn_select_kernel<<<1, 1024, 0, st>>>(idx->seed.as<uint32_t>(), S, h);
    RTD_LAUNCH_CHECK();
    // Inside a stream capture the kernels run at each launch of the graph,
    // not now: an eager search afterwards must still compute the seed.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    RTD_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs == cudaStreamCaptureStatusNone) idx->nn_seeded = true;
    return RTD_OK;
}

namespace {

template <typename K>
rtd_status build_typed(rtd_index *idx, const float *d_xyz, uint64_t n, cudaStream_t st) {
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    uint32_t *d_err = &h->err;
    const int kbits = sizeof(K) == 4 ? 30 : idx->morton_bits;
    const float scale = sizeof(K) == 4 ? 1023.0f : (float)((1u << (kbits / 3)) - 1u);
    RTD_TRY(idx->keys.reserve(n * sizeof(K)));
    RTD_TRY(idx->keys_alt.reserve(n * sizeof(K)));
    RTD_TRY(idx->vals.reserve(n * sizeof(uint32_t)));
    RTD_TRY(idx->vals_alt.reserve(n * sizeof(uint32_t)));
    const int g = grid_for(n, BLOCK, 148 * 8);
    RTD_LAUNCH_CHAINED(morton_kernel<K>, dim3(g), dim3(BLOCK), 0, st, d_xyz, n,
                       (const IndexHeader *)h, scale, idx->keys.as<K>(), aligned16(d_xyz));
    // the last pass gathers the points into idx->pts in key order
    K *skeys;
    if (sizeof(K) == 8 && kbits > 32 && kbits <= 48) {
        // 64-bit keys of up to 48 bits: the low bits as 64-bit keys, then
        // four passes over the top 32 bits as 32-bit keys
        RTD_TRY(idx->k32a.reserve(n * sizeof(uint32_t)));
        RTD_TRY(idx->k32b.reserve(n * sizeof(uint32_t)));
        RTD_TRY(radix_sort_split64(reinterpret_cast<const uint64_t *>(idx->keys.ptr),
                                   idx->keys_alt.as<uint64_t>(), idx->k32a.as<uint32_t>(),
                                   idx->k32b.as<uint32_t>(), idx->vals.as<uint32_t>(),
                                   idx->vals_alt.as<uint32_t>(), n, kbits, idx->sort, st, d_xyz,
                                   idx->pts.as<float4>(), idx->keys_alt.as<uint64_t>()));
        skeys = idx->keys_alt.as<K>();
    } else {
        bool in_alt = false;
        RTD_TRY(radix_sort_pairs<K>(idx->keys.as<K>(), idx->keys_alt.as<K>(),
                                    idx->vals.as<uint32_t>(), idx->vals_alt.as<uint32_t>(), true, n,
                                    0, kbits, idx->sort, d_err, st, &in_alt, d_xyz,
                                    idx->pts.as<float4>()));
        skeys = in_alt ? idx->keys_alt.as<K>() : idx->keys.as<K>();
    }
    idx->skeys = skeys;
    idx->mark(EV_BUILD_SORTED, st);
    // the sorted keys are ready: side-stream work may wait on this
    if (idx->ev_sorted) RTD_CUDA(cudaEventRecord(idx->ev_sorted, st));
    return build_tree_sorted<K>(idx, skeys, n, st);
}

}  // namespace

// Karras tree, leaf collapse and child boxes over keys already sorted, with
// idx->pts holding the points in key order.
template <typename K>
rtd_status build_tree_sorted(rtd_index *idx, const K *skeys, uint64_t n, cudaStream_t st,
                             bool ranges) {
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    uint32_t *d_err = &h->err;
    if (n < 2 || n <= idx->leaf_size) return RTD_OK;
    const uint64_t ni = n - 1;
    for (rtd::DevBuf *b : {&idx->flags, &idx->cidx, &idx->csel})
        RTD_TRY(b->reserve(ni * sizeof(uint32_t)));
    if (ranges)
        for (rtd::DevBuf *b : {&idx->kfirst, &idx->klast}) RTD_TRY(b->reserve(ni * sizeof(uint32_t)));
    // box pyramid over the sorted points (levels until one has <= 8 entries)
    Pyramid P;
    P.pts = idx->pts.as<float4>();
    uint64_t sizes[PYR_MAX + 1] = {n}, offs[PYR_MAX + 1] = {0}, total = 0;
    int nlev = 0;
    while (sizes[nlev] > PYR_B && nlev < PYR_MAX) {
        ++nlev;
        sizes[nlev] = ceil_div(sizes[nlev - 1], PYR_B);
        offs[nlev] = total;
        total += sizes[nlev];
    }
    P.nlev = nlev;
    P.n = (uint32_t)n;
    RTD_TRY(idx->pyramid.reserve((total ? total : 1) * 2 * sizeof(float4)));
    float4 *pyr = idx->pyramid.as<float4>();
    P.pyr = pyr;
    float4 *lv[PYR_MAX + 1] = {};
    for (int j = 1; j <= nlev; ++j) lv[j] = pyr + 2 * offs[j];
    // The pyramid (from the points) runs on the tree stream while the flags
    // and their scan (from the keys) run on st; the node kernel needs both.
    RTD_TRY(ensure_side_stream(idx));
    cudaStream_t ts = idx->tree_stream;
    RTD_CUDA(cudaEventRecord(idx->ev_tree_fork, st));
    RTD_CUDA(cudaStreamWaitEvent(ts, idx->ev_tree_fork, 0));
    // three levels per launch: 1-3 from the points, 4-6 from level 3, ...
    cudaError_t pe = cudaSuccess;
    for (int j = 1; j <= nlev && pe == cudaSuccess; j += 3) {
        float4 *o2 = j + 1 <= nlev ? lv[j + 1] : nullptr;
        float4 *o3 = j + 2 <= nlev ? lv[j + 2] : nullptr;
        const unsigned g = (unsigned)ceil_div(sizes[j - 1], 512);
        if (j == 1) pyramid_fold_kernel<true><<<g, 512, 0, ts>>>(P.pts, n, lv[1], o2, o3);
        else pyramid_fold_kernel<false><<<g, 512, 0, ts>>>(lv[j - 1], sizes[j - 1], lv[j], o2, o3);
        note_launch();
        pe = cudaGetLastError();
    }
    RTD_CUDA(cudaEventRecord(idx->ev_tree_join, ts));
    const unsigned gi = (unsigned)ceil_div(ni, (uint64_t)FLAG_TILE);
    note_launch();
    cudaError_t fe = launch_chained(karras_flag_kernel<K>, dim3(gi), dim3(BLOCK), 0, st, skeys,
                                    (int64_t)n, idx->leaf_size, idx->flags.as<uint32_t>());
    const rtd_status sr =
        fe != cudaSuccess ? RTD_OK
                          : exclusive_scan_select_u32(idx->flags.as<uint32_t>(), idx->cidx.as<uint32_t>(),
                                                      idx->csel.as<uint32_t>(), ni, &h->n_internal,
                                                      idx->scan, d_err, st);
    RTD_CUDA(cudaStreamWaitEvent(st, idx->ev_tree_join, 0));   // also on the error paths
    if (pe != cudaSuccess) return cuda_fail(pe, "pyramid_fold_kernel launch");
    if (fe != cudaSuccess) return cuda_fail(fe, "karras_flag_kernel launch");
    RTD_TRY(sr);
    // grid for about (n - 1) / leaf_size kept nodes, the count of a balanced
    // tree; the kernel strides over however many there are (up to
    // n - 1 - leaf_size in a chain-shaped tree)
    const uint64_t kept_max = ni / idx->leaf_size + 1 < ni ? ni / idx->leaf_size + 1 : ni;
    RTD_LAUNCH_CHAINED(node_kernel<K>, dim3(grid_for(kept_max, BLOCK, 148 * 8)), dim3(BLOCK), 0, st,
                       skeys, n, (const IndexHeader *)h, (const uint32_t *)idx->csel.as<uint32_t>(),
                       (const uint32_t *)idx->cidx.as<uint32_t>(), idx->leaf_size, P,
                       idx->nodes.as<BvhNode>(), ranges ? idx->kfirst.as<uint32_t>() : nullptr,
                       ranges ? idx->klast.as<uint32_t>() : nullptr);
    return RTD_OK;
}

template rtd_status build_tree_sorted<uint32_t>(rtd_index *, const uint32_t *, uint64_t,
                                                cudaStream_t, bool);
template rtd_status build_tree_sorted<uint64_t>(rtd_index *, const uint64_t *, uint64_t,
                                                cudaStream_t, bool);

rtd_status ensure_side_stream(rtd_index *idx) {
    if (idx->side_stream) return RTD_OK;
    RTD_CUDA(cudaStreamCreateWithFlags(&idx->tree_stream, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&idx->ev_fork, &idx->ev_join, &idx->ev_seed_fork, &idx->ev_seed_join,
                           &idx->ev_sorted, &idx->ev_tree_fork, &idx->ev_tree_join})
        RTD_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    // created last: its presence means every stream and event exists
    RTD_CUDA(cudaStreamCreateWithFlags(&idx->side_stream, cudaStreamNonBlocking));
    return RTD_OK;
}

rtd_status index_build(rtd_index *idx, const float *d_xyz, uint64_t n, const rtd_schedule *s,
                       cudaStream_t st) {
    if (!idx) return fail(RTD_ERR_INVALID_ARGUMENT, "index is NULL");
    if (n > 0 && !d_xyz) return fail(RTD_ERR_INVALID_ARGUMENT, "points pointer is NULL");
    if (n >= (1ull << 30) - 1) return fail(RTD_ERR_INVALID_ARGUMENT, "at most 2^30-2 points");
    rtd_schedule def;
    rtd_schedule_default(&def);
    if (!s) s = &def;
    if (s->leaf_size < 1 || s->leaf_size > 64)
        return fail(RTD_ERR_INVALID_ARGUMENT, "leaf_size must be in [1, 64]");
    int mb = (int)s->morton_bits;
    // auto: 48-bit cubic keys (16 bits per axis); measured as fast to search as
    // 63-bit keys on the clustered and sheet workloads, with two fewer sort passes
    if (mb == 0) mb = 48;
    if (mb != 30 && (mb < 33 || mb > 63 || mb % 3 != 0))
        return fail(RTD_ERR_INVALID_ARGUMENT, "morton_bits must be 30 or a multiple of 3 in [33, 63]");
    RTD_CUDA(cudaGetDevice(&idx->device));
    idx->rtoken.valid = false;
    idx->skeys = nullptr;
    idx->n = n;
    idx->leaf_size = s->leaf_size;
    idx->morton_bits = mb;
    RTD_TRY(idx->hdr.reserve(sizeof(IndexHeader)));
    RTD_TRY(idx->pts.reserve((n ? n : 1) * sizeof(float4)));
    RTD_TRY(idx->nodes.reserve((n > 1 ? n - 1 : 1) * sizeof(BvhNode)));
    RTD_TRY(idx->top.reserve(TOP_MAX * sizeof(BvhNode)));
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    for (bool &e : idx->ev_set) e = false;
    idx->mark(EV_BUILD0, st);
    RTD_LAUNCH_CHAINED(hdr_init_kernel, dim3(1), dim3(1), 0, st, h);
    if (n > 0) {
        RTD_LAUNCH_CHAINED(bbox_kernel, dim3(grid_for(n, BLOCK, 148 * 4)), dim3(BLOCK), 0, st, d_xyz,
                           n, h, aligned16(d_xyz));
        // the radius-seed sample reads only the input points: it runs on the
        // side stream while the keys are made and sorted
        RTD_TRY(ensure_side_stream(idx));
        RTD_CUDA(cudaEventRecord(idx->ev_seed_fork, st));
        RTD_CUDA(cudaStreamWaitEvent(idx->side_stream, idx->ev_seed_fork, 0));
        const rtd_status rs = build_seed(idx, d_xyz, n, idx->side_stream);
        RTD_CUDA(cudaEventRecord(idx->ev_seed_join, idx->side_stream));
        const rtd_status rb = mb == 30 ? build_typed<uint32_t>(idx, d_xyz, n, st)
                                       : build_typed<uint64_t>(idx, d_xyz, n, st);
        RTD_CUDA(cudaStreamWaitEvent(st, idx->ev_seed_join, 0));   // also on the error paths
        RTD_TRY(rs);
        RTD_TRY(rb);
    }
    RTD_LAUNCH_CHAINED(stage_top_kernel, dim3(1), dim3(32), 0, st, h,
                       (const BvhNode *)idx->nodes.as<BvhNode>(), idx->top.as<BvhNode>(), n,
                       idx->leaf_size);
    idx->mark(EV_BUILD1, st);
    return RTD_OK;
}

// ------------------------------------------------------- query ordering
namespace {
// Processing-order keys of the queries: 30-bit Morton codes; with chunks > 1
// the query's chunk (i * chunks / nq) takes the top cbits bits of a 32-bit
// key and the code loses its cbits - 2 lowest bits if it must.
__global__ void __launch_bounds__(BLOCK) query_morton_kernel(const float *__restrict__ q,
                                                             uint64_t nq, const IndexHeader *h,
                                                             uint32_t chunks, int cbits,
                                                             uint32_t *__restrict__ keys) {
    const SceneNorm s = scene_norm_cubic(h);   // processing order only
    const int drop = cbits > 2 ? cbits - 2 : 0;
    for (uint64_t i = (uint64_t)blockIdx.x * BLOCK + threadIdx.x; i < nq;
         i += (uint64_t)gridDim.x * BLOCK) {
        const uint32_t code = morton30(quantize(q[3 * i], s.lo[0], s.ext[0], 1023.0f),
                                       quantize(q[3 * i + 1], s.lo[1], s.ext[1], 1023.0f),
                                       quantize(q[3 * i + 2], s.lo[2], s.ext[2], 1023.0f));
        keys[i] = cbits ? ((uint32_t)(i * chunks / nq) << (32 - cbits)) | (code >> drop) : code;
    }
}
}  // namespace

rtd_status order_queries(rtd_index *idx, const float *d_q, uint64_t nq, bool morton,
                         const uint32_t **perm, cudaStream_t st) {
    *perm = nullptr;
    idx->rtoken.valid = false;   // the query-order buffers are about to change
    if (!morton || nq < 2) return RTD_OK;
    if (nq >= (1ull << 30)) return fail(RTD_ERR_INVALID_ARGUMENT, "at most 2^30-1 queries");
    RTD_TRY(idx->qkeys.reserve(nq * 4));
    RTD_TRY(idx->qkeys_alt.reserve(nq * 4));
    RTD_TRY(idx->qperm.reserve(nq * 4));
    RTD_TRY(idx->qperm_alt.reserve(nq * 4));
    IndexHeader *h = idx->hdr.as<IndexHeader>();
    query_morton_kernel<<<grid_for(nq, BLOCK, 148 * 8), BLOCK, 0, st>>>(d_q, nq, h, 1u, 0,
                                                                        idx->qkeys.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    bool in_alt = false;
    RTD_TRY(radix_sort_pairs<uint32_t>(idx->qkeys.as<uint32_t>(), idx->qkeys_alt.as<uint32_t>(),
                                       idx->qperm.as<uint32_t>(), idx->qperm_alt.as<uint32_t>(),
                                       true, nq, 0, 30, idx->sort, &h->err, st, &in_alt));
    *perm = in_alt ? idx->qperm_alt.as<uint32_t>() : idx->qperm.as<uint32_t>();
    return RTD_OK;
}

rtd_status order_queries_own(QueryOrderScratch &qs, const float *d_q, uint64_t nq,
                             const uint32_t **perm, cudaStream_t st, uint32_t chunks) {
    *perm = nullptr;
    if (nq < 2) return RTD_OK;
    if (nq >= (1ull << 30)) return fail(RTD_ERR_INVALID_ARGUMENT, "at most 2^30-1 queries");
    if (chunks < 1 || chunks > (uint32_t)MAX_CHUNKS) return fail(RTD_ERR_INVALID_ARGUMENT, "bad chunk count");
    RTD_TRY(qs.hdr.reserve(sizeof(IndexHeader)));
    RTD_TRY(qs.keys.reserve(nq * 4));
    RTD_TRY(qs.keys_alt.reserve(nq * 4));
    RTD_TRY(qs.perm.reserve(nq * 4));
    RTD_TRY(qs.perm_alt.reserve(nq * 4));
    IndexHeader *h = qs.hdr.as<IndexHeader>();
    hdr_init_kernel<<<1, 1, 0, st>>>(h);
    RTD_LAUNCH_CHECK();
    bbox_kernel<<<grid_for(nq, BLOCK, 148 * 4), BLOCK, 0, st>>>(d_q, nq, h, aligned16(d_q));
    RTD_LAUNCH_CHECK();
    int cbits = 0;
    while ((1u << cbits) < chunks) ++cbits;
    query_morton_kernel<<<grid_for(nq, BLOCK, 148 * 8), BLOCK, 0, st>>>(d_q, nq, h, chunks, cbits,
                                                                        qs.keys.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    bool in_alt = false;
    RTD_TRY(radix_sort_pairs<uint32_t>(qs.keys.as<uint32_t>(), qs.keys_alt.as<uint32_t>(),
                                       qs.perm.as<uint32_t>(), qs.perm_alt.as<uint32_t>(), true,
                                       nq, 0, cbits ? 32 : 30, qs.sort, &h->err, st, &in_alt));
    *perm = in_alt ? qs.perm_alt.as<uint32_t>() : qs.perm.as<uint32_t>();
    return RTD_OK;
}

}  // namespace rtd
