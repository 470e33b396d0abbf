/*
 * oracle.c -- CPU restatement of rt-dsl's spatial-search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls
 * this file: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline arm use it, and only as the checker (or as the timed CPU port of
 * the reference's own CPU search).  The product path is the CUDA library
 * built from rt-dsl_b200/csrc and fails loudly when that library is absent.
 *
 * Parity pinning.  The reference (cashmanjack/rt-dsl, a Rust + OptiX
 * workspace) cannot be built here: no cargo/rustc, no OptiX SDK, and its
 * gprt-optix/host/CMakeLists.txt is missing.  It ships no golden vectors and
 * no unit tests.  The kNN / range restatement below is therefore pinned
 * against the reference's own validation route instead: scipy's cKDTree,
 * which gprt-sandbox/validate_full.py:20-22 uses as ground truth (golden
 * fixtures in tests/golden/, generated by tests/golden/make_golden.py).
 * The Barnes-Hut restatement follows gprt-core/src/lib.rs:427-539 and the
 * intended walk of gprt-macros/src/lib.rs:760-806; the reference's BH device
 * code does not compile as shipped, so the BH walk is "parity unpinned"
 * beyond the physics check of gprt-sandbox/verify_physics.py (sum of force
 * magnitudes vs an FP64 direct sum), which tests/ repeats on this code.
 *
 * Arithmetic contract.  Compiled with -ffp-contract=off and without
 * -ffast-math, so every float expression below rounds exactly as written
 * (IEEE binary32, round-to-nearest-even, no fused multiply-add).  The CUDA
 * kernels use __fadd_rn/__fmul_rn/__fsub_rn/__fdiv_rn/__fsqrt_rn for the
 * same expressions, which makes neighbour IDs and the reference-law
 * Barnes-Hut forces bit-comparable.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#if defined(FLT_EVAL_METHOD) && FLT_EVAL_METHOD != 0
#error "oracle needs FLT_EVAL_METHOD == 0 (SSE float arithmetic)"
#endif

#define ORC_EMPTY 0xFFFFFFFFu

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------
 * Canonical FP32 squared-distance key.
 * gprt-macros/src/lib.rs:338-339: dx = o.x - sphere.x; ...;
 * dist_sq = dx*dx + dy*dy + dz*dz  (query minus point, left to right).
 * ---------------------------------------------------------------------- */
static inline float orc_key(const float *q, const float *p) {
    float dx = q[0] - p[0];
    float dy = q[1] - p[1];
    float dz = q[2] - p[2];
    float s = dx * dx;
    s = s + dy * dy;
    s = s + dz * dz;
    return s;
}

float orc_key_public(const float *q, const float *p) { return orc_key(q, p); }

/* (key, id) lexicographic order; NaN keys are never selected. */
static inline int orc_less(float ka, uint32_t ia, float kb, uint32_t ib) {
    return (ka < kb) || (ka == kb && ia < ib);
}

/* ------------------------------------------------------------------------
 * Morton codes, gprt-core/src/morton.rs:4-48.
 * ---------------------------------------------------------------------- */
static uint32_t orc_expand_bits(uint32_t x) {
    x &= 0x000003ffu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

uint32_t orc_morton3(uint32_t x, uint32_t y, uint32_t z) {
    return (orc_expand_bits(x) << 2) | (orc_expand_bits(y) << 1) | orc_expand_bits(z);
}

/* Rust `f32 as u32`: saturating, NaN -> 0. */
static uint32_t orc_f2u_sat(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

/* compute_morton_codes (morton.rs:19-48): per-axis extent clamped to >=1e-6,
 * ((p - min) / extent * 1023) as u32, min 1023. */
void orc_morton_codes(const float *xyz, int64_t n, uint32_t *out) {
    if (n <= 0) return;
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            float v = xyz[3 * i + a];
            mn[a] = fminf(mn[a], v);
            mx[a] = fmaxf(mx[a], v);
        }
    float ext[3];
    for (int a = 0; a < 3; ++a) ext[a] = fmaxf(mx[a] - mn[a], 1e-6f);
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c[3];
        for (int a = 0; a < 3; ++a) {
            uint32_t u = orc_f2u_sat((xyz[3 * i + a] - mn[a]) / ext[a] * 1023.0f);
            c[a] = u < 1023u ? u : 1023u;
        }
        out[i] = orc_morton3(c[0], c[1], c[2]);
    }
}

/* ------------------------------------------------------------------------
 * Exact kNN by brute force: the k smallest (key, id) pairs per query,
 * ascending.  Slots past the number of finite-or-inf keys hold ORC_EMPTY /
 * +inf.  This is the contract the in-kernel radius expansion of k_nn!
 * (gprt-macros/src/lib.rs:462-595) converges to once every query holds k
 * hits; the reference breaks distance ties in OptiX traversal order, which
 * is unspecified, so ties go to the lower point index here.
 * ---------------------------------------------------------------------- */
void orc_knn(const float *pts, int64_t n, const float *q, int64_t nq, int k,
             uint32_t *ids, float *d2) {
#pragma omp parallel
    {
        float *bk = (float *)malloc(sizeof(float) * (size_t)(k > 0 ? k : 1));
        uint32_t *bi = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(k > 0 ? k : 1));
#pragma omp for schedule(dynamic, 16)
        for (int64_t qi = 0; qi < nq; ++qi) {
            for (int j = 0; j < k; ++j) { bk[j] = INFINITY; bi[j] = ORC_EMPTY; }
            const float *qq = q + 3 * qi;
            for (int64_t p = 0; p < n; ++p) {
                float key = orc_key(qq, pts + 3 * p);
                if (!(key <= INFINITY)) continue;           /* NaN */
                if (k == 0 || !orc_less(key, (uint32_t)p, bk[k - 1], bi[k - 1])) continue;
                int j = k - 1;
                while (j > 0 && orc_less(key, (uint32_t)p, bk[j - 1], bi[j - 1])) {
                    bk[j] = bk[j - 1]; bi[j] = bi[j - 1]; --j;
                }
                bk[j] = key; bi[j] = (uint32_t)p;
            }
            for (int j = 0; j < k; ++j) {
                ids[qi * k + j] = bi[j];
                if (d2) d2[qi * k + j] = bk[j];
            }
        }
        free(bk); free(bi);
    }
}

/* For each query, how many of the k selected neighbours would change if the
 * ranking used exact FP64 distances instead of the FP32 key (the
 * "FP32-ambiguity count"): returns the number of queries whose FP64 top-k
 * set differs from ids[]. */
int64_t orc_knn_fp64_ambiguity(const float *pts, int64_t n, const float *q, int64_t nq,
                               int k, const uint32_t *ids) {
    int64_t diff = 0;
#pragma omp parallel reduction(+ : diff)
    {
        double *bk = (double *)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1));
        uint32_t *bi = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(k > 0 ? k : 1));
#pragma omp for schedule(dynamic, 16)
        for (int64_t qi = 0; qi < nq; ++qi) {
            for (int j = 0; j < k; ++j) { bk[j] = INFINITY; bi[j] = ORC_EMPTY; }
            const float *qq = q + 3 * qi;
            for (int64_t p = 0; p < n; ++p) {
                double dx = (double)qq[0] - pts[3 * p], dy = (double)qq[1] - pts[3 * p + 1],
                       dz = (double)qq[2] - pts[3 * p + 2];
                double key = dx * dx + dy * dy + dz * dz;
                if (!(key <= INFINITY)) continue;
                if (k == 0 || !((key < bk[k - 1]) || (key == bk[k - 1] && (uint32_t)p < bi[k - 1]))) continue;
                int j = k - 1;
                while (j > 0 && ((key < bk[j - 1]) || (key == bk[j - 1] && (uint32_t)p < bi[j - 1]))) {
                    bk[j] = bk[j - 1]; bi[j] = bi[j - 1]; --j;
                }
                bk[j] = key; bi[j] = (uint32_t)p;
            }
            /* set comparison (order-insensitive) */
            int same = 1;
            for (int a = 0; a < k && same; ++a) {
                int found = 0;
                for (int b = 0; b < k; ++b) if (bi[a] == ids[qi * k + b]) { found = 1; break; }
                same = found;
            }
            diff += same ? 0 : 1;
        }
        free(bk); free(bi);
    }
    return diff;
}

/* ------------------------------------------------------------------------
 * Fixed-radius range query.  Membership follows the intersection program
 * gprt-macros/src/lib.rs:334-345: dist_sq <= r*r with r*r rounded to FP32
 * (raygen lib.rs:283 passes __float_as_uint(r_val * r_val)).  The reference
 * pushes prim ids per query with atomicAdd (lib.rs:287-295); the restatement
 * returns per-query counts and the (query, id) pairs sorted by query, id.
 * ---------------------------------------------------------------------- */
int64_t orc_range_count(const float *pts, int64_t n, const float *q, int64_t nq, float r,
                        uint32_t *counts) {
    const float r2 = r * r;
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
    for (int64_t qi = 0; qi < nq; ++qi) {
        uint32_t c = 0;
        for (int64_t p = 0; p < n; ++p)
            if (orc_key(q + 3 * qi, pts + 3 * p) <= r2) ++c;
        counts[qi] = c;
        total += c;
    }
    return total;
}

/* offsets[qi] = exclusive prefix of counts; pairs is 2*total u32 (q, id). */
void orc_range_pairs(const float *pts, int64_t n, const float *q, int64_t nq, float r,
                     const uint64_t *offsets, uint32_t *pairs) {
    const float r2 = r * r;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t qi = 0; qi < nq; ++qi) {
        uint64_t o = offsets[qi];
        for (int64_t p = 0; p < n; ++p)
            if (orc_key(q + 3 * qi, pts + 3 * p) <= r2) {
                pairs[2 * o] = (uint32_t)qi;
                pairs[2 * o + 1] = (uint32_t)p;
                ++o;
            }
    }
}

/* ------------------------------------------------------------------------
 * Initial-radius heuristics.
 * (a) sampled-percentile, the k_nn! default (gprt-macros/src/lib.rs:425-451):
 *     <=100 queries at stride max(nq/100,1), each against <=1000 points at
 *     stride max(n/1000,1); per query the k-th smallest d2 with d2 > 1e-10;
 *     sorted sqrt-distances; radius = dists[min(int(len*p), len-1)] * 1.1.
 *     d2 there is (q.x-p.x).powi(2)+... which equals the key above.
 * (b) sampled nearest-neighbour: mult x the 95th-percentile 1-NN distance
 *     among a 4096-point stride sample of the data (points i*n/4096),
 *     excluding each sample point itself.
 * ---------------------------------------------------------------------- */
static int orc_cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

static int orc_cmp_float(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

float orc_radius_sampled_percentile(const float *pts, int64_t n, const float *q, int64_t nq,
                                    int k, float p) {
    if (nq <= 0 || n <= 0 || k <= 0) return 1.0f;
    int64_t qstep = nq / 100 > 1 ? nq / 100 : 1;
    int64_t pstep = n / 1000 > 1 ? n / 1000 : 1;
    float dists[100];
    int nd = 0;
    float *knn = (float *)malloc(sizeof(float) * (size_t)k);
    for (int64_t qi = 0, tq = 0; qi < nq && tq < 100; qi += qstep, ++tq) {
        for (int j = 0; j < k; ++j) knn[j] = FLT_MAX;
        for (int64_t pi = 0, tp = 0; pi < n && tp < 1000; pi += pstep, ++tp) {
            float d2 = orc_key(q + 3 * qi, pts + 3 * pi);
            if (d2 > 1e-10f && d2 < knn[k - 1]) {
                knn[k - 1] = d2;
                qsort(knn, (size_t)k, sizeof(float), orc_cmp_float);
            }
        }
        if (knn[k - 1] != FLT_MAX) dists[nd++] = sqrtf(knn[k - 1]);
    }
    free(knn);
    if (nd == 0) return 1.0f;
    qsort(dists, (size_t)nd, sizeof(float), orc_cmp_float);
    int64_t idx = (int64_t)((float)nd * p);
    if (idx > nd - 1) idx = nd - 1;
    if (idx < 0) idx = 0;
    return dists[idx] * 1.1f;
}

float orc_radius_sampled_nn(const float *pts, int64_t n, float mult) {
    if (n < 2) return 1.0f;
    int64_t s = n < 4096 ? n : 4096;
    float *d = (float *)malloc(sizeof(float) * (size_t)s);
    for (int64_t a = 0; a < s; ++a) {
        int64_t ia = a * n / s;
        float best = INFINITY;
        for (int64_t b = 0; b < s; ++b) {
            if (b == a) continue;
            int64_t ib = b * n / s;
            float key = orc_key(pts + 3 * ia, pts + 3 * ib);
            if (key < best) best = key;
        }
        d[a] = best;
    }
    qsort(d, (size_t)s, sizeof(float), orc_cmp_float);
    int64_t idx = (int64_t)(0.95f * (float)s);
    if (idx > s - 1) idx = s - 1;
    float r = sqrtf(d[idx]) * mult;
    free(d);
    if (!(r > 0.0f) || !(r < INFINITY)) r = 1.0f;
    return r;
}

/* ------------------------------------------------------------------------
 * The reference's own CPU search: gprt-core Scene::build (midpoint split,
 * leaf <= 2, gprt-core/src/lib.rs:134-210) and Scene::traverse (slab test of
 * Ray::query(origin, radius) = +x ray of length radius, lib.rs:37-55,
 * 212-258; Sphere::intersect dist_sq <= r*r, lib.rs:82-93), driven by the
 * k_nn! round loop (gprt-macros/src/lib.rs:462-595: <=30 rounds, radius *= M
 * per round, partial results from round 15, queries in Morton order when
 * use_morton_lbv).  Node bounds are point bounds grown by the current radius
 * at test time: Scene::build's split choices depend only on the sphere
 * centres (bounds grown by the same r on every axis keep the axis order and
 * the midpoints), so this equals rebuilding the Scene every round.
 * Used as the timed CPU baseline ("port").
 * ---------------------------------------------------------------------- */
typedef struct { float mn[3], mx[3]; uint32_t left_first, count; } orc_bvh_node;

typedef struct {
    orc_bvh_node *nodes; int64_t nn, cap;
    uint32_t *idx;
    const float *pts;
} orc_scene;

static void orc_scene_bounds(orc_scene *s, int64_t ni) {
    orc_bvh_node *nd = &s->nodes[ni];
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = 0; i < nd->count; ++i) {
        const float *p = s->pts + 3 * (size_t)s->idx[nd->left_first + i];
        for (int a = 0; a < 3; ++a) { mn[a] = fminf(mn[a], p[a]); mx[a] = fmaxf(mx[a], p[a]); }
    }
    memcpy(nd->mn, mn, sizeof mn); memcpy(nd->mx, mx, sizeof mx);
}

static int64_t orc_scene_push(orc_scene *s, uint32_t lf, uint32_t c) {
    if (s->nn == s->cap) {
        s->cap = s->cap ? 2 * s->cap : 1024;
        s->nodes = (orc_bvh_node *)realloc(s->nodes, sizeof(orc_bvh_node) * (size_t)s->cap);
    }
    s->nodes[s->nn].left_first = lf; s->nodes[s->nn].count = c;
    return s->nn++;
}

static void orc_scene_subdivide(orc_scene *s, int64_t root) {
    int64_t *work = (int64_t *)malloc(sizeof(int64_t) * 256);
    int64_t wcap = 256, wn = 0;
    work[wn++] = root;
    while (wn) {
        int64_t ni = work[--wn];
        uint32_t lf = s->nodes[ni].left_first, cnt = s->nodes[ni].count;
        if (cnt <= 2) continue;
        float ext[3], ctr[3];
        for (int a = 0; a < 3; ++a) {
            ext[a] = s->nodes[ni].mx[a] - s->nodes[ni].mn[a];
            ctr[a] = (s->nodes[ni].mn[a] + s->nodes[ni].mx[a]) * 0.5f;
        }
        int axis = 0;
        if (ext[1] > ext[0]) axis = 1;
        if (ext[2] > ext[1] && ext[2] > ext[0]) axis = 2;
        float split = ctr[axis];
        int64_t i = lf, j = (int64_t)lf + cnt - 1;
        while (i <= j) {
            float v = s->pts[3 * (size_t)s->idx[i] + axis];
            if (v < split) ++i;
            else {
                uint32_t t = s->idx[i]; s->idx[i] = s->idx[j]; s->idx[j] = t;
                if (j == 0) break;
                --j;
            }
        }
        uint32_t lc = (uint32_t)(i - lf);
        if (lc == 0 || lc == cnt) continue;
        int64_t l = orc_scene_push(s, lf, lc);
        orc_scene_push(s, (uint32_t)i, cnt - lc);
        s->nodes[ni].left_first = (uint32_t)l;
        s->nodes[ni].count = 0;
        orc_scene_bounds(s, l);
        orc_scene_bounds(s, l + 1);
        if (wn + 2 > wcap) { wcap *= 2; work = (int64_t *)realloc(work, sizeof(int64_t) * (size_t)wcap); }
        work[wn++] = l + 1;
        work[wn++] = l;
    }
    free(work);
}

/* Rust f32::min / f32::max ignore a NaN operand, like fminf/fmaxf. */
static int orc_ray_box(const orc_bvh_node *nd, float r, const float *o, float tmax0) {
    float tmin = 0.0f, tmax = tmax0;
    const float inv[3] = {1.0f, INFINITY, INFINITY};
    for (int a = 0; a < 3; ++a) {
        float t1 = ((nd->mn[a] - r) - o[a]) * inv[a];
        float t2 = ((nd->mx[a] + r) - o[a]) * inv[a];
        tmin = fmaxf(tmin, fminf(t1, t2));
        tmax = fminf(tmax, fmaxf(t1, t2));
    }
    return tmax >= tmin && tmax > 0.0f;
}

/* Scene::build over n points (midpoint split, leaf <= 2). */
static void orc_scene_build(orc_scene *s, const float *pts, int64_t n) {
    memset(s, 0, sizeof *s);
    s->pts = pts;
    if (n <= 0) return;
    s->idx = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) s->idx[i] = (uint32_t)i;
    orc_scene_push(s, 0, (uint32_t)n);
    orc_scene_bounds(s, 0);
    orc_scene_subdivide(s, 0);
}

/* The reference's fixed-radius search on its CPU BVH: Scene::build, then
 * one Scene::traverse per query at radius r (the global-push programs'
 * single launch, gprt-macros/src/lib.rs:276-295, where each hit with
 * dist_sq <= r*r is pushed to the query's buffer).  Every hit id is stored
 * (per-thread buffer, like the push slab); counts[q] = hits of query q.
 * Returns the total.  Timed CPU baseline of the range query ("port"). */
int64_t orc_cpu_bvh_range(const float *pts, int64_t n, const float *q, int64_t nq, float r,
                          uint32_t *counts) {
    orc_scene s;
    orc_scene_build(&s, pts, n);
    const float r2 = r * r;
    int64_t total = 0;
#pragma omp parallel reduction(+ : total)
    {
        int64_t scap = 256, bcap = 4096, nb = 0;
        int64_t *stack = (int64_t *)malloc(sizeof(int64_t) * (size_t)scap);
        uint32_t *buf = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)bcap);
#pragma omp for schedule(dynamic, 64)
        for (int64_t qi = 0; qi < nq; ++qi) {
            const float *o = q + 3 * qi;
            uint32_t hits = 0;
            int64_t sp = 0;
            nb = 0;
            if (s.nn) stack[sp++] = 0;
            while (sp) {
                const orc_bvh_node *nd = &s.nodes[stack[--sp]];
                if (!orc_ray_box(nd, r, o, r)) continue;
                if (nd->count > 0) {
                    for (uint32_t i = 0; i < nd->count; ++i) {
                        uint32_t pid = s.idx[nd->left_first + i];
                        if (!(orc_key(o, pts + 3 * (size_t)pid) <= r2)) continue;
                        if (nb == bcap) {
                            bcap *= 2;
                            buf = (uint32_t *)realloc(buf, sizeof(uint32_t) * (size_t)bcap);
                        }
                        buf[nb++] = pid;
                        ++hits;
                    }
                } else {
                    if (sp + 2 > scap) { scap *= 2; stack = (int64_t *)realloc(stack, sizeof(int64_t) * (size_t)scap); }
                    stack[sp++] = nd->left_first;
                    stack[sp++] = nd->left_first + 1;
                }
            }
            counts[qi] = hits;
            total += hits;
        }
        free(stack); free(buf);
    }
    free(s.nodes); free(s.idx);
    return total;
}

/* Returns the number of rounds run.  ids/d2 are nq*k, (key, id)-ascending,
 * ORC_EMPTY/+inf where a query ended with fewer than k hits. */
int orc_cpu_bvh_knn(const float *pts, int64_t n, const float *q, int64_t nq, int k,
                    float radius0, float mult, int use_morton, uint32_t *ids, float *d2) {
    orc_scene s;
    orc_scene_build(&s, pts, n);
    int rounds = 0;
    int64_t *active = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nq > 0 ? nq : 1));
    int64_t na = nq;
    if (use_morton && nq > 0) {
        uint32_t *codes = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nq);
        orc_morton_codes(q, nq, codes);
        /* stable counting order by code: sort_by_key is stable (morton.rs:54) */
        uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)nq);
        for (int64_t i = 0; i < nq; ++i) tmp[i] = ((uint64_t)codes[i] << 32) | (uint64_t)i;
        qsort(tmp, (size_t)nq, sizeof(uint64_t), orc_cmp_u64);
        for (int64_t i = 0; i < nq; ++i) active[i] = (int64_t)(tmp[i] & 0xFFFFFFFFu);
        free(tmp); free(codes);
    } else {
        for (int64_t i = 0; i < nq; ++i) active[i] = i;
    }
    for (int64_t i = 0; i < nq * (int64_t)k; ++i) { ids[i] = ORC_EMPTY; if (d2) d2[i] = INFINITY; }
    float radius = radius0;
    int64_t *next = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nq > 0 ? nq : 1));
    unsigned char *keep = (unsigned char *)malloc((size_t)(nq > 0 ? nq : 1));
    while (na > 0 && rounds < 30) {
        ++rounds;
        const float r2 = radius * radius;
#pragma omp parallel
        {
            float *bk = (float *)malloc(sizeof(float) * (size_t)(k > 0 ? k : 1));
            uint32_t *bi = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(k > 0 ? k : 1));
            int64_t scap = 256;
            int64_t *stack = (int64_t *)malloc(sizeof(int64_t) * (size_t)scap);
#pragma omp for schedule(dynamic, 64)
            for (int64_t a = 0; a < na; ++a) {
                int64_t qi = active[a];
                const float *o = q + 3 * qi;
                int hits = 0;
                for (int j = 0; j < k; ++j) { bk[j] = INFINITY; bi[j] = ORC_EMPTY; }
                int64_t sp = 0;
                if (s.nn) stack[sp++] = 0;
                while (sp) {
                    int64_t ni = stack[--sp];
                    const orc_bvh_node *nd = &s.nodes[ni];
                    if (!orc_ray_box(nd, radius, o, radius)) continue;
                    if (nd->count > 0) {
                        for (uint32_t i = 0; i < nd->count; ++i) {
                            uint32_t pid = s.idx[nd->left_first + i];
                            float key = orc_key(o, pts + 3 * (size_t)pid);
                            if (!(key <= r2)) continue;
                            ++hits;
                            if (k == 0 || !orc_less(key, pid, bk[k - 1], bi[k - 1])) continue;
                            int j = k - 1;
                            while (j > 0 && orc_less(key, pid, bk[j - 1], bi[j - 1])) {
                                bk[j] = bk[j - 1]; bi[j] = bi[j - 1]; --j;
                            }
                            bk[j] = key; bi[j] = pid;
                        }
                    } else {
                        if (sp + 2 > scap) { scap *= 2; stack = (int64_t *)realloc(stack, sizeof(int64_t) * (size_t)scap); }
                        stack[sp++] = nd->left_first;
                        stack[sp++] = nd->left_first + 1;
                    }
                }
                int done = hits >= k || rounds >= 15;
                keep[a] = (unsigned char)!done;
                if (done) {
                    for (int j = 0; j < k; ++j) {
                        ids[qi * k + j] = bi[j];
                        if (d2) d2[qi * k + j] = bk[j];
                    }
                }
            }
            free(bk); free(bi); free(stack);
        }
        int64_t nn2 = 0;
        for (int64_t a = 0; a < na; ++a) if (keep[a]) next[nn2++] = active[a];
        int64_t *t = active; active = next; next = t;
        na = nn2;
        radius *= mult;
    }
    free(active); free(next); free(keep);
    free(s.nodes); free(s.idx);
    return rounds;
}

/* ------------------------------------------------------------------------
 * Barnes-Hut, reference tree: BarnesHutTree::build (gprt-core/src/lib.rs:
 * 427-469), build_recursive (340-424), compute_com (471-501) and
 * flatten_dfs (503-539).  BUCKET_SIZE = 128, MIN_SPLIT_SIZE = 1e-5
 * (lib.rs:275-276) are parameters here (bucket, min_width).
 * The reference orders bodies with sort_unstable_by_key(morton) (lib.rs:446)
 * whose order among equal codes is unspecified; the restatement uses the
 * stable order (code, original index).
 * ---------------------------------------------------------------------- */
typedef struct {
    float com[3]; float mass; float width;
    uint32_t is_leaf, next_idx, autorope, bucket_start, num_particles;
} orc_flat_node;   /* FlatNode, gprt-core/src/lib.rs:299-308 (40 B) */

typedef struct {
    float mn[3], mx[3];
    int32_t child[8]; int nchild;
    float com[3]; float mass;
    int64_t start, count;   /* count = bodies for leaves, 0 for internal */
} orc_oct;

typedef struct {
    const float *pos; const float *mass;
    orc_oct *arena; int64_t na, cap;
    uint32_t *scratch;
    uint32_t bucket; float min_width;
} orc_bh_builder;

static int64_t orc_bh_rec(orc_bh_builder *b, uint32_t *ind, int64_t cnt, const float mn[3],
                          const float mx[3], float width, int64_t abs_start) {
    if (b->na == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 1024;
        b->arena = (orc_oct *)realloc(b->arena, sizeof(orc_oct) * (size_t)b->cap);
    }
    int64_t ni = b->na++;
    orc_oct *o = &b->arena[ni];
    int leaf = cnt <= (int64_t)b->bucket || width < b->min_width;
    memcpy(o->mn, mn, 3 * sizeof(float)); memcpy(o->mx, mx, 3 * sizeof(float));
    o->nchild = 0; o->com[0] = o->com[1] = o->com[2] = 0.0f; o->mass = 0.0f;
    o->start = abs_start; o->count = leaf ? cnt : 0;
    if (leaf) return ni;
    float c[3];
    for (int a = 0; a < 3; ++a) c[a] = (mn[a] + mx[a]) * 0.5f;   /* AABB::center */
    int64_t counts[8] = {0};
    for (int64_t i = 0; i < cnt; ++i) {
        const float *p = b->pos + 3 * (size_t)ind[i];
        int oc = (p[0] >= c[0] ? 1 : 0) | (p[1] >= c[1] ? 2 : 0) | (p[2] >= c[2] ? 4 : 0);
        counts[oc]++;
    }
    int64_t off[8]; off[0] = 0;
    for (int i = 1; i < 8; ++i) off[i] = off[i - 1] + counts[i - 1];
    uint32_t *scr = b->scratch + abs_start;
    for (int64_t i = 0; i < cnt; ++i) {
        const float *p = b->pos + 3 * (size_t)ind[i];
        int oc = (p[0] >= c[0] ? 1 : 0) | (p[1] >= c[1] ? 2 : 0) | (p[2] >= c[2] ? 4 : 0);
        scr[off[oc]++] = ind[i];
    }
    memcpy(ind, scr, sizeof(uint32_t) * (size_t)cnt);
    float cw = width * 0.5f;
    int64_t rel = 0, absn = abs_start;
    int32_t kids[8]; int nk = 0;
    for (int oc = 0; oc < 8; ++oc) {
        int64_t cc = counts[oc];
        if (cc == 0) continue;
        float cmn[3], cmx[3];
        cmn[0] = (oc & 1) ? c[0] : mn[0]; cmx[0] = (oc & 1) ? mx[0] : c[0];
        cmn[1] = (oc & 2) ? c[1] : mn[1]; cmx[1] = (oc & 2) ? mx[1] : c[1];
        cmn[2] = (oc & 4) ? c[2] : mn[2]; cmx[2] = (oc & 4) ? mx[2] : c[2];
        kids[nk++] = (int32_t)orc_bh_rec(b, ind + rel, cc, cmn, cmx, cw, absn);
        rel += cc; absn += cc;
    }
    o = &b->arena[ni];   /* arena may have moved */
    memcpy(o->child, kids, sizeof(int32_t) * (size_t)nk);
    o->nchild = nk;
    return ni;
}

static void orc_bh_com(orc_bh_builder *b, int64_t ni, const uint32_t *ind) {
    orc_oct *o = &b->arena[ni];
    float tm = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
    if (o->nchild == 0) {
        for (int64_t i = 0; i < o->count; ++i) {
            uint32_t bi = ind[o->start + i];
            float m = b->mass[bi];
            const float *p = b->pos + 3 * (size_t)bi;
            tm = tm + m;
            for (int a = 0; a < 3; ++a) c[a] = c[a] + p[a] * m;
        }
    } else {
        for (int j = 0; j < o->nchild; ++j) {
            orc_bh_com(b, o->child[j], ind);
            o = &b->arena[ni];
            const orc_oct *ch = &b->arena[o->child[j]];
            tm = tm + ch->mass;
            for (int a = 0; a < 3; ++a) c[a] = c[a] + ch->com[a] * ch->mass;
        }
    }
    o->mass = tm;
    if (tm > 0.0f) for (int a = 0; a < 3; ++a) o->com[a] = c[a] / tm;
    else for (int a = 0; a < 3; ++a) o->com[a] = 0.0f;
}

static int64_t orc_bh_flatten(const orc_bh_builder *b, int64_t ni, orc_flat_node *out, int64_t *nout,
                              uint32_t *order_out, int64_t *nbod, const uint32_t *ind) {
    int64_t me = (*nout)++;
    const orc_oct *o = &b->arena[ni];
    float w = fmaxf(fmaxf(o->mx[0] - o->mn[0], o->mx[1] - o->mn[1]), o->mx[2] - o->mn[2]);
    uint32_t bs = 0, np = (uint32_t)o->count;
    if (np > 0) {
        bs = (uint32_t)*nbod;
        for (int64_t i = 0; i < o->count; ++i) order_out[(*nbod)++] = ind[o->start + i];
    }
    orc_flat_node *f = &out[me];
    for (int a = 0; a < 3; ++a) f->com[a] = o->com[a];
    f->mass = o->mass; f->width = w;
    f->is_leaf = o->nchild == 0 ? 1u : 0u;
    f->next_idx = (uint32_t)(me + 1);
    f->bucket_start = bs; f->num_particles = np;
    for (int j = 0; j < o->nchild; ++j) orc_bh_flatten(b, o->child[j], out, nout, order_out, nbod, ind);
    out[me].autorope = (uint32_t)*nout;
    return *nout - me;
}

/* Builds the reference tree.  nodes_out must hold 2*n+1 entries (an upper
 * bound), order_out n entries (flat body order: order_out[i] is the original
 * index of the i-th body of flat_bodies).  Returns the node count. */
int64_t orc_bh_build(const float *pos, const float *mass, int64_t n, uint32_t bucket,
                     float min_width, orc_flat_node *nodes_out, uint32_t *order_out,
                     float *root_out /* 7 floats: min xyz, max xyz, width */) {
    if (n <= 0) return 0;
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            /* Vec3::min/max = f32::min/max per component */
            mn[a] = fminf(mn[a], pos[3 * i + a]);
            mx[a] = fmaxf(mx[a], pos[3 * i + a]);
        }
    float ext[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    float me = fmaxf(fmaxf(ext[0], ext[1]), ext[2]);
    float ctr[3], rmn[3], rmx[3];
    for (int a = 0; a < 3; ++a) {
        ctr[a] = (mn[a] + mx[a]) * 0.5f;
        rmn[a] = ctr[a] - me / 2.0f;
        rmx[a] = ctr[a] + me / 2.0f;
    }
    if (root_out) {
        for (int a = 0; a < 3; ++a) { root_out[a] = rmn[a]; root_out[3 + a] = rmx[a]; }
        root_out[6] = me;
    }
    float scale = me > 0.0f ? 1023.0f / me : 0.0f;
    uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        uint32_t lx = orc_f2u_sat((pos[3 * i] - mn[0]) * scale);
        uint32_t ly = orc_f2u_sat((pos[3 * i + 1] - mn[1]) * scale);
        uint32_t lz = orc_f2u_sat((pos[3 * i + 2] - mn[2]) * scale);
        keys[i] = ((uint64_t)orc_morton3(lx, ly, lz) << 32) | (uint64_t)i;
    }
    qsort(keys, (size_t)n, sizeof(uint64_t), orc_cmp_u64);
    uint32_t *ind = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) ind[i] = (uint32_t)(keys[i] & 0xFFFFFFFFu);
    free(keys);
    orc_bh_builder b; memset(&b, 0, sizeof b);
    b.pos = pos; b.mass = mass; b.bucket = bucket; b.min_width = min_width;
    b.scratch = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    orc_bh_rec(&b, ind, n, rmn, rmx, me, 0);
    orc_bh_com(&b, 0, ind);
    int64_t nout = 0, nbod = 0;
    orc_bh_flatten(&b, 0, nodes_out, &nout, order_out, &nbod, ind);
    free(b.arena); free(b.scratch); free(ind);
    return nout;
}

/* gprt_dot, assumed a.x*b.x + a.y*b.y + a.z*b.z (left to right). */
static inline float orc_dot3(float x, float y, float z) {
    float s = x * x;
    s = s + y * y;
    s = s + z * z;
    return s;
}

/* The intended reference walk (gprt-macros/src/lib.rs:760-806), one body:
 * stackless pre-order walk over next_idx/autorope.  A node is accepted
 * ("hit") when width < max(1e-6, theta*d) + 1e-5, d = |com - x_i|.
 * Leaves: direct sum over the bucket (bodies of the flattened order, which
 * fixes lib.rs:829 indexing the unsorted array).  Accepted internal nodes:
 * monopole.  Law: G*m_i*m_j*delta / (r2*sqrt(r2+1e-6)), skipped when
 * r2 <= 1e-10.  Forces are returned in original body order. */
/* One body of the walk: force on caller body i (fb = bodies in flat order
 * as (x, y, z, m)). */
static void orc_bh_ref_body(const float *pos, const float *mass, int64_t i,
                            const orc_flat_node *nodes, int64_t nn, const float *fb, float theta,
                            float G, float *out) {
    const float px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const float gm = G * mass[i];
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    uint32_t p = 0;
    while ((int64_t)p < nn) {
        const orc_flat_node *nd = &nodes[p];
        float dx = nd->com[0] - px, dy = nd->com[1] - py, dz = nd->com[2] - pz;
        float dist_sq = orc_dot3(dx, dy, dz);
        float d = sqrtf(dist_sq);
        float tmax = fmaxf(1e-6f, theta * d) + 1e-5f;
        int hit = nd->width < tmax;
        if (nd->is_leaf) {
            for (uint32_t j = 0; j < nd->num_particles; ++j) {
                const float *b = fb + 4 * (size_t)(nd->bucket_start + j);
                float ex = b[0] - px, ey = b[1] - py, ez = b[2] - pz;
                float d2 = orc_dot3(ex, ey, ez);
                if (d2 > 1e-10f) {
                    float denom = d2 * sqrtf(d2 + 1e-6f);
                    float fm = (gm * b[3]) / denom;
                    sx = sx + ex * fm; sy = sy + ey * fm; sz = sz + ez * fm;
                }
            }
            p = hit ? nd->autorope : nd->next_idx;
        } else if (hit) {
            if (dist_sq > 1e-10f) {
                float denom = dist_sq * sqrtf(dist_sq + 1e-6f);
                float fm = (gm * nd->mass) / denom;
                sx = sx + dx * fm; sy = sy + dy * fm; sz = sz + dz * fm;
            }
            p = nd->autorope;
        } else {
            p = nd->next_idx;
        }
    }
    out[0] = sx; out[1] = sy; out[2] = sz;
}

static float *orc_bh_flat_bodies(const float *pos, const float *mass, int64_t n,
                                 const uint32_t *order) {
    float *fb = (float *)malloc(sizeof(float) * 4 * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) {
        uint32_t o = order[i];
        fb[4 * i] = pos[3 * o]; fb[4 * i + 1] = pos[3 * o + 1]; fb[4 * i + 2] = pos[3 * o + 2];
        fb[4 * i + 3] = mass[o];
    }
    return fb;
}

void orc_bh_ref_forces(const float *pos, const float *mass, int64_t n, const orc_flat_node *nodes,
                       int64_t nn, const uint32_t *order, float theta, float G, float *force) {
    float *fb = orc_bh_flat_bodies(pos, mass, n, order);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i)
        orc_bh_ref_body(pos, mass, i, nodes, nn, fb, theta, G, force + 3 * i);
    free(fb);
}

/* The same walk for the listed caller bodies only (force[3*t] for
 * targets[t]): the check of a large tree on a sample of its bodies. */
void orc_bh_ref_forces_at(const float *pos, const float *mass, int64_t n,
                          const orc_flat_node *nodes, int64_t nn, const uint32_t *order,
                          float theta, float G, const int64_t *targets, int64_t nt, float *force) {
    float *fb = orc_bh_flat_bodies(pos, mass, n, order);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < nt; ++t)
        orc_bh_ref_body(pos, mass, targets[t], nodes, nn, fb, theta, G, force + 3 * t);
    free(fb);
}

/* FP64 direct sum with the reference law (skip r2 <= 1e-10), for the
 * BH-vs-direct error of reference-law runs; only the listed targets. */
void orc_direct_ref_f64(const float *pos, const float *mass, int64_t n, const int64_t *targets,
                        int64_t nt, double G, double *force) {
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t t = 0; t < nt; ++t) {
        int64_t i = targets[t];
        double sx = 0, sy = 0, sz = 0;
        for (int64_t j = 0; j < n; ++j) {
            double ex = (double)pos[3 * j] - pos[3 * i], ey = (double)pos[3 * j + 1] - pos[3 * i + 1],
                   ez = (double)pos[3 * j + 2] - pos[3 * i + 2];
            double d2 = ex * ex + ey * ey + ez * ez;
            if (d2 > 1e-10) {
                double f = G * mass[i] * mass[j] / (d2 * sqrt(d2 + 1e-6));
                sx += ex * f; sy += ey * f; sz += ez * f;
            }
        }
        force[3 * t] = sx; force[3 * t + 1] = sy; force[3 * t + 2] = sz;
    }
}

/* ------------------------------------------------------------------------
 * Plummer-law Barnes-Hut (the build's physics mode; no reference
 * counterpart beyond the tree).  The tree is the reference tree built by
 * orc_bh_build (with its own bucket size).  A node is accepted for body i
 * when RN(width*width) < RN(theta2 * d2), d2 = |COM - x_i|^2 summed left to
 * right (all FP32, rounded per operation, theta2 = RN(theta*theta)): the
 * decision the GPU walk makes.  Accepted nodes interact as monopole (+
 * traceless quadrupole) multipoles about their COM, rejected leaves by
 * direct summation, rejected internal nodes are opened.
 * orc_bh_plummer_eval takes the decisions from the FP32 tree and the FP32
 * positions of one configuration, and evaluates phi, a and
 * L = sum(phi) + 0.5*sum|a|^2 in FP64 for FP64 (possibly perturbed)
 * positions and masses, with cell moments recomputed from them over the
 * fixed tree membership: the function whose derivative the GPU adjoint
 * computes, so central finite differences of it check the adjoint.
 * ---------------------------------------------------------------------- */

typedef struct { double c[3]; double m; double q[6]; } orc_cell64;

/* FP64 cell moments over each node's flat body range. */
static void orc_cells64(const orc_flat_node *nodes, int64_t nn, const double *pos,
                        const double *mass, int64_t n, orc_cell64 *cells) {
    int64_t *first = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nn + 1));
    int64_t nxt = n;
    for (int64_t i = nn - 1; i >= 0; --i) {   /* first body of the subtree */
        if (nodes[i].is_leaf) nxt = nodes[i].bucket_start;
        first[i] = nxt;
    }
    first[nn] = n;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < nn; ++i) {
        int64_t s = first[i];
        int64_t e = nodes[i].autorope < (uint32_t)nn ? first[nodes[i].autorope] : n;
        double m = 0, c[3] = {0, 0, 0}, q[6] = {0, 0, 0, 0, 0, 0};
        for (int64_t j = s; j < e; ++j) {
            m += mass[j];
            for (int a = 0; a < 3; ++a) c[a] += mass[j] * pos[3 * j + a];
        }
        if (m > 0) for (int a = 0; a < 3; ++a) c[a] /= m;
        for (int64_t j = s; j < e; ++j) {
            double dx = pos[3 * j] - c[0], dy = pos[3 * j + 1] - c[1], dz = pos[3 * j + 2] - c[2];
            double r2 = dx * dx + dy * dy + dz * dz, w = mass[j];
            q[0] += w * (3 * dx * dx - r2); q[1] += w * (3 * dy * dy - r2); q[2] += w * (3 * dz * dz - r2);
            q[3] += w * 3 * dx * dy; q[4] += w * 3 * dx * dz; q[5] += w * 3 * dy * dz;
        }
        orc_cell64 *o = &cells[i];
        memcpy(o->c, c, sizeof c); o->m = m; memcpy(o->q, q, sizeof q);
    }
    free(first);
}

/* pos32: the FP32 flat-order positions the decisions use; pos/mass: FP64
 * flat-order values.  Returns L; phi/acc optional (flat order). */
double orc_bh_plummer_eval(const orc_flat_node *nodes, int64_t nn, const float *pos32,
                           const double *pos, const double *mass, int64_t n, float theta,
                           double eps, double G, int quad, double *phi, double *acc) {
    orc_cell64 *cells = (orc_cell64 *)malloc(sizeof(orc_cell64) * (size_t)(nn > 0 ? nn : 1));
    orc_cells64(nodes, nn, pos, mass, n, cells);
    const double e2 = eps * eps;
    const float th2 = theta * theta;
    double L = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : L)
    for (int64_t i = 0; i < n; ++i) {
        const double *x = pos + 3 * i;
        const float *x32 = pos32 + 3 * i;
        double ph = 0, ax = 0, ay = 0, az = 0;
        int64_t p = 0;
        while (p < nn) {
            const orc_flat_node *nd = &nodes[p];
            float d2 = orc_dot3(nd->com[0] - x32[0], nd->com[1] - x32[1], nd->com[2] - x32[2]);
            if (nd->width * nd->width < th2 * d2) {
                const orc_cell64 *c = &cells[p];
                double rx = x[0] - c->c[0], ry = x[1] - c->c[1], rz = x[2] - c->c[2];
                double s2 = rx * rx + ry * ry + rz * rz + e2;
                double i1 = 1.0 / sqrt(s2), i2 = i1 * i1, i3 = i1 * i2;
                ph -= c->m * i1;
                ax -= c->m * rx * i3; ay -= c->m * ry * i3; az -= c->m * rz * i3;
                if (quad) {
                    const double *Q = c->q;
                    double qx = Q[0] * rx + Q[3] * ry + Q[4] * rz;
                    double qy = Q[3] * rx + Q[1] * ry + Q[5] * rz;
                    double qz = Q[4] * rx + Q[5] * ry + Q[2] * rz;
                    double q = rx * qx + ry * qy + rz * qz;
                    double i5 = i3 * i2, i7 = i5 * i2;
                    ph -= 0.5 * q * i5;
                    ax += qx * i5 - 2.5 * q * rx * i7;
                    ay += qy * i5 - 2.5 * q * ry * i7;
                    az += qz * i5 - 2.5 * q * rz * i7;
                }
                p = nd->autorope;
            } else if (nd->is_leaf) {
                int64_t s = nd->bucket_start, cnt = nd->num_particles;
                for (int64_t j = s; j < s + cnt; ++j) {
                    if (j == i) continue;
                    double rx = x[0] - pos[3 * j], ry = x[1] - pos[3 * j + 1], rz = x[2] - pos[3 * j + 2];
                    double s2 = rx * rx + ry * ry + rz * rz + e2;
                    double i1 = 1.0 / sqrt(s2), i3 = i1 * i1 * i1;
                    ph -= mass[j] * i1;
                    ax -= mass[j] * rx * i3; ay -= mass[j] * ry * i3; az -= mass[j] * rz * i3;
                }
                p = p + 1;
            } else {
                p = p + 1;
            }
        }
        ph *= G; ax *= G; ay *= G; az *= G;
        if (phi) phi[i] = ph;
        if (acc) { acc[3 * i] = ax; acc[3 * i + 1] = ay; acc[3 * i + 2] = az; }
        L += ph + 0.5 * (ax * ax + ay * ay + az * az);
    }
    free(cells);
    return L;
}

/* FP64 Plummer direct sum: phi, acc (n, n*3) and, if g_pos != NULL, the
 * gradient of L = sum(phi) + 0.5*sum|a|^2 with respect to positions and
 * masses.  Returns L. */
double orc_direct_plummer_f64(const double *pos, const double *mass, int64_t n, double eps,
                              double G, double *phi, double *acc, double *g_pos, double *g_mass) {
    const double e2 = eps * eps;
    double L = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : L)
    for (int64_t i = 0; i < n; ++i) {
        double ph = 0, ax = 0, ay = 0, az = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            double rx = pos[3 * i] - pos[3 * j], ry = pos[3 * i + 1] - pos[3 * j + 1],
                   rz = pos[3 * i + 2] - pos[3 * j + 2];
            double s2 = rx * rx + ry * ry + rz * rz + e2;
            double i1 = 1.0 / sqrt(s2), i3 = i1 * i1 * i1;
            ph -= mass[j] * i1;
            ax -= mass[j] * rx * i3; ay -= mass[j] * ry * i3; az -= mass[j] * rz * i3;
        }
        phi[i] = G * ph;
        acc[3 * i] = G * ax; acc[3 * i + 1] = G * ay; acc[3 * i + 2] = G * az;
        L += G * ph + 0.5 * G * G * (ax * ax + ay * ay + az * az);
    }
    if (!g_pos) return L;
    /* u_i = 1, v_i = a_i; pair term as field point k and as source k */
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t k = 0; k < n; ++k) {
        double gx = 0, gy = 0, gz = 0, gm = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == k) continue;
            /* k as field point, j as source */
            {
                const double *v = acc + 3 * k;
                double rx = pos[3 * k] - pos[3 * j], ry = pos[3 * k + 1] - pos[3 * j + 1],
                       rz = pos[3 * k + 2] - pos[3 * j + 2];
                double s2 = rx * rx + ry * ry + rz * rz + e2;
                double i1 = 1.0 / sqrt(s2), i3 = i1 * i1 * i1, i5 = i3 * i1 * i1;
                double vr = v[0] * rx + v[1] * ry + v[2] * rz, m = mass[j];
                gx += G * (m * rx * i3 - m * (v[0] * i3 - 3 * vr * rx * i5));
                gy += G * (m * ry * i3 - m * (v[1] * i3 - 3 * vr * ry * i5));
                gz += G * (m * rz * i3 - m * (v[2] * i3 - 3 * vr * rz * i5));
            }
            /* j as field point, k as source */
            {
                const double *v = acc + 3 * j;
                double rx = pos[3 * j] - pos[3 * k], ry = pos[3 * j + 1] - pos[3 * k + 1],
                       rz = pos[3 * j + 2] - pos[3 * k + 2];
                double s2 = rx * rx + ry * ry + rz * rz + e2;
                double i1 = 1.0 / sqrt(s2), i3 = i1 * i1 * i1, i5 = i3 * i1 * i1;
                double vr = v[0] * rx + v[1] * ry + v[2] * rz, m = mass[k];
                gx -= G * (m * rx * i3 - m * (v[0] * i3 - 3 * vr * rx * i5));
                gy -= G * (m * ry * i3 - m * (v[1] * i3 - 3 * vr * ry * i5));
                gz -= G * (m * rz * i3 - m * (v[2] * i3 - 3 * vr * rz * i5));
                gm += G * (-i1 - vr * i3);
            }
        }
        g_pos[3 * k] = gx; g_pos[3 * k + 1] = gy; g_pos[3 * k + 2] = gz;
        if (g_mass) g_mass[k] = gm;
    }
    return L;
}

/* FP64 direct sum of the Plummer potential and acceleration (as
 * orc_direct_plummer_f64) at the listed targets only, from FP32 inputs:
 * the BH-vs-direct error of a large run on a subsample of its bodies. */
void orc_direct_plummer_at_f64(const float *pos, const float *mass, int64_t n, double eps,
                               double G, const int64_t *targets, int64_t nt, double *phi,
                               double *acc) {
    const double e2 = eps * eps;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t i = targets[t];
        const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
        double ph = 0, ax = 0, ay = 0, az = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            double rx = px - pos[3 * j], ry = py - pos[3 * j + 1], rz = pz - pos[3 * j + 2];
            double s2 = rx * rx + ry * ry + rz * rz + e2;
            double i1 = 1.0 / sqrt(s2), i3 = i1 * i1 * i1;
            double m = mass[j];
            ph -= m * i1;
            ax -= m * rx * i3; ay -= m * ry * i3; az -= m * rz * i3;
        }
        phi[t] = G * ph;
        acc[3 * t] = G * ax; acc[3 * t + 1] = G * ay; acc[3 * t + 2] = G * az;
    }
}

/* ------------------------------------------------------------------------
 * DBSCAN over the range-query membership (FP32 key <= RN(eps*eps), the
 * point itself included).  The reference advertises DBSCAN on top of its
 * push-to-buffer range search (README.md:13) but ships no implementation;
 * this follows the published algorithm (Ester et al., 1996) with the
 * labelling order of scikit-learn's DBSCAN, the reference validators'
 * library:
 *   - core point: at least min_pts neighbours;
 *   - clusters are numbered 0, 1, ... in the order of their smallest core
 *     point, expanded one at a time;
 *   - a non-core neighbour of a core point takes the first cluster that
 *     reaches it, i.e. the smallest label among its core neighbours;
 *   - everything else is noise (-1).
 * Brute force, O(n^2): test sizes only.  Returns the number of clusters.
 * ---------------------------------------------------------------------- */
int64_t orc_dbscan(const float *pts, int64_t n, float eps, uint32_t min_pts, int32_t *labels) {
    const float r2 = eps * eps;
    uint8_t *core = (uint8_t *)calloc((size_t)(n > 0 ? n : 1), 1);
    int64_t *stack = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c = 0;
        for (int64_t j = 0; j < n; ++j)
            if (orc_key(pts + 3 * i, pts + 3 * j) <= r2) ++c;
        core[i] = c >= min_pts;
    }
    for (int64_t i = 0; i < n; ++i) labels[i] = -1;
    int32_t next = 0;
    for (int64_t s = 0; s < n; ++s) {
        if (labels[s] != -1 || !core[s]) continue;
        // a point takes the label of the cluster whose expansion first
        // reaches it; labelling it when it is pushed keeps each point on the
        // stack at most once (only one cluster expands at a time, so the
        // label is the same as labelling it when popped)
        int64_t sp = 0;
        labels[s] = next;
        stack[sp++] = s;
        while (sp > 0) {
            const int64_t i = stack[--sp];
            if (!core[i]) continue;
            for (int64_t j = 0; j < n; ++j)
                if (labels[j] == -1 && orc_key(pts + 3 * i, pts + 3 * j) <= r2) {
                    labels[j] = next;
                    stack[sp++] = j;
                }
        }
        ++next;
    }
    free(core);
    free(stack);
    return next;
}

/* ------------------------------------------------------------------------
 * Exact k-NN and range membership at full size: a k-d tree over the points
 * that returns exactly what the brute-force orc_knn / orc_range_* return
 * (the k smallest (FP32 key, id) pairs; every id with key <= RN(r*r)), in
 * O(log n) per query, so the large configurations can be checked on every
 * query rather than a sample.
 *
 * Pruning is exact, with no tolerance.  For a box [lo, hi] and a query q,
 * the box key is the FP32 key of the clamped point c = clamp(q, lo, hi),
 * computed with the same rounded operations as orc_key.  For any point p in
 * the box, |q_a - p_a| >= |q_a - c_a| on each axis, and round-to-nearest is
 * monotone, so |RN(q_a - p_a)| >= |RN(q_a - c_a)|; squaring and the two
 * rounded additions are monotone in non-negative operands, so
 * key(q, p) >= key(q, c).  A subtree is skipped only when its box key is
 * strictly greater than the current k-th key (an equal key with a lower id
 * could still enter) or than RN(r*r).  NaN anywhere makes a comparison
 * false, so such a box is never skipped.
 *
 * Layout: balanced tree in heap order (node i has children 2i+1, 2i+2),
 * median split along the widest axis, leaves of <= ORC_KD_LEAF points.
 * Points with a NaN coordinate are left out: their key is NaN for every
 * query and neither brute-force routine selects them.
 * ---------------------------------------------------------------------- */
#define ORC_KD_LEAF 16

typedef struct { float lo[3], hi[3]; uint32_t begin, end; } orc_kd_node;

typedef struct orc_kdtree {
    int64_t n;            /* points in the tree (NaN points excluded) */
    int depth;            /* leaves sit at this depth (root = 0) */
    int64_t n_nodes;
    orc_kd_node *nodes;
    float *xyz;           /* points in tree order */
    uint32_t *ids;        /* original index of each tree-order point */
} orc_kdtree;

static void orc_kd_select(float *xyz, uint32_t *ids, int64_t lo, int64_t hi, int64_t kth,
                          int axis) {
    /* quickselect on [lo, hi): element kth in place, smaller (or equal)
     * coordinates before it, larger (or equal) after */
    while (hi - lo > 1) {
        const int64_t m = lo + (hi - lo) / 2;
        float a = xyz[3 * lo + axis], b = xyz[3 * m + axis], c = xyz[3 * (hi - 1) + axis];
        float pivot = (a < b) ? ((b < c) ? b : (a < c ? c : a)) : ((a < c) ? a : (b < c ? c : b));
        int64_t i = lo, j = hi - 1;
        while (i <= j) {
            while (xyz[3 * i + axis] < pivot) ++i;
            while (xyz[3 * j + axis] > pivot) --j;
            if (i <= j) {
                for (int t = 0; t < 3; ++t) {
                    float v = xyz[3 * i + t]; xyz[3 * i + t] = xyz[3 * j + t]; xyz[3 * j + t] = v;
                }
                uint32_t u = ids[i]; ids[i] = ids[j]; ids[j] = u;
                ++i; --j;
            }
        }
        if (kth <= j) hi = j + 1;
        else if (kth >= i) lo = i;
        else return;
    }
}

static void orc_kd_build_node(orc_kdtree *t, int64_t ni, int d, int64_t b, int64_t e) {
    orc_kd_node *nd = &t->nodes[ni];
    nd->begin = (uint32_t)b; nd->end = (uint32_t)e;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = b; i < e; ++i)
        for (int a = 0; a < 3; ++a) {
            float v = t->xyz[3 * i + a];
            if (v < lo[a]) lo[a] = v;
            if (v > hi[a]) hi[a] = v;
        }
    memcpy(nd->lo, lo, sizeof lo); memcpy(nd->hi, hi, sizeof hi);
    if (d == t->depth) return;
    int axis = 0;
    float ext0 = hi[0] - lo[0], ext1 = hi[1] - lo[1], ext2 = hi[2] - lo[2];
    if (ext1 > ext0) axis = 1;
    if (ext2 > ext0 && ext2 > ext1) axis = 2;
    const int64_t mid = b + (e - b) / 2;
    orc_kd_select(t->xyz, t->ids, b, e, mid, axis);
    if (e - b > 65536) {
#pragma omp task
        orc_kd_build_node(t, 2 * ni + 1, d + 1, b, mid);
#pragma omp task
        orc_kd_build_node(t, 2 * ni + 2, d + 1, mid, e);
#pragma omp taskwait
    } else {
        orc_kd_build_node(t, 2 * ni + 1, d + 1, b, mid);
        orc_kd_build_node(t, 2 * ni + 2, d + 1, mid, e);
    }
}

orc_kdtree *orc_kd_build(const float *pts, int64_t n) {
    orc_kdtree *t = (orc_kdtree *)calloc(1, sizeof(orc_kdtree));
    t->xyz = (float *)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
    t->ids = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) {
        const float *p = pts + 3 * i;
        if (isnan(p[0]) || isnan(p[1]) || isnan(p[2])) continue;
        t->xyz[3 * m] = p[0]; t->xyz[3 * m + 1] = p[1]; t->xyz[3 * m + 2] = p[2];
        t->ids[m] = (uint32_t)i;
        ++m;
    }
    t->n = m;
    if (m == 0) return t;
    int depth = 0;
    while ((m + ((int64_t)1 << depth) - 1) >> depth > ORC_KD_LEAF) ++depth;
    t->depth = depth;
    t->n_nodes = ((int64_t)2 << depth) - 1;
    t->nodes = (orc_kd_node *)malloc(sizeof(orc_kd_node) * (size_t)t->n_nodes);
#pragma omp parallel
#pragma omp single
    orc_kd_build_node(t, 0, 0, 0, m);
    return t;
}

void orc_kd_free(orc_kdtree *t) {
    if (!t) return;
    free(t->nodes); free(t->xyz); free(t->ids); free(t);
}

int64_t orc_kd_size(const orc_kdtree *t) { return t ? t->n : 0; }

/* FP32 key of the box point nearest to q (a lower bound of every key in
 * the box, see above). */
static inline float orc_kd_box_key(const orc_kd_node *nd, const float *q) {
    float c[3];
    for (int a = 0; a < 3; ++a) {
        float v = q[a];
        if (v < nd->lo[a]) v = nd->lo[a];
        if (v > nd->hi[a]) v = nd->hi[a];
        c[a] = v;
    }
    return orc_key(q, c);
}

/* Max-heap on (key, id) for k above ORC_KD_LIST (the root is the k-th). */
#define ORC_KD_LIST 64
static void orc_heap_sift_down(float *hk, uint32_t *hi, int64_t n, int64_t i) {
    while (1) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < n && orc_less(hk[m], hi[m], hk[l], hi[l])) m = l;
        if (r < n && orc_less(hk[m], hi[m], hk[r], hi[r])) m = r;
        if (m == i) return;
        float tk = hk[i]; hk[i] = hk[m]; hk[m] = tk;
        uint32_t ti = hi[i]; hi[i] = hi[m]; hi[m] = ti;
        i = m;
    }
}

typedef struct { float *bk; uint32_t *bi; int64_t cnt; int k; } orc_klist;

static inline float orc_klist_worst(const orc_klist *L, uint32_t *wid) {
    if (L->cnt < L->k) { *wid = ORC_EMPTY; return INFINITY; }
    if (L->k <= ORC_KD_LIST) { *wid = L->bi[L->k - 1]; return L->bk[L->k - 1]; }
    *wid = L->bi[0]; return L->bk[0];
}

static inline void orc_klist_add(orc_klist *L, float key, uint32_t id) {
    const int k = L->k;
    if (k <= ORC_KD_LIST) {
        /* sorted array, unused slots hold (+inf, EMPTY) */
        if (!orc_less(key, id, L->bk[k - 1], L->bi[k - 1])) return;
        int j = k - 1;
        while (j > 0 && orc_less(key, id, L->bk[j - 1], L->bi[j - 1])) {
            L->bk[j] = L->bk[j - 1]; L->bi[j] = L->bi[j - 1]; --j;
        }
        L->bk[j] = key; L->bi[j] = id;
        if (L->cnt < k) ++L->cnt;
        return;
    }
    if (L->cnt < k) {   /* heap insert (sift up) */
        int64_t i = L->cnt++;
        L->bk[i] = key; L->bi[i] = id;
        while (i > 0) {
            int64_t p = (i - 1) / 2;
            if (!orc_less(L->bk[p], L->bi[p], L->bk[i], L->bi[i])) break;
            float tk = L->bk[i]; L->bk[i] = L->bk[p]; L->bk[p] = tk;
            uint32_t ti = L->bi[i]; L->bi[i] = L->bi[p]; L->bi[p] = ti;
            i = p;
        }
        return;
    }
    if (!orc_less(key, id, L->bk[0], L->bi[0])) return;
    L->bk[0] = key; L->bi[0] = id;
    orc_heap_sift_down(L->bk, L->bi, k, 0);
}

/* Writes the list ascending into ids/d2 (k slots, EMPTY / +inf padded). */
static void orc_klist_out(orc_klist *L, uint32_t *ids, float *d2) {
    const int k = L->k;
    if (k > ORC_KD_LIST) {   /* heap sort in place: pop the max to the end */
        int64_t n = L->cnt;
        while (n > 1) {
            float tk = L->bk[0]; L->bk[0] = L->bk[n - 1]; L->bk[n - 1] = tk;
            uint32_t ti = L->bi[0]; L->bi[0] = L->bi[n - 1]; L->bi[n - 1] = ti;
            --n;
            orc_heap_sift_down(L->bk, L->bi, n, 0);
        }
        for (int64_t j = L->cnt; j < k; ++j) { L->bk[j] = INFINITY; L->bi[j] = ORC_EMPTY; }
    }
    for (int j = 0; j < k; ++j) {
        ids[j] = L->bi[j];
        if (d2) d2[j] = L->bk[j];
    }
}

static void orc_kd_knn_one(const orc_kdtree *t, const float *q, orc_klist *L, int64_t *stack) {
    const int k = L->k;
    L->cnt = 0;
    for (int j = 0; j < (k <= ORC_KD_LIST ? k : 0); ++j) { L->bk[j] = INFINITY; L->bi[j] = ORC_EMPTY; }
    if (t->n == 0 || isnan(q[0]) || isnan(q[1]) || isnan(q[2])) return;
    int64_t sp = 0;
    stack[sp++] = 0;
    const int64_t first_leaf = ((int64_t)1 << t->depth) - 1;
    while (sp) {
        const int64_t ni = stack[--sp];
        const orc_kd_node *nd = &t->nodes[ni];
        uint32_t wid;
        const float worst = orc_klist_worst(L, &wid);
        if (orc_kd_box_key(nd, q) > worst) continue;
        if (ni >= first_leaf) {
            for (uint32_t i = nd->begin; i < nd->end; ++i) {
                const float key = orc_key(q, t->xyz + 3 * (size_t)i);
                if (!(key <= INFINITY)) continue;   /* NaN */
                orc_klist_add(L, key, t->ids[i]);
            }
            continue;
        }
        const int64_t l = 2 * ni + 1, r = l + 1;
        const float kl = orc_kd_box_key(&t->nodes[l], q), kr = orc_kd_box_key(&t->nodes[r], q);
        /* near child on top of the stack */
        if (kl <= kr) { stack[sp++] = r; stack[sp++] = l; }
        else { stack[sp++] = l; stack[sp++] = r; }
    }
}

/* Exact k-NN of nq queries: identical to orc_knn's output. */
void orc_kd_knn(const orc_kdtree *t, const float *q, int64_t nq, int k, uint32_t *ids, float *d2) {
    if (k <= 0) return;
#pragma omp parallel
    {
        orc_klist L;
        L.k = k;
        L.bk = (float *)malloc(sizeof(float) * (size_t)k);
        L.bi = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)k);
        int64_t *stack = (int64_t *)malloc(sizeof(int64_t) * (size_t)(2 * t->depth + 4));
#pragma omp for schedule(dynamic, 64)
        for (int64_t qi = 0; qi < nq; ++qi) {
            orc_kd_knn_one(t, q + 3 * qi, &L, stack);
            orc_klist_out(&L, ids + qi * (int64_t)k, d2 ? d2 + qi * (int64_t)k : NULL);
        }
        free(L.bk); free(L.bi); free(stack);
    }
}

/* Visits every tree point with key <= r2 for query q; returns the count and,
 * when out != NULL, writes their ids (unsorted). */
static int64_t orc_kd_range_one(const orc_kdtree *t, const float *q, float r2, uint32_t *out,
                                int64_t *stack) {
    if (t->n == 0) return 0;
    int64_t sp = 0, c = 0;
    stack[sp++] = 0;
    const int64_t first_leaf = ((int64_t)1 << t->depth) - 1;
    while (sp) {
        const int64_t ni = stack[--sp];
        const orc_kd_node *nd = &t->nodes[ni];
        if (orc_kd_box_key(nd, q) > r2) continue;
        if (ni >= first_leaf) {
            for (uint32_t i = nd->begin; i < nd->end; ++i)
                if (orc_key(q, t->xyz + 3 * (size_t)i) <= r2) {
                    if (out) out[c] = t->ids[i];
                    ++c;
                }
            continue;
        }
        stack[sp++] = 2 * ni + 2;
        stack[sp++] = 2 * ni + 1;
    }
    return c;
}

static int orc_cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}

/* Range counts (membership key <= RN(r*r), as orc_range_count). */
int64_t orc_kd_range_count(const orc_kdtree *t, const float *q, int64_t nq, float r,
                           uint32_t *counts) {
    const float r2 = r * r;
    int64_t total = 0;
#pragma omp parallel reduction(+ : total)
    {
        int64_t *stack = (int64_t *)malloc(sizeof(int64_t) * (size_t)(2 * t->depth + 4));
#pragma omp for schedule(dynamic, 64)
        for (int64_t qi = 0; qi < nq; ++qi) {
            const int64_t c = orc_kd_range_one(t, q + 3 * qi, r2, NULL, stack);
            counts[qi] = (uint32_t)c;
            total += c;
        }
        free(stack);
    }
    return total;
}

/* (query, id) pairs sorted by (query, id) at the exclusive offsets of the
 * counts, as orc_range_pairs. */
void orc_kd_range_pairs(const orc_kdtree *t, const float *q, int64_t nq, float r,
                        const uint64_t *offsets, uint32_t *pairs) {
    const float r2 = r * r;
#pragma omp parallel
    {
        int64_t *stack = (int64_t *)malloc(sizeof(int64_t) * (size_t)(2 * t->depth + 4));
        int64_t cap = 1024;
        uint32_t *buf = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)cap);
#pragma omp for schedule(dynamic, 64)
        for (int64_t qi = 0; qi < nq; ++qi) {
            int64_t c = orc_kd_range_one(t, q + 3 * qi, r2, NULL, stack);
            if (c > cap) {
                cap = c;
                buf = (uint32_t *)realloc(buf, sizeof(uint32_t) * (size_t)cap);
            }
            orc_kd_range_one(t, q + 3 * qi, r2, buf, stack);
            qsort(buf, (size_t)c, sizeof(uint32_t), orc_cmp_u32);
            uint64_t o = offsets[qi];
            for (int64_t j = 0; j < c; ++j) {
                pairs[2 * (o + j)] = (uint32_t)qi;
                pairs[2 * (o + j) + 1] = buf[j];
            }
        }
        free(stack); free(buf);
    }
}
