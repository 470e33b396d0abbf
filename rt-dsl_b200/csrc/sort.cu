// sort.cu -- LSD radix sort of (key, u32 value) pairs and exclusive scan,
// both as a count kernel and a scatter kernel over fixed tiles (sort.cuh).
#include "sort.cuh"
#include "scan.cuh"

namespace rtd {

namespace {

constexpr int RS_BLOCK = 256;
constexpr int RS_WARPS = RS_BLOCK / 32;
constexpr int RS_ITEMS = 12;
constexpr int RS_TILE = RS_BLOCK * RS_ITEMS;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread over a 256-thread block.
// s_warp must hold RS_WARPS + 1 entries; ends with __syncthreads().
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t v, uint32_t *s_warp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < RS_WARPS ? s_warp[lane] : 0u;
        uint32_t iw = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, iw, o);
            if (lane >= o) iw += y;
        }
        if (lane < RS_WARPS) s_warp[lane] = iw - w;
        if (lane == RS_WARPS - 1) s_warp[RS_WARPS] = iw;
    }
    __syncthreads();
    uint32_t r = s_warp[warp] + x - v;
    __syncthreads();
    return r;
}

// Lanes of the warp whose 8-bit digit equals this lane's: one ballot per bit.
__device__ __forceinline__ uint32_t digit_peers(uint32_t dig) {
    uint32_t peers = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const bool bit = (dig >> b) & 1u;
        const uint32_t m = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? m : ~m;
    }
    return peers;
}

// For digit d of tile `tile`: the digit's count in the earlier tiles (the
// earlier tiles of its group, the earlier groups of its super group and the
// earlier super groups) in *before, and its count over all tiles (the sum
// of the super-group rows, or of the group rows when there is one super
// group) in *total.  Rows are 256 words apart.
__device__ __forceinline__ void digit_counts(const uint32_t *tcount, const uint32_t *gsum,
                                             const uint32_t *ssum, uint64_t tile, uint32_t groups,
                                             uint32_t supers, uint32_t d, uint32_t *before,
                                             uint32_t *total) {
    const uint64_t g = tile / GROUP_TILES, s = tile / SUPER_TILES;
    const uint32_t rt = (uint32_t)(tile % GROUP_TILES), rg = (uint32_t)(g % 32);
    const uint32_t *tp = tcount + g * GROUP_TILES * 256 + d;
    uint32_t a = 0, b = 0, c = 0, t = 0;
#pragma unroll
    for (uint32_t j = 0; j < GROUP_TILES; ++j) a += j < rt ? tp[j * 256] : 0u;
    if (supers == 1) {
#pragma unroll
        for (uint32_t j = 0; j < 32; ++j) {
            const uint32_t v = j < groups ? gsum[j * 256 + d] : 0u;
            t += v;
            b += j < rg ? v : 0u;
        }
    } else {
        const uint32_t *gp = gsum + s * 32 * 256 + d;
#pragma unroll
        for (uint32_t j = 0; j < 32; ++j) b += j < rg ? gp[j * 256] : 0u;
        for (uint32_t j = 0; j < supers; ++j) {
            const uint32_t v = ssum[j * 256 + d];
            t += v;
            c += j < s ? v : 0u;
        }
    }
    *before = a + b + c;
    *total = t;
}

// Counts of one pass: the digit histogram of each tile of RS_TILE keys in
// tcount[tile][d], added into its group's row of gsum and, when there is
// more than one super group, into its super group's row of ssum.  Each
// warp counts its keys in a private shared row with shared-memory atomics
// (measured faster here than ballot-matched counting).
template <typename K>
__global__ void __launch_bounds__(RS_BLOCK) rs_count_kernel(const K *__restrict__ kin, uint64_t n,
                                                            int shift, uint32_t *__restrict__ tcount,
                                                            uint32_t *gsum, uint32_t *ssum,
                                                            int supers) {
    chain_wait();
    __shared__ uint32_t s_wh[RS_WARPS][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < RS_WARPS * 256; i += RS_BLOCK) (&s_wh[0][0])[i] = 0;
    const uint64_t tile = blockIdx.x;
    const uint64_t wbase = tile * RS_TILE + (uint64_t)warp * RS_ITEMS * 32;
    K key[RS_ITEMS];
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint64_t idx = wbase + (uint64_t)i * 32 + lane;
        key[i] = idx < n ? kin[idx] : K(0);
    }
    __syncthreads();
    uint32_t *wh = s_wh[warp];
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const bool ok = wbase + (uint64_t)i * 32 + lane < n;
        const uint32_t dig = (uint32_t)(key[i] >> shift) & 255u;
        if (ok) atomicAdd(&wh[dig], 1u);
    }
    __syncthreads();
    const uint32_t d = (uint32_t)tid;
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) c += s_wh[w][d];
    tcount[tile * 256 + d] = c;
    if (c) {
        atomicAdd(&gsum[(tile / GROUP_TILES) * 256 + d], c);
        if (supers > 1) atomicAdd(&ssum[(tile / SUPER_TILES) * 256 + d], c);
    }
}

// Values of the split sort with the low key bits packed above the index:
// with bits != 0, the first pass makes v = index | (key & low_mask) << bits
// (index < 2^bits), and the last pass takes the index and rebuilds the full
// key (top << low) | (v >> bits) without reading the keys again.  With
// bits = 0 values are plain indices.
struct ValuePack {
    uint32_t bits = 0, low = 0;
    uint64_t low_mask = 0;
    __device__ __forceinline__ uint32_t make(uint64_t idx, uint64_t key) const {
        return bits ? (uint32_t)idx | ((uint32_t)(key & low_mask) << bits) : (uint32_t)idx;
    }
    __device__ __forceinline__ uint32_t index(uint32_t v) const {
        return bits ? v & ((1u << bits) - 1u) : v;
    }
    __device__ __forceinline__ uint64_t key(uint64_t top, uint32_t v) const {
        return (top << low) | (uint64_t)(v >> bits);
    }
};

// Scatter of one pass over 8 bits at `shift`: the tile's keys are ranked
// in registers (stable: warp, item, lane order), staged in shared memory
// grouped by digit, and each digit run is written contiguously from the
// digit's global start plus the count of the digit in earlier tiles (the
// count kernel's levels).  Outputs at the key's new slot dst: kout[dst] =
// key (kout may be null); with kout32, kout32[dst] = the key's bits from
// shift32 up (a 64-bit key becoming the 32-bit key of later passes); with
// gk_out, gk_out[dst] = gk_in[v] for the key's value v; and vout[dst] = v,
// or with gout (the last pass) the point gxyz[v] with v in w instead.
template <typename K>
__global__ void __launch_bounds__(RS_BLOCK) rs_scatter_kernel(
    const K *__restrict__ kin, K *__restrict__ kout, const uint32_t *__restrict__ vin,
    uint32_t *__restrict__ vout, uint64_t n, int shift, const uint32_t *__restrict__ tcount,
    const uint32_t *__restrict__ gsum, const uint32_t *__restrict__ ssum, uint32_t groups,
    uint32_t supers, const float *__restrict__ gxyz, float4 *__restrict__ gout,
    uint32_t *__restrict__ kout32, int shift32, const uint64_t *__restrict__ gk_in,
    uint64_t *__restrict__ gk_out, const ValuePack pk) {
    chain_wait();
    extern __shared__ __align__(16) unsigned char rs_smem[];
    K *s_keys = reinterpret_cast<K *>(rs_smem);
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + RS_TILE);
    uint32_t *s_wh = s_vals + RS_TILE;            // [RS_WARPS][256]
    uint32_t *s_excl = s_wh + RS_WARPS * 256;     // [256] tile-local digit start
    uint32_t *s_base = s_excl + 256;              // [256] global dest of local pos 0 (mod 2^32)
    uint32_t *s_misc = s_base + 256;              // [RS_WARPS + 1]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < RS_WARPS * 256; i += RS_BLOCK) s_wh[i] = 0;
    const uint64_t tile = blockIdx.x;
    const uint64_t base = tile * RS_TILE;

    K key[RS_ITEMS];
    uint32_t val[RS_ITEMS], rank[RS_ITEMS];
    const uint64_t wbase = base + (uint64_t)warp * RS_ITEMS * 32;
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint64_t idx = wbase + (uint64_t)i * 32 + lane;
        const bool ok = idx < n;
        key[i] = ok ? kin[idx] : ~K(0);
        val[i] = ok ? (vin ? vin[idx] : pk.make(idx, (uint64_t)key[i])) : 0u;
    }
    const uint32_t d = (uint32_t)tid;
    uint32_t before, total;
    digit_counts(tcount, gsum, ssum, tile, groups, supers, d, &before, &total);
    // the digit's global start: exclusive scan of the digit totals
    const uint32_t digit_start = block_excl_scan256(total, s_misc);
    const uint32_t lt = lanemask_lt();
    uint32_t *wh = s_wh + warp * 256;
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint32_t dig = (uint32_t)(key[i] >> shift) & 255u;
        const uint32_t peers = digit_peers(dig);
        const uint32_t below = __popc(peers & lt);
        const uint32_t cnt = wh[dig];
        rank[i] = cnt + below;
        __syncwarp();
        if (below == 0) wh[dig] = cnt + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // Per digit (thread = digit): exclusive scan over warps, tile total.
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) {
        const uint32_t t = s_wh[w * 256 + d];
        s_wh[w * 256 + d] = run;
        run += t;
    }
    const uint32_t excl_local = block_excl_scan256(run, s_misc);
    s_excl[d] = excl_local;
    s_base[d] = digit_start + before - excl_local;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint32_t dig = (uint32_t)(key[i] >> shift) & 255u;
        const uint32_t lp = s_excl[dig] + s_wh[warp * 256 + dig] + rank[i];
        s_keys[lp] = key[i];
        s_vals[lp] = val[i];
    }
    __syncthreads();
    const uint64_t rem = n - base;
    const uint32_t valid = rem < (uint64_t)RS_TILE ? (uint32_t)rem : (uint32_t)RS_TILE;
    if (gout) {
        // Last pass with a gather: the points (and keys) are read at random,
        // so GATHER slots' loads are issued together before their stores.
        constexpr int GATHER = 4;
        for (uint32_t j0 = tid; j0 < valid; j0 += GATHER * RS_BLOCK) {
            uint32_t v[GATHER], dst[GATHER];
            float x[GATHER], y[GATHER], z[GATHER];
            uint64_t gk[GATHER];
#pragma unroll
            for (int u = 0; u < GATHER; ++u) {
                const uint32_t j = j0 + u * RS_BLOCK;
                const uint32_t jj = j < valid ? j : j0;   // a repeat of slot j0: not stored
                const K k = s_keys[jj];
                dst[u] = s_base[(uint32_t)(k >> shift) & 255u] + jj;
                const uint32_t w = s_vals[jj];
                v[u] = pk.index(w);
                const uint64_t o = v[u];
                x[u] = gxyz[3 * o];
                y[u] = gxyz[3 * o + 1];
                z[u] = gxyz[3 * o + 2];
                gk[u] = !gk_out ? 0ull : pk.bits ? pk.key((uint64_t)k, w) : gk_in[o];
                if (j < valid) {
                    if (kout) kout[dst[u]] = k;
                    if (kout32) kout32[dst[u]] = (uint32_t)((uint64_t)k >> shift32);
                }
            }
#pragma unroll
            for (int u = 0; u < GATHER; ++u) {
                if (j0 + u * RS_BLOCK < valid) {
                    gout[dst[u]] = make_float4(x[u], y[u], z[u], __uint_as_float(v[u]));
                    if (gk_out) gk_out[dst[u]] = gk[u];
                }
            }
        }
        return;
    }
    for (uint32_t j = tid; j < valid; j += RS_BLOCK) {
        const K k = s_keys[j];
        const uint32_t dj = (uint32_t)(k >> shift) & 255u;
        const uint32_t dst = s_base[dj] + j;
        if (kout) kout[dst] = k;
        if (kout32) kout32[dst] = (uint32_t)((uint64_t)k >> shift32);
        const uint32_t w = s_vals[j];
        if (gk_out) {   // the last pass: full keys, values unpacked
            const uint32_t v = pk.index(w);
            gk_out[dst] = pk.bits ? pk.key((uint64_t)k, w) : gk_in[v];
            vout[dst] = v;
        } else {
            vout[dst] = w;
        }
    }
}

size_t rs_scatter_smem(size_t key_bytes) {
    return RS_TILE * (key_bytes + 4) + (RS_WARPS * 256 + 512 + RS_WARPS + 1) * 4;
}

// Count rows for `passes` passes over n keys: every pass's tile rows, then
// every pass's group and super rows (zeroed together: the count kernels add
// into them).
struct PassRows {
    Levels L;
    uint32_t *tc = nullptr, *sc = nullptr;
    explicit PassRows(uint64_t n) : L(ceil_div(n, RS_TILE)) {}
    rtd_status reserve(SortScratch &scr, int passes, cudaStream_t stream) {
        const size_t trows = (size_t)passes * L.tiles, srows = (size_t)passes * (L.groups + L.supers);
        RTD_TRY(scr.counts.reserve((trows + srows) * 256 * sizeof(uint32_t)));
        tc = scr.counts.as<uint32_t>();
        sc = tc + trows * 256;
        RTD_TRY(zero_words(sc, srows * 256, stream));
        return RTD_OK;
    }
};

// Outputs of one pass besides the values (see rs_scatter_kernel).
template <typename K> struct PassOut {
    K *kout = nullptr;
    uint32_t *kout32 = nullptr;
    int shift32 = 0;
    const float *gxyz = nullptr;
    float4 *gout = nullptr;
    const uint64_t *gk_in = nullptr;
    uint64_t *gk_out = nullptr;
    ValuePack pk;
};

// Count + scatter of pass p (its count rows) over bits [shift, shift + 8).
template <typename K>
rtd_status run_pass(const PassRows &R, int p, const K *kin, const uint32_t *vin, uint32_t *vout,
                    uint64_t n, int shift, const PassOut<K> &o, cudaStream_t stream) {
    const Levels &L = R.L;
    uint32_t *tcount = R.tc + (size_t)p * L.tiles * 256;
    uint32_t *gsum = R.sc + (size_t)p * (L.groups + L.supers) * 256;
    uint32_t *ssum = gsum + L.groups * 256;
    RTD_LAUNCH_CHAINED(rs_count_kernel<K>, dim3((unsigned)L.tiles), dim3(RS_BLOCK), 0, stream, kin,
                       n, shift, tcount, gsum, ssum, (int)L.supers);
    const size_t smem = rs_scatter_smem(sizeof(K));
    RTD_CUDA(cudaFuncSetAttribute(rs_scatter_kernel<K>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    RTD_LAUNCH_CHAINED(rs_scatter_kernel<K>, dim3((unsigned)L.tiles), dim3(RS_BLOCK), smem, stream,
                       kin, o.kout, vin, vout, n, shift, tcount, gsum, ssum, (uint32_t)L.groups,
                       (uint32_t)L.supers, o.gxyz, o.gout, o.kout32, o.shift32, o.gk_in, o.gk_out,
                       o.pk);
    return RTD_OK;
}

}  // namespace

template <typename K>
rtd_status radix_sort_pairs(K *keys, K *keys_alt, uint32_t *vals, uint32_t *vals_alt,
                            bool vals_iota, uint64_t n, int begin_bit, int end_bit,
                            SortScratch &scr, uint32_t *d_err, cudaStream_t stream, bool *in_alt,
                            const float *gather_xyz, float4 *gather_out) {
    (void)d_err;   // no pass waits on another tile: nothing can time out
    *in_alt = false;
    if (n == 0) return RTD_OK;
    if (n >= (1ull << 30)) return fail(RTD_ERR_INVALID_ARGUMENT, "radix sort: n must be < 2^30");
    const int passes = (end_bit - begin_bit + 7) / 8;
    if (passes <= 0 || passes > 8 || end_bit > (int)(8 * sizeof(K)))
        return fail(RTD_ERR_INVALID_ARGUMENT, "radix sort: bad bit range");
    PassRows R(n);
    RTD_TRY(R.reserve(scr, passes, stream));
    K *kin = keys, *kout = keys_alt;
    uint32_t *vin = vals, *vout = vals_alt;
    for (int p = 0; p < passes; ++p) {
        PassOut<K> o;
        o.kout = kout;
        if (p == passes - 1) {
            o.gxyz = gather_xyz;
            o.gout = gather_out;
        }
        // Pass 0 with vals_iota generates the values 0..n-1 on the fly.
        RTD_TRY(run_pass<K>(R, p, kin, (p == 0 && vals_iota) ? nullptr : vin, vout, n,
                            begin_bit + 8 * p, o, stream));
        K *tk = kin; kin = kout; kout = tk;
        uint32_t *tv = vin; vin = vout; vout = tv;
        *in_alt = !*in_alt;
    }
    return RTD_OK;
}

rtd_status radix_sort_split64(const uint64_t *keys, uint64_t *keys_alt, uint32_t *k32a,
                              uint32_t *k32b, uint32_t *vals, uint32_t *vals_alt, uint64_t n,
                              int key_bits, SortScratch &scr, cudaStream_t stream,
                              const float *gather_xyz, float4 *gather_out,
                              uint64_t *sorted_keys, uint32_t **sorted_vals) {
    if (n == 0) return RTD_OK;
    if (n >= (1ull << 30)) return fail(RTD_ERR_INVALID_ARGUMENT, "radix sort: n must be < 2^30");
    if (key_bits <= 32 || key_bits > 48)
        return fail(RTD_ERR_INVALID_ARGUMENT, "split radix sort: key_bits must be in (32, 48]");
    const int low = key_bits - 32;          // bits [0, low) sort as 64-bit keys
    const int lp = (low + 7) / 8;           // 1 or 2 passes
    // the low key bits ride above the index in the values when they fit
    ValuePack pk;
    uint32_t ib = 1;
    while (ib < 32 && (1ull << ib) < n) ++ib;
    if (ib + (uint32_t)low <= 32) {
        pk.bits = ib;
        pk.low = (uint32_t)low;
        pk.low_mask = (1ull << low) - 1ull;
    }
    PassRows R(n);
    RTD_TRY(R.reserve(scr, lp + 4, stream));
    const uint32_t *vin = nullptr;          // pass 0: values 0..n-1 on the fly
    uint32_t *vout = vals;
    // low passes; the last writes the top 32 bits as the next passes' keys
    const uint64_t *kin = keys;
    for (int p = 0; p < lp; ++p) {
        PassOut<uint64_t> o;
        if (p == 0) o.pk = pk;   // makes the values
        if (p == lp - 1) {
            o.kout32 = k32a;
            o.shift32 = low;
        } else {
            o.kout = keys_alt;
        }
        RTD_TRY(run_pass<uint64_t>(R, p, kin, vin, vout, n, 8 * p, o, stream));
        kin = keys_alt;
        vin = vout;
        vout = vout == vals ? vals_alt : vals;
    }
    // top passes on 32-bit keys; the last gathers the points and the full keys
    uint32_t *k32in = k32a, *k32out = k32b;
    for (int p = 0; p < 4; ++p) {
        PassOut<uint32_t> o;
        if (p == 3) {
            o.gxyz = gather_xyz;
            o.gout = gather_out;
            o.gk_in = keys;
            o.gk_out = sorted_keys;
            o.pk = pk;   // unpacks the values, rebuilds the keys
        } else {
            o.kout = k32out;
        }
        RTD_TRY(run_pass<uint32_t>(R, lp + p, k32in, vin, vout, n, 8 * p, o, stream));
        if (p == 3 && sorted_vals) *sorted_vals = gather_out ? nullptr : vout;
        uint32_t *t = k32in; k32in = k32out; k32out = t;
        vin = vout;
        vout = vout == vals ? vals_alt : vals;
    }
    return RTD_OK;
}

template rtd_status radix_sort_pairs<uint32_t>(uint32_t *, uint32_t *, uint32_t *, uint32_t *,
                                               bool, uint64_t, int, int, SortScratch &,
                                               uint32_t *, cudaStream_t, bool *, const float *,
                                               float4 *);
template rtd_status radix_sort_pairs<uint64_t>(uint64_t *, uint64_t *, uint32_t *, uint32_t *,
                                               bool, uint64_t, int, int, SortScratch &,
                                               uint32_t *, cudaStream_t, bool *, const float *,
                                               float4 *);

rtd_status exclusive_scan_u32(const uint32_t *in, uint64_t *out, uint64_t n, uint64_t *d_total,
                              ScanScratch &scr, uint32_t *d_err, cudaStream_t stream) {
    (void)d_err;
    return scan_impl<ArrayIn, uint64_t>(ArrayIn{in}, out, n, d_total, scr, stream);
}
rtd_status exclusive_scan_u32_32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total,
                                 ScanScratch &scr, uint32_t *d_err, cudaStream_t stream) {
    (void)d_err;
    return scan_impl<ArrayIn, uint32_t>(ArrayIn{in}, out, n, d_total, scr, stream);
}
rtd_status exclusive_scan_select_u32(const uint32_t *in, uint32_t *out, uint32_t *select,
                                     uint64_t n, uint32_t *d_total, ScanScratch &scr,
                                     uint32_t *d_err, cudaStream_t stream) {
    (void)d_err;
    return scan_impl<ArrayIn, uint32_t>(ArrayIn{in}, out, n, d_total, scr, stream, select);
}

}  // namespace rtd
