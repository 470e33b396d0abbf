// sort.cu -- onesweep radix sort and decoupled look-back scan (see sort.cuh).
#include "sort.cuh"

namespace rtd {

namespace {

constexpr int RS_BLOCK = 256;
constexpr int RS_WARPS = RS_BLOCK / 32;
constexpr int RS_ITEMS = 12;
constexpr int RS_TILE = RS_BLOCK * RS_ITEMS;
constexpr uint32_t FLAG_AGG = 1u << 30;
constexpr uint32_t FLAG_INC = 2u << 30;
constexpr uint32_t VALUE_MASK = (1u << 30) - 1;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread over a 256-thread block.
// s_warp must hold RS_WARPS entries; ends with __syncthreads().
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t v, uint32_t *s_warp,
                                                       uint32_t *total) {
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
    if (total) *total = s_warp[RS_WARPS];
    __syncthreads();
    return r;
}

template <typename K>
__global__ void __launch_bounds__(RS_BLOCK) rs_hist_kernel(const K *__restrict__ keys, uint64_t n,
                                                           int begin_bit, int passes,
                                                           uint32_t *__restrict__ hist) {
    __shared__ uint32_t sh[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += RS_BLOCK) (&sh[0][0])[i] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * RS_BLOCK + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * RS_BLOCK) {
        K k = keys[i];
        for (int p = 0; p < passes; ++p)
            atomicAdd(&sh[p][(uint32_t)(k >> (begin_bit + 8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += RS_BLOCK) {
        uint32_t c = (&sh[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// In place: hist[p][d] counts -> exclusive offsets.
__global__ void __launch_bounds__(RS_BLOCK) rs_hist_scan_kernel(uint32_t *hist, int passes) {
    __shared__ uint32_t s_warp[RS_WARPS + 1];
    for (int p = 0; p < passes; ++p) {
        uint32_t v = hist[p * 256 + threadIdx.x];
        uint32_t e = block_excl_scan256(v, s_warp, nullptr);
        hist[p * 256 + threadIdx.x] = e;
    }
}

template <typename K>
__global__ void __launch_bounds__(RS_BLOCK) rs_pass_kernel(
    const K *__restrict__ kin, K *__restrict__ kout, const uint32_t *__restrict__ vin,
    uint32_t *__restrict__ vout, uint64_t n, int shift, const uint32_t *__restrict__ digit_off,
    uint32_t *status, uint32_t *tile_counter, uint32_t *d_err, const float *__restrict__ gxyz,
    float4 *__restrict__ gout) {
    extern __shared__ __align__(16) unsigned char rs_smem[];
    K *s_keys = reinterpret_cast<K *>(rs_smem);
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + RS_TILE);
    uint32_t *s_wh = s_vals + RS_TILE;            // [RS_WARPS][256]
    uint32_t *s_excl = s_wh + RS_WARPS * 256;     // [256] tile-local digit start
    uint32_t *s_base = s_excl + 256;              // [256] global dest of local pos 0 (mod 2^32)
    uint32_t *s_misc = s_base + 256;              // [RS_WARPS + 2]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_misc[RS_WARPS + 1] = atomicAdd(tile_counter, 1u);
    for (int i = tid; i < RS_WARPS * 256; i += RS_BLOCK) s_wh[i] = 0;
    __syncthreads();
    const uint32_t tile = s_misc[RS_WARPS + 1];
    const uint64_t base = (uint64_t)tile * RS_TILE;

    K key[RS_ITEMS];
    uint32_t val[RS_ITEMS], dig[RS_ITEMS], rank[RS_ITEMS];
    const uint64_t wbase = base + (uint64_t)warp * RS_ITEMS * 32;
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        uint64_t idx = wbase + (uint64_t)i * 32 + lane;
        bool ok = idx < n;
        key[i] = ok ? kin[idx] : ~K(0);
        val[i] = ok ? (vin ? vin[idx] : (uint32_t)idx) : 0u;
        dig[i] = (uint32_t)(key[i] >> shift) & 255u;
    }
    const uint32_t lt = lanemask_lt();
    uint32_t *wh = s_wh + warp * 256;
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        // lanes holding the same digit: one ballot per digit bit
        uint32_t peers = 0xffffffffu;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const bool bit = (dig[i] >> b) & 1u;
            const uint32_t m = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? m : ~m;
        }
        uint32_t before = __popc(peers & lt);
        uint32_t cnt = wh[dig[i]];
        rank[i] = cnt + before;
        __syncwarp();
        if (before == 0) wh[dig[i]] = cnt + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // Per digit (thread = digit): exclusive scan over warps, tile total.
    const uint32_t d = (uint32_t)tid;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) {
        uint32_t t = s_wh[w * 256 + d];
        s_wh[w * 256 + d] = run;
        run += t;
    }
    const uint32_t tile_cnt = run;
    volatile uint32_t *st = status;
    if (tile == 0) st[d] = FLAG_INC | tile_cnt;
    else st[(uint64_t)tile * 256 + d] = FLAG_AGG | tile_cnt;

    uint32_t excl_local = block_excl_scan256(tile_cnt, s_misc, nullptr);
    s_excl[d] = excl_local;

    // Look back over earlier tiles, 8 status words in flight at a time:
    // sum their counts up to the nearest inclusive prefix.
    uint32_t prev = 0;
    if (tile > 0) {
        int64_t t = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (true) {
            uint32_t w[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
                w[j] = (t - j >= 0) ? (uint32_t)st[(uint64_t)(t - j) * 256 + d] : (2u << 30);
            int used = 0;
            bool done = false;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (done || used < j) continue;
                uint32_t f = w[j] & ~VALUE_MASK;
                if (f == 0) continue;          // not published yet: retry from here
                prev += w[j] & VALUE_MASK;
                used = j + 1;
                if (f == FLAG_INC) done = true;
            }
            if (done) break;
            t -= used;
            if (used < 8 && !spin_more(spins, SPIN_LIMIT)) {
                atomicOr(d_err, DEVERR_TIMEOUT);
                break;
            }
        }
        st[(uint64_t)tile * 256 + d] = FLAG_INC | ((prev + tile_cnt) & VALUE_MASK);
    }
    s_base[d] = digit_off[d] + prev - excl_local;
    __syncthreads();

#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        uint32_t lp = s_excl[dig[i]] + s_wh[warp * 256 + dig[i]] + rank[i];
        s_keys[lp] = key[i];
        s_vals[lp] = val[i];
    }
    __syncthreads();
    const uint64_t rem = n - base;
    const uint32_t valid = rem < (uint64_t)RS_TILE ? (uint32_t)rem : (uint32_t)RS_TILE;
    for (uint32_t j = tid; j < valid; j += RS_BLOCK) {
        K k = s_keys[j];
        uint32_t dj = (uint32_t)(k >> shift) & 255u;
        uint32_t dst = s_base[dj] + j;
        kout[dst] = k;
        const uint32_t v = s_vals[j];
        if (gout) {   // last pass with a gather: the point itself, its index in w
            const uint64_t o = v;
            gout[dst] = make_float4(gxyz[3 * o], gxyz[3 * o + 1], gxyz[3 * o + 2], __uint_as_float(v));
        } else {
            vout[dst] = v;
        }
    }
}

size_t rs_pass_smem(size_t key_bytes) {
    return RS_TILE * (key_bytes + 4) + (RS_WARPS * 256 + 512 + RS_WARPS + 2) * 4;
}

// ----------------------------------------------------------------- scan
constexpr int SC_BLOCK = 256;
constexpr int SC_ITEMS = 8;
constexpr int SC_TILE = SC_BLOCK * SC_ITEMS;
constexpr uint64_t SC_AGG = 1ull << 62;
constexpr uint64_t SC_INC = 2ull << 62;
constexpr uint64_t SC_MASK = (1ull << 62) - 1;

// With select != nullptr, also select[out[i]] = i for every i with in[i] != 0
// (stream compaction of the indices of flagged entries).
template <typename OutT>
__global__ void __launch_bounds__(SC_BLOCK) scan_kernel(const uint32_t *__restrict__ in,
                                                        OutT *__restrict__ out, uint64_t n,
                                                        OutT *d_total, uint64_t *status,
                                                        uint32_t *counter, uint32_t ntiles,
                                                        uint32_t *d_err, uint32_t *select) {
    __shared__ uint64_t s_io[SC_TILE];
    __shared__ uint64_t s_warp[SC_BLOCK / 32 + 1];
    __shared__ uint64_t s_prefix;
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * SC_TILE;
    for (int i = tid; i < SC_TILE; i += SC_BLOCK) {
        uint64_t idx = base + i;
        s_io[i] = idx < n ? (uint64_t)in[idx] : 0ull;
    }
    __syncthreads();
    uint64_t v[SC_ITEMS];
    uint64_t sum = 0;
#pragma unroll
    for (int i = 0; i < SC_ITEMS; ++i) {
        v[i] = s_io[tid * SC_ITEMS + i];
        sum += v[i];
    }
    // block exclusive scan of 64-bit sums
    uint64_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < SC_BLOCK / 32 ? s_warp[lane] : 0ull;
        uint64_t iw = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, iw, o);
            if (lane >= o) iw += y;
        }
        if (lane < SC_BLOCK / 32) s_warp[lane] = iw - w;
        if (lane == SC_BLOCK / 32 - 1) s_warp[SC_BLOCK / 32] = iw;
    }
    __syncthreads();
    const uint64_t excl = s_warp[warp] + x - sum;
    const uint64_t agg = s_warp[SC_BLOCK / 32];
    // Warp-cooperative look-back: lane j reads tile (t - j); the nearest
    // inclusive prefix ends the sum.
    if (warp == 0) {
        volatile uint64_t *st = status;
        uint64_t prev = 0;
        if (tile == 0) {
            if (lane == 0) st[0] = SC_INC | (agg & SC_MASK);
        } else {
            if (lane == 0) st[tile] = SC_AGG | (agg & SC_MASK);
            int64_t t = (int64_t)tile - 1;
            uint32_t spins = 0;
            while (true) {
                const int64_t ti = t - lane;
                uint64_t w = ti >= 0 ? (uint64_t)st[ti] : (2ull << 62);
                while (__any_sync(0xffffffffu, (w & ~SC_MASK) == 0)) {
                    if (!spin_more(spins, SPIN_LIMIT)) break;
                    if ((w & ~SC_MASK) == 0) w = st[ti];
                }
                if (spins > SPIN_LIMIT) {
                    if (lane == 0) atomicOr(d_err, DEVERR_TIMEOUT);
                    break;
                }
                const uint32_t inc = __ballot_sync(0xffffffffu, (w & ~SC_MASK) == SC_INC);
                const int stop = inc ? __ffs(inc) - 1 : 31;
                uint64_t v = lane <= stop ? (w & SC_MASK) : 0ull;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                prev += v;
                if (inc) break;
                t -= 32;
            }
            if (lane == 0) st[tile] = SC_INC | ((prev + agg) & SC_MASK);
        }
        if (lane == 0) {
            s_prefix = prev;
            if (tile == ntiles - 1 && d_total) *d_total = (OutT)(prev + agg);
        }
    }
    __syncthreads();
    uint64_t run = s_prefix + excl;
#pragma unroll
    for (int i = 0; i < SC_ITEMS; ++i) {
        s_io[tid * SC_ITEMS + i] = run;
        if (select && v[i]) select[run] = (uint32_t)(base + (uint64_t)tid * SC_ITEMS + i);
        run += v[i];
    }
    __syncthreads();
    for (int i = tid; i < SC_TILE; i += SC_BLOCK) {
        uint64_t idx = base + i;
        if (idx < n) out[idx] = (OutT)s_io[i];
    }
}

template <typename OutT>
rtd_status scan_impl(const uint32_t *in, OutT *out, uint64_t n, OutT *d_total, ScanScratch &scr,
                     uint32_t *d_err, cudaStream_t stream, uint32_t *select = nullptr) {
    if (n == 0) {
        if (d_total) RTD_CUDA(cudaMemsetAsync(d_total, 0, sizeof(OutT), stream));
        return RTD_OK;
    }
    uint64_t ntiles = ceil_div(n, SC_TILE);
    if (ntiles >= (1ull << 31)) return fail(RTD_ERR_INVALID_ARGUMENT, "scan: input too large");
    RTD_TRY(scr.status.reserve(ntiles * sizeof(uint64_t)));
    RTD_TRY(scr.counter.reserve(sizeof(uint32_t)));
    RTD_CUDA(cudaMemsetAsync(scr.status.ptr, 0, ntiles * sizeof(uint64_t), stream));
    RTD_CUDA(cudaMemsetAsync(scr.counter.ptr, 0, sizeof(uint32_t), stream));
    scan_kernel<OutT><<<(unsigned)ntiles, SC_BLOCK, 0, stream>>>(
        in, out, n, d_total, scr.status.as<uint64_t>(), scr.counter.as<uint32_t>(),
        (uint32_t)ntiles, d_err, select);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

}  // namespace

template <typename K>
rtd_status radix_sort_pairs(K *keys, K *keys_alt, uint32_t *vals, uint32_t *vals_alt,
                            bool vals_iota, uint64_t n, int begin_bit, int end_bit,
                            SortScratch &scr, uint32_t *d_err, cudaStream_t stream, bool *in_alt,
                            const float *gather_xyz, float4 *gather_out) {
    *in_alt = false;
    if (n == 0) return RTD_OK;
    if (n >= (1ull << 30)) return fail(RTD_ERR_INVALID_ARGUMENT, "radix sort: n must be < 2^30");
    const int passes = (end_bit - begin_bit + 7) / 8;
    if (passes <= 0 || passes > 8 || end_bit > (int)(8 * sizeof(K)))
        return fail(RTD_ERR_INVALID_ARGUMENT, "radix sort: bad bit range");
    const uint64_t ntiles = ceil_div(n, RS_TILE);
    RTD_TRY(scr.hist.reserve((size_t)passes * 256 * sizeof(uint32_t)));
    RTD_TRY(scr.status.reserve((size_t)passes * ntiles * 256 * sizeof(uint32_t)));
    RTD_TRY(scr.counters.reserve((size_t)passes * sizeof(uint32_t)));
    RTD_CUDA(cudaMemsetAsync(scr.hist.ptr, 0, (size_t)passes * 256 * 4, stream));
    RTD_CUDA(cudaMemsetAsync(scr.status.ptr, 0, (size_t)passes * ntiles * 256 * 4, stream));
    RTD_CUDA(cudaMemsetAsync(scr.counters.ptr, 0, (size_t)passes * 4, stream));
    rs_hist_kernel<K><<<grid_for(n, RS_BLOCK, 148 * 4), RS_BLOCK, 0, stream>>>(
        keys, n, begin_bit, passes, scr.hist.as<uint32_t>());
    RTD_LAUNCH_CHECK();
    rs_hist_scan_kernel<<<1, RS_BLOCK, 0, stream>>>(scr.hist.as<uint32_t>(), passes);
    RTD_LAUNCH_CHECK();
    const size_t smem = rs_pass_smem(sizeof(K));
    RTD_CUDA(cudaFuncSetAttribute(rs_pass_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    K *kin = keys, *kout = keys_alt;
    uint32_t *vin = vals, *vout = vals_alt;
    for (int p = 0; p < passes; ++p) {
        // Pass 0 with vals_iota generates the values 0..n-1 on the fly.
        rs_pass_kernel<K><<<(unsigned)ntiles, RS_BLOCK, smem, stream>>>(
            kin, kout, (p == 0 && vals_iota) ? nullptr : vin, vout, n, begin_bit + 8 * p,
            scr.hist.as<uint32_t>() + p * 256,
            scr.status.as<uint32_t>() + (size_t)p * ntiles * 256, scr.counters.as<uint32_t>() + p,
            d_err, gather_xyz, p == passes - 1 ? gather_out : nullptr);
        RTD_LAUNCH_CHECK();
        K *tk = kin; kin = kout; kout = tk;
        uint32_t *tv = vin; vin = vout; vout = tv;
        *in_alt = !*in_alt;
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
    return scan_impl<uint64_t>(in, out, n, d_total, scr, d_err, stream);
}
rtd_status exclusive_scan_u32_32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total,
                                 ScanScratch &scr, uint32_t *d_err, cudaStream_t stream) {
    return scan_impl<uint32_t>(in, out, n, d_total, scr, d_err, stream);
}
rtd_status exclusive_scan_select_u32(const uint32_t *in, uint32_t *out, uint32_t *select,
                                     uint64_t n, uint32_t *d_total, ScanScratch &scr,
                                     uint32_t *d_err, cudaStream_t stream) {
    return scan_impl<uint32_t>(in, out, n, d_total, scr, d_err, stream, select);
}

}  // namespace rtd
