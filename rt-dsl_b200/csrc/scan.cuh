// scan.cuh -- exclusive scan as a count kernel and an apply kernel over
// fixed tiles, for any input read through a functor (sort.cu scans arrays;
// lbvh.cu scans the Karras keep flags computed from the sorted keys).
//
// The count kernel writes each tile's sum and adds it into the sums of its
// group (32 tiles) and super group (32 groups); the apply kernel takes the
// tile's prefix from those three levels (at most 31 + 31 entries and the
// earlier super groups), so no tile waits on another.
#pragma once

#include "sort.cuh"

namespace rtd {
namespace {

// Prefix levels of the tile counts: 32 tiles make a group, 32 groups a
// super group.  A tile's prefix is the sum of at most 31 tile entries, 31
// group entries and the super-group entries before it, all written by an
// earlier kernel.
constexpr uint32_t GROUP_TILES = 32;
constexpr uint32_t SUPER_TILES = GROUP_TILES * 32;

struct Levels {
    uint64_t tiles, groups, supers;
    explicit Levels(uint64_t t)
        : tiles(t), groups(ceil_div(t, GROUP_TILES)), supers(ceil_div(t, SUPER_TILES)) {}
};

// Zeroes words [0, count) of p: a chained kernel in place of a memset, so
// that the kernels on either side stay chained.
__global__ void __launch_bounds__(256) zero_words_kernel(uint32_t *p, uint64_t count) {
    chain_wait();
    for (uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * 256)
        p[i] = 0u;
}
inline rtd_status zero_words(uint32_t *p, uint64_t count, cudaStream_t stream) {
    if (count == 0) return RTD_OK;
    RTD_LAUNCH_CHAINED(zero_words_kernel, dim3(grid_for(count, 256, 148 * 4)), dim3(256), 0, stream, p,
                       count);
    return RTD_OK;
}

// Scan input: an array.
struct ArrayIn {
    const uint32_t *in;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return in[i]; }
};

constexpr int SC_BLOCK = 256;
constexpr int SC_ITEMS = 8;
constexpr int SC_TILE = SC_BLOCK * SC_ITEMS;

// Scan counts: each tile's sum in tsum[tile], added into its group's sum
// and, with more than one super group, its super group's.
template <typename In>
__global__ void __launch_bounds__(SC_BLOCK) scan_count_kernel(const In in, uint64_t n,
                                                              uint64_t *__restrict__ tsum,
                                                              unsigned long long *gsum,
                                                              unsigned long long *ssum, int supers) {
    chain_wait();
    __shared__ uint64_t s_warp[SC_BLOCK / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t tile = blockIdx.x, base = tile * SC_TILE;
    uint64_t sum = 0;
#pragma unroll
    for (int i = 0; i < SC_ITEMS; ++i) {
        const uint64_t idx = base + (uint64_t)i * SC_BLOCK + tid;
        if (idx < n) sum += in(idx);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) s_warp[warp] = sum;
    __syncthreads();
    if (tid == 0) {
        uint64_t t = 0;
#pragma unroll
        for (int w = 0; w < SC_BLOCK / 32; ++w) t += s_warp[w];
        tsum[tile] = t;
        if (t) {
            atomicAdd(&gsum[tile / GROUP_TILES], (unsigned long long)t);
            if (supers > 1) atomicAdd(&ssum[tile / SUPER_TILES], (unsigned long long)t);
        }
    }
}

// Scan output: out[i] = prefix of the tile (the sums of the earlier tiles
// of its group, earlier groups of its super group and earlier super groups)
// + the block's exclusive scan within the tile.  With select != nullptr,
// also select[out[i]] = i for every i with in(i) != 0 (stream compaction
// of the indices of flagged entries).
template <typename In, typename OutT>
__global__ void __launch_bounds__(SC_BLOCK) scan_apply_kernel(
    const In in, OutT *__restrict__ out, uint64_t n, OutT *d_total,
    const uint64_t *__restrict__ tsum, const uint64_t *__restrict__ gsum,
    const uint64_t *__restrict__ ssum, uint64_t ntiles, uint32_t *select) {
    chain_wait();
    __shared__ uint64_t s_io[SC_TILE];
    __shared__ uint64_t s_warp[SC_BLOCK / 32 + 1];
    __shared__ uint64_t s_prefix;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t tile = blockIdx.x, base = tile * SC_TILE;
    if (warp == 0) {
        // lane j reads tile entry j and group entry j of the levels; the
        // super groups are strided over the lanes
        const uint64_t g = tile / GROUP_TILES, s = tile / SUPER_TILES;
        const uint32_t rt = (uint32_t)(tile % GROUP_TILES), rg = (uint32_t)(g % 32);
        uint64_t v = 0;
        if ((uint32_t)lane < rt) v += tsum[g * GROUP_TILES + lane];
        if ((uint32_t)lane < rg) v += gsum[s * 32 + lane];
        for (uint64_t j = lane; j < s; j += 32) v += ssum[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s_prefix = v;
    }
    for (int i = tid; i < SC_TILE; i += SC_BLOCK) {
        uint64_t idx = base + i;
        s_io[i] = idx < n ? (uint64_t)in(idx) : 0ull;
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
    const uint64_t prefix = s_prefix;
    if (tid == 0 && tile == ntiles - 1 && d_total) *d_total = (OutT)(prefix + s_warp[SC_BLOCK / 32]);
    uint64_t run = prefix + s_warp[warp] + x - sum;
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

// Exclusive scan of in(0 .. n) into out (and *d_total, device), with the
// stream compaction above when select != nullptr.
template <typename In, typename OutT>
rtd_status scan_impl(const In in, OutT *out, uint64_t n, OutT *d_total, ScanScratch &scr,
                     cudaStream_t stream, uint32_t *select = nullptr) {
    if (n == 0) {
        if (d_total) RTD_CUDA(cudaMemsetAsync(d_total, 0, sizeof(OutT), stream));
        return RTD_OK;
    }
    const Levels L(ceil_div(n, SC_TILE));
    if (L.tiles >= (1ull << 31)) return fail(RTD_ERR_INVALID_ARGUMENT, "scan: input too large");
    RTD_TRY(scr.sums.reserve((L.tiles + L.groups + L.supers) * sizeof(uint64_t)));
    uint64_t *tsum = scr.sums.as<uint64_t>();
    uint64_t *gsum = tsum + L.tiles, *ssum = gsum + L.groups;
    RTD_TRY(zero_words(reinterpret_cast<uint32_t *>(gsum), 2 * (L.groups + L.supers), stream));
    RTD_LAUNCH_CHAINED(scan_count_kernel<In>, dim3((unsigned)L.tiles), dim3(SC_BLOCK), 0, stream, in,
                       n, tsum, reinterpret_cast<unsigned long long *>(gsum),
                       reinterpret_cast<unsigned long long *>(ssum), (int)L.supers);
    RTD_LAUNCH_CHAINED((scan_apply_kernel<In, OutT>), dim3((unsigned)L.tiles), dim3(SC_BLOCK), 0,
                       stream, in, out, n, d_total, (const uint64_t *)tsum, (const uint64_t *)gsum,
                       (const uint64_t *)ssum, L.tiles, select);
    return RTD_OK;
}

}  // namespace
}  // namespace rtd
