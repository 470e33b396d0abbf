// sort.cuh -- LSD radix sort of (key, u32 value) pairs and an exclusive
// scan, each pass as a count kernel and a scatter kernel over fixed tiles.
//
// Radix sort: each 8-bit pass runs two kernels.  The count kernel writes
// every tile's digit histogram and adds it into the sums of its group (32
// tiles) and super group (32 groups).  The scatter kernel ranks a tile's
// keys with warp ballots, takes each digit's count in the earlier tiles
// from those three levels (at most 31 + 31 entries and the earlier super
// groups, all written by the count kernel) and the digit's global start
// from a block scan of the digit totals (the group or super-group sums),
// and writes each digit run contiguously through shared memory.  No tile
// waits on another, so there is nothing to time out and no chain of waits
// when every tile is resident at once.
#pragma once

#include "common.cuh"

namespace rtd {

struct SortScratch {
    DevBuf counts;    // passes * (tiles + groups + super groups) * 256 u32
};

// Sorts n pairs by bits [begin_bit, end_bit) of the key.  keys/vals hold the
// input; keys_alt/vals_alt are scratch of the same size (all four buffers
// are required).  With vals_iota the input values are taken to be 0..n-1
// and vals is not read.  On return *in_alt tells whether the sorted result
// is in the *_alt buffers.  n must be < 2^30.  With gather_out, the last
// pass writes gather_out[i] = (x, y, z, bits of v) of the i-th sorted value
// v from the xyz triples gather_xyz instead of the sorted values.  d_err
// (the caller's device error word) is not written: no pass waits on
// another tile, so none can give up.
template <typename K>
rtd_status radix_sort_pairs(K *keys, K *keys_alt, uint32_t *vals, uint32_t *vals_alt,
                            bool vals_iota, uint64_t n, int begin_bit, int end_bit,
                            SortScratch &scr, uint32_t *d_err, cudaStream_t stream, bool *in_alt,
                            const float *gather_xyz = nullptr, float4 *gather_out = nullptr);

// Sorts n 64-bit keys of key_bits bits, 32 < key_bits <= 48, with their
// indices as values (stable): one or two passes over the low key_bits - 32
// bits move the 64-bit keys, whose last writes the top 32 bits to k32a, and
// four passes over those 32-bit keys (k32a / k32b) finish the order.  The
// last pass writes sorted_keys[i] = keys[v] for the i-th sorted index v,
// and the index itself to *sorted_vals (one of vals / vals_alt) or, with
// gather_out, the point gather_xyz[v] with v in w (as radix_sort_pairs).
// keys is not modified; keys_alt is scratch for two low passes; all
// buffers hold n entries.
rtd_status radix_sort_split64(const uint64_t *keys, uint64_t *keys_alt, uint32_t *k32a,
                              uint32_t *k32b, uint32_t *vals, uint32_t *vals_alt, uint64_t n,
                              int key_bits, SortScratch &scr, cudaStream_t stream,
                              const float *gather_xyz, float4 *gather_out,
                              uint64_t *sorted_keys, uint32_t **sorted_vals = nullptr);

// out[i] = sum(in[0..i)), out has n entries; *d_total (device) = sum(in).
// As for the sort, d_err is not written.
struct ScanScratch {
    DevBuf sums;      // tiles + groups + super groups u64
};
rtd_status exclusive_scan_u32(const uint32_t *in, uint64_t *out, uint64_t n, uint64_t *d_total,
                              ScanScratch &scr, uint32_t *d_err, cudaStream_t stream);
// Same, 32-bit output (caller guarantees the sum fits).
rtd_status exclusive_scan_u32_32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total,
                                 ScanScratch &scr, uint32_t *d_err, cudaStream_t stream);
// Same for 0/1 flags, also writing select[out[i]] = i where in[i] != 0:
// the indices of the flagged entries in order.
rtd_status exclusive_scan_select_u32(const uint32_t *in, uint32_t *out, uint32_t *select,
                                     uint64_t n, uint32_t *d_total, ScanScratch &scr,
                                     uint32_t *d_err, cudaStream_t stream);

}  // namespace rtd
