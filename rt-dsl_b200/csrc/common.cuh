// common.cuh -- shared helpers for the rt-dsl B200 kernels: status plumbing,
// exact-rounding arithmetic, ordered-float atomics, launch geometry.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <string>
#include <utility>

#include "rtdsl.h"

namespace rtd {

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
rtd_status fail(rtd_status s, const std::string &msg);
rtd_status cuda_fail(cudaError_t e, const char *what);

#define RTD_CUDA(call)                                                  \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return ::rtd::cuda_fail(e_, #call);      \
    } while (0)

// Counts a kernel launch and reports a launch error.
void note_launch();
#define RTD_LAUNCH_CHECK()                                              \
    do {                                                                \
        ::rtd::note_launch();                                           \
        cudaError_t e_ = cudaGetLastError();                            \
        if (e_ != cudaSuccess) return ::rtd::cuda_fail(e_, "kernel launch"); \
    } while (0)

#define RTD_TRY(call)                                                   \
    do {                                                                \
        rtd_status s_ = (call);                                         \
        if (s_ != RTD_OK) return s_;                                    \
    } while (0)

// ------------------------------------------------------- chained launches
// The kernels of one dependent chain (the index build, the search) launch
// with programmatic stream serialization: a kernel's blocks may be
// scheduled while the previous kernel in the stream finishes, and wait in
// chain_wait() (griddepcontrol.wait) until that kernel has completed and
// its writes are visible.  A kernel launched this way calls chain_wait()
// before it reads or writes anything; launched the plain way, the wait
// returns at once.
__device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                  cudaStream_t st, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
#define RTD_LAUNCH_CHAINED(kernel, grid, block, smem, st, ...)                           \
    do {                                                                                \
        ::rtd::note_launch();                                                           \
        cudaError_t e_ = ::rtd::launch_chained(kernel, grid, block, smem, st, __VA_ARGS__); \
        if (e_ != cudaSuccess) return ::rtd::cuda_fail(e_, "kernel launch");           \
    } while (0)

// Device-side error flags (bit mask), written by kernels whose bounded
// loops or waits give up; read by the host at synchronisation points.
enum : uint32_t {
    DEVERR_TIMEOUT = 1u << 0,       // a spin-wait hit its iteration limit
    DEVERR_STACK = 1u << 1,         // traversal stack would overflow
    DEVERR_NOT_CONVERGED = 1u << 2, // radius expansion ran out of rounds
    DEVERR_OVERFLOW = 1u << 3,      // output buffer too small
    DEVERR_DEPTH = 1u << 4,         // tree deeper than the key supports
    DEVERR_MISMATCH = 1u << 5,      // a fill found other hit counts than its count pass
};
rtd_status status_from_deverr(uint32_t flags);

// ---------------------------------------------------------------- sizes
constexpr int NUM_SMS_HINT = 148;
inline int grid_for(uint64_t n, int block, int max_blocks = 148 * 16) {
    uint64_t g = (n + (uint64_t)block - 1) / (uint64_t)block;
    if (g < 1) g = 1;
    if (g > (uint64_t)max_blocks) g = (uint64_t)max_blocks;
    return (int)g;
}
inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Growable device buffer owned by a handle.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    rtd_status reserve(size_t want);
    void release();
    template <typename T> T *as() const { return reinterpret_cast<T *>(ptr); }
    ~DevBuf() { release(); }
};

// ------------------------------------------------ exact FP32 arithmetic
// The squared-distance key of the reference intersection program
// (gprt-macros/src/lib.rs:338-339), q minus p, summed left to right, with
// every operation rounded separately (no FMA contraction).
__device__ __forceinline__ float exact_key(float qx, float qy, float qz, float px, float py,
                                           float pz) {
    float dx = __fsub_rn(qx, px), dy = __fsub_rn(qy, py), dz = __fsub_rn(qz, pz);
    float s = __fmul_rn(dx, dx);
    s = __fadd_rn(s, __fmul_rn(dy, dy));
    s = __fadd_rn(s, __fmul_rn(dz, dz));
    return s;
}

// Lower bound of exact_key over every point inside [lo, hi]: rounding is
// monotone, so each rounded per-axis gap is <= the rounded |q - p|.
__device__ __forceinline__ float box_min_key(float qx, float qy, float qz, float lx, float ly,
                                             float lz, float hx, float hy, float hz) {
    float dx = fmaxf(fmaxf(__fsub_rn(lx, qx), __fsub_rn(qx, hx)), 0.0f);
    float dy = fmaxf(fmaxf(__fsub_rn(ly, qy), __fsub_rn(qy, hy)), 0.0f);
    float dz = fmaxf(fmaxf(__fsub_rn(lz, qz), __fsub_rn(qz, hz)), 0.0f);
    float s = __fmul_rn(dx, dx);
    s = __fadd_rn(s, __fmul_rn(dy, dy));
    s = __fadd_rn(s, __fmul_rn(dz, dz));
    return s;
}

// Upper bound of exact_key over every point inside [lo, hi].
__device__ __forceinline__ float box_max_key(float qx, float qy, float qz, float lx, float ly,
                                             float lz, float hx, float hy, float hz) {
    float dx = fmaxf(fabsf(__fsub_rn(qx, lx)), fabsf(__fsub_rn(qx, hx)));
    float dy = fmaxf(fabsf(__fsub_rn(qy, ly)), fabsf(__fsub_rn(qy, hy)));
    float dz = fmaxf(fabsf(__fsub_rn(qz, lz)), fabsf(__fsub_rn(qz, hz)));
    float s = __fmul_rn(dx, dx);
    s = __fadd_rn(s, __fmul_rn(dy, dy));
    s = __fadd_rn(s, __fmul_rn(dz, dz));
    return s;
}

// (key, id) lexicographic order.
__device__ __forceinline__ bool key_less(float ka, uint32_t ia, float kb, uint32_t ib) {
    return (ka < kb) || (ka == kb && ia < ib);
}

// ------------------------------------------- order-preserving float<->u32
__device__ __forceinline__ uint32_t float_flip(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ inline float float_unflip(uint32_t u) {
    uint32_t v = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(v);
#else
    float f;
    memcpy(&f, &v, 4);
    return f;
#endif
}

// ------------------------------------------------------- Morton codes
// expand_bits / morton, gprt-core/src/morton.rs:4-16 (x<<2 | y<<1 | z).
__host__ __device__ inline uint32_t expand_bits10(uint32_t x) {
    x &= 0x000003ffu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
__host__ __device__ inline uint32_t morton30(uint32_t x, uint32_t y, uint32_t z) {
    return (expand_bits10(x) << 2) | (expand_bits10(y) << 1) | expand_bits10(z);
}
// 21 bits per axis -> 63-bit code, same x<<2 | y<<1 | z interleave.
__host__ __device__ inline uint64_t expand_bits21(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}
__host__ __device__ inline uint64_t morton63(uint32_t x, uint32_t y, uint32_t z) {
    return (expand_bits21(x) << 2) | (expand_bits21(y) << 1) | expand_bits21(z);
}

// Quantise ((v - lo) / ext * scale) as u32 with Rust `as u32` saturation
// (NaN and negatives -> 0), clamped to scale.
__device__ __forceinline__ uint32_t quantize(float v, float lo, float ext, float scale) {
    float t = __fmul_rn(__fdiv_rn(__fsub_rn(v, lo), ext), scale);
    if (!(t > 0.0f)) return 0u;
    if (t >= scale) return (uint32_t)scale;
    return (uint32_t)t;
}

// Bounded spin-waits.  A device wait on another block's progress must count
// its retries with spin_more, which backs off and returns false once
// `limit` retries have run out; the waiter then sets DEVERR_TIMEOUT and
// stops waiting, so a wait that can never complete ends the kernel instead
// of hanging the GPU.  (The radix sort and the scans run each pass as a
// count kernel and a scatter kernel and wait on no other block.)
constexpr uint32_t SPIN_LIMIT = 1u << 24;
__device__ __forceinline__ bool spin_more(uint32_t &spins, uint32_t limit) {
    if (++spins > limit) return false;
    __nanosleep(20);
    return true;
}

}  // namespace rtd
