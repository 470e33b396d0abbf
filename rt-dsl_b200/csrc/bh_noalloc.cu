// bh_noalloc.cu -- the Plummer-law Barnes-Hut forward walk without any
// device allocation.
//
// The walk keeps a traversal stack per warp in global memory.
// rtd_bh_forward reserves that stack from the CUDA allocator the first time
// a tree needs it; some callers cannot let a library call cudaMalloc: a host
// whose memory manager owns all device memory and hands out only its own
// buffers, or a step loop that must not stall on the device-wide
// synchronisation cudaMalloc / cudaFree can cause.  rtd_bh_forward_noalloc
// runs the same walk kernel on a stack that lives in the fixed array below,
// which the CUDA module loader places on each device that loads this
// library's code and keeps there until the process exits.
#include <mutex>

#include <rtdsl.h>

#include "bh.cuh"

namespace rtd {
rtd_status bh_forward_on_stack(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                               uint2 *stack, uint64_t max_warps, cudaStream_t st);
}  // namespace rtd

using namespace rtd;

// 592 warp stacks (148 SMs x one block of 4 warps) of BH_STACK_CAP = 8192
// entries of 8 bytes: 37 MiB per device.
static constexpr uint64_t NOALLOC_WARPS = 592;
static __device__ __align__(256) uint2 g_noalloc_walk_stack[NOALLOC_WARPS * BH_STACK_CAP];

namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
uint2 *g_stack_addr[MAX_DEVICES] = {};   // device address of the array, per device

// Device address of the stack array on the current device.  The host symbol
// g_noalloc_walk_stack is only a stand-in for it; the address is looked up
// once per device, with that device current.
rtd_status stack_address(uint2 **out) {
    int dev = 0;
    RTD_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES)
        return fail(RTD_ERR_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_stack_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_walk_stack);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
        g_stack_addr[dev] = static_cast<uint2 *>(p);
    }
    *out = g_stack_addr[dev];
    return RTD_OK;
}
}  // namespace

extern "C" rtd_status rtd_bh_forward_noalloc(rtd_bh *b, const rtd_bh_params *p, float *d_out,
                                             float *d_phi, rtd_stream stream) {
    if (!b) return fail(RTD_ERR_INVALID_ARGUMENT, "bh is NULL");
    uint2 *stack = nullptr;
    RTD_TRY(stack_address(&stack));
    return bh_forward_on_stack(b, p, d_out, d_phi, stack, NOALLOC_WARPS, (cudaStream_t)stream);
}
