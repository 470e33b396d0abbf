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
#include <rtdsl.h>

#include "bh.cuh"

namespace rtd {
rtd_status bh_forward_on_stack(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                               uint2 *stack, uint64_t max_warps, cudaStream_t st);
}  // namespace rtd

using namespace rtd;

// 592 warp stacks (148 SMs x one block of 4 warps) of BH_STACK_CAP_MAX = 8192
// entries of 8 bytes: 37 MiB per device.
static constexpr uint64_t NOALLOC_WARPS = 592;
static __device__ __align__(256) uint2 g_noalloc_walk_stack[NOALLOC_WARPS * BH_STACK_CAP_MAX];

namespace {
// Device address of the stack array in the current context.  The host
// symbol g_noalloc_walk_stack is only a stand-in for it.  The address is
// looked up on every call, with the caller's device current: a table
// lookup in the CUDA runtime once the module is loaded, and always the
// address in the context the walk will run in (a cached address would go
// stale after cudaDeviceReset, or under another context of the same device).
// The first lookup in a context loads this file's module, which places the
// 37 MiB array on the device: that is the one time the entry point takes
// device memory, through the module loader rather than cudaMalloc.
rtd_status stack_address(uint2 **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_walk_stack);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
    *out = static_cast<uint2 *>(p);
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
