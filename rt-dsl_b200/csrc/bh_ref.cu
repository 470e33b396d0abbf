// bh_ref.cu -- the reference-law Barnes-Hut walk over the octree of
// bh_tree.cu: the intended walk of the reference's OptiX programs
// (gprt-macros/src/lib.rs:760-806), one thread per body, stackless over
// next = p + 1 / autorope, every operation rounded separately so the forces
// are bit-identical to the CPU restatement.
#include <rtdsl.h>

#include "bh.cuh"

namespace rtd {
namespace {

// ----------------------------------------------------- reference law
__device__ __forceinline__ float dot3_rn(float x, float y, float z) {
    float s = __fmul_rn(x, x);
    s = __fadd_rn(s, __fmul_rn(y, y));
    s = __fadd_rn(s, __fmul_rn(z, z));
    return s;
}

__global__ void __launch_bounds__(128) bh_ref_walk_kernel(const BhView v, float theta, float G,
                                                          float *__restrict__ out) {
    const uint32_t n_nodes = v.hdr->n_nodes;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < v.n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 me = v.fbody[i];
        const float px = me.x, py = me.y, pz = me.z;
        const float gm = __fmul_rn(G, me.w);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        uint32_t p = 0;
        while (p < n_nodes) {
            const float4 a = __ldg(&v.node_a[p]);
            const uint4 b = __ldg(&v.node_b[p]);
            const float dx = __fsub_rn(a.x, px), dy = __fsub_rn(a.y, py), dz = __fsub_rn(a.z, pz);
            const float dist_sq = dot3_rn(dx, dy, dz);
            const float d = __fsqrt_rn(dist_sq);
            const float tmax = __fadd_rn(fmaxf(1e-6f, __fmul_rn(theta, d)), 1e-5f);
            const bool hit = __uint_as_float(b.w) < tmax;
            if (b.z & BH_LEAF_BIT) {
                const uint32_t s = b.y, c = b.z & ~BH_LEAF_BIT;
                for (uint32_t j = 0; j < c; ++j) {
                    const float4 o = __ldg(&v.fbody[s + j]);
                    const float ex = __fsub_rn(o.x, px), ey = __fsub_rn(o.y, py), ez = __fsub_rn(o.z, pz);
                    const float d2 = dot3_rn(ex, ey, ez);
                    if (d2 > 1e-10f) {
                        const float denom = __fmul_rn(d2, __fsqrt_rn(__fadd_rn(d2, 1e-6f)));
                        const float fm = __fdiv_rn(__fmul_rn(gm, o.w), denom);
                        sx = __fadd_rn(sx, __fmul_rn(ex, fm));
                        sy = __fadd_rn(sy, __fmul_rn(ey, fm));
                        sz = __fadd_rn(sz, __fmul_rn(ez, fm));
                    }
                }
                p = hit ? b.x : p + 1;
            } else if (hit) {
                if (dist_sq > 1e-10f) {
                    const float denom = __fmul_rn(dist_sq, __fsqrt_rn(__fadd_rn(dist_sq, 1e-6f)));
                    const float fm = __fdiv_rn(__fmul_rn(gm, a.w), denom);
                    sx = __fadd_rn(sx, __fmul_rn(dx, fm));
                    sy = __fadd_rn(sy, __fmul_rn(dy, fm));
                    sz = __fadd_rn(sz, __fmul_rn(dz, fm));
                }
                p = b.x;
            } else {
                p = p + 1;
            }
        }
        const uint32_t o = v.order[i];
        out[3 * (uint64_t)o] = sx;
        out[3 * (uint64_t)o + 1] = sy;
        out[3 * (uint64_t)o + 2] = sz;
    }
}

}  // namespace

rtd_status bh_ref_forward(rtd_bh *b, const rtd_bh_params *p, float *d_out, cudaStream_t st) {
    const BhView v = bh_view(b);
    bh_ref_walk_kernel<<<grid_for(b->n, 128, 1 << 20), 128, 0, st>>>(v, p->theta, p->G, d_out);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

}  // namespace rtd
