// bh_walk.cu -- Barnes-Hut tree walks over the octree of bh_tree.cu.
//
//  * Reference law: the intended walk of the reference's OptiX programs
//    (gprt-macros/src/lib.rs:760-806), one thread per body, stackless over
//    next = p + 1 / autorope, every operation rounded separately so the
//    forces are bit-identical to the CPU restatement.
//  * Plummer law, forward: one warp per 32 consecutive bodies (flat order),
//    one shared walk with a group MAC (width^2 < theta^2 * dist^2(COM,
//    group box)); node and leaf-body loads are warp-uniform broadcasts and
//    each lane accumulates its own acceleration and potential.
//  * Plummer law, adjoint: the same walk and decisions; each lane adds the
//    derivative of its interactions with respect to its own position and
//    the warp reduces the source-side derivatives (body position and mass,
//    or cell COM / mass / quadrupole) before one vector atomic per source.
//    A top-down pass then turns cell derivatives into body derivatives:
//    with Q about the COM the first moment vanishes, so for cell C and
//    member body j
//        dL/dx_j += m_j (g_c/M - 2 B c + 2 B x_j)
//        dL/dm_j += g_M + g_c.(x_j - c)/M + (x_j-c)^T B (x_j-c)
//    with B = 3 sym(G_Q) - tr(G_Q) I; these sums split into per-node
//    constants that accumulate along root-to-leaf paths.
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

// ------------------------------------------------------ Plummer law
struct Group {
    float lo[3], hi[3];
};

__device__ __forceinline__ Group group_box(float x, float y, float z, bool valid) {
    Group g;
    float p[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
        float lo = valid ? p[a] : INFINITY, hi = valid ? p[a] : -INFINITY;
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        g.lo[a] = lo;
        g.hi[a] = hi;
    }
    return g;
}

// Group MAC: accept the cell when width^2 < theta^2 * dist^2(COM, group box).
__device__ __forceinline__ bool group_accept(const Group &g, float cx, float cy, float cz,
                                             float width, float theta2) {
    float tx = fmaxf(fmaxf(__fsub_rn(g.lo[0], cx), __fsub_rn(cx, g.hi[0])), 0.0f);
    float ty = fmaxf(fmaxf(__fsub_rn(g.lo[1], cy), __fsub_rn(cy, g.hi[1])), 0.0f);
    float tz = fmaxf(fmaxf(__fsub_rn(g.lo[2], cz), __fsub_rn(cz, g.hi[2])), 0.0f);
    float d2 = dot3_rn(tx, ty, tz);
    return __fmul_rn(width, width) < __fmul_rn(theta2, d2);
}

__device__ __forceinline__ float warp_sum(float x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

template <bool QUAD>
__global__ void __launch_bounds__(128) bh_plummer_fwd_kernel(const BhView v, float theta2,
                                                             float eps2, float G,
                                                             float *__restrict__ acc_out,
                                                             float *__restrict__ phi_out) {
    const uint32_t n_nodes = v.hdr->n_nodes;
    const int lane = threadIdx.x & 31;
    const uint64_t ngroups = (v.n + BH_GROUP - 1) / BH_GROUP;
    for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups;
         g += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint64_t i = g * BH_GROUP + lane;
        const bool valid = i < v.n;
        const float4 me = valid ? v.fbody[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const Group box = group_box(me.x, me.y, me.z, valid);
        float ax = 0.f, ay = 0.f, az = 0.f, phi = 0.f;
        uint32_t p = 0;
        while (p < n_nodes) {
            const float4 a = __ldg(&v.node_a[p]);
            const uint4 b = __ldg(&v.node_b[p]);
            if (group_accept(box, a.x, a.y, a.z, __uint_as_float(b.w), theta2)) {
                const float rx = me.x - a.x, ry = me.y - a.y, rz = me.z - a.z;
                const float s = rx * rx + ry * ry + rz * rz + eps2;
                const float i1 = rsqrtf(s), i2 = i1 * i1, i3 = i1 * i2;
                phi -= a.w * i1;
                ax -= a.w * rx * i3;
                ay -= a.w * ry * i3;
                az -= a.w * rz * i3;
                if (QUAD) {
                    const float4 q0 = __ldg(&v.node_q[2 * p]), q1 = __ldg(&v.node_q[2 * p + 1]);
                    const float qx = q0.x * rx + q0.w * ry + q1.x * rz;
                    const float qy = q0.w * rx + q0.y * ry + q1.y * rz;
                    const float qz = q1.x * rx + q1.y * ry + q0.z * rz;
                    const float q = rx * qx + ry * qy + rz * qz;
                    const float i5 = i3 * i2, i7 = i5 * i2;
                    phi -= 0.5f * q * i5;
                    ax += qx * i5 - 2.5f * q * rx * i7;
                    ay += qy * i5 - 2.5f * q * ry * i7;
                    az += qz * i5 - 2.5f * q * rz * i7;
                }
                p = b.x;
            } else if (b.z & BH_LEAF_BIT) {
                const uint32_t s0 = b.y, c = b.z & ~BH_LEAF_BIT;
                for (uint32_t j = 0; j < c; ++j) {
                    const float4 o = __ldg(&v.fbody[s0 + j]);
                    if (s0 + j == i) continue;
                    const float rx = me.x - o.x, ry = me.y - o.y, rz = me.z - o.z;
                    const float s = rx * rx + ry * ry + rz * rz + eps2;
                    const float i1 = rsqrtf(s), i3 = i1 * i1 * i1;
                    phi -= o.w * i1;
                    ax -= o.w * rx * i3;
                    ay -= o.w * ry * i3;
                    az -= o.w * rz * i3;
                }
                p = p + 1;
            } else {
                p = p + 1;
            }
        }
        if (valid) {
            const uint32_t o = v.order[i];
            acc_out[3 * (uint64_t)o] = G * ax;
            acc_out[3 * (uint64_t)o + 1] = G * ay;
            acc_out[3 * (uint64_t)o + 2] = G * az;
            if (phi_out) phi_out[o] = G * phi;
        }
    }
}

// Cell-gradient record (12 floats = 3 float4): g_c.xyz, g_M | G_Q xx yy zz xy | xz yz, 0, 0.
template <bool QUAD>
__global__ void __launch_bounds__(128) bh_plummer_adj_kernel(
    const BhView v, float theta2, float eps2, float G, const float *__restrict__ g_acc,
    const float *__restrict__ g_phi, float4 *__restrict__ cell_grad,
    float4 *__restrict__ body_grad /* flat: dL/dx, dL/dm */) {
    const uint32_t n_nodes = v.hdr->n_nodes;
    const int lane = threadIdx.x & 31;
    const uint64_t ngroups = (v.n + BH_GROUP - 1) / BH_GROUP;
    for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups;
         g += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint64_t i = g * BH_GROUP + lane;
        const bool valid = i < v.n;
        const float4 me = valid ? v.fbody[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const Group box = group_box(me.x, me.y, me.z, valid);
        float vx = 0.f, vy = 0.f, vz = 0.f, u = 0.f;
        if (valid) {
            const uint32_t o = v.order[i];
            vx = g_acc[3 * (uint64_t)o];
            vy = g_acc[3 * (uint64_t)o + 1];
            vz = g_acc[3 * (uint64_t)o + 2];
            u = g_phi ? g_phi[o] : 0.f;
        }
        float gx = 0.f, gy = 0.f, gz = 0.f;
        uint32_t p = 0;
        while (p < n_nodes) {
            const float4 a = __ldg(&v.node_a[p]);
            const uint4 b = __ldg(&v.node_b[p]);
            if (group_accept(box, a.x, a.y, a.z, __uint_as_float(b.w), theta2)) {
                const float rx = me.x - a.x, ry = me.y - a.y, rz = me.z - a.z;
                const float s = rx * rx + ry * ry + rz * rz + eps2;
                const float i1 = rsqrtf(s), i2 = i1 * i1, i3 = i1 * i2, i5 = i3 * i2;
                const float M = a.w;
                const float vr = vx * rx + vy * ry + vz * rz;
                // monopole: a = -M r i3, phi = -M i1
                float grx = u * M * rx * i3 - M * (vx * i3 - 3.f * vr * rx * i5);
                float gry = u * M * ry * i3 - M * (vy * i3 - 3.f * vr * ry * i5);
                float grz = u * M * rz * i3 - M * (vz * i3 - 3.f * vr * rz * i5);
                float gM = -u * i1 - vr * i3;
                float gq[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (QUAD) {
                    const float4 q0 = __ldg(&v.node_q[2 * p]), q1 = __ldg(&v.node_q[2 * p + 1]);
                    const float Qxx = q0.x, Qyy = q0.y, Qzz = q0.z, Qxy = q0.w, Qxz = q1.x, Qyz = q1.y;
                    const float qrx = Qxx * rx + Qxy * ry + Qxz * rz;
                    const float qry = Qxy * rx + Qyy * ry + Qyz * rz;
                    const float qrz = Qxz * rx + Qyz * ry + Qzz * rz;
                    const float qvx = Qxx * vx + Qxy * vy + Qxz * vz;
                    const float qvy = Qxy * vx + Qyy * vy + Qyz * vz;
                    const float qvz = Qxz * vx + Qyz * vy + Qzz * vz;
                    const float q = rx * qrx + ry * qry + rz * qrz;
                    const float vqr = vx * qrx + vy * qry + vz * qrz;
                    const float i7 = i5 * i2, i9 = i7 * i2;
                    // a_Q = Qr i5 - 2.5 q r i7, phi_Q = -0.5 q i5
                    const float ax_q = qrx * i5 - 2.5f * q * rx * i7;
                    const float ay_q = qry * i5 - 2.5f * q * ry * i7;
                    const float az_q = qrz * i5 - 2.5f * q * rz * i7;
                    // -u dphi_Q/dr = u a_Q ... (dphi/dr = -a), so u*dphi_Q/dr = -u a_Q
                    grx += -u * ax_q;
                    gry += -u * ay_q;
                    grz += -u * az_q;
                    // d(v.a_Q)/dr = Qv i5 - 5 vQr r i7 - 2.5(2 Qr vr i7 + q v i7 - 7 q vr r i9)
                    grx += qvx * i5 - 5.f * vqr * rx * i7 - 2.5f * (2.f * qrx * vr * i7 + q * vx * i7 - 7.f * q * vr * rx * i9);
                    gry += qvy * i5 - 5.f * vqr * ry * i7 - 2.5f * (2.f * qry * vr * i7 + q * vy * i7 - 7.f * q * vr * ry * i9);
                    grz += qvz * i5 - 5.f * vqr * rz * i7 - 2.5f * (2.f * qrz * vr * i7 + q * vz * i7 - 7.f * q * vr * rz * i9);
                    // dL/dQ (symmetric part): -0.5 u i5 rr^T + i5 sym(v r^T) - 2.5 vr i7 rr^T
                    const float cr = -0.5f * u * i5 - 2.5f * vr * i7;
                    gq[0] = cr * rx * rx + i5 * vx * rx;
                    gq[1] = cr * ry * ry + i5 * vy * ry;
                    gq[2] = cr * rz * rz + i5 * vz * rz;
                    gq[3] = cr * rx * ry + 0.5f * i5 * (vx * ry + vy * rx);
                    gq[4] = cr * rx * rz + 0.5f * i5 * (vx * rz + vz * rx);
                    gq[5] = cr * ry * rz + 0.5f * i5 * (vy * rz + vz * ry);
                }
                // monopole phi term: u * dphi_M/dr = u * M r i3 (already in grx)
                gx += G * grx;
                gy += G * gry;
                gz += G * grz;
                // source side, reduced over the warp (invalid lanes contribute 0)
                float sx = valid ? -G * grx : 0.f, sy = valid ? -G * gry : 0.f,
                      sz = valid ? -G * grz : 0.f, sm = valid ? G * gM : 0.f;
                sx = warp_sum(sx); sy = warp_sum(sy); sz = warp_sum(sz); sm = warp_sum(sm);
                if (QUAD)
                    for (int t = 0; t < 6; ++t) gq[t] = warp_sum(valid ? G * gq[t] : 0.f);
                if (lane == 0) {
                    atomicAdd(&cell_grad[3 * p], make_float4(sx, sy, sz, sm));
                    if (QUAD) {
                        atomicAdd(&cell_grad[3 * p + 1], make_float4(gq[0], gq[1], gq[2], gq[3]));
                        atomicAdd(&cell_grad[3 * p + 2], make_float4(gq[4], gq[5], 0.f, 0.f));
                    }
                }
                p = b.x;
            } else if (b.z & BH_LEAF_BIT) {
                const uint32_t s0 = b.y, c = b.z & ~BH_LEAF_BIT;
                for (uint32_t j = 0; j < c; ++j) {
                    const float4 o = __ldg(&v.fbody[s0 + j]);
                    const bool use = valid && (s0 + j != i);
                    const float rx = me.x - o.x, ry = me.y - o.y, rz = me.z - o.z;
                    const float s = rx * rx + ry * ry + rz * rz + eps2;
                    const float i1 = rsqrtf(s), i2 = i1 * i1, i3 = i1 * i2, i5 = i3 * i2;
                    const float vr = vx * rx + vy * ry + vz * rz;
                    const float m = o.w;
                    float grx = G * (u * m * rx * i3 - m * (vx * i3 - 3.f * vr * rx * i5));
                    float gry = G * (u * m * ry * i3 - m * (vy * i3 - 3.f * vr * ry * i5));
                    float grz = G * (u * m * rz * i3 - m * (vz * i3 - 3.f * vr * rz * i5));
                    float gm = G * (-u * i1 - vr * i3);
                    if (!use) { grx = gry = grz = gm = 0.f; }
                    gx += grx;
                    gy += gry;
                    gz += grz;
                    const float sx = warp_sum(-grx), sy = warp_sum(-gry), sz = warp_sum(-grz),
                                sm = warp_sum(gm);
                    if (lane == 0) atomicAdd(&body_grad[s0 + j], make_float4(sx, sy, sz, sm));
                }
                p = p + 1;
            } else {
                p = p + 1;
            }
        }
        if (valid) atomicAdd(&body_grad[i], make_float4(gx, gy, gz, 0.f));
    }
}

// Top-down: per node the constants of the cell-to-body rule, summed along
// root-to-node paths; then each leaf applies its path sums to its bodies.
// prefix record (12 floats): Pvec.xyz, Pconst | Pmat xx yy zz xy | xz yz.
__device__ __forceinline__ void cell_constants(const float4 a, const float4 *cg, float out[10]) {
    const float4 g0 = cg[0], g1 = cg[1], g2 = cg[2];
    const float M = a.w, cx = a.x, cy = a.y, cz = a.z;
    const float Gxx = g1.x, Gyy = g1.y, Gzz = g1.z, Gxy = g1.w, Gxz = g2.x, Gyz = g2.y;
    const float tr = Gxx + Gyy + Gzz;
    const float Bxx = 3.f * Gxx - tr, Byy = 3.f * Gyy - tr, Bzz = 3.f * Gzz - tr;
    const float Bxy = 3.f * Gxy, Bxz = 3.f * Gxz, Byz = 3.f * Gyz;
    const float Bcx = Bxx * cx + Bxy * cy + Bxz * cz;
    const float Bcy = Bxy * cx + Byy * cy + Byz * cz;
    const float Bcz = Bxz * cx + Byz * cy + Bzz * cz;
    const float invM = M > 0.f ? 1.f / M : 0.f;
    out[0] = g0.x * invM - 2.f * Bcx;
    out[1] = g0.y * invM - 2.f * Bcy;
    out[2] = g0.z * invM - 2.f * Bcz;
    out[3] = g0.w - (g0.x * cx + g0.y * cy + g0.z * cz) * invM + (cx * Bcx + cy * Bcy + cz * Bcz);
    out[4] = Bxx; out[5] = Byy; out[6] = Bzz; out[7] = Bxy; out[8] = Bxz; out[9] = Byz;
}

__global__ void __launch_bounds__(1024) bh_prefix_kernel(const BhView v,
                                                         const uint32_t *__restrict__ level_nodes,
                                                         const float4 *__restrict__ cell_grad,
                                                         float4 *prefix) {
    const BhHeader *h = v.hdr;
    for (int l = 0; l <= BH_MAX_LEVEL + 1; ++l) {
        const uint32_t off = h->level_off[l], cnt = h->level_count[l];
        for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) {
            const uint32_t i = level_nodes[off + t];
            float own[10];
            cell_constants(v.node_a[i], cell_grad + 3 * i, own);
            // prefix[i] holds the parent's path sum (zero at the root)
            float4 p0 = l == 0 ? make_float4(0.f, 0.f, 0.f, 0.f) : prefix[3 * i];
            float4 p1 = l == 0 ? make_float4(0.f, 0.f, 0.f, 0.f) : prefix[3 * i + 1];
            float4 p2 = l == 0 ? make_float4(0.f, 0.f, 0.f, 0.f) : prefix[3 * i + 2];
            p0 = make_float4(p0.x + own[0], p0.y + own[1], p0.z + own[2], p0.w + own[3]);
            p1 = make_float4(p1.x + own[4], p1.y + own[5], p1.z + own[6], p1.w + own[7]);
            p2 = make_float4(p2.x + own[8], p2.y + own[9], 0.f, 0.f);
            prefix[3 * i] = p0;
            prefix[3 * i + 1] = p1;
            prefix[3 * i + 2] = p2;
            const uint4 b = v.node_b[i];
            if (!(b.z & BH_LEAF_BIT))
                for (uint32_t c = i + 1; c < b.x; c = v.node_b[c].x) {
                    prefix[3 * c] = p0;
                    prefix[3 * c + 1] = p1;
                    prefix[3 * c + 2] = p2;
                }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(128) bh_finish_grad_kernel(const BhView v,
                                                             const float4 *__restrict__ prefix,
                                                             const float4 *__restrict__ body_grad,
                                                             float *__restrict__ g_pos,
                                                             float *__restrict__ g_mass) {
    const uint32_t n_nodes = v.hdr->n_nodes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x) {
        const uint4 b = v.node_b[i];
        if (!(b.z & BH_LEAF_BIT)) continue;
        const float4 p0 = prefix[3 * i], p1 = prefix[3 * i + 1], p2 = prefix[3 * i + 2];
        const float Pxx = p1.x, Pyy = p1.y, Pzz = p1.z, Pxy = p1.w, Pxz = p2.x, Pyz = p2.y;
        const uint32_t s0 = b.y, c = b.z & ~BH_LEAF_BIT;
        for (uint32_t k = 0; k < c; ++k) {
            const float4 o = v.fbody[s0 + k];
            const float Px = Pxx * o.x + Pxy * o.y + Pxz * o.z;
            const float Py = Pxy * o.x + Pyy * o.y + Pyz * o.z;
            const float Pz = Pxz * o.x + Pyz * o.y + Pzz * o.z;
            const float4 bg = body_grad[s0 + k];
            const uint32_t orig = v.order[s0 + k];
            g_pos[3 * (uint64_t)orig] = bg.x + o.w * (p0.x + 2.f * Px);
            g_pos[3 * (uint64_t)orig + 1] = bg.y + o.w * (p0.y + 2.f * Py);
            g_pos[3 * (uint64_t)orig + 2] = bg.z + o.w * (p0.z + 2.f * Pz);
            if (g_mass)
                g_mass[orig] = bg.w + p0.w + (p0.x * o.x + p0.y * o.y + p0.z * o.z) +
                               (o.x * Px + o.y * Py + o.z * Pz);
        }
    }
}

}  // namespace

rtd_status bh_forward(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                      cudaStream_t st) {
    if (!b || !b->built) return fail(RTD_ERR_INVALID_ARGUMENT, "bh tree not built");
    if (b->n && !d_out) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL output");
    rtd_bh_params def;
    rtd_bh_params_default(&def);
    if (!p) p = &def;
    if (b->n == 0) return RTD_OK;
    const BhView v = bh_view(b);
    if (p->law == RTD_BH_LAW_REFERENCE) {
        bh_ref_walk_kernel<<<grid_for(b->n, 128, 1 << 20), 128, 0, st>>>(v, p->theta, p->G, d_out);
    } else if (p->law == RTD_BH_LAW_PLUMMER) {
        const uint64_t warps = (b->n + BH_GROUP - 1) / BH_GROUP;
        const int grid = grid_for(warps * 32, 128, 1 << 20);
        const float th2 = p->theta * p->theta, e2 = p->eps * p->eps;
        if (p->quadrupole)
            bh_plummer_fwd_kernel<true><<<grid, 128, 0, st>>>(v, th2, e2, p->G, d_out, d_phi);
        else
            bh_plummer_fwd_kernel<false><<<grid, 128, 0, st>>>(v, th2, e2, p->G, d_out, d_phi);
    } else {
        return fail(RTD_ERR_INVALID_ARGUMENT, "unknown law");
    }
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

rtd_status bh_backward(rtd_bh *b, const rtd_bh_params *p, const float *g_acc, const float *g_phi,
                       float *g_pos, float *g_mass, cudaStream_t st) {
    if (!b || !b->built) return fail(RTD_ERR_INVALID_ARGUMENT, "bh tree not built");
    rtd_bh_params def;
    rtd_bh_params_default(&def);
    if (!p) p = &def;
    if (p->law != RTD_BH_LAW_PLUMMER)
        return fail(RTD_ERR_UNSUPPORTED, "the adjoint is defined for the Plummer law");
    if (b->n == 0) return RTD_OK;
    if (!g_acc || !g_pos) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL gradient buffer");
    const uint64_t n = b->n;
    RTD_TRY(b->cell_grad.reserve(n * 3 * sizeof(float4) + 64 * sizeof(uint32_t)));
    RTD_TRY(b->prefix.reserve(n * 3 * sizeof(float4)));
    RTD_TRY(b->gpos_flat.reserve(n * sizeof(float4)));
    // cell_grad also holds the build's level counters at its start; they
    // are not needed after the build.
    RTD_CUDA(cudaMemsetAsync(b->cell_grad.ptr, 0, n * 3 * sizeof(float4), st));
    RTD_CUDA(cudaMemsetAsync(b->gpos_flat.ptr, 0, n * sizeof(float4), st));
    const BhView v = bh_view(b);
    const uint64_t warps = (n + BH_GROUP - 1) / BH_GROUP;
    const int grid = grid_for(warps * 32, 128, 1 << 20);
    const float th2 = p->theta * p->theta, e2 = p->eps * p->eps;
    if (p->quadrupole)
        bh_plummer_adj_kernel<true><<<grid, 128, 0, st>>>(v, th2, e2, p->G, g_acc, g_phi,
                                                          b->cell_grad.as<float4>(),
                                                          b->gpos_flat.as<float4>());
    else
        bh_plummer_adj_kernel<false><<<grid, 128, 0, st>>>(v, th2, e2, p->G, g_acc, g_phi,
                                                           b->cell_grad.as<float4>(),
                                                           b->gpos_flat.as<float4>());
    RTD_LAUNCH_CHECK();
    bh_prefix_kernel<<<1, 1024, 0, st>>>(v, b->level_nodes.as<uint32_t>(),
                                          b->cell_grad.as<float4>(), b->prefix.as<float4>());
    RTD_LAUNCH_CHECK();
    bh_finish_grad_kernel<<<grid_for(n, 128, 1 << 20), 128, 0, st>>>(
        v, b->prefix.as<float4>(), b->gpos_flat.as<float4>(), g_pos, g_mass);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

}  // namespace rtd
