// bh_plummer.cu -- Plummer-law Barnes-Hut walks (forward and adjoint).
//
// Physics: phi_i = -G sum_j m_j / sqrt(|x_i - x_j|^2 + eps^2), a_i =
// -grad phi_i; accepted cells act as monopole + traceless quadrupole about
// their COM with the same softened distance.  A cell is accepted for body
// i when width^2 < theta^2 |COM - x_i|^2 (each operation rounded, so the
// CPU oracle makes identical decisions); rejected leaves are summed
// directly, rejected internal cells opened.
//
// Execution: a warp takes a group of <= 32 bodies (packed sibling leaves,
// so spatially compact) and walks the tree once for all of them.  Stack
// entries carry the mask of lanes that still need the node; per step up to
// 32 entries are loaded in parallel and each is tested by every lane in its
// mask.  Accepted cells and the bodies of rejected leaves go to per-warp
// lists with their lane masks; every 32 entries form a tile staged in
// shared memory and evaluated by all lanes from broadcast reads.
//
// Adjoint (dL/dx, dL/dm for upstream dL/da, dL/dphi): per tile, pass 1
// (lane = body) adds d/dx_i of the body's interactions; pass 2 (lane =
// source) sums the source-side derivatives over the group's bodies and
// issues one vector atomic per source.  Cell derivatives (COM, mass,
// quadrupole) are then pushed to the bodies by a top-down pass: with Q
// about the COM the first moment vanishes, so for a cell C holding body j
//     dL/dx_j += m_j (g_c/M - 2 B c + 2 B x_j)
//     dL/dm_j += g_M + g_c.(x_j - c)/M + (x_j - c)^T B (x_j - c)
// with B = 3 sym(G_Q) - tr(G_Q) I; both split into per-node constants that
// add up along root-to-leaf paths.
#include <rtdsl.h>

#include "bh.cuh"

namespace rtd {
namespace {

constexpr int WW = 4;   // warps per block

// Adjoint: source-side derivatives of RED_CELLS cells (3 float4 each) or
// RED_BODIES bodies (1 float4 each) per chunk, one row per lane.

constexpr int RED_CELLS = 3;
constexpr int RED_BODIES = 9;

struct WarpTile {
    float4 cell[32][3];   // (com, M), (Qxx Qyy Qzz Qxy), (Qxz Qyz 0 0)
    uint32_t cmask_t[32];
    float4 body[32];      // (x, y, z, m)
    uint32_t bid[32];
    uint32_t bmask_t[32];
    uint32_t clist[32], cmask[32];
    uint32_t blist[64], bmask[64];
};

// The adjoint's per-chunk table: red[j][lane] = lane's share of source j.
struct WarpRed {
    float4 red[RED_CELLS * 3][32];
};
static_assert(RED_BODIES <= RED_CELLS * 3, "body chunk fits the cell chunk's table");

// Sum of each of `rows` table rows over its 32 entries, L lanes per row:
// lane l takes row l / L and the entries seg, seg + L, seg + 2L, ... of
// it (seg = l % L), rotated by the row so that the lanes of one load phase
// read different banks; the row's lanes then add up by shuffles.  On
// return `owner` marks the row's first lane, which holds the sum.
template <int L>
__device__ __forceinline__ float4 table_row_sum(const WarpRed &R, int rows, int lane, int &row,
                                                bool &owner) {
    constexpr int T = (32 + L - 1) / L;
    row = lane / L;
    const int seg = lane - row * L;
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    if (row < rows) {
#pragma unroll
        for (int i = 0; i < T; ++i) {
            int ii = i + row;
            if (ii >= T) ii -= T;
            const int j = seg + L * ii;
            if (j < 32) {
                const float4 e = R.red[row][j];
                t.x += e.x; t.y += e.y; t.z += e.z; t.w += e.w;
            }
        }
    }
    const float4 t0 = t;
#pragma unroll
    for (int d = 1; d < L; ++d) {
        t.x += __shfl_down_sync(0xffffffffu, t0.x, d);
        t.y += __shfl_down_sync(0xffffffffu, t0.y, d);
        t.z += __shfl_down_sync(0xffffffffu, t0.z, d);
        t.w += __shfl_down_sync(0xffffffffu, t0.w, d);
    }
    owner = row < rows && seg == 0;
    return t;
}

__device__ __forceinline__ float dot3_rn(float x, float y, float z) {
    float s = __fmul_rn(x, x);
    s = __fadd_rn(s, __fmul_rn(y, y));
    s = __fadd_rn(s, __fmul_rn(z, z));
    return s;
}

// Per-body MAC: accept when width^2 < theta^2 * |COM - x|^2.
__device__ __forceinline__ bool body_accept(float x, float y, float z, float cx, float cy, float cz,
                                            float width, float theta2) {
    const float d2 = dot3_rn(__fsub_rn(cx, x), __fsub_rn(cy, y), __fsub_rn(cz, z));
    return __fmul_rn(width, width) < __fmul_rn(theta2, d2);
}

__device__ __forceinline__ uint32_t lane_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Forward interaction of field point r = x - c with a cell (G omitted).
template <bool QUAD>
__device__ __forceinline__ void cell_fwd(float rx, float ry, float rz, const float4 &c,
                                         const float4 &q0, const float4 &q1, float eps2,
                                         float &ax, float &ay, float &az, float &phi) {
    const float s = rx * rx + ry * ry + rz * rz + eps2;
    const float i1 = rsqrtf(s), i2 = i1 * i1, i3 = i1 * i2;
    phi -= c.w * i1;
    ax -= c.w * rx * i3;
    ay -= c.w * ry * i3;
    az -= c.w * rz * i3;
    if (QUAD) {
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
}

// Derivatives of u*phi + v.a for one cell interaction (G omitted):
// g_r = d/dr (r = x - c), gM = d/dM, gq = d/dQ (symmetric part, 6 comps).
template <bool QUAD>
__device__ __forceinline__ void cell_adj(float rx, float ry, float rz, const float4 &c,
                                         const float4 &q0, const float4 &q1, float eps2, float u,
                                         float vx, float vy, float vz, float &grx, float &gry,
                                         float &grz, float &gM, float gq[6]) {
    const float s = rx * rx + ry * ry + rz * rz + eps2;
    const float i1 = rsqrtf(s), i2 = i1 * i1, i3 = i1 * i2, i5 = i3 * i2;
    const float M = c.w;
    const float vr = vx * rx + vy * ry + vz * rz;
    grx = u * M * rx * i3 - M * (vx * i3 - 3.f * vr * rx * i5);
    gry = u * M * ry * i3 - M * (vy * i3 - 3.f * vr * ry * i5);
    grz = u * M * rz * i3 - M * (vz * i3 - 3.f * vr * rz * i5);
    gM = -u * i1 - vr * i3;
    if (QUAD) {
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
        // phi_Q = -q i5 / 2, a_Q = Qr i5 - 2.5 q r i7: u dphi_Q/dr = -u a_Q
        const float k1 = 2.5f * q * i7;
        grx -= u * (qrx * i5 - k1 * rx);
        gry -= u * (qry * i5 - k1 * ry);
        grz -= u * (qrz * i5 - k1 * rz);
        // d(v.a_Q)/dr = Qv i5 - 5 vQr i7 r - 5 vr i7 Qr - 2.5 q i7 v + 17.5 q vr i9 r
        const float kr = -5.f * vqr * i7 + 17.5f * q * vr * i9;
        const float kq = -5.f * vr * i7;
        const float kv = -2.5f * q * i7;
        grx += qvx * i5 + kr * rx + kq * qrx + kv * vx;
        gry += qvy * i5 + kr * ry + kq * qry + kv * vy;
        grz += qvz * i5 + kr * rz + kq * qrz + kv * vz;
        // dL/dQ: -u i5 rr^T / 2 + i5 sym(v r^T) - 2.5 vr i7 rr^T
        const float cr = -0.5f * u * i5 - 2.5f * vr * i7;
        gq[0] = cr * rx * rx + i5 * vx * rx;
        gq[1] = cr * ry * ry + i5 * vy * ry;
        gq[2] = cr * rz * rz + i5 * vz * rz;
        gq[3] = cr * rx * ry + 0.5f * i5 * (vx * ry + vy * rx);
        gq[4] = cr * rx * rz + 0.5f * i5 * (vx * rz + vz * rx);
        gq[5] = cr * ry * rz + 0.5f * i5 * (vy * rz + vz * ry);
    }
}

// Derivatives of u*phi + v.a for one body-body interaction (G omitted),
// r = x_target - x_source, source mass m: g_r and d/dm.
__device__ __forceinline__ void body_adj(float rx, float ry, float rz, float m, float eps2, float u,
                                         float vx, float vy, float vz, float &grx, float &gry,
                                         float &grz, float &gm) {
    const float s = rx * rx + ry * ry + rz * rz + eps2;
    const float i1 = rsqrtf(s), i2 = i1 * i1, i3 = i1 * i2, i5 = i3 * i2;
    const float vr = vx * rx + vy * ry + vz * rz;
    grx = u * m * rx * i3 - m * (vx * i3 - 3.f * vr * rx * i5);
    gry = u * m * ry * i3 - m * (vy * i3 - 3.f * vr * ry * i5);
    grz = u * m * rz * i3 - m * (vz * i3 - 3.f * vr * rz * i5);
    gm = -u * i1 - vr * i3;
}

// The adjoint walk holds more state: bounded to 6 blocks of 4 warps per SM
// (79 registers, no spills) instead of the 5 its unbounded 93 registers give.
template <bool QUAD, bool ADJ>
__global__ void __launch_bounds__(WW * 32, ADJ ? 6 : 0) bh_walk_kernel(
    const BhView v, float theta2, float eps2, float G, const float *__restrict__ g_acc,
    const float *__restrict__ g_phi, float *__restrict__ acc_out, float *__restrict__ phi_out,
    float4 *__restrict__ cell_grad, float4 *__restrict__ body_grad, uint2 *__restrict__ stack,
    uint32_t stack_entries, const IlogView lg, BhHeader *hm) {
    __shared__ WarpTile tiles[WW];
    __shared__ WarpRed reds[ADJ ? WW : 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpTile &T = tiles[warp];
    WarpRed &R = reds[ADJ ? warp : 0];
    const uint64_t gw = (uint64_t)blockIdx.x * WW + warp;
    uint2 *stk = stack + gw * BH_STACK_CAP_MAX;   // this warp's slice
    const uint32_t ngroups = v.hdr->n_groups, n_nodes = v.hdr->n_nodes;
    const uint32_t lt = lane_lt();
    const uint32_t *child = reinterpret_cast<const uint32_t *>(v.child8);
    uint32_t max_sp = 0;
    while (true) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(&hm->group_counter, 1u);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= ngroups) break;
        const uint2 gr = v.groups[g];
        const uint32_t gs = gr.x, gc = gr.y;
        const uint32_t i = gs + lane;
        const bool valid = (uint32_t)lane < gc;
        const float4 me = valid ? v.fbody[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        float ax = 0.f, ay = 0.f, az = 0.f, phi = 0.f;   // forward sums / adjoint d/dx_i
        float vx = 0.f, vy = 0.f, vz = 0.f, u = 0.f;
        if (ADJ) {
            if (valid) {
                const uint32_t o = v.order[i];
                vx = g_acc[3 * (uint64_t)o];
                vy = g_acc[3 * (uint64_t)o + 1];
                vz = g_acc[3 * (uint64_t)o + 2];
                u = g_phi ? g_phi[o] : 0.f;
            }
        }
        int cn = 0, bn = 0, sp = 0;
        const uint32_t all = __ballot_sync(0xffffffffu, valid);
        // The adjoint replays the group's tiles from the forward's log when
        // the log holds them all; otherwise it walks the tree.
        const uint2 lgg = (ADJ && lg.group) ? lg.group[g] : make_uint2(ILOG_NONE, ILOG_NONE);
        const uint32_t logged = lgg.y;
        if (n_nodes > 0 && logged == ILOG_NONE) {
            if (lane == 0) stk[0] = make_uint2(0u, all);
            sp = 1;
        }
        __syncwarp();
        // forward: every evaluated tile (cnt entries of clist/cmask or
        // blist/bmask) appended to the group's chain of log pages, while the
        // pool has pages (all warp-uniform)
        uint32_t nt = 0, page = ILOG_NONE, first = ILOG_NONE;
        bool lok = !ADJ && lg.group != nullptr;
        auto log_tile = [&](int cnt, bool bodies) {
            if (ADJ || !lg.group) return;
            const uint32_t pos = nt % ILOG_PAGE;
            if (pos == 0 && lok) {
                uint32_t pg = 0;
                if (lane == 0) pg = atomicAdd(&hm->ilog_used, 1u);
                pg = __shfl_sync(0xffffffffu, pg, 0);
                if (pg >= lg.pages) {
                    lok = false;
                } else {
                    if (page == ILOG_NONE) first = pg;
                    else if (lane == 0) lg.next[page] = pg;
                    page = pg;
                }
            }
            if (lok) {
                const uint64_t slot = (uint64_t)page * ILOG_PAGE + pos;
                if (lane < cnt)
                    lg.entries[slot * 32 + lane] = bodies ? make_uint2(T.blist[lane], T.bmask[lane])
                                                          : make_uint2(T.clist[lane], T.cmask[lane]);
                if (lane == 0) lg.counts[slot] = (uint8_t)(cnt | (bodies ? 0x80 : 0));
            }
            ++nt;
        };

        auto eval_cells = [&](int cnt) {
            log_tile(cnt, false);
            uint32_t nid = 0, cm = 0;
            if (lane < cnt) {
                nid = T.clist[lane];
                cm = T.cmask[lane];
                T.cell[lane][0] = __ldg(&v.node_a[nid]);
                if (QUAD) {
                    T.cell[lane][1] = __ldg(&v.node_q[2 * nid]);
                    T.cell[lane][2] = __ldg(&v.node_q[2 * nid + 1]);
                }
                T.cmask_t[lane] = cm;
            }
            __syncwarp();
            const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (!ADJ) {
                for (int k = 0; k < cnt; ++k) {   // lane = body
                    if (!((T.cmask_t[k] >> lane) & 1u)) continue;
                    const float4 c = T.cell[k][0];
                    const float4 q0 = QUAD ? T.cell[k][1] : z4, q1 = QUAD ? T.cell[k][2] : z4;
                    cell_fwd<QUAD>(me.x - c.x, me.y - c.y, me.z - c.z, c, q0, q1, eps2, ax, ay, az, phi);
                }
            } else {
                // One evaluation per (body, cell) pair, lane = body: the
                // body's derivative stays in its registers, the cell's (COM,
                // mass, quadrupole; d/dc = -d/dx) goes to the chunk table, one
                // row per (cell, part), and each row is summed over the lanes
                // by a few lanes each (table_row_sum).
                constexpr int PARTS = QUAD ? 3 : 1;
                for (int k0 = 0; k0 < cnt; k0 += RED_CELLS) {
                    const int kn = cnt - k0 < RED_CELLS ? cnt - k0 : RED_CELLS;
                    for (int kk = 0; kk < kn; ++kk) {
                        const int k = k0 + kk;
                        float4 r0 = z4, r1 = z4, r2 = z4;
                        if ((T.cmask_t[k] >> lane) & 1u) {
                            const float4 c = T.cell[k][0];
                            const float4 q0 = QUAD ? T.cell[k][1] : z4, q1 = QUAD ? T.cell[k][2] : z4;
                            float grx, gry, grz, gM, gq[6];
                            cell_adj<QUAD>(me.x - c.x, me.y - c.y, me.z - c.z, c, q0, q1, eps2, u,
                                           vx, vy, vz, grx, gry, grz, gM, gq);
                            ax += grx; ay += gry; az += grz;
                            r0 = make_float4(-grx, -gry, -grz, gM);
                            if (QUAD) {
                                r1 = make_float4(gq[0], gq[1], gq[2], gq[3]);
                                r2 = make_float4(gq[4], gq[5], 0.f, 0.f);
                            }
                        }
                        R.red[PARTS * kk][lane] = r0;
                        if (QUAD) {
                            R.red[PARTS * kk + 1][lane] = r1;
                            R.red[PARTS * kk + 2][lane] = r2;
                        }
                    }
                    __syncwarp();
                    int row;
                    bool owner;
                    const float4 t = table_row_sum<32 / (RED_CELLS * PARTS)>(R, kn * PARTS, lane,
                                                                             row, owner);
                    if (owner) {
                        const int kk = row / PARTS, part = row - kk * PARTS;
                        const uint32_t cid = T.clist[k0 + kk];
                        atomicAdd(&cell_grad[3 * cid + part], make_float4(G * t.x, G * t.y, G * t.z, G * t.w));
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
        };
        auto eval_bodies = [&](int cnt) {
            log_tile(cnt, true);
            uint32_t bid = 0, bm = 0;
            if (lane < cnt) {
                bid = T.blist[lane];
                bm = T.bmask[lane];
                T.body[lane] = __ldg(&v.fbody[bid]);
                T.bid[lane] = bid;
                T.bmask_t[lane] = bm;
            }
            __syncwarp();
            if (!ADJ) {
                for (int k = 0; k < cnt; ++k) {   // lane = target
                    if (!((T.bmask_t[k] >> lane) & 1u) || T.bid[k] == i) continue;
                    const float4 o = T.body[k];
                    const float rx = me.x - o.x, ry = me.y - o.y, rz = me.z - o.z;
                    const float s = rx * rx + ry * ry + rz * rz + eps2;
                    const float i1 = rsqrtf(s), i3 = i1 * i1 * i1;
                    phi -= o.w * i1;
                    ax -= o.w * rx * i3;
                    ay -= o.w * ry * i3;
                    az -= o.w * rz * i3;
                }
            } else {
                // as for cells: one evaluation per (target, source) pair,
                // the source's derivative summed over the lanes
                const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
                for (int k0 = 0; k0 < cnt; k0 += RED_BODIES) {
                    const int kn = cnt - k0 < RED_BODIES ? cnt - k0 : RED_BODIES;
                    for (int kk = 0; kk < kn; ++kk) {
                        const int k = k0 + kk;
                        float4 r = z4;
                        if (((T.bmask_t[k] >> lane) & 1u) && T.bid[k] != i) {
                            const float4 o = T.body[k];
                            float grx, gry, grz, gm;
                            body_adj(me.x - o.x, me.y - o.y, me.z - o.z, o.w, eps2, u, vx, vy, vz,
                                     grx, gry, grz, gm);
                            ax += grx; ay += gry; az += grz;
                            r = make_float4(-grx, -gry, -grz, gm);
                        }
                        R.red[kk][lane] = r;
                    }
                    __syncwarp();
                    int row;
                    bool owner;
                    const float4 t = table_row_sum<32 / RED_BODIES>(R, kn, lane, row, owner);
                    if (owner)
                        atomicAdd(&body_grad[T.bid[k0 + row]], make_float4(G * t.x, G * t.y, G * t.z, G * t.w));
                    __syncwarp();
                }
            }
            __syncwarp();
        };

        if (logged != ILOG_NONE && logged > 0) {
            // replay: each logged tile back into the lists, evaluated as
            // the walk evaluated it (same tiles, same order).  A page's
            // tile counts come in one load (lane l: tile l) with the next
            // page's id, and each tile's entries are loaded while the tile
            // before it is evaluated.
            uint32_t pg = lgg.x;
            uint32_t c_lane = lane < (int)ILOG_PAGE ? lg.counts[(uint64_t)pg * ILOG_PAGE + lane] : 0u;
            uint32_t pg_next = logged > ILOG_PAGE ? lg.next[pg] : ILOG_NONE;
            uint2 e = lg.entries[(uint64_t)pg * ILOG_PAGE * 32 + lane];
            for (uint32_t t = 0; t < logged; ++t) {
                const uint32_t pos = t % ILOG_PAGE;
                if (pos == 0 && t > 0) {
                    pg = pg_next;
                    c_lane = lane < (int)ILOG_PAGE ? lg.counts[(uint64_t)pg * ILOG_PAGE + lane] : 0u;
                    pg_next = t + ILOG_PAGE < logged ? lg.next[pg] : ILOG_NONE;
                }
                const uint32_t c = __shfl_sync(0xffffffffu, c_lane, (int)pos);
                const int cnt = (int)(c & 0x7F);
                uint2 en = make_uint2(0u, 0u);
                if (t + 1 < logged) {
                    const uint32_t pos1 = (t + 1) % ILOG_PAGE;
                    const uint32_t pg1 = pos1 == 0 ? pg_next : pg;
                    en = lg.entries[((uint64_t)pg1 * ILOG_PAGE + pos1) * 32 + lane];
                }
                if (lane < cnt) {
                    if (c & 0x80) { T.blist[lane] = e.x; T.bmask[lane] = e.y; }
                    else { T.clist[lane] = e.x; T.cmask[lane] = e.y; }
                }
                __syncwarp();
                if (c & 0x80) eval_bodies(cnt);
                else eval_cells(cnt);
                e = en;
            }
        }
        while (sp > 0) {
            const int t = sp < 32 ? sp : 32;
            sp -= t;
            uint2 e = make_uint2(0u, 0u);
            float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
            uint4 b = make_uint4(0u, 0u, 0u, 0u);
            if (lane < t) {
                e = stk[sp + lane];
                a = __ldg(&v.node_a[e.x]);
                b = __ldg(&v.node_b[e.x]);
            }
            __syncwarp();
            for (int k = 0; k < t; ++k) {
                const uint32_t nk = __shfl_sync(0xffffffffu, e.x, k);
                const uint32_t mk = __shfl_sync(0xffffffffu, e.y, k);
                const float cx = __shfl_sync(0xffffffffu, a.x, k);
                const float cy = __shfl_sync(0xffffffffu, a.y, k);
                const float cz = __shfl_sync(0xffffffffu, a.z, k);
                const uint32_t bz = __shfl_sync(0xffffffffu, b.z, k);
                const uint32_t bw = __shfl_sync(0xffffffffu, b.w, k);
                const bool in = (mk >> lane) & 1u;
                const bool acc = in && body_accept(me.x, me.y, me.z, cx, cy, cz, __uint_as_float(bw), theta2);
                const uint32_t A = __ballot_sync(0xffffffffu, acc);
                const uint32_t R = mk & ~A;
                if (A) {
                    if (lane == 0) { T.clist[cn] = nk; T.cmask[cn] = A; }
                    ++cn;
                    __syncwarp();
                    if (cn == 32) { eval_cells(32); cn = 0; }
                }
                if (!R) continue;
                if (bz & BH_LEAF_BIT) {
                    const uint32_t bs = __shfl_sync(0xffffffffu, b.y, k);
                    const uint32_t bc = bz & ~BH_LEAF_BIT;
                    for (uint32_t off = 0; off < bc; off += 32) {
                        const uint32_t kk = bc - off < 32u ? bc - off : 32u;
                        if ((uint32_t)lane < kk) {
                            T.blist[bn + lane] = bs + off + lane;
                            T.bmask[bn + lane] = R;
                        }
                        bn += (int)kk;
                        __syncwarp();
                        if (bn >= 32) {
                            eval_bodies(32);
                            if (lane < bn - 32) {
                                T.blist[lane] = T.blist[32 + lane];
                                T.bmask[lane] = T.bmask[32 + lane];
                            }
                            bn -= 32;
                            __syncwarp();
                        }
                    }
                } else {
                    const uint32_t c = lane < 8 ? __ldg(&child[8 * (uint64_t)nk + lane]) : 0xFFFFFFFFu;
                    const uint32_t pm = __ballot_sync(0xffffffffu, c != 0xFFFFFFFFu);
                    const int np = __popc(pm);
                    if ((uint32_t)(sp + np) <= stack_entries) {
                        if (c != 0xFFFFFFFFu) stk[sp + __popc(pm & lt)] = make_uint2(c, R);
                        sp += np;
                    } else if (lane == 0) {
                        atomicOr(&hm->err, DEVERR_STACK);
                    }
                    __syncwarp();
                }
            }
            max_sp = max(max_sp, (uint32_t)sp);
        }
        if (cn > 0) eval_cells(cn);
        if (bn > 0) eval_bodies(bn);
        if (!ADJ && lg.group && lane == 0) {
            lg.group[g] = make_uint2(first, lok ? nt : ILOG_NONE);
            atomicAdd(&hm->ilog_need, (nt + ILOG_PAGE - 1) / ILOG_PAGE);
        }
        if (valid) {
            if (!ADJ) {
                const uint32_t o = v.order[i];
                acc_out[3 * (uint64_t)o] = G * ax;
                acc_out[3 * (uint64_t)o + 1] = G * ay;
                acc_out[3 * (uint64_t)o + 2] = G * az;
                if (phi_out) phi_out[o] = G * phi;
            } else {
                atomicAdd(&body_grad[i], make_float4(G * ax, G * ay, G * az, 0.f));
            }
        }
        __syncwarp();
    }
    if (lane == 0) atomicMax(&hm->max_stack, max_sp);
}

// Per-node constants of the cell-to-body rule (Pvec.xyz, Pconst | Pmat xx
// yy zz xy | xz yz) from the cell's derivatives (g_c, g_M | G_Q).
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

// Top-down path sums of the per-node constants (one block, level by level).
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
            const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
            float4 p0 = l == 0 ? z : prefix[3 * i];      // the parent's path sum
            float4 p1 = l == 0 ? z : prefix[3 * i + 1];
            float4 p2 = l == 0 ? z : prefix[3 * i + 2];
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

template <bool QUAD, bool ADJ>
rtd_status launch_walk(rtd_bh *b, const rtd_bh_params *p, const float *g_acc, const float *g_phi,
                       float *acc, float *phi, const IlogView &lg, cudaStream_t st) {
    int dev = 0, sms = 148, per_sm = 4;
    RTD_CUDA(cudaGetDevice(&dev));
    RTD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RTD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bh_walk_kernel<QUAD, ADJ>,
                                                           WW * 32, 0));
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = (uint64_t)sms * (uint64_t)per_sm;
    const uint64_t need = (b->n + WW - 1) / WW;   // groups <= bodies
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    const uint64_t warps = blocks * WW;
    if (b->stack_warps < warps) {
        RTD_TRY(b->stack.reserve(warps * BH_STACK_CAP_MAX * sizeof(uint2)));
        b->stack_warps = warps;
    }
    BhHeader *h = b->hdr.as<BhHeader>();
    RTD_CUDA(cudaMemsetAsync(&h->group_counter, 0, sizeof(uint32_t), st));
    const BhView v = bh_view(b);
    bh_walk_kernel<QUAD, ADJ><<<(unsigned)blocks, WW * 32, 0, st>>>(
        v, p->theta * p->theta, p->eps * p->eps, p->G, g_acc, g_phi, acc, phi,
        b->cell_grad.as<float4>(), b->gpos_flat.as<float4>(), b->stack.as<uint2>(),
        bh_stack_entries(), lg, h);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

}  // namespace

rtd_status bh_ref_forward(rtd_bh *b, const rtd_bh_params *p, float *d_out, cudaStream_t st);

// The interaction log for a forward: pinned hint and event on first use,
// the pool grown to the last logging forward's need once its copy has
// landed (grown only), the per-group array for up to n groups, and the
// page counters cleared.
static rtd_status ilog_prepare(rtd_bh *b, cudaStream_t st, IlogView &lg) {
    if (!b->ilog_hint) {
        RTD_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&b->ilog_hint), sizeof(uint32_t),
                               cudaHostAllocDefault));
        *b->ilog_hint = 0;
    }
    if (!b->ilog_ev) RTD_CUDA(cudaEventCreateWithFlags(&b->ilog_ev, cudaEventDisableTiming));
    const cudaError_t q = cudaEventQuery(b->ilog_ev);
    if (q == cudaSuccess && *b->ilog_hint > b->ilog_pages) {
        const uint64_t want = (uint64_t)*b->ilog_hint + *b->ilog_hint / 16 + 64;
        RTD_TRY(b->ilog_entries.reserve(want * ILOG_PAGE * 32 * sizeof(uint2)));
        RTD_TRY(b->ilog_counts.reserve(want * ILOG_PAGE));
        RTD_TRY(b->ilog_next.reserve(want * sizeof(uint32_t)));
        b->ilog_pages = (uint32_t)want;
    } else if (q != cudaSuccess && q != cudaErrorNotReady) {
        return cuda_fail(q, "cudaEventQuery");
    }
    cudaGetLastError();   // a not-ready query leaves no error behind
    RTD_TRY(b->ilog_group.reserve(b->n * sizeof(uint2) + 64));
    BhHeader *h = b->hdr.as<BhHeader>();
    RTD_CUDA(cudaMemsetAsync(&h->ilog_used, 0, 2 * sizeof(uint32_t), st));
    lg.entries = b->ilog_entries.as<uint2>();
    lg.counts = b->ilog_counts.as<uint8_t>();
    lg.next = b->ilog_next.as<uint32_t>();
    lg.group = b->ilog_group.as<uint2>();
    lg.pages = b->ilog_pages;
    return RTD_OK;
}

rtd_status bh_forward(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                      cudaStream_t st) {
    if (!b || !b->built) return fail(RTD_ERR_INVALID_ARGUMENT, "bh tree not built");
    if (b->n && !d_out) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL output");
    rtd_bh_params def;
    rtd_bh_params_default(&def);
    if (!p) p = &def;
    if (b->n == 0) return RTD_OK;
    if (p->law == RTD_BH_LAW_REFERENCE) return bh_ref_forward(b, p, d_out, st);
    if (p->law != RTD_BH_LAW_PLUMMER) return fail(RTD_ERR_INVALID_ARGUMENT, "unknown law");
    if (!b->plummer_ready)
        return fail(RTD_ERR_INVALID_ARGUMENT, "tree was not built for the Plummer law");
    if (p->quadrupole && !b->has_quad)
        return fail(RTD_ERR_INVALID_ARGUMENT, "tree was built without quadrupoles");
    IlogView lg{};
    if (b->backward_seen) RTD_TRY(ilog_prepare(b, st, lg));
    b->ilog_valid = false;
    if (p->quadrupole) RTD_TRY((launch_walk<true, false>(b, p, nullptr, nullptr, d_out, d_phi, lg, st)));
    else RTD_TRY((launch_walk<false, false>(b, p, nullptr, nullptr, d_out, d_phi, lg, st)));
    if (lg.group) {
        // the pages this forward needed, for sizing the next one's pool
        RTD_CUDA(cudaMemcpyAsync(b->ilog_hint, &b->hdr.as<BhHeader>()->ilog_need, sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st));
        RTD_CUDA(cudaEventRecord(b->ilog_ev, st));
        b->ilog_valid = lg.pages > 0;
        b->ilog_theta = p->theta;
        b->ilog_quad = p->quadrupole;
    }
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
    if (!b->plummer_ready)
        return fail(RTD_ERR_INVALID_ARGUMENT, "tree was not built for the Plummer law");
    if (p->quadrupole && !b->has_quad)
        return fail(RTD_ERR_INVALID_ARGUMENT, "tree was built without quadrupoles");
    const uint64_t n = b->n;
    RTD_TRY(b->cell_grad.reserve(n * 3 * sizeof(float4) + 64 * sizeof(uint32_t)));
    RTD_TRY(b->prefix.reserve(n * 3 * sizeof(float4)));
    RTD_TRY(b->gpos_flat.reserve(n * sizeof(float4)));
    RTD_CUDA(cudaMemsetAsync(b->cell_grad.ptr, 0, n * 3 * sizeof(float4), st));
    RTD_CUDA(cudaMemsetAsync(b->gpos_flat.ptr, 0, n * sizeof(float4), st));
    // replay the last forward's interaction log when it was taken on this
    // tree with these parameters; otherwise walk
    IlogView lg{};
    if (b->ilog_valid && b->ilog_theta == p->theta && b->ilog_quad == p->quadrupole) {
        lg.entries = b->ilog_entries.as<uint2>();
        lg.counts = b->ilog_counts.as<uint8_t>();
        lg.next = b->ilog_next.as<uint32_t>();
        lg.group = b->ilog_group.as<uint2>();
        lg.pages = b->ilog_pages;
    }
    b->backward_seen = true;
    if (p->quadrupole) RTD_TRY((launch_walk<true, true>(b, p, g_acc, g_phi, nullptr, nullptr, lg, st)));
    else RTD_TRY((launch_walk<false, true>(b, p, g_acc, g_phi, nullptr, nullptr, lg, st)));
    const BhView v = bh_view(b);
    bh_prefix_kernel<<<1, 1024, 0, st>>>(v, b->level_nodes.as<uint32_t>(), b->cell_grad.as<float4>(),
                                          b->prefix.as<float4>());
    RTD_LAUNCH_CHECK();
    bh_finish_grad_kernel<<<grid_for(n, 128, 1 << 20), 128, 0, st>>>(
        v, b->prefix.as<float4>(), b->gpos_flat.as<float4>(), g_pos, g_mass);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

namespace {

// Forward walk on a traversal stack supplied by the caller: `stack` holds
// max_warps slices of BH_STACK_CAP_MAX entries and the launch is capped to that
// many warps.  Nothing is allocated.
template <bool QUAD>
rtd_status launch_walk_on_stack(rtd_bh *b, const rtd_bh_params *p, float *acc, float *phi,
                                uint2 *stack, uint64_t max_warps, cudaStream_t st) {
    int dev = 0, sms = 148, per_sm = 4;
    RTD_CUDA(cudaGetDevice(&dev));
    RTD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RTD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bh_walk_kernel<QUAD, false>,
                                                           WW * 32, 0));
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = (uint64_t)sms * (uint64_t)per_sm;
    const uint64_t need = (b->n + WW - 1) / WW;
    if (blocks > need) blocks = need;
    if (blocks > max_warps / WW) blocks = max_warps / WW;
    if (blocks < 1) return fail(RTD_ERR_INVALID_ARGUMENT, "stack holds less than one block of warps");
    BhHeader *h = b->hdr.as<BhHeader>();
    RTD_CUDA(cudaMemsetAsync(&h->group_counter, 0, sizeof(uint32_t), st));
    const BhView v = bh_view(b);
    bh_walk_kernel<QUAD, false><<<(unsigned)blocks, WW * 32, 0, st>>>(
        v, p->theta * p->theta, p->eps * p->eps, p->G, nullptr, nullptr, acc, phi, nullptr,
        nullptr, stack, bh_stack_entries(), IlogView{}, h);
    RTD_LAUNCH_CHECK();
    return RTD_OK;
}

}  // namespace

// Plummer-law forward walk with the traversal stack given by the caller
// (max_warps slices of BH_STACK_CAP_MAX uint2 entries); same checks and results
// as bh_forward for the Plummer law.
rtd_status bh_forward_on_stack(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                               uint2 *stack, uint64_t max_warps, cudaStream_t st) {
    if (!b || !b->built) return fail(RTD_ERR_INVALID_ARGUMENT, "bh tree not built");
    if (b->n && !d_out) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL output");
    if (!stack) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL stack");
    rtd_bh_params def;
    rtd_bh_params_default(&def);
    if (!p) p = &def;
    if (p->law != RTD_BH_LAW_PLUMMER)
        return fail(RTD_ERR_UNSUPPORTED, "this walk implements the Plummer law only");
    if (b->n == 0) return RTD_OK;
    if (!b->plummer_ready)
        return fail(RTD_ERR_INVALID_ARGUMENT, "tree was not built for the Plummer law");
    if (p->quadrupole && !b->has_quad)
        return fail(RTD_ERR_INVALID_ARGUMENT, "tree was built without quadrupoles");
    if (p->quadrupole) return launch_walk_on_stack<true>(b, p, d_out, d_phi, stack, max_warps, st);
    return launch_walk_on_stack<false>(b, p, d_out, d_phi, stack, max_warps, st);
}

}  // namespace rtd

namespace rtd {
namespace {

// Interaction counts of the Plummer walk for every stride-th flat body: the
// same per-body MAC over the pre-order tree (autoropes), counting accepted
// cells and the bodies of opened leaves.  out[0] += cells, out[1] += bodies.
__global__ void bh_count_kernel(const BhView v, float theta2, uint64_t stride,
                                unsigned long long *out) {
    const uint32_t n_nodes = v.hdr->n_nodes;
    unsigned long long cells = 0, bodies = 0;
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s * stride < v.n;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const float4 me = v.fbody[s * stride];
        uint32_t p = 0;
        while (p < n_nodes) {
            const float4 a = __ldg(&v.node_a[p]);
            const uint4 b = __ldg(&v.node_b[p]);
            if (body_accept(me.x, me.y, me.z, a.x, a.y, a.z, __uint_as_float(b.w), theta2)) {
                ++cells;
                p = b.x;
            } else {
                if (b.z & BH_LEAF_BIT) bodies += b.z & ~BH_LEAF_BIT;
                ++p;
            }
        }
    }
    atomicAdd(&out[0], cells);
    atomicAdd(&out[1], bodies);
}

}  // namespace

rtd_status bh_interaction_counts(rtd_bh *b, float theta, uint64_t stride, uint64_t *h_cells,
                                 uint64_t *h_bodies, uint64_t *h_sampled, cudaStream_t st) {
    if (!b || !b->built) return fail(RTD_ERR_INVALID_ARGUMENT, "bh tree not built");
    if (stride < 1) return fail(RTD_ERR_INVALID_ARGUMENT, "stride must be >= 1");
    RTD_TRY(b->cell_grad.reserve(2 * sizeof(unsigned long long)));
    unsigned long long *d = b->cell_grad.as<unsigned long long>();
    RTD_CUDA(cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), st));
    const uint64_t ns = b->n ? (b->n + stride - 1) / stride : 0;
    if (ns) {
        bh_count_kernel<<<grid_for(ns, 128, 148 * 8), 128, 0, st>>>(bh_view(b), theta * theta,
                                                                     stride, d);
        RTD_LAUNCH_CHECK();
    }
    unsigned long long h[2] = {0, 0};
    RTD_CUDA(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    if (h_cells) *h_cells = h[0];
    if (h_bodies) *h_bodies = h[1];
    if (h_sampled) *h_sampled = ns;
    return RTD_OK;
}

}  // namespace rtd
