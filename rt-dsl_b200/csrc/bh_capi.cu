// bh_capi.cu -- extern "C" Barnes-Hut entry points of include/rtdsl.h.
#include <new>
#include <vector>

#include "bh.cuh"
#include "index.cuh"

namespace rtd {

rtd_status bh_forward(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                      cudaStream_t st);
rtd_status bh_backward(rtd_bh *b, const rtd_bh_params *p, const float *g_acc, const float *g_phi,
                       float *g_pos, float *g_mass, cudaStream_t st);

rtd_status check_bh_errors(rtd_bh *b, cudaStream_t st) {
    if (!b->hdr.ptr) return RTD_OK;
    uint32_t f = 0;
    BhHeader *h = b->hdr.as<BhHeader>();
    RTD_CUDA(cudaMemcpyAsync(&f, &h->err, sizeof(f), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    if (f) RTD_CUDA(cudaMemsetAsync(&h->err, 0, sizeof(uint32_t), st));
    if (f & DEVERR_DEPTH)
        return fail(RTD_ERR_UNSUPPORTED, "octree cell still above the bucket size 21 levels down");
    return status_from_deverr(f);
}

namespace {
// gprt-core Body {pos, mass, velocity} (28 B) -> positions and masses.
__global__ void split_bodies_kernel(const float *__restrict__ bodies, uint64_t n,
                                    float *__restrict__ pos, float *__restrict__ mass) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float *b = bodies + 7 * i;
        pos[3 * i] = b[0];
        pos[3 * i + 1] = b[1];
        pos[3 * i + 2] = b[2];
        mass[i] = b[3];
    }
}
}  // namespace

}  // namespace rtd

using namespace rtd;

rtd_context_bh *context_bh(rtd_context *ctx);
cudaStream_t context_stream(rtd_context *ctx);

rtd_bh::~rtd_bh() {
    if (ilog_hint) cudaFreeHost(ilog_hint);
    if (ilog_ev) cudaEventDestroy(ilog_ev);
}

extern "C" {

void rtd_bh_params_default(rtd_bh_params *p) {
    if (!p) return;
    p->theta = 0.5f;
    p->G = 6.674e-11f;
    p->eps = 1e-3f;
    p->law = RTD_BH_LAW_REFERENCE;
    p->quadrupole = 1;
    p->bucket = 128;
    p->min_width = 1e-5f;
}

rtd_status rtd_bh_create(rtd_bh **out) {
    if (!out) return fail(RTD_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = new (std::nothrow) rtd_bh();
    if (!*out) return fail(RTD_ERR_OUT_OF_MEMORY, "host allocation failed");
    return RTD_OK;
}

rtd_status rtd_bh_destroy(rtd_bh *b) {
    delete b;
    return RTD_OK;
}

rtd_status rtd_bh_build(rtd_bh *b, const float *d_pos, const float *d_mass, uint64_t n,
                        const rtd_bh_params *p, rtd_stream stream) {
    return bh_build(b, d_pos, d_mass, n, p, (cudaStream_t)stream);
}

rtd_status rtd_bh_release(rtd_bh *b) {
    if (!b) return fail(RTD_ERR_INVALID_ARGUMENT, "bh handle is NULL");
    for (DevBuf *d : {&b->mkeys, &b->mkeys_alt, &b->mvals, &b->mvals_alt, &b->pkeys, &b->pkeys_alt,
                      &b->pvals, &b->pvals_alt, &b->lcp, &b->wmin, &b->lam, &b->nn, &b->base,
                      &b->heads, &b->leaf_head, &b->leaf_of, &b->fkeys, &b->fkeys_alt, &b->fvals,
                      &b->fvals_alt, &b->node_start, &b->node_level, &b->level_nodes, &b->order,
                      &b->fbody, &b->node_a, &b->node_b, &b->node_q, &b->child8, &b->leaf_node,
                      &b->groups, &b->stack, &b->cell_grad, &b->prefix, &b->gpos_flat,
                      &b->gmass_flat})
        d->release();
    for (DevBuf *d : {&b->ilog_entries, &b->ilog_counts, &b->ilog_next, &b->ilog_group})
        d->release();
    b->stack_warps = 0;
    b->plummer_ready = false;
    b->has_quad = false;
    b->ilog_pages = 0;
    b->ilog_valid = false;
    b->sort.counts.release();
    b->scan.sums.release();
    b->built = false;
    return RTD_OK;
}

rtd_status rtd_bh_forward(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                          rtd_stream stream) {
    return bh_forward(b, p, d_out, d_phi, (cudaStream_t)stream);
}

rtd_status rtd_bh_backward(rtd_bh *b, const rtd_bh_params *p, const float *d_g_acc,
                           const float *d_g_phi, float *d_g_pos, float *d_g_mass,
                           rtd_stream stream) {
    return bh_backward(b, p, d_g_acc, d_g_phi, d_g_pos, d_g_mass, (cudaStream_t)stream);
}

rtd_status rtd_bh_info_get(rtd_bh *b, rtd_bh_info *info, rtd_stream stream) {
    if (!b || !info) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL argument");
    memset(info, 0, sizeof(*info));
    info->n_bodies = b->n;
    if (!b->hdr.ptr || !b->built) return RTD_OK;
    BhHeader h;
    cudaStream_t st = (cudaStream_t)stream;
    RTD_CUDA(cudaMemcpyAsync(&h, b->hdr.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    info->n_nodes = h.n_nodes;
    info->n_leaves = h.n_leaves;
    for (int l = 0; l <= BH_MAX_LEVEL + 1; ++l)
        if (h.level_count[l]) info->depth = (uint32_t)l;
    for (int a = 0; a < 3; ++a) {
        info->root_min[a] = h.root_min[a];
        info->root_max[a] = h.root_max[a];
    }
    info->max_stack = h.max_stack;
    info->log_pages = b->ilog_valid ? (h.ilog_used < b->ilog_pages ? h.ilog_used : b->ilog_pages) : 0;
    return check_bh_errors(b, st);
}

rtd_status rtd_bh_export(rtd_bh *b, void *h_flat_nodes, uint32_t *h_order, rtd_stream stream) {
    if (!b || !b->built) return fail(RTD_ERR_INVALID_ARGUMENT, "bh tree not built");
    cudaStream_t st = (cudaStream_t)stream;
    RTD_TRY(check_bh_errors(b, st));
    BhHeader h;
    RTD_CUDA(cudaMemcpyAsync(&h, b->hdr.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    const uint32_t nn = b->n ? h.n_nodes : 0;
    std::vector<float4> a(nn);
    std::vector<uint4> bb(nn);
    if (nn) {
        RTD_CUDA(cudaMemcpyAsync(a.data(), b->node_a.ptr, nn * sizeof(float4), cudaMemcpyDeviceToHost, st));
        RTD_CUDA(cudaMemcpyAsync(bb.data(), b->node_b.ptr, nn * sizeof(uint4), cudaMemcpyDeviceToHost, st));
    }
    if (h_order && b->n)
        RTD_CUDA(cudaMemcpyAsync(h_order, b->order.ptr, b->n * 4, cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    if (h_flat_nodes) {
        // FlatNode: com (3 f32), mass, width, is_leaf, next_idx, autorope, bucket_start, num_particles
        unsigned char *out = static_cast<unsigned char *>(h_flat_nodes);
        for (uint32_t i = 0; i < nn; ++i) {
            float f[5] = {a[i].x, a[i].y, a[i].z, a[i].w, 0.f};
            memcpy(&f[4], &bb[i].w, 4);
            const bool leaf = (bb[i].z & BH_LEAF_BIT) != 0;
            uint32_t u[5] = {leaf ? 1u : 0u, i + 1, bb[i].x, leaf ? bb[i].y : 0u,
                             leaf ? (bb[i].z & ~BH_LEAF_BIT) : 0u};
            memcpy(out + 40 * (size_t)i, f, 20);
            memcpy(out + 40 * (size_t)i + 20, u, 20);
        }
    }
    return RTD_OK;
}

rtd_status rtd_barnes_hut_host(rtd_context *ctx, const rtd_body *bodies, uint64_t n, float theta,
                               float G, rtd_vec3 *out_forces) {
    if (!ctx) return fail(RTD_ERR_INVALID_ARGUMENT, "context is NULL");
    if (n && (!bodies || !out_forces)) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL host buffer");
    static_assert(sizeof(rtd_body) == 28, "Body is 28 bytes");
    rtd_context_bh *c = context_bh(ctx);
    if (!c) return fail(RTD_ERR_OUT_OF_MEMORY, "host allocation failed");
    cudaStream_t st = context_stream(ctx);
    RTD_TRY(c->bodies.reserve(n * sizeof(rtd_body)));
    RTD_TRY(c->pos.reserve(n * 12));
    RTD_TRY(c->mass.reserve(n * 4));
    RTD_TRY(c->out.reserve(n * 12));
    if (n) {
        RTD_CUDA(cudaMemcpyAsync(c->bodies.ptr, bodies, n * sizeof(rtd_body), cudaMemcpyHostToDevice, st));
        split_bodies_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(
            c->bodies.as<float>(), n, c->pos.as<float>(), c->mass.as<float>());
        RTD_LAUNCH_CHECK();
    }
    rtd_bh_params p;
    rtd_bh_params_default(&p);
    p.theta = theta;
    p.G = G;
    RTD_TRY(bh_build(&c->bh, c->pos.as<float>(), c->mass.as<float>(), n, &p, st));
    RTD_TRY(bh_forward(&c->bh, &p, c->out.as<float>(), nullptr, st));
    if (n) RTD_CUDA(cudaMemcpyAsync(out_forces, c->out.ptr, n * 12, cudaMemcpyDeviceToHost, st));
    RTD_CUDA(cudaStreamSynchronize(st));
    return check_bh_errors(&c->bh, st);
}

}  // extern "C"

namespace rtd {
rtd_status bh_interaction_counts(rtd_bh *b, float theta, uint64_t stride, uint64_t *h_cells,
                                 uint64_t *h_bodies, uint64_t *h_sampled, cudaStream_t st);
}  // namespace rtd

extern "C" rtd_status rtd_bh_interaction_counts(rtd_bh *b, float theta, uint64_t stride,
                                                uint64_t *cells, uint64_t *bodies,
                                                uint64_t *sampled, rtd_stream stream) {
    return rtd::bh_interaction_counts(b, theta, stride, cells, bodies, sampled,
                                      (cudaStream_t)stream);
}
