// bh_integrate.cu -- time integration of the Barnes-Hut bodies.
//
// The reference's Body carries a velocity (gprt-core/src/lib.rs:311-317)
// that nothing advances.  Here a kick-drift-kick leapfrog steps positions
// and velocities with the Plummer-law accelerations, rebuilding the tree
// from the same Morton pipeline every step:
//   v += a(x) dt/2;  x += v dt;  rebuild;  a = a(x);  v += a dt/2.
// The acceleration buffer carries a(x) from one call to the next.
#include <rtdsl.h>

#include "bh.cuh"

namespace rtd {

rtd_status bh_forward(rtd_bh *b, const rtd_bh_params *p, float *d_out, float *d_phi,
                      cudaStream_t st);

namespace {

__global__ void kick_kernel(float *__restrict__ vel, const float *__restrict__ acc, uint64_t n3,
                            float half_dt) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3;
         i += (uint64_t)gridDim.x * blockDim.x)
        vel[i] = fmaf(acc[i], half_dt, vel[i]);
}

__global__ void drift_kernel(float *__restrict__ pos, const float *__restrict__ vel, uint64_t n3,
                             float dt) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3;
         i += (uint64_t)gridDim.x * blockDim.x)
        pos[i] = fmaf(vel[i], dt, pos[i]);
}

}  // namespace
}  // namespace rtd

using namespace rtd;

extern "C" rtd_status rtd_bh_leapfrog(rtd_bh *b, const rtd_bh_params *p, float *d_pos,
                                      float *d_vel, const float *d_mass, uint64_t n, float dt,
                                      uint32_t steps, float *d_acc, int acc_valid,
                                      rtd_stream stream) {
    if (!b) return fail(RTD_ERR_INVALID_ARGUMENT, "bh handle is NULL");
    rtd_bh_params def;
    rtd_bh_params_default(&def);
    def.law = RTD_BH_LAW_PLUMMER;
    if (!p) p = &def;
    if (p->law != RTD_BH_LAW_PLUMMER)
        return fail(RTD_ERR_UNSUPPORTED, "the leapfrog integrates the Plummer law");
    if (!(dt == dt) || !(fabsf(dt) < INFINITY)) return fail(RTD_ERR_INVALID_ARGUMENT, "dt must be finite");
    if (n == 0 || steps == 0) return RTD_OK;
    if (!d_pos || !d_vel || !d_mass || !d_acc) return fail(RTD_ERR_INVALID_ARGUMENT, "NULL device buffer");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t n3 = 3 * n;
    const int g = grid_for(n3, 256, 148 * 8);
    if (!acc_valid) {
        RTD_TRY(bh_build(b, d_pos, d_mass, n, p, st));
        RTD_TRY(bh_forward(b, p, d_acc, nullptr, st));
    }
    for (uint32_t s = 0; s < steps; ++s) {
        kick_kernel<<<g, 256, 0, st>>>(d_vel, d_acc, n3, 0.5f * dt);
        RTD_LAUNCH_CHECK();
        drift_kernel<<<g, 256, 0, st>>>(d_pos, d_vel, n3, dt);
        RTD_LAUNCH_CHECK();
        RTD_TRY(bh_build(b, d_pos, d_mass, n, p, st));
        RTD_TRY(bh_forward(b, p, d_acc, nullptr, st));
        kick_kernel<<<g, 256, 0, st>>>(d_vel, d_acc, n3, 0.5f * dt);
        RTD_LAUNCH_CHECK();
    }
    return RTD_OK;
}
