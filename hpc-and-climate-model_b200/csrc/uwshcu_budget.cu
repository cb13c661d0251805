// uwshcu_budget.cu -- column energy and water budgets of a compute_uwshcu call on the device.
//
// check_energy_chng (check_energy.F90:321-395) as CAM applies it after the shallow scheme
// (tphysbc.F90:446-447: flx_vap = 0, flx_cnd = precip + rliq, flx_ice = snow, flx_sen = 0), on the
// state before the call and the state advanced by dt with the call's tendencies:
//   te = sum_k [ 0.5 (u^2 + v^2) + s + (latvap + latice) qv + latice ql ] dp/g
//   tw = sum_k (qv + ql + qi) dp/g
//   te_rer = (te_before + te_tnd dt - te_after) / te_before,  te_tnd = -(flx_cnd - snow) 1000 latice
//   tw_rer = (tw_before + tw_tnd dt - tw_after) / tw_before,  tw_tnd = -flx_cnd 1000
// CAM flags |te_rer| > 1e-14 and |tw_rer| > 1e-10.  Sums run over CAM's level order (top to bottom);
// the unit is built without FMA contraction, so the results are those of the same expressions
// evaluated in order on the host.
#include <cuda_runtime.h>

#include "uwshcu_common.cuh"

namespace {

__global__ void uw_budget_kernel(int mix, int mkx, int iend, int inv, double dt, double latvap,
                                 double latice, double g, const double* __restrict__ s0,
                                 const double* __restrict__ qv0, const double* __restrict__ ql0,
                                 const double* __restrict__ qi0, const double* __restrict__ u0,
                                 const double* __restrict__ v0, const double* __restrict__ dp0,
                                 const double* __restrict__ sten, const double* __restrict__ qvten,
                                 const double* __restrict__ qlten, const double* __restrict__ qiten,
                                 const double* __restrict__ uten, const double* __restrict__ vten,
                                 const double* __restrict__ precip, const double* __restrict__ snow,
                                 const double* __restrict__ rliq, double* __restrict__ te_rer,
                                 double* __restrict__ tw_rer)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= iend) return;
    double te0 = 0.0, tw0 = 0.0, te1 = 0.0, tw1 = 0.0;
    for (int j = 0; j < mkx; j++) {
        // CAM level order: top first.  Bottom-up arrays (inv = 0) hold the top layer in row mkx-1.
        const size_t r = (size_t)(inv ? j : mkx - 1 - j) * mix + i;
        const double dp = dp0[r];
        const double u = u0[r], v = v0[r], sv = s0[r], qv = qv0[r], ql = ql0[r], qi = qi0[r];
        const double u1 = u + uten[r] * dt, v1 = v + vten[r] * dt, s1 = sv + sten[r] * dt;
        const double qv1 = qv + qvten[r] * dt, ql1 = ql + qlten[r] * dt, qi1 = qi + qiten[r] * dt;
        te0 = te0 + 0.5 * (u * u + v * v) * dp / g + sv * dp / g + (latvap + latice) * qv * dp / g + latice * ql * dp / g;
        tw0 = tw0 + (qv + ql + qi) * dp / g;
        te1 = te1 + 0.5 * (u1 * u1 + v1 * v1) * dp / g + s1 * dp / g + (latvap + latice) * qv1 * dp / g + latice * ql1 * dp / g;
        tw1 = tw1 + (qv1 + ql1 + qi1) * dp / g;
    }
    const double flx_cnd = precip[i] + rliq[i];
    const double te_tnd = -(flx_cnd - snow[i]) * 1000.0 * latice;
    const double tw_tnd = -flx_cnd * 1000.0;
    te_rer[i] = ((te0 + te_tnd * dt) - te1) / te0;
    tw_rer[i] = tw0 > 0.0 ? ((tw0 + tw_tnd * dt) - tw1) / tw0 : 0.0;
}

}  // namespace

extern "C" cudaError_t uw_budget_launch(int mix, int mkx, int iend, int inv, double dt, double latvap,
                                        double latice, double g, const double* s0, const double* qv0,
                                        const double* ql0, const double* qi0, const double* u0,
                                        const double* v0, const double* dp0, const double* sten,
                                        const double* qvten, const double* qlten, const double* qiten,
                                        const double* uten, const double* vten, const double* precip,
                                        const double* snow, const double* rliq, double* te_rer,
                                        double* tw_rer, cudaStream_t stream)
{
    if (iend <= 0) return cudaSuccess;
    uw_budget_kernel<<<(iend + 255) / 256, 256, 0, stream>>>(mix, mkx, iend, inv, dt, latvap, latice, g, s0, qv0,
                                                             ql0, qi0, u0, v0, dp0, sten, qvten, qlten, qiten,
                                                             uten, vten, precip, snow, rliq, te_rer, tw_rer);
    return cudaGetLastError();
}
