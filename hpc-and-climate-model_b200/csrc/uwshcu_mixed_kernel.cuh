// uwshcu_mixed_kernel.cuh -- mixed-precision sm_100a kernel of compute_uwshcu (uwshcu.F90:478-4664),
// one thread per column, same schedule and column algorithm as the FP64 kernel.
//
// Precision map.  FP32 ("bulk"): exner functions, the saturation lookups of the buoyancy sorting and
// the evaporation (qsat), CIN integrands (single_cin/getbuoy), entrainment/detrainment mixing, the
// updraft profiles, penetrative entrainment, fluxbelowinv, the flux and tendency assembly, findsp.
// FP64 islands: the conden saturation adjustment (Newton iteration and its saturation lookups), the
// quadratic roots of the mixing-fraction and penetration solves, the LCL inversion (qsinvert), the
// implicit-CIN quantities (cin sums, del_CIN, compute_alpha) and compute_mumin2, and the
// positive_moisture fixer with its column sums.  Vertical FP32 sums (tkeavg, the rain/snow
// fluxes, the evaporated fluxes, rliq) are Kahan-compensated.  Inputs and outputs keep the FP64 ABI.
//
// The FP64 islands use algebraically equal but cheaper forms than the Fortran (one division per
// Newton step instead of six, FMA contraction allowed) and stop the conden iteration once the
// temperature change is below 1e-9 K (each lane at its own step, so results do not depend on which
// columns share a warp); this kernel is checked against the FP64 oracle with error
// statistics, not bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include "uwshcu_common.cuh"
#include "uw_state.cuh"

namespace {

__constant__ UwConst c;
__constant__ double c_estbl[UW_TBL];

typedef float R;

#define MX(a, b) ((a) > (b) ? (a) : (b))
#define MN(a, b) ((a) < (b) ? (a) : (b))

// Compensated (Kahan) FP32 sum.
struct Kahan {
    float s = 0.f, e = 0.f;
    __device__ __forceinline__ void reset() { s = 0.f; e = 0.f; }
    __device__ __forceinline__ void add(float x)
    {
        float y = x - e;
        float t = s + y;
        e = (t - s) - y;
        s = t;
    }
};
// Kahan sums in the hand-off state of the sorted schedule (uw_state.cuh): two words (the scalar
// overloads there stay visible next to these).
using ::uw_st_get;
using ::uw_st_put;
__device__ __forceinline__ void uw_st_put(double* st, size_t& w, size_t cs, const Kahan& x)
{
    st[w++ * cs] = (double)x.s;
    st[w++ * cs] = (double)x.e;
}
__device__ __forceinline__ void uw_st_get(const double* st, size_t& w, size_t cs, Kahan& x)
{
    x.s = (float)st[w++ * cs];
    x.e = (float)st[w++ * cs];
}

__device__ __forceinline__ float estblf_f(float td, const float* __restrict__ tf)
{
    const float tmin = (float)c.tmin, tmax = (float)c.tmax;
    float e = MX(MN(td, tmax), tmin);
    int i = (int)(e - tmin) + 1;
    float ai = truncf(e - tmin);
    return (tmin + ai - e + 1.0f) * tf[i - 1] - (tmin + ai - e) * tf[i];
}

__device__ __forceinline__ double estblf_d(double td, const double* __restrict__ td_)
{
    double e = MX(MN(td, c.tmax), c.tmin);
    int i = (int)(e - c.tmin) + 1;
    double ai = trunc(e - c.tmin);
    return (c.tmin + ai - e + 1.0) * td_[i - 1] - (c.tmin + ai - e) * td_[i];
}

// qs of vqsatd (wv_saturation.F90:482-609) in FP32.
__device__ __forceinline__ float qsat_qs(float t, float p, const double* __restrict__ tbld, const float* __restrict__ tblf)
{
    (void)tbld;
    float es = estblf_f(t, tblf);
    float qs = (float)c.epsqs * es / (p - (float)c.omeps * es);
    qs = MN(1.0f, qs);
    if (qs < 0.0f) qs = 1.0f;
    return qs;
}

// vqsatd with gam, FP64 (used by the LCL inversion).
__device__ __forceinline__ void qsat3_d(double t, double p, double& es, double& qs, double& gam,
                                        const double* __restrict__ tbld)
{
    es = estblf_d(t, tbld);
    qs = c.epsqs * es / (p - c.omeps * es);
    qs = MN(1.0, qs);
    if (qs < 0.0) {
        qs = 1.0;
        es = p;
    }
    double hltalt, desdt;
    if (c.icephs && c.ttrice != 0.0) {
        double tc = t - c.tmelt;
        bool lflg = (tc >= -c.ttrice && tc < 0.0);
        double weight = MN(-tc * c.trinv, 1.0);
        hltalt = (t < c.tmelt) ? c.hlatv + weight * c.hlatf : c.hlatv - 2369.0 * tc;
        double tterm = lflg ? c.pcf[0] + tc * (c.pcf[1] + tc * (c.pcf[2] + tc * (c.pcf[3] + tc * c.pcf[4]))) : 0.0;
        desdt = hltalt * es / (c.rgasv * t * t) + tterm * c.trinv;
    } else {
        double hlatsb = c.icephs ? c.hlatv + c.hlatf : c.hlatv;
        hltalt = (t < c.tmelt) ? hlatsb : c.hlatv - 2369.0 * (t - c.tmelt);
        desdt = hltalt * es / (c.rgasv * t * t);
    }
    gam = hltalt * qs * p * desdt / (c.cpws * es * (p - c.omeps * es));
    if (qs == 1.0) gam = 0.0;
}

__device__ __forceinline__ float exnf(float p) { return powf(p / (float)c.p00, (float)c.rovcp); }

// conden (uwshcu.F90:4718-4785): FP64 saturation adjustment from FP32 (p, exner, thl, qt).
__device__ __noinline__ int conden(R p, R ex, R thl, R qt, R& th, R& qv, R& ql, R& qi,
                                      const double* __restrict__ tbld, const float* __restrict__ tblf)
{
    (void)tblf;
    const double pd = p, qtd = qt;
    const double tc = (double)thl * (double)ex;
    const double nu = MX(MN((268.0 - tc) * 0.05, 1.0), 0.0);
    const double leff = (1.0 - nu) * c.xlv + nu * c.xls;
    double es = estblf_d(tc, tbld);
    double rvls = MN(1.0, c.epsqs * es / (pd - c.omeps * es));
    if (rvls < 0.0) rvls = 1.0;
    if (rvls >= qtd) {
        qv = qt;
        ql = 0.0f;
        qi = 0.0f;
        th = thl;       // tc / ex
        return 0;
    }
    const double cpl = c.cp / leff;
    const double a = c.ep2 * leff / c.r;
    double temps = tc;
    bool done = false;
#pragma unroll 1
    for (int it = 0; it < 10; it++) {
        if (!done) {
            const double rt = 1.0 / temps;
            const double dT = ((tc - temps) * cpl + qtd - rvls) / (cpl + a * rvls * rt * rt);
            temps += dT;
            es = estblf_d(temps, tbld);
            rvls = MN(1.0, c.epsqs * es / (pd - c.omeps * es));
            if (rvls < 0.0) rvls = 1.0;
            done = fabs(dT) < 1.e-9;
        }
        if (__all_sync(__activemask(), done)) break;
    }
    const double qc = MX(qtd - rvls, 0.0);
    qv = (R)(qtd - qc);
    ql = (R)(qc * (1.0 - nu));
    qi = (R)(nu * qc);
    th = (R)(temps / (double)ex);
    return (fabs((temps - (leff / c.cp) * qc) - tc) >= 1.0) ? 1 : 0;
}

// roots (uwshcu.F90:4787-4829), FP64.
__device__ __forceinline__ int roots(double a, double b, double cc, double& r1, double& r2)
{
    int status = 0;
    if (a == 0.0) {
        if (b == 0.0) status = 1;
        else r1 = -cc / b;
        r2 = r1;
    } else {
        if (b == 0.0) {
            if (a * cc > 0.0) status = 2;
            else r1 = sqrt(-cc / a);
            r2 = -r1;
        } else {
            if ((b * b - 4.0 * a * cc) < 0.0) {
                status = 3;
            } else {
                double q = -0.5 * (b + copysign(1.0, b) * sqrt(b * b - 4.0 * a * cc));
                r1 = q / a;
                r2 = cc / q;
            }
        }
    }
    return status;
}

template <int KP>
__device__ __forceinline__ void slope(int mkx, const R* field, const R* p0, R* sl)
{
    R below = (field[2] - field[1]) / (p0[2] - p0[1]);
#pragma unroll 1
    for (int k = 2; k <= mkx; k++) {
        R above = (field[k] - field[k - 1]) / (p0[k] - p0[k - 1]);
        if (above > 0.0f) sl[k - 1] = MX(0.0f, MN(above, below));
        else sl[k - 1] = MN(0.0f, MX(above, below));
        below = above;
    }
    sl[mkx] = sl[mkx - 1];
}

// qsinvert (uwshcu.F90:4863-4929), FP64 Newton iteration for the LCL pressure.
__device__ R qsinvert(R qt_, R thl_, R psfc_, R exsfc_, const double* __restrict__ tbld, const float* __restrict__ tblf)
{
    (void)tblf;
    (void)exsfc_;
    const double qt = qt_, thl = thl_, psfc = psfc_;
    const double psmin = 100.0 * 100.0, dpsmax = 1.0;
    double es, qs, gam;
    double Ti = thl * pow(psfc / c.p00, c.rovcp);
    qsat3_d(Ti, psfc, es, qs, gam, tbld);
    double rhi = qt / qs;
    if (rhi <= 0.01) return (R)psmin;
    double TLCL = 55.0 + 1.0 / (1.0 / (Ti - 55.0) - log(rhi) / 2840.0);
    double PiLCL = TLCL / thl;
    double ps = c.p00 * pow(PiLCL, 1.0 / c.rovcp);
#pragma unroll 1
    for (int i = 1; i <= 10; i++) {
        double Pis = pow(ps / c.p00, c.rovcp);
        double Ts = thl * Pis;
        qsat3_d(Ts, ps, es, qs, gam, tbld);
        double err = qt - qs;
        double nu = MX(MN((268.0 - Ts) / 20.0, 1.0), 0.0);
        double leff = (1.0 - nu) * c.xlv + nu * c.xls;
        double dlnqsdT = gam * (c.cp / leff) / qs;
        double dPisdps = c.rovcp * Pis / ps;
        double dlnqsdps = -1.0 / (ps - (1.0 - c.ep2) * es);
        double derrdps = -qs * (dlnqsdT * thl * dPisdps + dlnqsdps);
        double dps = -err / derrdps;
        ps = ps + dps;
        if (ps < 0.0) return (R)psmin;
        if (fabs(dps) <= dpsmax) return (R)ps;
    }
    return (R)psmin;
}

// compute_alpha (uwshcu.F90:4931-4950), FP64.
__device__ double compute_alpha(double del_CIN, double ke)
{
    double x0 = 0.0;
#pragma unroll 1
    for (int it = 0; it < 10; it++) {
        double e = exp(-x0 * ke * del_CIN);
        x0 = x0 - (e - x0) / (-ke * del_CIN * e - 1.0);
    }
    return x0;
}

// compute_mumin2 (uwshcu.F90:4952-4979), FP64.
__device__ R compute_mumin2(R mulcl_, R rmaxfrac_, R mulow_)
{
    const double mulcl = mulcl_, rmaxfrac = rmaxfrac_;
    double x0 = mulow_;
#pragma unroll 1
    for (int it = 0; it < 10; it++) {
        double ex = exp(-(x0 * x0));
        double ef = erfc(x0);
        double exf = ex / ef;
        double t1 = ex / 2.0 / rmaxfrac;
        double t2 = mulcl * 2.5066 / 2.0;
        double f = 0.5 * (exf * exf) - 0.5 * (t1 * t1) - (t2 * t2);
        double fs = (2.0 * (exf * exf)) * (exf / sqrt(3.141592) - x0) + (0.5 * x0 * (ex * ex)) / (rmaxfrac * rmaxfrac);
        x0 = x0 - f / fs;
    }
    return (R)x0;
}

// compute_ppen (uwshcu.F90:4981-5028), FP32.
__device__ R compute_ppen(R wtwb, R D, R bogbot, R bogtop, R rho0j, R dpen)
{
    R x0;
    R SB = (bogtop - bogbot) / dpen;
    R s00 = bogbot / rho0j - D * wtwb;
    if (D * dpen < 1.e-8f) {
        if (s00 >= 0.0f) x0 = dpen;
        else x0 = MX(0.0f, MN(dpen, -0.5f * wtwb / s00));
    } else {
        if (s00 >= 0.0f) x0 = dpen;
        else x0 = 0.0f;
        const R q = 1.0f / (D * rho0j);
        const R b2 = bogbot - SB / (2.0f * D);
#pragma unroll 1
        for (int it = 0; it < 5; it++) {
            R e = expf(-2.0f * D * x0);
            R f = e * (wtwb - b2 * q) + (SB * x0 + b2) * q;
            R fs = -2.0f * D * e * (wtwb - b2 * q) + SB * q;
            if (fs >= 0.0f) fs = MX(fs, 1.e-10f);
            else fs = MN(fs, -1.e-10f);
            x0 = x0 - f / fs;
        }
    }
    return -MX(0.0f, MN(dpen, x0));
}

__device__ __forceinline__ R single_cin(R pbot, R exb, R thv0bot, R ptop, R ext, R thv0top, R thvubot, R thvutop)
{
    const R r = (R)c.r;
    return ((1.0f - thvubot / thv0bot) + (1.0f - thvutop / thv0top)) * (pbot - ptop) /
           (pbot / (r * thv0bot * exb) + ptop / (r * thv0top * ext));
}

// getbuoy (uwshcu.F90:4672-4702): FP32 integrand, FP64 CIN accumulator.
__device__ __forceinline__ void getbuoy(R pbot, R exb, R thv0bot, R ptop, R ext, R thv0top, R thvubot,
                                        R thvutop, R& plfc, double& cin)
{
    const R r = (R)c.r;
    if (thvubot > thv0bot && thvutop > thv0top) {
        plfc = pbot;
    } else if (thvubot <= thv0bot && thvutop <= thv0top) {
        cin = cin - ((thvubot / thv0bot - 1.0f) + (thvutop / thv0top - 1.0f)) * (pbot - ptop) /
                        (pbot / (r * thv0bot * exb) + ptop / (r * thv0top * ext));
    } else if (thvubot > thv0bot && thvutop <= thv0top) {
        R frc = (thvutop / thv0top - 1.0f) / ((thvutop / thv0top - 1.0f) - (thvubot / thv0bot - 1.0f));
        cin = cin - (thvutop / thv0top - 1.0f) * ((ptop + frc * (pbot - ptop)) - ptop) /
                        (pbot / (r * thv0bot * exb) + ptop / (r * thv0top * ext));
    } else {
        R frc = (thvubot / thv0bot - 1.0f) / ((thvubot / thv0bot - 1.0f) - (thvutop / thv0top - 1.0f));
        plfc = pbot - frc * (pbot - ptop);
        cin = cin - (thvubot / thv0bot - 1.0f) * (pbot - plfc) /
                        (pbot / (r * thv0bot * exb) + ptop / (r * thv0top * ext));
    }
}

__device__ __forceinline__ void fluxbelowinv(R cbmf, const R* ps0, int kinv, R dt, R xsrc, R xmean, R xtopin,
                                             R xbotin, R* xflx)
{
    R xtop, xbot;
    R dp = ps0[kinv - 1] - ps0[kinv];
    if (fabsf(xbotin - xtopin) <= 1.e-13f) {
        xbot = xbotin - 1.e-13f;
        xtop = xtopin + 1.e-13f;
    } else {
        xbot = xbotin;
        xtop = xtopin;
    }
    R xtop_ori = xtop, xbot_ori = xbot;
    R rcbmf = (cbmf * (R)c.g * dt) / dp;
    R rpeff = (xmean - xtop) / (xbot - xtop);
    rpeff = MN(MX(0.0f, rpeff), 1.0f);
    if (rpeff == 0.0f || rpeff == 1.0f) {
        xbot = xmean;
        xtop = xmean;
    }
    R rr = rpeff / rcbmf;
    R pinv = ps0[kinv - 1] - rpeff * dp;
    const R s = cbmf * (xsrc - xbot) / (ps0[0] - pinv);
#pragma unroll 1
    for (int k = 0; k <= kinv - 1; k++) xflx[k] = s * (ps0[0] - ps0[k]);
    if (rr <= 1.0f) xflx[kinv - 1] = xflx[kinv - 1] - (1.0f - rr) * cbmf * (xtop_ori - xbot_ori);
}

// findsp (uwshcu.F90:5164-5454) for one point, FP32.
__device__ R findsp_point(R q, R t, R p, unsigned int& errbits, const double* __restrict__ tbld, const float* __restrict__ tblf)
{
    (void)tbld;
    const R epsqs = (R)c.epsqs, omeps = 1.0f - epsqs, trinv = 1.0f / (R)c.ttrice, cpws = (R)c.cpws;
    const R hlatv = (R)c.hlatv, hlatf = (R)c.hlatf, ttrice = (R)c.ttrice, rgasv = (R)c.rgasv;
    const R c3 = 287.04f * (7.5f * 2.302585093f) / cpws, dttol = 1.e-4f, dqtol = 1.e-4f, tt0 = 273.15f;
    R dtt = 0.0f, dq = 0.0f, enin, enout = 1.0f, tsp, qsp, hltalt = 0.0f;
    int doit = 0;
    R tlim = MN(MX(t, 173.0f), 373.0f);
    R es = estblf_f(tlim, tblf);
    R denom = p - omeps * es;
    R qs = epsqs * es / denom;
    if (p > 5.0f * es && qs > 0.0f && qs < 0.5f) {
        qs = MN(qs, 1.0f);
        R tc = tlim - tt0;
        R weight = MN(-tc * trinv, 1.0f);
        hltalt = (tlim < tt0) ? hlatv + weight * hlatf : hlatv - 2369.0f * tc;
        enin = cpws * tlim + hltalt * q;
        R c1 = hltalt * c3;
        R c2 = (tlim + 36.0f) * (tlim + 36.0f);
        R qvd = c2 / (c2 + c1 * qs) * (q - qs);
        tsp = tlim + ((hltalt / cpws) * qvd);
        es = estblf_f(tsp, tblf);
        qsp = MN(epsqs * es / (p - omeps * es), 1.0f);
    } else {
        doit = 1;
        tsp = tlim;
        qsp = q;
        enin = 1.0f;
    }
#pragma unroll 1
    for (int l = 1; l <= 8 && doit == 0; l++) {
        es = estblf_f(tsp, tblf);
        qs = MN(epsqs * es / (p - omeps * es), 1.0f);
        R tc = tsp - tt0;
        bool lflg = (tc >= -ttrice && tc < 0.0f);
        R weight = MN(-tc * trinv, 1.0f);
        hltalt = (tsp < tt0) ? hlatv + weight * hlatf : hlatv - 2369.0f * tc;
        R tterm = lflg ? (R)c.pcf[0] + tc * ((R)c.pcf[1] + tc * ((R)c.pcf[2] + tc * ((R)c.pcf[3] + tc * (R)c.pcf[4]))) : 0.0f;
        R desdt = hltalt * es / (rgasv * tsp * tsp) + tterm * trinv;
        R dqsdt = (epsqs + omeps * qs) / (p - omeps * es) * desdt;
        R gg = enin - (cpws * tsp + hltalt * qsp);
        R dgdt = -(cpws + hltalt * dqsdt);
        R t1 = tsp - gg / dgdt;
        dtt = fabsf(t1 - tsp) / t1;
        tsp = MX(t1, (R)c.tmin);
        es = estblf_f(tsp, tblf);
        R q1 = MN(epsqs * es / (p - omeps * es), 1.0f);
        dq = fabsf(q1 - qsp) / MX(q1, 1.e-12f);
        qsp = q1;
        if (dtt < dttol && dq < dqtol) doit = 2;
        enout = cpws * tsp + hltalt * qsp;
        if (tsp < 174.16f) doit = 4;
    }
    if (doit == 0 && (dtt > dttol || dq > dqtol)) errbits |= UW_ERRBIT_FINDSP;
    if (doit == 2 && fabsf((enin - enout) / (enin + enout)) > 1.e-4f) errbits |= UW_ERRBIT_ENTHALPY;
    return qsp;
}

}  // namespace

#define UW_MODE_ALL 0
#define UW_MODE_TRIGGER 1
#define UW_MODE_LIST 2

// ------------------------------------------------------------------------------------------------
// The column kernel.  KP bounds the level arrays (mkx + 1 <= KP), NC the tracer count.
//
// MODE selects what a launch does:
//   UW_MODE_ALL      every column 0..iend-1 runs the whole scheme (single pass);
//   UW_MODE_TRIGGER  every column runs up to the end of the iteration-1 closure (uwshcu.F90:2184).
//                    Columns that leave the scheme on the way write their final outputs (the
//                    label-333 zeroes); the others are appended to the worklist `wl` (warp ballot,
//                    one atomicAdd per warp) and write nothing;
//   UW_MODE_LIST     thread t runs the whole scheme for column wl[t], t < *wl_count;
//   UW_MODE_LIST1    as UW_MODE_LIST, except that a column taking the implicit-CIN branch of
//                    iteration 2 (uwshcu.F90:1759-1889) stores its state in the hand-off region
//                    A.hand (a free slot permitting) and stops there;
//   UW_MODE_RESUME   thread t continues hand-off slot order[t] from that point to the end.
// The worklist path recomputes the phase-1 part of a convecting column instead of storing it: the
// heavy buoyancy-sorting work then runs in warps made only of convecting columns.  The split at the
// CIN decision drops the columns that end in iteration 1 or take the explicit-CIN branch from the
// warps of iteration 2, and sorts the rest by their iteration-1 updraft depth, which predicts the
// iteration-2 depth (lanes whose updraft has stopped wait for the deepest one in their warp).
#define UW_MODE_LIST1 3
#define UW_MODE_RESUME 4
#define UW_MODE_IS_LIST(m) ((m) == UW_MODE_LIST || (m) == UW_MODE_LIST1 || (m) == UW_MODE_RESUME)

// The column code and the kernels have internal linkage: every unit that includes a column-code
// header (FP64, fast, mixed, tangent) carries its own copies under the same names.
namespace {

// One column per lane: column i_in of A when `active` (in UW_MODE_RESUME, i_in is a hand-off slot).
// All 32 lanes of the warp must call it together (it starts with a warp ballot).  `tbl` is the saturation table in shared memory.  In
// UW_MODE_TRIGGER, convecting columns are appended to wl / *wl_count.
// FAST = 1: the fast-FP64 precision mode (conden_fast in place of conden), not bit-exact.
// ZW = 1: compute_zwshcu (zwshcu.F90), which reads A.omega and the zw_* options; compiled out of the
// compute_uwshcu instantiations.
template <int KP, int NC, int MODE, int FAST, int ZW = 0>
__device__ __forceinline__ void uw_column(const UwArgs& A, const double* __restrict__ tbld, const float* __restrict__ tblf, const int i_in,
                                          const bool active, int* __restrict__ wl, int* __restrict__ wl_count)
{
    const int i = (MODE == UW_MODE_RESUME && active) ? A.hand->col[i_in] : i_in;
#define CONDEN(...) conden(__VA_ARGS__)
    bool cand = false;
    // lanes of this warp that run a column; UW_SYNC() joins them where every one of them arrives
    const unsigned live = __ballot_sync(0xffffffffu, active);
#define UW_SYNC() __syncwarp(live)
    if (active) {

    const int mix = A.mix, mkx = A.mkx, ncnst = A.ncnst;
    const R dt = A.dt;
    const R xlv = c.xlv, xls = c.xls, cp = c.cp, zvir = c.zvir, r = c.r, g = c.g, p00 = c.p00,
                 rovcp = c.rovcp, rpen = c.rpen;
    const R rle = c.rle, rkm = c.rkm, rkfre = 1.0f, rmaxfrac = 0.10f, mumin1 = 0.906f, rbuoy = 1.0f,
                 rdrag = 1.0f, epsvarw = 5.e-4f, PGFc = 0.7f, criqc = c.criqc, frc_rasn = 1.0f, kevp = 2.e-6f;
    const int ixnumliq = c.ixnumliq, ixnumice = c.ixnumice;

    // Row of level k in the caller's arrays: bottom-up (compute_uwshcu) or CAM's top-down order
    // (compute_uwshcu_inv, uwshcu.F90:380-469, where interface k and layer k both sit at row mkx-k).
    const int inv = A.inv;
#define RI(k) (inv ? (mkx - (k)) : (k))
#define RL(k) (inv ? (mkx - (k)) : ((k) - 1))
#define GI(a, k) ((R)__ldg(&A.a[(size_t)RI(k) * mix + i]))
#define GL(a, k) ((R)__ldg(&A.a[(size_t)RL(k) * mix + i]))
#define GT(m, k) ((R)__ldg(&A.tr0[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]))
#define OI(a, k) A.a[(size_t)RI(k) * mix + i]
#define OL(a, k) A.a[(size_t)RL(k) * mix + i]
#define OT(m, k) A.trten[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]
#define CNT(x) (inv ? (double)(mkx + 1) - (double)(x) : (double)(x))
#define DLV(j, k) A.diag_level[((size_t)(j) * (mkx + 1) + (k)) * mix + i]
// per-level diagnostics of the current state, levels bottom-up in both level orders
// (uwshcu.F90:1945-1990 and :4383-4433)
#define PUT_DIAG_LEVEL()                                                                                  \
    if (A.diag_level) {                                                                                   \
        for (int k = 0; k <= mkx; k++) {                                                                  \
            DLV(UW_DL_UFRC, k) = ufrc[k];                                                                 \
            DLV(UW_DL_QTU, k) = qtu[k];                                                                   \
            DLV(UW_DL_THLU, k) = thlu[k];                                                                 \
            DLV(UW_DL_THVU, k) = thvu[k];                                                                 \
            DLV(UW_DL_UU, k) = uu[k];                                                                     \
            DLV(UW_DL_VU, k) = vu[k];                                                                     \
            DLV(UW_DL_UEMF, k) = UEMF(k);                                                                 \
            DLV(UW_DL_FLXRAIN, k) = flxrain[k];                                                           \
            DLV(UW_DL_FLXSNOW, k) = flxsnow[k];                                                           \
        }                                                                                                 \
        for (int j = UW_DL_FER; j < UW_NDL; j++) DLV(j, 0) = 0.0f;                                         \
        for (int k = 1; k <= mkx; k++) {                                                                  \
            DLV(UW_DL_FER, k) = fer[k];                                                                   \
            DLV(UW_DL_FDR, k) = fdr[k];                                                                   \
            DLV(UW_DL_DWTEN, k) = dwten[k];                                                               \
            DLV(UW_DL_DITEN, k) = diten[k];                                                               \
        }                                                                                                 \
    }

    // ---- thread-private profiles ---------------------------------------------------------------
    R ps0[KP], p0[KP], dp0[KP], zs0[KP], exn0[KP], exns0[KP];
    R qv0[KP], ql0[KP], qi0[KP], t0[KP], s0[KP], qt0[KP], thl0[KP];
    R ssthl0[KP], ssqt0[KP], ssu0[KP], ssv0[KP], sstr0[NC][KP];
    R thv0bot[KP], thv0top[KP], thvl0bot[KP], thvl0top[KP];
    R thv0bot_o[KP], thv0top_o[KP], thvl0bot_o[KP], thvl0top_o[KP];
    R umf[KP], emf[KP], thlu[KP], qtu[KP], uu[KP], vu[KP], thvu[KP], wu[KP], ufrc[KP], rei[KP];
    R fer[KP], fdr[KP], dwten[KP], diten[KP], tru[NC][KP];
    R thlu_emf[KP], qtu_emf[KP], uu_emf[KP], vu_emf[KP], tru_emf[NC][KP];
    R slflx[KP], qtflx[KP], uflx[KP], vflx[KP], trflx[NC][KP], xflx[KP];
    R qlten_sink[KP], qiten_sink[KP], nlten_sink[KP], niten_sink[KP];
    R uten[KP], vten[KP], uf[KP], vf[KP], qrten[KP], qsten[KP], slten[KP], qtten[KP];
    R qlten[KP], qiten[KP], qvten[KP], sten[KP], qc[KP], qc_l[KP], qc_i[KP], evapc[KP];
    R flxrain[KP], flxsnow[KP], cufrc[KP], qcu[KP], qlu[KP], qiu[KP], trten[NC][KP];
    R qw0[KP], trflx_d[KP], trflx_u[KP];
    R trsrc[NC], tre[NC];

    unsigned int errbits = 0;
    int xflags = 0, lflags = 0;
    bool id_exit = false;
    // stop: the column leaves the scheme (the Fortran's `go to 333`); every later section skips.
    bool stop = false;
    int kinv = 0, klcl = 0, klfc = 0, krel = 0, kbup = 0, kpen = 0;
    int kinv_s = 0, klcl_s = 0, klfc_s = 0, krel_s = 0, kbup_s = 0, kpen_s = 0;
    double cin = 0, cinlcl = 0;
    R plcl = 0, plfc = 0, prel = 0, exlcl = 1.0f, exprel = 1.0f, tkeavg = 0,
           thvlmin = 0, qtsrc = 0, thlsrc = 0, thvlsrc = 0, usrc = 0, vsrc = 0, thv0lcl = 0, thv0rel = 0;
    double cin_i = 0, cinlcl_i = 0, ke = 0;
    R kinv_o_d = 0;
    int kinv_o = 0, klcl_o = 0, klfc_o = 0;
    R plcl_o = 0, plfc_o = 0, tkeavg_o = 0, thvlmin_o = 0, qtsrc_o = 0, thvlsrc_o = 0, thlsrc_o = 0,
           usrc_o = 0, vsrc_o = 0, thv0lcl_o = 0, trsrc_o[NC];
    R cin_s = -1.0f, cinlcl_s = -1.0f, plcl_s = 0, plfc_s = 0, pinv_s = 0, pbup_s = 0, ppen_s = 0,
           tkeavg_s = 0;
    R cbmf = 0, wlcl = 0, ufrclcl = 0, ppen = 0, precip = 0, snow = 0, cush, cnt, cnb;
    Kahan rliq;
    R thlu_top = 0, qtu_top = 0, exntop = 1.0f, drage = 0, bogbot = 0, bogtop = 0, rho0j = 0,
           wtwb = 0, wtw = 0;
    double xs1 = 0, xs2 = 0, xc1 = 0, xc2 = 0;
    R thj = 0, qvj = 0, qlj = 0, qij = 0;
    Kahan rainflx, snowflx;
    (void)kinv_o_d;
    const R pblh = __ldg(&A.pblh[i]);
    R tscaleh_r = 0.0f;   // UW_MODE_RESUME: tscaleh of the iteration handed over
    bool handed = false;      // UW_MODE_LIST1: the column continues in UW_MODE_RESUME

    if constexpr (MODE != UW_MODE_RESUME) {   // uniform

    // ---- output initialisation (uwshcu.F90:1087-1124) ------------------------------------------
    if (MODE != UW_MODE_TRIGGER) {
    for (int k = 0; k <= mkx; k++) {
        OI(umf, k) = 0.0f;
        OI(slflx, k) = 0.0f;
        OI(qtflx, k) = 0.0f;
        OI(flxprc1, k) = 0.0f;
        OI(flxsnow1, k) = 0.0f;
        OI(wu, k) = 0.0f;
    }
    for (int k = 1; k <= mkx; k++) {
        OL(qvten, k) = 0.0f; OL(qlten, k) = 0.0f; OL(qiten, k) = 0.0f; OL(sten, k) = 0.0f;
        OL(uten, k) = 0.0f; OL(vten, k) = 0.0f; OL(qrten, k) = 0.0f; OL(qsten, k) = 0.0f;
        OL(evapc, k) = 0.0f; OL(cufrc, k) = 0.0f; OL(qcu, k) = 0.0f; OL(qlu, k) = 0.0f;
        OL(qiu, k) = 0.0f; OL(qc, k) = 0.0f;
        for (int m = 1; m <= ncnst; m++) OT(m, k) = 0.0f;
    }
    A.precip[i] = 0.0f;
    A.snow[i] = 0.0f;
    A.cbmf[i] = 0.0f;
    A.rliq[i] = 0.0f;
    A.cnt[i] = CNT((R)mkx);
    A.cnb[i] = CNT(0.0f);
    }

    // ---- inputs and findsp (uwshcu.F90:1216-1259), and non-finite inputs ----------------------
    // Non-finite inputs have no counterpart in the Fortran, where a NaN or Inf propagates into the
    // column's outputs or stops the model in findsp: a column with a non-finite value in any input
    // the scheme reads takes the exit path (label-333 outputs), is marked UW_X_NONFINITE and sets
    // only that status bit (no findsp at or above the bad level, no conden).  The values are checked
    // as they are loaded; z0 and tke, which the scheme reads later and only at some levels, once here.
    bool nonfinite = !uw_isfinite(pblh) || !uw_isfinite(A.cush[i]);
    for (int k = 0; k <= mkx; k++) {
        ps0[k] = GI(ps0, k);
        zs0[k] = GI(zs0, k);
        nonfinite |= !uw_isfinite(ps0[k]) || !uw_isfinite(zs0[k]) || !uw_isfinite(GI(tke, k));
        exns0[k] = powf(ps0[k] / p00, rovcp);
    }
    for (int k = 1; k <= mkx; k++) {
        p0[k] = GL(p0, k);
        dp0[k] = GL(dp0, k);
        qv0[k] = GL(qv0, k);
        ql0[k] = GL(ql0, k);
        qi0[k] = GL(qi0, k);
        t0[k] = GL(t0, k);
        s0[k] = GL(s0, k);
        nonfinite |= !uw_isfinite(p0[k]) || !uw_isfinite(dp0[k]) || !uw_isfinite(qv0[k]) || !uw_isfinite(ql0[k]) ||
                     !uw_isfinite(qi0[k]) || !uw_isfinite(t0[k]) || !uw_isfinite(s0[k]) || !uw_isfinite(GL(z0, k));
        exn0[k] = powf(p0[k] / p00, rovcp);
        qt0[k] = (qv0[k] + ql0[k] + qi0[k]);
        thl0[k] = (t0[k] - xlv * ql0[k] / cp - xls * qi0[k] / cp) / exn0[k];
        qw0[k] = nonfinite ? 0.0f : findsp_point(qv0[k], t0[k], p0[k], errbits, tbld, tblf);
    }
    cush = A.cush[i];
    {
        R tmpf[KP];
        slope<KP>(mkx, thl0, p0, ssthl0);
        slope<KP>(mkx, qt0, p0, ssqt0);
        for (int k = 1; k <= mkx; k++) {
            tmpf[k] = GL(u0, k);
            nonfinite |= !uw_isfinite(tmpf[k]);
        }
        slope<KP>(mkx, tmpf, p0, ssu0);
        for (int k = 1; k <= mkx; k++) {
            tmpf[k] = GL(v0, k);
            nonfinite |= !uw_isfinite(tmpf[k]);
        }
        slope<KP>(mkx, tmpf, p0, ssv0);
        for (int m = 1; m <= ncnst; m++) {
            for (int k = 1; k <= mkx; k++) {
                tmpf[k] = GT(m, k);
                nonfinite |= !uw_isfinite(tmpf[k]);
            }
            slope<KP>(mkx, tmpf, p0, sstr0[m - 1]);
        }
    }
    if (nonfinite) {
        xflags |= UW_X_NONFINITE;
        errbits = UW_ERRBIT_NONFINITE;   // findsp of the levels below the bad one reports nothing
        id_exit = true;
        stop = true;
    }
    // thv0 at layer bottom/top (:1275-1299)
    for (int k = 1; k <= mkx && !nonfinite; k++) {
        R thl0bot = thl0[k] + ssthl0[k] * (ps0[k - 1] - p0[k]);
        R qt0bot = qt0[k] + ssqt0[k] * (ps0[k - 1] - p0[k]);
        if (CONDEN(ps0[k - 1], exns0[k - 1], thl0bot, qt0bot, thj, qvj, qlj, qij, tbld, tblf)) {
            xflags |= UW_X_CONDEN;
            id_exit = true;
            stop = true;
            break;
        }
        thv0bot[k] = thj * (1.0f + zvir * qvj - qlj - qij);
        thvl0bot[k] = thl0bot * (1.0f + zvir * qt0bot);
        R thl0top = thl0[k] + ssthl0[k] * (ps0[k] - p0[k]);
        R qt0top = qt0[k] + ssqt0[k] * (ps0[k] - p0[k]);
        if (CONDEN(ps0[k], exns0[k], thl0top, qt0top, thj, qvj, qlj, qij, tbld, tblf)) {
            xflags |= UW_X_CONDEN;
            id_exit = true;
            stop = true;
            break;
        }
        thv0top[k] = thj * (1.0f + zvir * qvj - qlj - qij);
        thvl0top[k] = thl0top * (1.0f + zvir * qt0top);
        thv0bot_o[k] = thv0bot[k];
        thv0top_o[k] = thv0top[k];
        thvl0bot_o[k] = thvl0bot[k];
        thvl0top_o[k] = thvl0top[k];
    }
    if (!stop) {
    // per-column initialisation (:1333-1408)
    for (int k = 0; k <= mkx; k++) {
        umf[k] = 0.0f; emf[k] = 0.0f; slflx[k] = 0.0f; qtflx[k] = 0.0f; uflx[k] = 0.0f; vflx[k] = 0.0f;
        ufrc[k] = 0.0f; thlu[k] = 0.0f; qtu[k] = 0.0f; uu[k] = 0.0f; vu[k] = 0.0f; wu[k] = 0.0f;
        thvu[k] = 0.0f; thlu_emf[k] = 0.0f; qtu_emf[k] = 0.0f; uu_emf[k] = 0.0f; vu_emf[k] = 0.0f;
        for (int m = 0; m < ncnst; m++) {
            trflx[m][k] = 0.0f;
            tru[m][k] = 0.0f;
            tru_emf[m][k] = 0.0f;
        }
    }
    for (int k = 1; k <= mkx; k++) {
        qvten[k] = 0.0f; qlten[k] = 0.0f; qiten[k] = 0.0f; sten[k] = 0.0f; uten[k] = 0.0f; vten[k] = 0.0f;
        qrten[k] = 0.0f; qsten[k] = 0.0f; dwten[k] = 0.0f; diten[k] = 0.0f; evapc[k] = 0.0f;
        cufrc[k] = 0.0f; qcu[k] = 0.0f; qlu[k] = 0.0f; qiu[k] = 0.0f; fer[k] = 0.0f; fdr[k] = 0.0f;
        qc[k] = 0.0f; qc_l[k] = 0.0f; qc_i[k] = 0.0f; qtten[k] = 0.0f; slten[k] = 0.0f;
        qlten_sink[k] = 0.0f; qiten_sink[k] = 0.0f; nlten_sink[k] = 0.0f; niten_sink[k] = 0.0f;
        rei[k] = 0.0f; uf[k] = 0.0f; vf[k] = 0.0f;
        for (int m = 0; m < ncnst; m++) trten[m][k] = 0.0f;
    }
    cnt = (R)mkx;
    cnb = 0.0f;
    }
    } else {   // uniform
        // the state UW_MODE_LIST1 stored at the implicit-CIN branch of iteration 2 (uw_state.cuh),
        // and the arrays that the set-up and that branch's restore build from the inputs, rebuilt
        // with the same operations
        UW_LOAD_STATE(A.hand->state + i_in, (size_t)A.hand->cap, tscaleh_r);
        for (int k = 0; k <= mkx; k++) {
            ps0[k] = GI(ps0, k);
            zs0[k] = GI(zs0, k);
        }
        for (int k = 1; k <= mkx; k++) {
            p0[k] = GL(p0, k);
            dp0[k] = GL(dp0, k);
        }
        {
            R tmpf[KP];
            for (int k = 1; k <= mkx; k++) tmpf[k] = GL(u0, k);
            slope<KP>(mkx, tmpf, p0, ssu0);
            for (int k = 1; k <= mkx; k++) tmpf[k] = GL(v0, k);
            slope<KP>(mkx, tmpf, p0, ssv0);
            for (int m = 1; m <= ncnst; m++) {
                for (int k = 1; k <= mkx; k++) tmpf[k] = GT(m, k);
                slope<KP>(mkx, tmpf, p0, sstr0[m - 1]);
            }
        }
        for (int k = 1; k <= mkx; k++) {
            qv0[k] = GL(qv0, k);
            ql0[k] = GL(ql0, k);
            qi0[k] = GL(qi0, k);
            t0[k] = GL(t0, k);
            s0[k] = GL(s0, k);
            qt0[k] = (qv0[k] + ql0[k] + qi0[k]);
            thl0[k] = (t0[k] - xlv * ql0[k] / cp - xls * qi0[k] / cp) / exn0[k];
            thv0bot[k] = thv0bot_o[k];
            thv0top[k] = thv0top_o[k];
            thvl0bot[k] = thvl0bot_o[k];
            thvl0top[k] = thvl0top_o[k];
        }
        slope<KP>(mkx, thl0, p0, ssthl0);
        slope<KP>(mkx, qt0, p0, ssqt0);
        for (int k = 0; k <= mkx; k++) {
            umf[k] = 0.0f; emf[k] = 0.0f; slflx[k] = 0.0f; qtflx[k] = 0.0f; uflx[k] = 0.0f;
            vflx[k] = 0.0f; ufrc[k] = 0.0f; thlu[k] = 0.0f; qtu[k] = 0.0f; uu[k] = 0.0f;
            vu[k] = 0.0f; wu[k] = 0.0f; thvu[k] = 0.0f; thlu_emf[k] = 0.0f; qtu_emf[k] = 0.0f;
            uu_emf[k] = 0.0f; vu_emf[k] = 0.0f;
            for (int m = 0; m < ncnst; m++) {
                trflx[m][k] = 0.0f;
                tru[m][k] = 0.0f;
                tru_emf[m][k] = 0.0f;
            }
        }
        for (int k = 1; k <= mkx; k++) {
            qvten[k] = 0.0f; qlten[k] = 0.0f; qiten[k] = 0.0f; sten[k] = 0.0f; uten[k] = 0.0f;
            vten[k] = 0.0f; qrten[k] = 0.0f; qsten[k] = 0.0f; dwten[k] = 0.0f; diten[k] = 0.0f;
            evapc[k] = 0.0f; cufrc[k] = 0.0f; qcu[k] = 0.0f; qlu[k] = 0.0f; qiu[k] = 0.0f;
            fer[k] = 0.0f; fdr[k] = 0.0f; qc[k] = 0.0f; qc_l[k] = 0.0f; qc_i[k] = 0.0f;
            qtten[k] = 0.0f; slten[k] = 0.0f;
            for (int m = 0; m < ncnst; m++) trten[m][k] = 0.0f;
        }
    }

    UW_SYNC();

    // ---- implicit-CIN loop (uwshcu.F90:1421-4331) --------------------------------------------
    // Lockstep skeleton.  Every lane of the warp runs the same iterations of this loop and of every
    // level loop inside it: a column's own level range and its exits are per-lane predicates.  Each
    // section is `if (!stop) do { ... } while (0);`, so an exit (`stop = true; break;`) skips the
    // rest of the section and every later one, and the lanes meet again at UW_SYNC() between
    // sections.  (Lanes that leave a loop at different iterations otherwise run apart for the rest
    // of the column: the worklist kernel ran with 1.9f of 32 lanes active.)  Loops marked `uniform`
    // have the same trip count on every live lane; UW_SYNC() appears only directly inside them.
    for (int iter = (MODE == UW_MODE_RESUME ? 2 : 1); iter <= (MODE == UW_MODE_TRIGGER ? 1 : 2); iter++) {   // uniform
        R tscaleh = tscaleh_r;
        if constexpr (MODE != UW_MODE_RESUME) {   // uniform
        if (!stop) do {
        tscaleh = cush;
        cush = -1.0f;

        // kinv (:1455-1468): the first interface from the top whose layer brackets pblh + 5
        kinv = 1;
        {
            bool found = false;
            for (int k = mkx - 1; k >= 1; k--) {
                if (!found && (pblh + 5.0f - zs0[k]) * (pblh + 5.0f - zs0[k + 1]) < 0.0f) {
                    kinv = k + 1;
                    found = true;
                }
            }
        }
        if (kinv <= 1) {
            xflags |= UW_X_KINV1;
            id_exit = true;
            stop = true;
            break;
        }
        // tkeavg, thvlmin (:1484-1499)
        {
            Kahan dpsum, tksum;
            thvlmin = 1000.0f;
            for (int k = 0; k <= mkx; k++) {
                if (k > kinv - 1) continue;
                R dpi;
                if (k == 0) dpi = ps0[0] - p0[1];
                else if (k == (kinv - 1)) dpi = p0[kinv - 1] - ps0[kinv - 1];
                else dpi = p0[k] - p0[k + 1];
                dpsum.add(dpi);
                tksum.add(dpi * GI(tke, k));
                if (k != 0) thvlmin = MN(thvlmin, MN(thvl0bot[k], thvl0top[k]));
            }
            tkeavg = tksum.s / dpsum.s;
        }
        // source air (:1509-1516)
        qtsrc = qt0[1];
        thvlsrc = thvlmin;
        thlsrc = thvlsrc / (1.0f + zvir * qtsrc);
        usrc = GL(u0, kinv - 1) + ssu0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        vsrc = GL(v0, kinv - 1) + ssv0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        for (int m = 1; m <= ncnst; m++) trsrc[m - 1] = GT(m, 1);
        } while (0);
        UW_SYNC();
        // LCL (:1533-1549)
        if (!stop) do {
        plcl = qsinvert(qtsrc, thlsrc, ps0[0], exns0[0], tbld, tblf);
        klcl = mkx;
        {
            bool found = false;
            for (int k = 0; k <= mkx; k++) {
                if (!found && ps0[k] < plcl) {
                    klcl = k;
                    found = true;
                }
            }
        }
        klcl = MX(1, klcl);
        if (plcl < 30000.0f) {
            xflags |= UW_X_KLCLMKX;
            id_exit = true;
            stop = true;
            break;
        }
        exlcl = exnf(plcl);
        {
            R thl0lcl = thl0[klcl] + ssthl0[klcl] * (plcl - p0[klcl]);
            R qt0lcl = qt0[klcl] + ssqt0[klcl] * (plcl - p0[klcl]);
            if (CONDEN(plcl, exlcl, thl0lcl, qt0lcl, thj, qvj, qlj, qij, tbld, tblf)) {
                xflags |= UW_X_CONDEN;
                id_exit = true;
                stop = true;
            break;
            }
            thv0lcl = thj * (1.0f + zvir * qvj - qlj - qij);
        }
        } while (0);
        UW_SYNC();
        // CIN (:1592-1685).  One loop over k = kinv .. mkx-1 serves both cases of the Fortran (LCL at
        // or above kinv, LCL below kinv), with one conden call at ps0(k) per level for every lane.
        // When the LCL is below kinv the Fortran also calls conden at ps0(k-1) with the same source
        // air; above the first level that repeats the previous level's call bit for bit, so only
        // the first level makes it here.
        if (!stop) {
            cin = 0.0f;
            cinlcl = 0.0f;
            plfc = 0.0f;
            klfc = mkx;
        }
        {
            const bool lcl_above = (klcl >= kinv);
            R thvubot = 0.0f, thvutop = 0.0f;
            bool ldone = stop;
            for (int k = 2; k <= mkx - 1; k++) {   // uniform (kinv >= 2)
                if (!ldone && k >= kinv) do {
                    if (lcl_above && k < klcl) {
                        thvubot = thvlsrc;
                        thvutop = thvlsrc;
                        cin = cin + single_cin(ps0[k - 1], exns0[k - 1], thv0bot[k], ps0[k], exns0[k], thv0top[k], thvubot, thvutop);
                        break;
                    }
                    if (!lcl_above && k == kinv) {
                        if (CONDEN(ps0[k - 1], exns0[k - 1], thlsrc, qtsrc, thj, qvj, qlj, qij, tbld, tblf)) {
                            xflags |= UW_X_CONDEN;
                            id_exit = true;
                            stop = true;
                            break;
                        }
                        thvutop = thj * (1.0f + zvir * qvj - qlj - qij);
                    }
                    const bool atlcl = lcl_above && k == klcl;
                    if (atlcl) {
                        thvubot = thvlsrc;
                        thvutop = thvlsrc;
                        cin = cin + single_cin(ps0[k - 1], exns0[k - 1], thv0bot[k], plcl, exlcl, thv0lcl, thvubot, thvutop);
                        if (cin < 0.0f) lflags |= UW_L_CINLCL;
                        cinlcl = MX(cin, 0.0f);
                        cin = cinlcl;
                        thvubot = thvlsrc;
                    } else {
                        thvubot = thvutop;
                    }
                    if (CONDEN(ps0[k], exns0[k], thlsrc, qtsrc, thj, qvj, qlj, qij, tbld, tblf)) {
                        xflags |= UW_X_CONDEN;
                        id_exit = true;
                        stop = true;
                        break;
                    }
                    thvutop = thj * (1.0f + zvir * qvj - qlj - qij);
                    getbuoy(atlcl ? plcl : ps0[k - 1], atlcl ? exlcl : exns0[k - 1], atlcl ? thv0lcl : thv0bot[k],
                            ps0[k], exns0[k], thv0top[k], thvubot, thvutop, plfc, cin);
                    if (plfc > 0.0f) {
                        klfc = k;
                        ldone = true;
                    }
                } while (0);
                if (stop) ldone = true;
            }
        }
        UW_SYNC();
        if (!stop) do {
        // (label 35, :1676-1685)
        if (cin < 0.0f) lflags |= UW_L_CIN;
        cin = MX(0.0f, cin);
        if (klfc >= mkx) {
            klfc = mkx;
            xflags |= UW_X_KLFCMKX;
            id_exit = true;
            stop = true;
            break;
        }
        if (iter == 1) {
            cin_i = cin;
            cinlcl_i = cinlcl;
            ke = rbuoy / (rkfre * tkeavg + epsvarw);
            kinv_o = kinv; klcl_o = klcl; klfc_o = klfc; plcl_o = plcl; plfc_o = plfc;
            tkeavg_o = tkeavg; thvlmin_o = thvlmin; qtsrc_o = qtsrc; thvlsrc_o = thvlsrc;
            thlsrc_o = thlsrc; usrc_o = usrc; vsrc_o = vsrc; thv0lcl_o = thv0lcl;
            for (int m = 0; m < ncnst; m++) trsrc_o[m] = trsrc[m];
        } else {
            double del_CIN = cin - cin_i;
            if (del_CIN > 0.0f) {
                // implicit CIN: restore the iteration-1 state (:1759-1889)
                double alpha = compute_alpha(del_CIN, ke);
                cin = cin_i + alpha * del_CIN;
                cinlcl = cinlcl_i;
                kinv = kinv_o; klcl = klcl_o; klfc = klfc_o; plcl = plcl_o; plfc = plfc_o;
                tkeavg = tkeavg_o; thvlmin = thvlmin_o; qtsrc = qtsrc_o; thvlsrc = thvlsrc_o;
                thlsrc = thlsrc_o; usrc = usrc_o; vsrc = vsrc_o; thv0lcl = thv0lcl_o;
                for (int m = 0; m < ncnst; m++) trsrc[m] = trsrc_o[m];
                exlcl = exnf(plcl);
                for (int k = 1; k <= mkx; k++) {
                    qv0[k] = GL(qv0, k);
                    ql0[k] = GL(ql0, k);
                    qi0[k] = GL(qi0, k);
                    t0[k] = GL(t0, k);
                    s0[k] = GL(s0, k);
                    qt0[k] = (qv0[k] + ql0[k] + qi0[k]);
                    thl0[k] = (t0[k] - xlv * ql0[k] / cp - xls * qi0[k] / cp) / exn0[k];
                    thv0bot[k] = thv0bot_o[k];
                    thv0top[k] = thv0top_o[k];
                    thvl0bot[k] = thvl0bot_o[k];
                    thvl0top[k] = thvl0top_o[k];
                }
                slope<KP>(mkx, thl0, p0, ssthl0);
                slope<KP>(mkx, qt0, p0, ssqt0);
                for (int k = 0; k <= mkx; k++) {
                    umf[k] = 0.0f; emf[k] = 0.0f; slflx[k] = 0.0f; qtflx[k] = 0.0f; uflx[k] = 0.0f;
                    vflx[k] = 0.0f; ufrc[k] = 0.0f; thlu[k] = 0.0f; qtu[k] = 0.0f; uu[k] = 0.0f;
                    vu[k] = 0.0f; wu[k] = 0.0f; thvu[k] = 0.0f; thlu_emf[k] = 0.0f; qtu_emf[k] = 0.0f;
                    uu_emf[k] = 0.0f; vu_emf[k] = 0.0f;
                    for (int m = 0; m < ncnst; m++) {
                        trflx[m][k] = 0.0f;
                        tru[m][k] = 0.0f;
                        tru_emf[m][k] = 0.0f;
                    }
                }
                for (int k = 1; k <= mkx; k++) {
                    qvten[k] = 0.0f; qlten[k] = 0.0f; qiten[k] = 0.0f; sten[k] = 0.0f; uten[k] = 0.0f;
                    vten[k] = 0.0f; qrten[k] = 0.0f; qsten[k] = 0.0f; dwten[k] = 0.0f; diten[k] = 0.0f;
                    evapc[k] = 0.0f; cufrc[k] = 0.0f; qcu[k] = 0.0f; qlu[k] = 0.0f; qiu[k] = 0.0f;
                    fer[k] = 0.0f; fdr[k] = 0.0f; qc[k] = 0.0f; qc_l[k] = 0.0f; qc_i[k] = 0.0f;
                    qtten[k] = 0.0f; slten[k] = 0.0f;
                    for (int m = 0; m < ncnst; m++) trten[m][k] = 0.0f;
                }
                precip = 0.0f; snow = 0.0f; rliq.reset(); cbmf = 0.0f;
                cnt = (R)mkx; cnb = 0.0f; ufrclcl = 0.0f; wlcl = 0.0f;
            } else {
                // explicit CIN: the iteration-1 outputs already sit in the output slots (:1891-2011);
                // flxprc1/flxsnow1 keep their initial zeros on this path, wu_out gets wu.
                lflags |= UW_L_DELCIN;
                for (int k = 0; k <= mkx; k++) OI(wu, k) = wu[k];
                if (A.diag_real) {
                    A.diag_real[UW_DR_CIN * (size_t)mix + i] = cin_s;
                    A.diag_real[UW_DR_CINLCL * (size_t)mix + i] = cinlcl_s;
                    A.diag_real[UW_DR_PLCL * (size_t)mix + i] = plcl_s;
                    A.diag_real[UW_DR_PLFC * (size_t)mix + i] = plfc_s;
                    A.diag_real[UW_DR_PINV * (size_t)mix + i] = pinv_s;
                    A.diag_real[UW_DR_PBUP * (size_t)mix + i] = pbup_s;
                    A.diag_real[UW_DR_PPEN * (size_t)mix + i] = ppen_s;
                    A.diag_real[UW_DR_TKEAVG * (size_t)mix + i] = tkeavg_s;
                }
                kinv = kinv_s; klcl = klcl_s; klfc = klfc_s; krel = krel_s; kbup = kbup_s; kpen = kpen_s;
                id_exit = false;
                stop = true;
            break;
            }
        }

        } while (0);
        UW_SYNC();
        }   // MODE != UW_MODE_RESUME
        if constexpr (MODE == UW_MODE_LIST1) {   // uniform
        if (iter == 2) {   // uniform
            // implicit CIN: the rest of the column runs in the UW_MODE_RESUME launch; without a free
            // slot it goes on here
            const unsigned want = __ballot_sync(live, !stop);
            if (want) {
                const UwHand& H = *A.hand;
                const unsigned ln = threadIdx.x & 31u;
                const int leader = __ffs(want) - 1;
                int base = 0;
                if ((int)ln == leader) base = atomicAdd(H.count, __popc(want));
                base = __shfl_sync(live, base, leader);
                const int slot = base + __popc(want & ((1u << ln) - 1u));
                if (!stop && slot < H.cap) {
                    H.col[slot] = i;
                    H.key[slot] = UW_HAND_KEYS - 1 - MN(MX(kpen_s - krel_s, 0), UW_HAND_KEYS - 1);
                    UW_SAVE_STATE(H.state + slot, (size_t)H.cap, tscaleh);
                    handed = true;
                    stop = true;
                }
            }
        }
        }
        // ---- release level and closure (:2035-2184) ------------------------------------------
        if (!stop) do {
        if (klcl < kinv) {
            krel = kinv;
            prel = ps0[krel - 1];
            exprel = exns0[krel - 1];
            thv0rel = thv0bot[krel];
        } else {
            krel = klcl;
            prel = plcl;
            exprel = exlcl;
            thv0rel = thv0lcl;
        }
        {
            R wcrit = sqrtf(2.0f * cin * rbuoy);
            // compute_zwshcu computes rho0inv first and lowers wcrit by the large-scale ascent at
            // the PBL top (zwshcu.F90:2277, 2295-2303); the same value of rho0inv for both schemes
            R rho0inv = ps0[kinv - 1] / (r * thv0top[kinv - 1] * exns0[kinv - 1]);
            R sigmaw = sqrtf(rkfre * tkeavg + epsvarw);
            if constexpr (ZW) {
                if (c.zw_lf) {
                    const R tmp1 = MN(MX(-GL(omega, kinv - 1), 0.0f), 3.0f);
                    wcrit = wcrit - tmp1 / rho0inv / 9.8f;
                    wcrit = MX(wcrit, 0.0f);
                }
                wcrit = wcrit * c.zw_fwcrit;
            }
            R mu = wcrit / sigmaw / 1.4142f;
            if (mu >= 3.0f) {
                id_exit = true;
                stop = true;
            break;
            }
            cbmf = (rho0inv * sigmaw / 2.5066f) * expf(-(mu * mu));
            R cbmflimit = 0.9f * dp0[kinv - 1] / g / dt;
            R mumin0 = 0.0f;
            if (cbmf > cbmflimit) mumin0 = sqrtf(-logf(2.5066f * cbmflimit / rho0inv / sigmaw));
            mu = MX(MX(mu, mumin0), mumin1);
            R mulcl = sqrtf(2.0f * cinlcl * rbuoy) / 1.4142f / sigmaw;
            R ta = expf(-(mu * mu)) / 2.5066f, te = erfcf(mu);
            R mulclstar = sqrtf(MX(0.0f, 2.0f * (ta * ta) * (1.0f / (te * te) - 0.25f / (rmaxfrac * rmaxfrac))));
            if (mulcl > 1.e-8f && mulcl > mulclstar) {
                R mumin2 = compute_mumin2(mulcl, rmaxfrac, mu);
                if (mu > mumin2) errbits |= UW_ERRBIT_MU;
                mu = MX(mu, mumin2);
                if (mu == mumin2) lflags |= UW_L_UFRC;
            }
            if (mu == mumin0) lflags |= UW_L_CBMF;
            if (mu == mumin1) lflags |= UW_L_UFRC;
            cbmf = (rho0inv * sigmaw / 2.5066f) * expf(-(mu * mu));
            R winv = sigmaw * (2.0f / 2.5066f) * expf(-(mu * mu)) / erfcf(mu);
            wtw = winv * winv - 2.0f * cinlcl * rbuoy;
            if (wtw <= 0.0f) {
                xflags |= UW_X_WTW;
                id_exit = true;
                stop = true;
            break;
            }
            wlcl = sqrtf(wtw);
            ufrclcl = cbmf / wlcl / rho0inv;
            if (ufrclcl <= 0.0001f) {
                xflags |= UW_X_UFRC;
                id_exit = true;
                stop = true;
            break;
            }
            ufrc[krel - 1] = ufrclcl;
            for (int k = 0; k <= mkx; k++) {
                if (k < kinv - 1 || k > krel - 1) continue;
                umf[k] = cbmf;
                wu[k] = winv;
            }
        }
        } while (0);
        if (MODE == UW_MODE_TRIGGER) {
            // the column convects past the closure: hand it to the worklist pass
            if (!stop) {
                cand = true;
                stop = true;
            }
        }
        UW_SYNC();
        if (MODE != UW_MODE_TRIGGER) {   // uniform
        // updraft at the release level (:2205-2236)
        if (!stop) do {
        emf[krel - 1] = 0.0f;
        umf[krel - 1] = cbmf;
        wu[krel - 1] = wlcl;
        thlu[krel - 1] = thlsrc;
        qtu[krel - 1] = qtsrc;
        if (CONDEN(prel, exprel, thlsrc, qtsrc, thj, qvj, qlj, qij, tbld, tblf)) {
            xflags |= UW_X_CONDEN;
            id_exit = true;
            stop = true;
            break;
        }
        thvu[krel - 1] = thj * (1.0f + zvir * qvj - qlj - qij);
        {
            R uplus = 0.0f, vplus = 0.0f;
            if (krel == kinv) {
                uplus = PGFc * ssu0[kinv] * (prel - ps0[kinv - 1]);
                vplus = PGFc * ssv0[kinv] * (prel - ps0[kinv - 1]);
            } else {
                for (int k = 0; k <= mkx; k++) {
                    if (k < kinv || k > MX(krel - 1, kinv)) continue;
                    uplus = uplus + PGFc * ssu0[k] * (ps0[k] - ps0[k - 1]);
                    vplus = vplus + PGFc * ssv0[k] * (ps0[k] - ps0[k - 1]);
                }
                uplus = uplus + PGFc * ssu0[krel] * (prel - ps0[krel - 1]);
                vplus = vplus + PGFc * ssv0[krel] * (prel - ps0[krel - 1]);
            }
            uu[krel - 1] = usrc + uplus;
            vu[krel - 1] = vsrc + vplus;
        }
        for (int m = 0; m < ncnst; m++) tru[m][krel - 1] = trsrc[m];
        } while (0);
        UW_SYNC();

        {
            R scaleh = tscaleh;
            if (tscaleh < 0.0f) scaleh = 1000.0f;
            // ---- buoyancy-sorting updraft, iter_scaleh loop (:2306-2952) ----------------------
            for (int iter_scaleh = 1; iter_scaleh <= 3; iter_scaleh++) {   // uniform
                R pe = 0.0f, dpe = 0.0f, exne = 1.0f, thvebot = 0.0f, thle = 0.0f, qte = 0.0f, ue = 0.0f, ve = 0.0f;
                if (!stop) {
                    kbup = krel;
                    kpen = krel;
                    wtw = wlcl * wlcl;
                    pe = 0.5f * (prel + ps0[krel]);
                    dpe = prel - ps0[krel];
                    exne = exnf(pe);
                    thvebot = thv0rel;
                    thle = thl0[krel] + ssthl0[krel] * (pe - p0[krel]);
                    qte = qt0[krel] + ssqt0[krel] * (pe - p0[krel]);
                    ue = GL(u0, krel) + ssu0[krel] * (pe - p0[krel]);
                    ve = GL(v0, krel) + ssv0[krel] * (pe - p0[krel]);
                    for (int m = 0; m < ncnst; m++) tre[m] = GT(m + 1, krel) + sstr0[m][krel] * (pe - p0[krel]);
                }

                // levels k = krel .. mkx-1, taken by every lane as k = krel + j
                bool ldone = stop;
                for (int j = 0; j <= mkx - 2; j++) {   // uniform
                    const int k = krel + j;
                    if (k > mkx - 1) ldone = true;
                    if (!ldone) do {
                    const int km1 = k - 1;
                    R thlue = thlu[km1];
                    R qtue = qtu[km1];
                    R wue = wu[km1];
                    wtwb = wtw;
                    bool xdone = false;
                    // environment at the layer midpoint: the same in both iter_xc passes, so the
                    // second pass reuses the first one's conden and qsat results (same bits)
                    R thv0j = 0.0f, excess0 = 0.0f;
                    for (int iter_xc = 1; iter_xc <= 2; iter_xc++) {
                        if (!xdone && !stop) do {
                        wtw = wu[km1] * wu[km1];
                        if (iter_xc == 1) {
                            if (CONDEN(pe, exne, thle, qte, thj, qvj, qlj, qij, tbld, tblf)) {
                                xflags |= UW_X_CONDEN;
                                id_exit = true;
                                stop = true;
                                break;
                            }
                            thv0j = thj * (1.0f + zvir * qvj - qlj - qij);
                            excess0 = qte - qsat_qs(thle * exne, pe, tbld, tblf);
                        }
                        rho0j = pe / (r * thv0j * exne);
                        if (CONDEN(pe, exne, thlue, qtue, thj, qvj, qlj, qij, tbld, tblf)) {
                            xflags |= UW_X_CONDEN;
                            id_exit = true;
                            stop = true;
            break;
                        }
                        // condensate above criqc leaves the updraft; without it the Fortran's
                        // second conden call repeats the first one's arguments and results
                        if ((qlj + qij) > criqc) {
                            R exql = ((qlj + qij) - criqc) * qlj / (qlj + qij);
                            R exqi = ((qlj + qij) - criqc) * qij / (qlj + qij);
                            qtue = qtue - exql - exqi;
                            thlue = thlue + (xlv / cp / exne) * exql + (xls / cp / exne) * exqi;
                            if (CONDEN(pe, exne, thlue, qtue, thj, qvj, qlj, qij, tbld, tblf)) {
                                xflags |= UW_X_CONDEN;
                                id_exit = true;
                                stop = true;
                                break;
                            }
                        }
                        R thvj = thj * (1.0f + zvir * qvj - qlj - qij);
                        R excessu = qtue - qsat_qs(thlue * exne, pe, tbld, tblf);
                        R cridis = rle * scaleh;
                        R xc;
                        if ((excessu <= 0.0f && excess0 <= 0.0f) || (excessu >= 0.0f && excess0 >= 0.0f)) {
                            xc = MN(1.0f, MX(0.0f, 1.0f - 2.0f * rbuoy * g * cridis / (wue * wue) * (1.0f - thvj / thv0j)));
                        } else {
                            R xsat = excessu / (excessu - excess0);
                            R thlxsat = thlue + xsat * (thle - thlue);
                            R qtxsat = qtue + xsat * (qte - qtue);
                            if (CONDEN(pe, exne, thlxsat, qtxsat, thj, qvj, qlj, qij, tbld, tblf)) {
                                xflags |= UW_X_CONDEN;
                                id_exit = true;
                                stop = true;
            break;
                            }
                            R thvxsat = thj * (1.0f + zvir * qvj - qlj - qij);
                            R x_cu = 0.0f, x_en = 0.0f;
                            for (int kk = 1; kk <= 2; kk++) {
                                R thv_x0, thv_x1;
                                if (kk == 1) {
                                    thv_x0 = thvj;
                                    thv_x1 = (1.0f - 1.0f / xsat) * thvj + (1.0f / xsat) * thvxsat;
                                } else {
                                    thv_x1 = thv0j;
                                    thv_x0 = (xsat / (xsat - 1.0f)) * thv0j + (1.0f / (1.0f - xsat)) * thvxsat;
                                }
                                R aquad = wue * wue;
                                R bquad = 2.0f * rbuoy * g * cridis * (thv_x1 - thv_x0) / thv0j - 2.0f * (wue * wue);
                                R cquad = 2.0f * rbuoy * g * cridis * (thv_x0 - thv0j) / thv0j + (wue * wue);
                                if (kk == 1) {
                                    if ((bquad * bquad - 4.0f * aquad * cquad) >= 0.0f) {
                                        roots(aquad, bquad, cquad, xs1, xs2);
                                        x_cu = MN(1.0f, MX(0.0f, MN(xsat, MN(xs1, xs2))));
                                    } else {
                                        x_cu = xsat;
                                    }
                                } else {
                                    if ((bquad * bquad - 4.0f * aquad * cquad) >= 0.0f) {
                                        roots(aquad, bquad, cquad, xs1, xs2);
                                        x_en = MN(1.0f, MX(0.0f, MX(xsat, MN(xs1, xs2))));
                                    } else {
                                        x_en = 1.0f;
                                    }
                                }
                            }
                            if (x_cu == xsat) xc = MX(x_cu, x_en);
                            else xc = x_cu;
                        }
                        R ee2 = xc * xc;
                        R ud2 = 1.0f - 2.0f * xc + xc * xc;
                        rei[k] = (0.5f * rkm / GL(z0, k) / g / rho0j);
                        if (xc > 0.5f) rei[k] = MN(rei[k], 0.9f * logf(dp0[k] / g / dt / umf[km1] + 1.0f) / dpe / (2.0f * xc - 1.0f));
                        fer[k] = rei[k] * ee2;
                        fdr[k] = rei[k] * ud2;
                        // compute_zwshcu's entrainment option (zwshcu.F90:2818-2844)
                        if (ZW && c.zw_ent) {
                            bogbot = rbuoy * (thvu[km1] / thvebot - 1.0f) * g;
                            fer[k] = c.zw_ent0 * bogbot / MX(wue * wue, 1.0e-4f);
                            R fer_min = 0.0f;
                            if (bogbot > 1.e-4f) fer_min = 1.e-4f;
                            fer[k] = MN(MX(fer[k], fer_min), 3.0e-2f);
                        }
                        umf[k] = umf[km1] * expf(dpe * (fer[k] - fdr[k]));
                        emf[k] = 0.0f;
                        if (fer[k] * dpe < 1.e-4f) {
                            thlu[k] = thlu[km1] + (thle + ssthl0[k] * dpe / 2.0f - thlu[km1]) * fer[k] * dpe;
                            qtu[k] = qtu[km1] + (qte + ssqt0[k] * dpe / 2.0f - qtu[km1]) * fer[k] * dpe;
                            uu[k] = uu[km1] + (ue + ssu0[k] * dpe / 2.0f - uu[km1]) * fer[k] * dpe - PGFc * ssu0[k] * dpe;
                            vu[k] = vu[km1] + (ve + ssv0[k] * dpe / 2.0f - vu[km1]) * fer[k] * dpe - PGFc * ssv0[k] * dpe;
                            for (int m = 0; m < ncnst; m++)
                                tru[m][k] = tru[m][km1] + (tre[m] + sstr0[m][k] * dpe / 2.0f - tru[m][km1]) * fer[k] * dpe;
                        } else {
                            const R ef = expf(-fer[k] * dpe);
                            thlu[k] = (thle + ssthl0[k] / fer[k] - ssthl0[k] * dpe / 2.0f) -
                                      (thle + ssthl0[k] * dpe / 2.0f - thlu[km1] + ssthl0[k] / fer[k]) * ef;
                            qtu[k] = (qte + ssqt0[k] / fer[k] - ssqt0[k] * dpe / 2.0f) -
                                     (qte + ssqt0[k] * dpe / 2.0f - qtu[km1] + ssqt0[k] / fer[k]) * ef;
                            uu[k] = (ue + (1.0f - PGFc) * ssu0[k] / fer[k] - ssu0[k] * dpe / 2.0f) -
                                    (ue + ssu0[k] * dpe / 2.0f - uu[km1] + (1.0f - PGFc) * ssu0[k] / fer[k]) * ef;
                            vu[k] = (ve + (1.0f - PGFc) * ssv0[k] / fer[k] - ssv0[k] * dpe / 2.0f) -
                                    (ve + ssv0[k] * dpe / 2.0f - vu[km1] + (1.0f - PGFc) * ssv0[k] / fer[k]) * ef;
                            for (int m = 0; m < ncnst; m++)
                                tru[m][k] = (tre[m] + sstr0[m][k] / fer[k] - sstr0[m][k] * dpe / 2.0f) -
                                            (tre[m] + sstr0[m][k] * dpe / 2.0f - tru[m][km1] + sstr0[m][k] / fer[k]) * ef;
                        }
                        if (CONDEN(ps0[k], exns0[k], thlu[k], qtu[k], thj, qvj, qlj, qij, tbld, tblf)) {
                            xflags |= UW_X_CONDEN;
                            id_exit = true;
                            stop = true;
            break;
                        }
                        if ((qlj + qij) > criqc) {
                            R exql = ((qlj + qij) - criqc) * qlj / (qlj + qij);
                            R exqi = ((qlj + qij) - criqc) * qij / (qlj + qij);
                            qtu[k] = qtu[k] - exql - exqi;
                            thlu[k] = thlu[k] + (xlv / cp / exns0[k]) * exql + (xls / cp / exns0[k]) * exqi;
                            dwten[k] = exql;
                            diten[k] = exqi;
                            if (CONDEN(ps0[k], exns0[k], thlu[k], qtu[k], thj, qvj, qlj, qij, tbld, tblf)) {
                                xflags |= UW_X_CONDEN;
                                id_exit = true;
                                stop = true;
                                break;
                            }
                        } else {
                            // nothing removed: the Fortran's second conden call repeats the first
                            dwten[k] = 0.0f;
                            diten[k] = 0.0f;
                        }
                        thvu[k] = thj * (1.0f + zvir * qvj - qlj - qij);
                        bogbot = rbuoy * (thvu[km1] / thvebot - 1.0f);
                        bogtop = rbuoy * (thvu[k] / thv0top[k] - 1.0f);
                        R delbog = bogtop - bogbot;
                        drage = fer[k] * (1.0f + rdrag);
                        R expfac = expf(-2.0f * drage * dpe);
                        wtwb = wtw;
                        if (drage * dpe > 1.e-3f)
                            wtw = wtw * expfac + (delbog + (1.0f - expfac) * (bogbot + delbog / (-2.0f * drage * dpe))) / (rho0j * drage);
                        else
                            wtw = wtw + dpe * (bogbot + bogtop) / rho0j;
                        if (wtw > 0.0f) {
                            thlue = 0.5f * (thlu[km1] + thlu[k]);
                            qtue = 0.5f * (qtu[km1] + qtu[k]);
                            wue = 0.5f * sqrtf(MX(wtwb + wtw, 0.0f));
                        } else {
                            xdone = true;   // go to 111
                        }
                        } while (0);
                    }
                    if (stop) break;
                    // (label 111, :2726-2793)
                    if (umf[k] == 0.0f) wtw = -1.0f;
                    if (bogtop > 0.0f && wtw > 0.0f) kbup = k;
                    if (wtw <= 0.0f) {
                        kpen = k;
                        ldone = true;
                        break;   // go to 45
                    }
                    wu[k] = sqrtf(wtw);
                    if (wu[k] > 100.0f) {
                        xflags |= UW_X_WU;
                        id_exit = true;
                        stop = true;
            break;
                    }
                    {
                        R rhos0j = ps0[k] / (r * 0.5f * (thv0bot[k + 1] + thv0top[k]) * exns0[k]);
                        ufrc[k] = umf[k] / (rhos0j * wu[k]);
                        if (ufrc[k] > rmaxfrac) {
                            lflags |= UW_L_UFRC;
                            ufrc[k] = rmaxfrac;
                            umf[k] = rmaxfrac * rhos0j * wu[k];
                            fdr[k] = fer[k] - logf(umf[k] / umf[km1]) / dpe;
                        }
                    }
                    pe = p0[k + 1];
                    dpe = dp0[k + 1];
                    exne = exn0[k + 1];
                    thvebot = thv0bot[k + 1];
                    thle = thl0[k + 1];
                    qte = qt0[k + 1];
                    ue = GL(u0, k + 1);
                    ve = GL(v0, k + 1);
                    for (int m = 0; m < ncnst; m++) tre[m] = GT(m + 1, k + 1);
                    } while (0);
                    if (stop) ldone = true;
                    UW_SYNC();
                }
                UW_SYNC();
                // (label 45) penetration depth (:2884-2907)
                if (!stop) do {
                if (drage == 0.0f) {
                    R aquad = (bogtop - bogbot) / (ps0[kpen] - ps0[kpen - 1]);
                    R bquad = 2.0f * bogbot;
                    R cquad = -(wu[kpen - 1] * wu[kpen - 1]) * rho0j;
                    int status = roots(aquad, bquad, cquad, xc1, xc2);
                    if (status == 0) {
                        if (xc1 <= 0.0f && xc2 <= 0.0f) {
                            ppen = MX(xc1, xc2);
                            ppen = MN(0.0f, MX(-dp0[kpen], ppen));
                        } else if (xc1 > 0.0f && xc2 > 0.0f) {
                            ppen = -dp0[kpen];
                        } else {
                            ppen = MN(xc1, xc2);
                            ppen = MN(0.0f, MX(-dp0[kpen], ppen));
                        }
                    } else {
                        ppen = -dp0[kpen];
                    }
                } else {
                    ppen = compute_ppen(wtwb, drage, bogbot, bogtop, rho0j, dp0[kpen]);
                }
                if (ppen == -dp0[kpen] || ppen == 0.0f) lflags |= UW_L_PPEN;
                // condensate at the cumulus top (:2917-2942)
                if (fer[kpen] * (-ppen) < 1.e-4f) {
                    thlu_top = thlu[kpen - 1] + (thl0[kpen] + ssthl0[kpen] * (-ppen) / 2.0f - thlu[kpen - 1]) * fer[kpen] * (-ppen);
                    qtu_top = qtu[kpen - 1] + (qt0[kpen] + ssqt0[kpen] * (-ppen) / 2.0f - qtu[kpen - 1]) * fer[kpen] * (-ppen);
                } else {
                    const R ef = expf(-fer[kpen] * (-ppen));
                    thlu_top = (thl0[kpen] + ssthl0[kpen] / fer[kpen] - ssthl0[kpen] * (-ppen) / 2.0f) -
                               (thl0[kpen] + ssthl0[kpen] * (-ppen) / 2.0f - thlu[kpen - 1] + ssthl0[kpen] / fer[kpen]) * ef;
                    qtu_top = (qt0[kpen] + ssqt0[kpen] / fer[kpen] - ssqt0[kpen] * (-ppen) / 2.0f) -
                              (qt0[kpen] + ssqt0[kpen] * (-ppen) / 2.0f - qtu[kpen - 1] + ssqt0[kpen] / fer[kpen]) * ef;
                }
                exntop = powf((ps0[kpen - 1] + ppen) / p00, rovcp);
                if (CONDEN(ps0[kpen - 1] + ppen, exntop, thlu_top, qtu_top, thj, qvj, qlj, qij, tbld, tblf)) {
                    xflags |= UW_X_CONDEN;
                    id_exit = true;
                    stop = true;
            break;
                }
                if ((qlj + qij) > criqc) {
                    dwten[kpen] = ((qlj + qij) - criqc) * qlj / (qlj + qij);
                    diten[kpen] = ((qlj + qij) - criqc) * qij / (qlj + qij);
                    qtu_top = qtu_top - dwten[kpen] - diten[kpen];
                    thlu_top = thlu_top + (xlv / cp / exntop) * dwten[kpen] + (xls / cp / exntop) * diten[kpen];
                } else {
                    dwten[kpen] = 0.0f;
                    diten[kpen] = 0.0f;
                }
                {
                    R rhos0j = ps0[kpen - 1] / (r * 0.5f * (thv0bot[kpen] + thv0top[kpen - 1]) * exns0[kpen - 1]);
                    cush = zs0[kpen - 1] - ppen / rhos0j / g;
                }
                scaleh = cush;
                } while (0);
                UW_SYNC();
            }
        }
        // forcedCu filter (:2964-2992)
        if (!stop) do {
        if (kbup == krel) {
            lflags |= UW_L_SHCU;
            xflags |= UW_X_CUFILTER;
            id_exit = true;
            stop = true;
            break;
        }
        lflags &= ~UW_L_SHCU;
        for (int k = 0; k <= mkx; k++) {
            if (k < kpen) continue;
            umf[k] = 0.0f;
            emf[k] = 0.0f;
            ufrc[k] = 0.0f;
        }
        for (int k = 0; k <= mkx; k++) {
            if (k < kpen + 1) continue;
            dwten[k] = 0.0f;
            diten[k] = 0.0f;
            fer[k] = 0.0f;
            fdr[k] = 0.0f;
        }
        // penetrative entrainment (:3055-3183)
        for (int k = 0; k <= mkx; k++) {
            thlu_emf[k] = thlu[k];
            qtu_emf[k] = qtu[k];
            uu_emf[k] = uu[k];
            vu_emf[k] = vu[k];
            for (int m = 0; m < ncnst; m++) tru_emf[m][k] = tru[m][k];
        }
        for (int k = mkx; k >= 0; k--) {
            if (k > kpen - 1 || k < kbup) continue;
            R rhos0j = ps0[k] / (r * 0.5f * (thv0bot[k + 1] + thv0top[k]) * exns0[k]);
            if (k == kpen - 1) {
                if ((umf[k] * ppen * rei[kpen] * rpen) < -0.1f * rhos0j) lflags |= UW_L_EMF;
                if ((umf[k] * ppen * rei[kpen] * rpen) < -0.9f * dp0[kpen] / g / dt) lflags |= UW_L_EMF;
                emf[k] = MX(MX(umf[k] * ppen * rei[kpen] * rpen, -0.1f * rhos0j), -0.9f * dp0[kpen] / g / dt);
                thlu_emf[k] = thl0[kpen] + ssthl0[kpen] * (ps0[k] - p0[kpen]);
                qtu_emf[k] = qt0[kpen] + ssqt0[kpen] * (ps0[k] - p0[kpen]);
                uu_emf[k] = GL(u0, kpen) + ssu0[kpen] * (ps0[k] - p0[kpen]);
                vu_emf[k] = GL(v0, kpen) + ssv0[kpen] * (ps0[k] - p0[kpen]);
                for (int m = 0; m < ncnst; m++) tru_emf[m][k] = GT(m + 1, kpen) + sstr0[m][kpen] * (ps0[k] - p0[kpen]);
            } else {
                if ((emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen) < -0.1f * rhos0j) lflags |= UW_L_EMF;
                if ((emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen) < -0.9f * dp0[k + 1] / g / dt) lflags |= UW_L_EMF;
                emf[k] = MX(MX(emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen, -0.1f * rhos0j), -0.9f * dp0[k + 1] / g / dt);
                if (fabsf(emf[k]) > fabsf(emf[k + 1])) {
                    thlu_emf[k] = (thlu_emf[k + 1] * emf[k + 1] + thl0[k + 1] * (emf[k] - emf[k + 1])) / emf[k];
                    qtu_emf[k] = (qtu_emf[k + 1] * emf[k + 1] + qt0[k + 1] * (emf[k] - emf[k + 1])) / emf[k];
                    uu_emf[k] = (uu_emf[k + 1] * emf[k + 1] + GL(u0, k + 1) * (emf[k] - emf[k + 1])) / emf[k];
                    vu_emf[k] = (vu_emf[k + 1] * emf[k + 1] + GL(v0, k + 1) * (emf[k] - emf[k + 1])) / emf[k];
                    for (int m = 0; m < ncnst; m++)
                        tru_emf[m][k] = (tru_emf[m][k + 1] * emf[k + 1] + GT(m + 1, k + 1) * (emf[k] - emf[k + 1])) / emf[k];
                } else {
                    thlu_emf[k] = thl0[k + 1];
                    qtu_emf[k] = qt0[k + 1];
                    uu_emf[k] = GL(u0, k + 1);
                    vu_emf[k] = GL(v0, k + 1);
                    for (int m = 0; m < ncnst; m++) tru_emf[m][k] = GT(m + 1, k + 1);
                }
            }
        }
        // 1.f PBL fluxes (:3255-3290)
        {
            R xsrc = qtsrc, xmean = qt0[kinv];
            R xtop = qt0[kinv + 1] + ssqt0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
            R xbot = qt0[kinv - 1] + ssqt0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
            fluxbelowinv(cbmf, ps0, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
            for (int k = 0; k <= mkx; k++) if (k <= kinv - 1) qtflx[k] = xflx[k];
            xsrc = thlsrc;
            xmean = thl0[kinv];
            xtop = thl0[kinv + 1] + ssthl0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
            xbot = thl0[kinv - 1] + ssthl0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
            fluxbelowinv(cbmf, ps0, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
            for (int k = 0; k <= mkx; k++) if (k <= kinv - 1) slflx[k] = cp * exns0[k] * xflx[k];
            xsrc = usrc;
            xmean = GL(u0, kinv);
            xtop = GL(u0, kinv + 1) + ssu0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
            xbot = GL(u0, kinv - 1) + ssu0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
            fluxbelowinv(cbmf, ps0, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
            for (int k = 0; k <= mkx; k++) if (k <= kinv - 1) uflx[k] = xflx[k];
            xsrc = vsrc;
            xmean = GL(v0, kinv);
            xtop = GL(v0, kinv + 1) + ssv0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
            xbot = GL(v0, kinv - 1) + ssv0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
            fluxbelowinv(cbmf, ps0, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
            for (int k = 0; k <= mkx; k++) if (k <= kinv - 1) vflx[k] = xflx[k];
            for (int m = 0; m < ncnst; m++) {
                xsrc = trsrc[m];
                xmean = GT(m + 1, kinv);
                xtop = GT(m + 1, kinv + 1) + sstr0[m][kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
                xbot = GT(m + 1, kinv - 1) + sstr0[m][kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
                fluxbelowinv(cbmf, ps0, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
                for (int k = 0; k <= mkx; k++) if (k <= kinv - 1) trflx[m][k] = xflx[k];
            }
        }
        // 2.f non-buoyancy-sorting fluxes (:3300-3313)
        {
            R uplus = 0.0f, vplus = 0.0f;
            for (int k = 0; k <= mkx; k++) {
                if (k < kinv || k > krel - 1) continue;
                const int kp1 = k + 1;
                qtflx[k] = cbmf * (qtsrc - (qt0[kp1] + ssqt0[kp1] * (ps0[k] - p0[kp1])));
                slflx[k] = cbmf * (thlsrc - (thl0[kp1] + ssthl0[kp1] * (ps0[k] - p0[kp1]))) * cp * exns0[k];
                uplus = uplus + PGFc * ssu0[k] * (ps0[k] - ps0[k - 1]);
                vplus = vplus + PGFc * ssv0[k] * (ps0[k] - ps0[k - 1]);
                uflx[k] = cbmf * (usrc + uplus - (GL(u0, kp1) + ssu0[kp1] * (ps0[k] - p0[kp1])));
                vflx[k] = cbmf * (vsrc + vplus - (GL(v0, kp1) + ssv0[kp1] * (ps0[k] - p0[kp1])));
                for (int m = 0; m < ncnst; m++)
                    trflx[m][k] = cbmf * (trsrc[m] - (GT(m + 1, kp1) + sstr0[m][kp1] * (ps0[k] - p0[kp1])));
            }
        }
        // 3.f buoyancy-sorting fluxes (:3322-3331)
        for (int k = 0; k <= mkx; k++) {
            if (k < krel || k > kbup - 1) continue;
            const int kp1 = k + 1;
            slflx[k] = cp * exns0[k] * umf[k] * (thlu[k] - (thl0[kp1] + ssthl0[kp1] * (ps0[k] - p0[kp1])));
            qtflx[k] = umf[k] * (qtu[k] - (qt0[kp1] + ssqt0[kp1] * (ps0[k] - p0[kp1])));
            uflx[k] = umf[k] * (uu[k] - (GL(u0, kp1) + ssu0[kp1] * (ps0[k] - p0[kp1])));
            vflx[k] = umf[k] * (vu[k] - (GL(v0, kp1) + ssv0[kp1] * (ps0[k] - p0[kp1])));
            for (int m = 0; m < ncnst; m++)
                trflx[m][k] = umf[k] * (tru[m][k] - (GT(m + 1, kp1) + sstr0[m][kp1] * (ps0[k] - p0[kp1])));
        }
        // 4.f penetrative-entrainment fluxes (:3392-3401)
        for (int k = 0; k <= mkx; k++) {
            if (k < kbup || k > kpen - 1) continue;
            slflx[k] = cp * exns0[k] * emf[k] * (thlu_emf[k] - (thl0[k] + ssthl0[k] * (ps0[k] - p0[k])));
            qtflx[k] = emf[k] * (qtu_emf[k] - (qt0[k] + ssqt0[k] * (ps0[k] - p0[k])));
            uflx[k] = emf[k] * (uu_emf[k] - (GL(u0, k) + ssu0[k] * (ps0[k] - p0[k])));
            vflx[k] = emf[k] * (vu_emf[k] - (GL(v0, k) + ssv0[k] * (ps0[k] - p0[k])));
            for (int m = 0; m < ncnst; m++)
                trflx[m][k] = emf[k] * (tru_emf[m][k] - (GT(m + 1, k) + sstr0[m][k] * (ps0[k] - p0[k])));
        }
        } while (0);
        UW_SYNC();
        // condensate tendency by compensating subsidence (:3416-3476)
        {
            // uemf(k), evaluated on demand with the same expressions as :3416-3422
#define UEMF(kk)                                                                                          \
    ((kk) <= kinv - 2 ? cbmf * (ps0[0] - ps0[(kk)]) / (ps0[0] - ps0[kinv - 1])                             \
                      : ((kk) <= krel - 1 ? cbmf : ((kk) <= kbup - 1 ? umf[(kk)] : ((kk) <= kpen - 1 ? emf[(kk)] : 0.0f))))
            bool ldone = stop;
            for (int k = 1; k <= mkx; k++) {   // uniform
                if (k > kpen) ldone = true;
                if (!ldone) do {
                R comsub = 0.5f * (UEMF(k) + UEMF(k - 1));
                R thlten_sub, qtten_sub, qlten_sub, qiten_sub, nlten_sub, niten_sub;
                if (comsub >= 0.0f) {
                    if (k == mkx) {
                        thlten_sub = 0.0f; qtten_sub = 0.0f; qlten_sub = 0.0f; qiten_sub = 0.0f;
                        nlten_sub = 0.0f; niten_sub = 0.0f;
                    } else {
                        thlten_sub = g * comsub * (thl0[k + 1] - thl0[k]) / (p0[k] - p0[k + 1]);
                        qtten_sub = g * comsub * (qt0[k + 1] - qt0[k]) / (p0[k] - p0[k + 1]);
                        qlten_sub = g * comsub * (ql0[k + 1] - ql0[k]) / (p0[k] - p0[k + 1]);
                        qiten_sub = g * comsub * (qi0[k + 1] - qi0[k]) / (p0[k] - p0[k + 1]);
                        nlten_sub = g * comsub * (GT(ixnumliq, k + 1) - GT(ixnumliq, k)) / (p0[k] - p0[k + 1]);
                        niten_sub = g * comsub * (GT(ixnumice, k + 1) - GT(ixnumice, k)) / (p0[k] - p0[k + 1]);
                    }
                } else {
                    if (k == 1) {
                        thlten_sub = 0.0f; qtten_sub = 0.0f; qlten_sub = 0.0f; qiten_sub = 0.0f;
                        nlten_sub = 0.0f; niten_sub = 0.0f;
                    } else {
                        thlten_sub = g * comsub * (thl0[k] - thl0[k - 1]) / (p0[k - 1] - p0[k]);
                        qtten_sub = g * comsub * (qt0[k] - qt0[k - 1]) / (p0[k - 1] - p0[k]);
                        qlten_sub = g * comsub * (ql0[k] - ql0[k - 1]) / (p0[k - 1] - p0[k]);
                        qiten_sub = g * comsub * (qi0[k] - qi0[k - 1]) / (p0[k - 1] - p0[k]);
                        nlten_sub = g * comsub * (GT(ixnumliq, k) - GT(ixnumliq, k - 1)) / (p0[k - 1] - p0[k]);
                        niten_sub = g * comsub * (GT(ixnumice, k) - GT(ixnumice, k - 1)) / (p0[k - 1] - p0[k]);
                    }
                }
                R thl_prog = thl0[k] + thlten_sub * dt;
                R qt_prog = MX(qt0[k] + qtten_sub * dt, 1.e-12f);
                if (CONDEN(p0[k], exn0[k], thl_prog, qt_prog, thj, qvj, qlj, qij, tbld, tblf)) {
                    id_exit = true;
                    stop = true;
            break;
                }
                qlten_sink[k] = MX(qlten_sub, -ql0[k] / dt);
                qiten_sink[k] = MX(qiten_sub, -qi0[k] / dt);
                nlten_sink[k] = MX(nlten_sub, -GT(ixnumliq, k) / dt);
                niten_sink[k] = MX(niten_sub, -GT(ixnumice, k) / dt);
                } while (0);
                if (stop) ldone = true;
            }
        }
        UW_SYNC();
        if (!stop) do {
        // momentum tendency (:3488-3501)
        for (int k = 1; k <= mkx; k++) {
            if (k > kpen) continue;
            uten[k] = (uflx[k - 1] - uflx[k]) * g / dp0[k];
            vten[k] = (vflx[k - 1] - vflx[k]) * g / dp0[k];
            uf[k] = GL(u0, k) + uten[k] * dt;
            vf[k] = GL(v0, k) + vten[k] * dt;
        }
        // thermodynamic tendencies (:3511-3791)
        rliq.reset();
        rainflx.reset();
        snowflx.reset();
        } while (0);
        UW_SYNC();
        {
            R qlubelow = 0.0f, qiubelow = 0.0f;
            bool ldone = stop;
            for (int k = 1; k <= mkx; k++) {   // uniform
                if (k > kpen) ldone = true;
                if (!ldone) do {
                const int km1 = k - 1;
                dwten[k] = dwten[k] * 0.5f * (umf[k - 1] + umf[k]) * g / dp0[k];
                diten[k] = diten[k] * 0.5f * (umf[k - 1] + umf[k]) * g / dp0[k];
                qrten[k] = frc_rasn * dwten[k];
                qsten[k] = frc_rasn * diten[k];
                rainflx.add(qrten[k] * dp0[k] / g);
                snowflx.add(qsten[k] * dp0[k] / g);
                slten[k] = (slflx[km1] - slflx[k]) * g / dp0[k];
                if (k == 1) {
                    const R u1 = GL(u0, k), u2 = GL(u0, k + 1), v1 = GL(v0, k), v2 = GL(v0, k + 1);
                    slten[k] = slten[k] - g / 4.0f / dp0[k] *
                                              (uflx[k] * (uf[k + 1] - uf[k] + u2 - u1) +
                                               vflx[k] * (vf[k + 1] - vf[k] + v2 - v1));
                } else if (k >= 2 && k <= kpen - 1) {
                    const R um = GL(u0, k - 1), u1 = GL(u0, k), u2 = GL(u0, k + 1);
                    const R vm = GL(v0, k - 1), v1 = GL(v0, k), v2 = GL(v0, k + 1);
                    slten[k] = slten[k] - g / 4.0f / dp0[k] *
                                              (uflx[k] * (uf[k + 1] - uf[k] + u2 - u1) +
                                               uflx[k - 1] * (uf[k] - uf[k - 1] + u1 - um) +
                                               vflx[k] * (vf[k + 1] - vf[k] + v2 - v1) +
                                               vflx[k - 1] * (vf[k] - vf[k - 1] + v1 - vm));
                } else if (k == kpen) {
                    const R um = GL(u0, k - 1), u1 = GL(u0, k), vm = GL(v0, k - 1), v1 = GL(v0, k);
                    slten[k] = slten[k] - g / 4.0f / dp0[k] *
                                              (uflx[k - 1] * (uf[k] - uf[k - 1] + u1 - um) +
                                               vflx[k - 1] * (vf[k] - vf[k - 1] + v1 - vm));
                }
                qtten[k] = (qtflx[km1] - qtflx[k]) * g / dp0[k];

                R qlu_mid, qiu_mid;
                if (k < krel || k > kpen) {
                    qlu_mid = 0.0f;
                    qiu_mid = 0.0f;
                    qlj = 0.0f;
                    qij = 0.0f;
                } else {
                    // one conden call site for the release level, the cloud top and the levels between
                    const bool atrel = (k == krel), attop = (k != krel && k == kpen);
                    if (atrel) {
                        if (CONDEN(prel, exprel, thlu[krel - 1], qtu[krel - 1], thj, qvj, qlj, qij, tbld, tblf)) {
                            xflags |= UW_X_CONDEN;
                            id_exit = true;
                            stop = true;
                            break;
                        }
                        qlubelow = qlj;
                        qiubelow = qij;
                    }
                    if (CONDEN(attop ? ps0[k - 1] + ppen : ps0[k], attop ? exntop : exns0[k], attop ? thlu_top : thlu[k],
                               attop ? qtu_top : qtu[k], thj, qvj, qlj, qij, tbld, tblf)) {
                        xflags |= UW_X_CONDEN;
                        id_exit = true;
                        stop = true;
                        break;
                    }
                    if (atrel) {
                        qlu_mid = 0.5f * (qlubelow + qlj) * (prel - ps0[k]) / (ps0[k - 1] - ps0[k]);
                        qiu_mid = 0.5f * (qiubelow + qij) * (prel - ps0[k]) / (ps0[k - 1] - ps0[k]);
                    } else if (attop) {
                        qlu_mid = 0.5f * (qlubelow + qlj) * (-ppen) / (ps0[k - 1] - ps0[k]);
                        qiu_mid = 0.5f * (qiubelow + qij) * (-ppen) / (ps0[k - 1] - ps0[k]);
                    } else {
                        qlu_mid = 0.5f * (qlubelow + qlj);
                        qiu_mid = 0.5f * (qiubelow + qij);
                    }
                }
                qlubelow = qlj;
                qiubelow = qij;

                R qc_lm, qc_im, nc_lm, nc_im;
                qc_l[k] = (1.0f - frc_rasn) * dwten[k];
                qc_i[k] = (1.0f - frc_rasn) * diten[k];
                const R trl = GT(ixnumliq, k), tri = GT(ixnumice, k);
                if (k <= kbup) {
                    qc_l[k] = qc_l[k] + g * 0.5f * (umf[k - 1] + umf[k]) * fdr[k] * qlu_mid;
                    qc_i[k] = qc_i[k] + g * 0.5f * (umf[k - 1] + umf[k]) * fdr[k] * qiu_mid;
                    qc_lm = -g * 0.5f * (umf[k - 1] + umf[k]) * fdr[k] * ql0[k];
                    qc_im = -g * 0.5f * (umf[k - 1] + umf[k]) * fdr[k] * qi0[k];
                    nc_lm = -g * 0.5f * (umf[k - 1] + umf[k]) * fdr[k] * trl;
                    nc_im = -g * 0.5f * (umf[k - 1] + umf[k]) * fdr[k] * tri;
                } else {
                    qc_lm = 0.0f;
                    qc_im = 0.0f;
                    nc_lm = 0.0f;
                    nc_im = 0.0f;
                }
                if (k == kbup) {
                    qc_l[k] = qc_l[k] + g * umf[k] * qlj / (ps0[k - 1] - ps0[k]);
                    qc_i[k] = qc_i[k] + g * umf[k] * qij / (ps0[k - 1] - ps0[k]);
                    qc_lm = qc_lm - g * umf[k] * ql0[k] / (ps0[k - 1] - ps0[k]);
                    qc_im = qc_im - g * umf[k] * qi0[k] / (ps0[k - 1] - ps0[k]);
                    nc_lm = nc_lm - g * umf[k] * trl / (ps0[k - 1] - ps0[k]);
                    nc_im = nc_im - g * umf[k] * tri / (ps0[k - 1] - ps0[k]);
                    R ql_emf_kbup, qi_emf_kbup, thjj, qvjj;
                    if (CONDEN(p0[k], exn0[k], thlu_emf[k], qtu_emf[k], thjj, qvjj, ql_emf_kbup, qi_emf_kbup, tbld, tblf)) {
                        id_exit = true;
                        stop = true;
            break;
                    }
                    R nl_emf_kbup = (ql_emf_kbup > 0.0f) ? tru_emf[ixnumliq - 1][k] : 0.0f;
                    R ni_emf_kbup = (qi_emf_kbup > 0.0f) ? tru_emf[ixnumice - 1][k] : 0.0f;
                    qc_lm = qc_lm - g * emf[k] * (ql_emf_kbup - ql0[k]) / (ps0[k - 1] - ps0[k]);
                    qc_im = qc_im - g * emf[k] * (qi_emf_kbup - qi0[k]) / (ps0[k - 1] - ps0[k]);
                    nc_lm = nc_lm - g * emf[k] * (nl_emf_kbup - trl) / (ps0[k - 1] - ps0[k]);
                    nc_im = nc_im - g * emf[k] * (ni_emf_kbup - tri) / (ps0[k - 1] - ps0[k]);
                }
                qlten[k] = qc_l[k] + frc_rasn * dwten[k] + (MX(0.0f, ql0[k] + (qc_lm + qlten_sink[k]) * dt) - ql0[k]) / dt;
                qiten[k] = qc_i[k] + frc_rasn * diten[k] + (MX(0.0f, qi0[k] + (qc_im + qiten_sink[k]) * dt) - qi0[k]) / dt;
                trten[ixnumliq - 1][k] = MX(nc_lm + nlten_sink[k], -trl / dt);
                trten[ixnumice - 1][k] = MX(nc_im + niten_sink[k], -tri / dt);
                qvten[k] = qtten[k] - qlten[k] - qiten[k];
                sten[k] = slten[k] + xlv * qlten[k] + xls * qiten[k];
                qc[k] = qc_l[k] + qc_i[k];
                rliq.add(qc[k] * dp0[k] / g / 1000.0f);
                } while (0);
                if (stop) ldone = true;
            }
        }
        UW_SYNC();
        // evaporation and melting of precipitation (:3808-3934)
        if (!stop) do {
        {
            Kahan evpint_rain, evpint_snow;
            for (int k = 0; k <= mkx; k++) {
                flxrain[k] = 0.0f;
                flxsnow[k] = 0.0f;
            }
            for (int k = mkx; k >= 1; k--) {
                R snowmlt;
                if (t0[k] > 273.16f) snowmlt = MX(0.0f, flxsnow[k] * g / dp0[k]);
                else snowmlt = 0.0f;
                R qs1 = qsat_qs(t0[k], p0[k], tbld, tblf);
                R subsat = MX((1.0f - qv0[k] / qs1), 0.0f);
                R evprain = kevp * subsat * sqrtf(flxrain[k] + snowmlt * dp0[k] / g);
                R evpsnow = kevp * subsat * sqrtf(MX(flxsnow[k] - snowmlt * dp0[k] / g, 0.0f));
                R evplimit = MX(0.0f, (qw0[k] - qv0[k]) / dt);
                R evplimit_rain = MN(evplimit, (flxrain[k] + snowmlt * dp0[k] / g) * g / dp0[k]);
                evplimit_rain = MN(evplimit_rain, (rainflx.s - evpint_rain.s) * g / dp0[k]);
                evprain = MX(0.0f, MN(evplimit_rain, evprain));
                R evplimit_snow = MN(evplimit, MX(flxsnow[k] - snowmlt * dp0[k] / g, 0.0f) * g / dp0[k]);
                evplimit_snow = MN(evplimit_snow, (snowflx.s - evpint_snow.s) * g / dp0[k]);
                evpsnow = MX(0.0f, MN(evplimit_snow, evpsnow));
                if ((evprain + evpsnow) > evplimit) {
                    R tmp1 = evprain * evplimit / (evprain + evpsnow);
                    R tmp2 = evpsnow * evplimit / (evprain + evpsnow);
                    evprain = tmp1;
                    evpsnow = tmp2;
                }
                evapc[k] = evprain + evpsnow;
                evpint_rain.add(evprain * dp0[k] / g);
                evpint_snow.add(evpsnow * dp0[k] / g);
                R ntraprd = qrten[k] - evprain + snowmlt;
                R ntsnprd = qsten[k] - evpsnow - snowmlt;
                flxrain[k - 1] = flxrain[k] + ntraprd * dp0[k] / g;
                flxsnow[k - 1] = flxsnow[k] + ntsnprd * dp0[k] / g;
                flxrain[k - 1] = MX(flxrain[k - 1], 0.0f);
                flxsnow[k - 1] = MX(flxsnow[k - 1], 0.0f);
                qlten[k] = qlten[k] - qrten[k];
                qiten[k] = qiten[k] - qsten[k];
                qvten[k] = qvten[k] + evprain + evpsnow;
                qtten[k] = qlten[k] + qiten[k] + qvten[k];
                if ((qv0[k] + qvten[k] * dt) < c.qmin[0] || (ql0[k] + qlten[k] * dt) < c.qmin[1] ||
                    (qi0[k] + qiten[k] * dt) < c.qmin[2])
                    lflags |= UW_L_NEGCON;
                sten[k] = sten[k] - xlv * evprain - xls * evpsnow - (xls - xlv) * snowmlt;
                slten[k] = sten[k] - xlv * qlten[k] - xls * qiten[k];
            }
            precip = (flxrain[0] + flxsnow[0]) / 1000.0f;
            snow = flxsnow[0] / 1000.0f;
        }
        // remove detrained condensate (:3966-3981)
        for (int k = 1; k <= mkx; k++) {
            if (k > kpen) continue;
            qtten[k] = qtten[k] - qc[k];
            qlten[k] = qlten[k] - qc_l[k];
            qiten[k] = qiten[k] - qc_i[k];
            slten[k] = slten[k] + (xlv * qc_l[k] + xls * qc_i[k]);
            sten[k] = sten[k] - (xls - xlv) * qc_i[k];
        }
        // positive_moisture_single (uwshcu.F90:5096-5162 via :3995-4001), FP64 with FP64 column sums
        {
            const double qvmin = c.qmin[0], qlmin = c.qmin[1], qimin = c.qmin[2], dtd = dt;
            double qvs[KP], qvt[KP];
            for (int k = 1; k <= mkx; k++) {
                qvt[k] = qvten[k];
                qvs[k] = (double)qv0[k] + qvt[k] * dtd;
            }
            double dqv = 0.0;
            for (int k = mkx; k >= 1; k--) {
                double qlk = (double)ql0[k] + (double)qlten[k] * dtd;
                double qik = (double)qi0[k] + (double)qiten[k] * dtd;
                double dql = MX(0.0, qlmin - qlk);
                double dqi = MX(0.0, qimin - qik);
                qlten[k] = (R)((double)qlten[k] + dql / dtd);
                qiten[k] = (R)((double)qiten[k] + dqi / dtd);
                qvt[k] = qvt[k] - (dql + dqi) / dtd;
                sten[k] = (R)((double)sten[k] + c.xlv * (dql / dtd) + c.xls * (dqi / dtd));
                qvs[k] = qvs[k] - dql - dqi;
                dqv = MX(0.0, qvmin - qvs[k]);
                qvt[k] = qvt[k] + dqv / dtd;
                qvs[k] = qvs[k] + dqv;
                if (k != 1) {
                    qvs[k - 1] = qvs[k - 1] - dqv * (double)dp0[k] / (double)dp0[k - 1];
                    qvt[k - 1] = qvt[k - 1] - dqv * (double)dp0[k] / (double)dp0[k - 1] / dtd;
                }
                qvs[k] = MX(qvs[k], qvmin);
            }
            if (dqv > 1.e-20) {
                double sum = 0.0;
                for (int k = 1; k <= mkx; k++)
                    if (qvs[k] > 2.0 * qvmin) sum = sum + qvs[k] * (double)dp0[k];
                double aa = dqv * (double)dp0[1] / MX(1.e-20, sum);
                if (aa < 0.5) {
                    for (int k = 1; k <= mkx; k++) {
                        if (qvs[k] > 2.0 * qvmin) {
                            double dum = aa * qvs[k];
                            qvs[k] = qvs[k] - dum;
                            qvt[k] = qvt[k] - dum / dtd;
                        }
                    }
                }
            }
            for (int k = 1; k <= mkx; k++) qvten[k] = (R)qvt[k];
        }
        for (int k = 1; k <= mkx; k++) {
            qtten[k] = qvten[k] + qlten[k] + qiten[k];
            slten[k] = sten[k] - xlv * qlten[k] - xls * qiten[k];
        }
        // tracer tendencies (:4007-4076)
        for (int m = 4; m <= ncnst; m++) {
            if (m != ixnumliq && m != ixnumice) {
                const R trmin = c.qmin[m - 1];
                const bool wet = c.wet[m - 1] != 0;
                for (int k = 0; k <= mkx; k++) {
                    trflx_d[k] = 0.0f;
                    trflx_u[k] = 0.0f;
                }
                for (int k = 1; k <= mkx - 1; k++) {
                    R pdelx = wet ? dp0[k] : GL(dpdry0, k);
                    R dum = (GT(m, k) - trmin) * pdelx / g / dt + trflx[m - 1][k - 1] - trflx[m - 1][k] + trflx_d[k - 1];
                    trflx_d[k] = MN(0.0f, dum);
                }
                for (int k = mkx; k >= 2; k--) {
                    R pdelx = wet ? dp0[k] : GL(dpdry0, k);
                    R dum = (GT(m, k) - trmin) * pdelx / g / dt + trflx[m - 1][k - 1] - trflx[m - 1][k] +
                                 trflx_d[k - 1] - trflx_d[k] - trflx_u[k];
                    trflx_u[k - 1] = MX(0.0f, -dum);
                }
                for (int k = 1; k <= mkx; k++) {
                    R pdelx = wet ? dp0[k] : GL(dpdry0, k);
                    trten[m - 1][k] = (trflx[m - 1][k - 1] - trflx[m - 1][k] + trflx_d[k - 1] - trflx_d[k] +
                                       trflx_u[k - 1] - trflx_u[k]) * g / pdelx;
                }
            }
        }
        // in-cloud diagnostics (:4092-4158)
        if (CONDEN(prel, exprel, thlu[krel - 1], qtu[krel - 1], thj, qvj, qlj, qij, tbld, tblf)) {
            xflags |= UW_X_CONDEN;
            id_exit = true;
            stop = true;
            break;
        }
        } while (0);
        UW_SYNC();
        {
            R qcubelow = qlj + qij, qlubelow = qlj, qiubelow = qij;
            bool ldone = stop;
            for (int j = 0; j <= mkx; j++) {   // uniform
                const int k = krel + j;
                if (k > kpen) ldone = true;
                if (!ldone) do {
                const bool attop = (k == kpen);
                const int idc = CONDEN(attop ? ps0[k - 1] + ppen : ps0[k], attop ? exntop : exns0[k],
                                       attop ? thlu_top : thlu[k], attop ? qtu_top : qtu[k], thj, qvj, qlj, qij, tbld, tblf);
                if (idc) {
                    xflags |= UW_X_CONDEN;
                    id_exit = true;
                    stop = true;
                    break;
                }
                qcu[k] = 0.5f * (qcubelow + qlj + qij);
                qlu[k] = 0.5f * (qlubelow + qlj);
                qiu[k] = 0.5f * (qiubelow + qij);
                // compute_zwshcu's cloud-fraction option (zwshcu.F90:4413-4431, 4449)
                R zw_tmp2 = 0.0f, zw_tmp3 = 1.0f;
                if (ZW && c.zw_cloud_sh) {
                    zw_tmp3 = 0.5f * c.zw_ufrc0;
                    R tmp1 = (GL(z0, k) - GL(z0, krel)) / (GL(z0, kpen) - GL(z0, krel) + 10.0f);
                    tmp1 = 1.0f + c.zw_ufrcz * tmp1;
                    zw_tmp3 = zw_tmp3 * tmp1;
                    zw_tmp2 = fdr[k] * umf[k] * (zs0[k] - zs0[k - 1]) * dt / dp0[k] * 9.8f * c.zw_ufrcd;
                    zw_tmp2 = MN(1.0f - rmaxfrac, zw_tmp2);
                }
                cufrc[k] = (ufrc[k - 1] + ufrc[k]);
                if (k == krel) {
                    cufrc[k] = (ufrclcl + ufrc[k]) * (prel - ps0[k]) / (ps0[k - 1] - ps0[k]);
                } else if (k == kpen) {
                    cufrc[k] = (ufrc[k - 1] + 0.0f) * (-ppen) / (ps0[k - 1] - ps0[k]);
                    if ((qlj + qij) > criqc) {
                        qcu[k] = 0.5f * (qcubelow + criqc);
                        qlu[k] = 0.5f * (qlubelow + criqc * qlj / (qlj + qij));
                        qiu[k] = 0.5f * (qiubelow + criqc * qij / (qlj + qij));
                    }
                }
                if constexpr (ZW) cufrc[k] = zw_tmp3 * cufrc[k] + zw_tmp2;
                qcubelow = qlj + qij;
                qlubelow = qlj;
                qiubelow = qij;
                } while (0);
                if (stop) ldone = true;
            }
        }
        UW_SYNC();
        if (!stop) do {
        cnt = (R)kpen;
        cnb = (R)(krel - 1);

        if (iter == 1) {
            // Save the iteration-1 outputs into the output slots (the Fortran *_s copies, :4177-4277)
            for (int k = 0; k <= mkx; k++) {
                OI(umf, k) = umf[k];
                OI(slflx, k) = slflx[k];
                OI(qtflx, k) = qtflx[k];
            }
            for (int k = 1; k <= mkx; k++) {
                OL(qvten, k) = qvten[k]; OL(qlten, k) = qlten[k]; OL(qiten, k) = qiten[k];
                OL(sten, k) = sten[k]; OL(uten, k) = uten[k]; OL(vten, k) = vten[k];
                OL(qrten, k) = qrten[k]; OL(qsten, k) = qsten[k]; OL(evapc, k) = evapc[k];
                OL(cufrc, k) = cufrc[k]; OL(qcu, k) = qcu[k]; OL(qlu, k) = qlu[k];
                OL(qiu, k) = qiu[k]; OL(qc, k) = qc[k];
                for (int m = 1; m <= ncnst; m++) OT(m, k) = trten[m - 1][k];
            }
            A.precip[i] = precip;
            A.snow[i] = snow;
            A.cush[i] = cush;
            A.cbmf[i] = cbmf;
            A.rliq[i] = rliq.s;
            A.cnt[i] = CNT(cnt);
            A.cnb[i] = CNT(cnb);
            PUT_DIAG_LEVEL();
            cin_s = cin; cinlcl_s = cinlcl; plcl_s = plcl; pinv_s = ps0[kinv - 1]; plfc_s = plfc;
            pbup_s = ps0[kbup]; ppen_s = ps0[kpen - 1] + ppen; tkeavg_s = tkeavg;
            kinv_s = kinv; klcl_s = klcl; klfc_s = klfc; krel_s = krel; kbup_s = kbup; kpen_s = kpen;
            // advance the state for the second CIN estimate (:4177-4184, :4285-4327)
            for (int k = 1; k <= mkx; k++) {
                R qv0s = qv0[k] + qvten[k] * dt;
                R ql0s = ql0[k] + qlten[k] * dt;
                R qi0s = qi0[k] + qiten[k] * dt;
                R s0s = s0[k] + sten[k] * dt;
                R t0s = t0[k] + sten[k] * dt / cp;
                qv0[k] = qv0s;
                ql0[k] = ql0s;
                qi0[k] = qi0s;
                s0[k] = s0s;
                t0[k] = t0s;
                qt0[k] = (qv0[k] + ql0[k] + qi0[k]);
                thl0[k] = (t0[k] - xlv * ql0[k] / cp - xls * qi0[k] / cp) / exn0[k];
            }
            slope<KP>(mkx, thl0, p0, ssthl0);
            slope<KP>(mkx, qt0, p0, ssqt0);
        }
        } while (0);
        UW_SYNC();
        if (iter == 1) {   // uniform
            bool ldone = stop;
            for (int k = 1; k <= mkx; k++) {   // uniform
                if (!ldone) do {
                R thl0bot = thl0[k] + ssthl0[k] * (ps0[k - 1] - p0[k]);
                R qt0bot = qt0[k] + ssqt0[k] * (ps0[k - 1] - p0[k]);
                if (CONDEN(ps0[k - 1], exns0[k - 1], thl0bot, qt0bot, thj, qvj, qlj, qij, tbld, tblf)) {
                    xflags |= UW_X_CONDEN;
                    id_exit = true;
                    stop = true;
                    break;
                }
                thv0bot[k] = thj * (1.0f + zvir * qvj - qlj - qij);
                thvl0bot[k] = thl0bot * (1.0f + zvir * qt0bot);
                R thl0top = thl0[k] + ssthl0[k] * (ps0[k] - p0[k]);
                R qt0top = qt0[k] + ssqt0[k] * (ps0[k] - p0[k]);
                if (CONDEN(ps0[k], exns0[k], thl0top, qt0top, thj, qvj, qlj, qij, tbld, tblf)) {
                    xflags |= UW_X_CONDEN;
                    id_exit = true;
                    stop = true;
                    break;
                }
                thv0top[k] = thj * (1.0f + zvir * qvj - qlj - qij);
                thvl0top[k] = thl0top * (1.0f + zvir * qt0top);
                } while (0);
                if (stop) ldone = true;
            }
        }
        UW_SYNC();
        }   // MODE != UW_MODE_TRIGGER
    }

    // ---- final outputs (uwshcu.F90:4337-4370) --------------------------------------------------
    if (!stop) {
    for (int k = 0; k <= mkx; k++) {
        OI(umf, k) = umf[k];
        OI(wu, k) = wu[k];
        OI(slflx, k) = slflx[k];
        OI(qtflx, k) = qtflx[k];
        OI(flxprc1, k) = flxrain[k] + flxsnow[k];
        OI(flxsnow1, k) = flxsnow[k];
    }
    for (int k = 1; k <= mkx; k++) {
        OL(qvten, k) = qvten[k]; OL(qlten, k) = qlten[k]; OL(qiten, k) = qiten[k];
        OL(sten, k) = sten[k]; OL(uten, k) = uten[k]; OL(vten, k) = vten[k];
        OL(qrten, k) = qrten[k]; OL(qsten, k) = qsten[k]; OL(evapc, k) = evapc[k];
        OL(cufrc, k) = cufrc[k]; OL(qcu, k) = qcu[k]; OL(qlu, k) = qlu[k];
        OL(qiu, k) = qiu[k]; OL(qc, k) = qc[k];
        for (int m = 1; m <= ncnst; m++) OT(m, k) = trten[m - 1][k];
    }
    A.precip[i] = precip;
    A.snow[i] = snow;
    A.cush[i] = cush;
    A.cbmf[i] = cbmf;
    A.rliq[i] = rliq.s;
    A.cnt[i] = CNT(cnt);
    A.cnb[i] = CNT(cnb);
    if (A.diag_real) {
        A.diag_real[UW_DR_CIN * (size_t)mix + i] = cin;
        A.diag_real[UW_DR_CINLCL * (size_t)mix + i] = cinlcl;
        A.diag_real[UW_DR_PLCL * (size_t)mix + i] = plcl;
        A.diag_real[UW_DR_PLFC * (size_t)mix + i] = plfc;
        A.diag_real[UW_DR_PINV * (size_t)mix + i] = ps0[kinv - 1];
        A.diag_real[UW_DR_PBUP * (size_t)mix + i] = ps0[kbup];
        A.diag_real[UW_DR_PPEN * (size_t)mix + i] = ps0[kpen - 1] + ppen;
        A.diag_real[UW_DR_TKEAVG * (size_t)mix + i] = tkeavg;
    }
    PUT_DIAG_LEVEL();
    }

    // (label 333, :4448-4549)
    if (!cand && !handed) {
    if (id_exit) {
        xflags |= UW_X_UWCU;
        for (int k = 0; k <= mkx; k++) {
            OI(umf, k) = 0.0f;
            OI(wu, k) = 0.0f;
            OI(slflx, k) = 0.0f;
            OI(qtflx, k) = 0.0f;
            OI(flxprc1, k) = 0.0f;
            OI(flxsnow1, k) = 0.0f;
        }
        for (int k = 1; k <= mkx; k++) {
            OL(qvten, k) = 0.0f; OL(qlten, k) = 0.0f; OL(qiten, k) = 0.0f; OL(sten, k) = 0.0f;
            OL(uten, k) = 0.0f; OL(vten, k) = 0.0f; OL(qrten, k) = 0.0f; OL(qsten, k) = 0.0f;
            OL(evapc, k) = 0.0f; OL(cufrc, k) = 0.0f; OL(qcu, k) = 0.0f; OL(qlu, k) = 0.0f;
            OL(qiu, k) = 0.0f; OL(qc, k) = 0.0f;
            for (int m = 1; m <= ncnst; m++) OT(m, k) = 0.0f;
        }
        A.precip[i] = 0.0f;
        A.snow[i] = 0.0f;
        A.cush[i] = -1.0f;
        A.cbmf[i] = 0.0f;
        A.rliq[i] = 0.0f;
        A.cnt[i] = CNT(1.0f);
        A.cnb[i] = CNT((R)mkx);
        if (A.diag_real) {
            A.diag_real[UW_DR_CIN * (size_t)mix + i] = -1.0f;
            A.diag_real[UW_DR_CINLCL * (size_t)mix + i] = -1.0f;
            for (int j = UW_DR_PLCL; j < UW_NDR; j++) A.diag_real[j * (size_t)mix + i] = 0.0f;
        }
        if (A.diag_level)
            for (int j = 0; j < UW_NDL; j++)
                for (int k = 0; k <= mkx; k++) DLV(j, k) = 0.0f;
        kinv = klcl = klfc = krel = kbup = kpen = 0;
    }
    if (A.diag_int) {
        A.diag_int[UW_DI_EXIT * (size_t)mix + i] = xflags;
        A.diag_int[UW_DI_LIMIT * (size_t)mix + i] = lflags;
        A.diag_int[UW_DI_KINV * (size_t)mix + i] = kinv;
        A.diag_int[UW_DI_KLCL * (size_t)mix + i] = klcl;
        A.diag_int[UW_DI_KLFC * (size_t)mix + i] = klfc;
        A.diag_int[UW_DI_KREL * (size_t)mix + i] = krel;
        A.diag_int[UW_DI_KBUP * (size_t)mix + i] = kbup;
        A.diag_int[UW_DI_KPEN * (size_t)mix + i] = kpen;
    }
    // the column's place in the next call's first worklist launch (uwshcu_set_depth_order): the
    // explicit-CIN columns first, then by updraft depth
    if (A.depth_key) {
        const int depth = kpen - krel;
        A.depth_key[i] = ((lflags & UW_L_DELCIN) ? 0 : 64) + (depth < 0 ? 0 : (depth > 63 ? 63 : depth));
    }
    }
    if (errbits) atomicOr(A.err, errbits);
    }  // active
    if (MODE == UW_MODE_TRIGGER) {
        // warp-aggregated append of this warp's candidates
        const unsigned lane = threadIdx.x & 31u;
        const unsigned mask = __ballot_sync(0xffffffffu, cand);
        if (mask) {
            const int leader = __ffs(mask) - 1;
            int base = 0;
            if ((int)lane == leader) base = atomicAdd(wl_count, __popc(mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (cand) wl[base + __popc(mask & ((1u << lane) - 1u))] = i;
        }
    }
#undef UW_SYNC
#undef CONDEN
#undef RI
#undef RL
#undef CNT
#undef GI
#undef GL
#undef GT
#undef OI
#undef OL
#undef OT
#undef DLV
#undef PUT_DIAG_LEVEL
#undef UEMF
}

// ---- kernels ---------------------------------------------------------------------------------------

// Register caps (resident blocks of 128 per SM): the worklist launches at 72 registers (7 blocks;
// 1,048,576 x 30 columns: 103.9 ms against 115.6 ms at the FP64 kernel's 4 and 5 blocks, 109.8 ms
// at 6, 104.5 ms at 8), the trigger pass at 72 too (7 blocks: 103.1-103.4 ms against 104.8 ms at 5),
// the single pass at 168.
#define UW_LIST_MINB(m) ((m) == UW_MODE_RESUME ? 7 : (UW_MODE_IS_LIST(m) ? 7 : ((m) == UW_MODE_TRIGGER ? 7 : 3)))
template <int KP, int NC, int MODE>
__global__ void __launch_bounds__(128, UW_LIST_MINB(MODE))
uwshcu_mixed_kernel(const __grid_constant__ UwArgs A, int* __restrict__ wl, int* __restrict__ wl_count)
{
    __shared__ double tbld[UW_TBL];
    __shared__ float tblf[UW_TBL];
    for (int t = threadIdx.x; t < UW_TBL; t += blockDim.x) {
        tbld[t] = c_estbl[t];
        tblf[t] = (float)c_estbl[t];
    }
    __syncthreads();

    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    int i;
    bool active;
    if (MODE == UW_MODE_LIST || MODE == UW_MODE_LIST1) {
        active = tid < *wl_count;
        i = active ? wl[tid] : 0;
    } else if (MODE == UW_MODE_RESUME) {
        const int n = MN(*A.hand->count, A.hand->cap);
        active = tid < n;
        i = active ? A.hand->order[tid] : 0;   // a hand-off slot
    } else {
        active = tid < A.iend;
        i = tid;
    }
    uw_column<KP, NC, MODE, 0>(A, tbld, tblf, i, active, wl, wl_count);
}

// Batched trigger pass: every column of every member of B (members of one level/tracer class).
// Blocks [block_start[m], block_start[m+1]) cover member m; its convecting columns go to
// wl[m] / count[m].  FAST selects the column code of the fast-FP64 mode.
template <int KP, int NC, int FAST>
__global__ void __launch_bounds__(128, 5) uwshcu_batch_trigger(const __grid_constant__ UwBatch B)
{
    __shared__ double tbld[UW_TBL];
    __shared__ float tblf[UW_TBL];
    for (int t = threadIdx.x; t < UW_TBL; t += blockDim.x) {
        tbld[t] = c_estbl[t];
        tblf[t] = (float)c_estbl[t];
    }
    __syncthreads();

    int m = 0;
    while (m + 1 < B.nm && (int)blockIdx.x >= B.block_start[m + 1]) m++;
    const int tid = ((int)blockIdx.x - B.block_start[m]) * blockDim.x + threadIdx.x;
    const bool active = tid < B.m[m].iend;
    uw_column<KP, NC, UW_MODE_TRIGGER, FAST>(B.m[m], tbld, tblf, tid, active, B.wl[m], B.count + m);
}

// Batched worklist pass, persistent: each warp takes the next task (32 * B.chunk consecutive queue
// entries of one member) from the device counter *B.task_head until the queues are drained, so a
// warp never mixes members (their level counts differ).  Task t of member m covers entries
// [t * 32 * chunk, (t + 1) * 32 * chunk) of wl[m].  LMODE: UW_MODE_LIST, or UW_MODE_LIST1 for the
// sorted schedule (each member hands its implicit-CIN columns to its own region, B.m[m].hand).
template <int KP, int NC, int MINB, int FAST, int LMODE = UW_MODE_LIST>
__global__ void __launch_bounds__(128, MINB) uwshcu_batch_list(const __grid_constant__ UwBatch B)
{
    __shared__ double tbld[UW_TBL];
    __shared__ float tblf[UW_TBL];
    for (int t = threadIdx.x; t < UW_TBL; t += blockDim.x) {
        tbld[t] = c_estbl[t];
        tblf[t] = (float)c_estbl[t];
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int per_task = 32 * B.chunk;
    for (;;) {
        int task = 0;
        if (lane == 0) task = atomicAdd(B.task_head, 1);
        task = __shfl_sync(0xffffffffu, task, 0);
        int m = -1, first = 0;
        for (int j = 0; j < B.nm; j++) {
            const int nt = (B.count[j] + per_task - 1) / per_task;
            if (m < 0) {
                if (task < nt) {
                    m = j;
                    first = task * per_task;
                } else {
                    task -= nt;
                }
            }
        }
        if (m < 0) break;   // same task on every lane: the whole warp leaves
        const int n = B.count[m];
        for (int c = 0; c < B.chunk; c++) {
            const int idx = first + c * 32 + lane;
            const bool active = idx < n;
            const int i = active ? B.wl[m][idx] : 0;
            uw_column<KP, NC, LMODE, FAST>(B.m[m], tbld, tblf, i, active, nullptr, nullptr);
        }
    }
}

// Batched resume launch of the sorted schedule, persistent: each warp takes the next task (32
// consecutive entries of one member's hand-off slots in sorted order) from *B.task_head2 until every
// member's slots are done.  Member m has min(*count, cap) slots in its region B.m[m].hand.
template <int KP, int NC, int FAST>
__global__ void __launch_bounds__(128, 5) uwshcu_batch_resume(const __grid_constant__ UwBatch B)
{
    __shared__ double tbld[UW_TBL];
    __shared__ float tblf[UW_TBL];
    for (int t = threadIdx.x; t < UW_TBL; t += blockDim.x) {
        tbld[t] = c_estbl[t];
        tblf[t] = (float)c_estbl[t];
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    for (;;) {
        int task = 0;
        if (lane == 0) task = atomicAdd(B.task_head2, 1);
        task = __shfl_sync(0xffffffffu, task, 0);
        int m = -1, first = 0;
        for (int j = 0; j < B.nm; j++) {
            const int nt = (MN(*B.m[j].hand->count, B.m[j].hand->cap) + 31) / 32;
            if (m < 0) {
                if (task < nt) {
                    m = j;
                    first = task * 32;
                } else {
                    task -= nt;
                }
            }
        }
        if (m < 0) break;   // same task on every lane: the whole warp leaves
        const UwHand& H = *B.m[m].hand;
        const int idx = first + lane;
        const bool active = idx < MN(*H.count, H.cap);
        const int slot = active ? H.order[idx] : 0;
        uw_column<KP, NC, UW_MODE_RESUME, FAST>(B.m[m], tbld, tblf, slot, active, nullptr, nullptr);
    }
}

}  // namespace
