// uwshcu_tl_kernel.cuh -- tangent-linear (forward-mode) kernel of compute_uwshcu
// (uwshcu.F90:478-4664).  GENERATED by gen_tangent.py from uwshcu_fp64_kernel.cuh: do not edit;
// change the FP64 column code and regenerate.  See gen_tangent.py for what the generator does.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include "uwshcu_common.cuh"
#include "uwshcu.h"
#include "uw_math.h"
#include "uw_dual.h"
#include "uw_state.cuh"

namespace {

typedef uwshcu_tangent UwTangent;

__constant__ UwConst c;
__constant__ double c_estbl[UW_TBL];

#define MX(a, b) ((a) > (b) ? (a) : (b))
#define MN(a, b) ((a) < (b) ? (a) : (b))

// estblf (wv_saturation.F90:64-80).  e is clamped to [tmin, tmax] first (a NaN argument ends at
// tmax), so i stays in 1..203 and i+1 inside the 204 filled entries.
__device__ __forceinline__ Tl estblf(Tl td, const double* __restrict__ tbl)
{
    Tl e = MX(MN(td, c.tmax), c.tmin);
    int i = (int)(e - c.tmin) + 1;
    Tl ai = trunc(e - c.tmin);
    return (c.tmin + ai - e + 1.0) * tbl[i - 1] - (c.tmin + ai - e) * tbl[i];
}

// vqsatd with len = 1 (wv_saturation.F90:482-609) returning es, qs and gam.
__device__ __forceinline__ void qsat3(Tl t, Tl p, Tl& es, Tl& qs, Tl& gam,
                                      const double* __restrict__ tbl)
{
    es = estblf(t, tbl);
    qs = c.epsqs * es / (p - c.omeps * es);
    qs = MN(1.0, qs);
    if (qs < 0.0) {
        qs = 1.0;
        es = p;
    }
    Tl hltalt, desdt;
    if (c.icephs && c.ttrice != 0.0) {
        Tl tc = t - c.tmelt;
        bool lflg = (tc >= -c.ttrice && tc < 0.0);
        Tl weight = MN(-tc * c.trinv, 1.0);
        Tl hlatsb = c.hlatv + weight * c.hlatf;
        Tl hlatvp = c.hlatv - 2369.0 * tc;
        hltalt = (t < c.tmelt) ? hlatsb : hlatvp;
        Tl tterm = lflg ? c.pcf[0] + tc * (c.pcf[1] + tc * (c.pcf[2] + tc * (c.pcf[3] + tc * c.pcf[4]))) : 0.0;
        desdt = hltalt * es / (c.rgasv * t * t) + tterm * c.trinv;
    } else {
        Tl hlatvp = c.hlatv - 2369.0 * (t - c.tmelt);
        Tl hlatsb = c.icephs ? c.hlatv + c.hlatf : c.hlatv;
        hltalt = (t < c.tmelt) ? hlatsb : hlatvp;
        desdt = hltalt * es / (c.rgasv * t * t);
    }
    gam = hltalt * qs * p * desdt / (c.cpws * es * (p - c.omeps * es));
    if (qs == 1.0) gam = 0.0;
}

// The qs of vqsatd only (what conden and the buoyancy sorting consume).
__device__ __forceinline__ Tl qsat_qs(Tl t, Tl p, const double* __restrict__ tbl)
{
    Tl es = estblf(t, tbl);
    Tl qs = c.epsqs * es / (p - c.omeps * es);
    qs = MN(1.0, qs);
    if (qs < 0.0) qs = 1.0;
    return qs;
}

__device__ __forceinline__ Tl exnf(Tl p) { return uw_pow(p / c.p00, c.rovcp); }

// conden (uwshcu.F90:4718-4785) with ex = exnf(p) supplied by the caller.  Not inlined: the kernel
// calls it from ~30 sites, and one shared copy keeps the kernel inside the instruction cache
// (inlined, the stall on instruction fetch doubled the run time).
__device__ __noinline__ int conden(Tl p, Tl ex, Tl thl, Tl qt, Tl& th, Tl& qv,
                                      Tl& ql, Tl& qi, const double* __restrict__ tbl)
{
    Tl tc = thl * ex;
    Tl nu = MX(MN((268.0 - tc) / 20.0, 1.0), 0.0);
    Tl leff = (1.0 - nu) * c.xlv + nu * c.xls;
    Tl temps = tc;
    Tl rvls = qsat_qs(temps, p, tbl);
    int id_check = 0;
    if (rvls >= qt) {
        qv = qt;
        ql = 0.0;
        qi = 0.0;
        th = tc / ex;
    } else {
        Tl qs = rvls;
        // the Fortran's divisions by leff, r and (twice per step) temps go through their
        // correctly rounded reciprocals: the same quotients, bit for bit (uw_div_by)
        const Tl rleff = 1.0 / leff;
        const Tl cpl = uw_div_by(c.cp, leff, rleff);
#pragma unroll 1
        for (int it = 0; it < 10; it++) {
            const Tl rt = 1.0 / temps;
            temps = temps + (uw_div_by((tc - temps) * c.cp, leff, rleff) + qt - rvls) /
                                (cpl + uw_div_by(uw_div_by(uw_div_by(c.ep2 * leff * rvls, c.r, c.rinv), temps, rt), temps, rt));
            qs = qsat_qs(temps, p, tbl);
            rvls = qs;
        }
        Tl qc = MX(qt - qs, 0.0);
        qv = qt - qc;
        ql = qc * (1.0 - nu);
        qi = nu * qc;
        th = temps / ex;
        id_check = (fabs((temps - (leff / c.cp) * qc) - tc) >= 1.0) ? 1 : 0;
    }
    return id_check;
}

// conden for the fast-FP64 precision mode: the same saturation adjustment with one reciprocal of the
// temperature per Newton step (2 divisions instead of 5), each lane stopping after its first step
// smaller than 1e-10 T.  The Fortran always takes 10 steps; the steps shrink about 100x per
// iteration and fall below 1e-10 T after 5-7, so the result differs from conden by about 1e-12
// relative.  A lane's result depends only on its own column; the warp leaves the loop when every
// lane is done (__all_sync over the lanes active at the call), so the lanes stay together.
__device__ __noinline__ int conden_fast(Tl p, Tl ex, Tl thl, Tl qt, Tl& th, Tl& qv,
                                        Tl& ql, Tl& qi, const double* __restrict__ tbl)
{
    Tl tc = thl * ex;
    Tl nu = MX(MN((268.0 - tc) / 20.0, 1.0), 0.0);
    Tl leff = (1.0 - nu) * c.xlv + nu * c.xls;
    Tl temps = tc;
    Tl rvls = qsat_qs(temps, p, tbl);
    int id_check = 0;
    if (rvls >= qt) {
        qv = qt;
        ql = 0.0;
        qi = 0.0;
        th = tc / ex;
    } else {
        const Tl cpl = c.cp / leff;
        const Tl a2 = c.ep2 * leff / c.r;
        Tl qs = rvls;
        bool done = false;
#pragma unroll 1
        for (int it = 0; it < 10; it++) {
            if (!done) {
                const Tl rt = 1.0 / temps;
                const Tl dT = ((tc - temps) * cpl + qt - rvls) / (cpl + a2 * rvls * rt * rt);
                temps = temps + dT;
                qs = qsat_qs(temps, p, tbl);
                rvls = qs;
                done = fabs(dT) < 1.e-10 * temps;
            }
            if (__all_sync(__activemask(), done)) break;
        }
        Tl qc = MX(qt - qs, 0.0);
        qv = qt - qc;
        ql = qc * (1.0 - nu);
        qi = nu * qc;
        th = temps / ex;
        id_check = (fabs((temps - (leff / c.cp) * qc) - tc) >= 1.0) ? 1 : 0;
    }
    return id_check;
}

// roots (uwshcu.F90:4787-4829); r1/r2 keep the caller's values on the failure branches.
__device__ __forceinline__ int roots(Tl a, Tl b, Tl cc, Tl& r1, Tl& r2)
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
                Tl q = -0.5 * (b + copysign(1.0, b) * sqrt(b * b - 4.0 * a * cc));
                r1 = q / a;
                r2 = cc / q;
            }
        }
    }
    return status;
}

// slope (uwshcu.F90:4831-4861); field/p0/sl are 1-based local arrays.
template <int KP>
__device__ __forceinline__ void slope(int mkx, const Tl* field, const Tl* p0, Tl* sl)
{
    Tl below = (field[2] - field[1]) / (p0[2] - p0[1]);
#pragma unroll 1
    for (int k = 2; k <= mkx; k++) {
        Tl above = (field[k] - field[k - 1]) / (p0[k] - p0[k - 1]);
        if (above > 0.0) sl[k - 1] = MX(0.0, MN(above, below));
        else sl[k - 1] = MN(0.0, MX(above, below));
        below = above;
    }
    sl[mkx] = sl[mkx - 1];
}

// qsinvert (uwshcu.F90:4863-4929) with exsfc = exnf(psfc).
__device__ __noinline__ Tl qsinvert(Tl qt, Tl thl, Tl psfc, Tl exsfc, const double* __restrict__ tbl)
{
    const Tl psmin = 100.0 * 100.0, dpsmax = 1.0;
    Tl es, qs, gam;
    Tl Ti = thl * exsfc;
    qsat3(Ti, psfc, es, qs, gam, tbl);
    Tl rhi = qt / qs;
    // single exit, fixed trip count: every lane of a warp leaves together
    Tl result = psmin;
    if (!(rhi <= 0.01)) {
        Tl TLCL = 55.0 + 1.0 / (1.0 / (Ti - 55.0) - uw_log(rhi) / 2840.0);
        Tl PiLCL = TLCL / thl;
        Tl ps = c.p00 * uw_pow(PiLCL, 1.0 / c.rovcp);
        bool done = false;
#pragma unroll 1
        for (int i = 1; i <= 10; i++) {
            if (done) continue;
            Tl Pis = uw_pow(ps / c.p00, c.rovcp);
            Tl Ts = thl * Pis;
            qsat3(Ts, ps, es, qs, gam, tbl);
            Tl err = qt - qs;
            Tl nu = MX(MN((268.0 - Ts) / 20.0, 1.0), 0.0);
            Tl leff = (1.0 - nu) * c.xlv + nu * c.xls;
            Tl dlnqsdT = gam * (c.cp / leff) / qs;
            Tl dTdPis = thl;
            Tl dPisdps = c.rovcp * Pis / ps;
            Tl dlnqsdps = -1.0 / (ps - (1.0 - c.ep2) * es);
            Tl derrdps = -qs * (dlnqsdT * dTdPis * dPisdps + dlnqsdps);
            Tl dps = -err / derrdps;
            ps = ps + dps;
            if (ps < 0.0) {
                done = true;
            } else if (fabs(dps) <= dpsmax) {
                result = ps;
                done = true;
            }
        }
    }
    return result;
}

// compute_alpha (uwshcu.F90:4931-4950)
__device__ __noinline__ Tl compute_alpha(Tl del_CIN, Tl ke)
{
    Tl x0 = 0.0;
#pragma unroll 1
    for (int it = 0; it < 10; it++) {
        Tl x1 = x0 - (uw_exp(-x0 * ke * del_CIN) - x0) / (-ke * del_CIN * uw_exp(-x0 * ke * del_CIN) - 1.0);
        x0 = x1;
    }
    return x0;
}

// compute_mumin2 (uwshcu.F90:4952-4979)
__device__ __noinline__ Tl compute_mumin2(Tl mulcl, Tl rmaxfrac, Tl mulow)
{
    Tl x0 = mulow;
#pragma unroll 1
    for (int it = 0; it < 10; it++) {
        Tl ex = uw_exp(-(x0 * x0));
        Tl ef = uw_erfc(x0);
        Tl exf = ex / ef;
        Tl t1 = ex / 2.0 / rmaxfrac;
        Tl t2 = mulcl * 2.5066 / 2.0;
        Tl f = 0.5 * (exf * exf) - 0.5 * (t1 * t1) - (t2 * t2);
        Tl fs = (2.0 * (exf * exf)) * (exf / sqrt(3.141592) - x0) + (0.5 * x0 * (ex * ex)) / (rmaxfrac * rmaxfrac);
        Tl x1 = x0 - f / fs;
        x0 = x1;
    }
    return x0;
}

// compute_ppen (uwshcu.F90:4981-5028); the 1.e-8 at :4998 is a default-real literal.
__device__ __noinline__ Tl compute_ppen(Tl wtwb, Tl D, Tl bogbot, Tl bogtop, Tl rho0j, Tl dpen)
{
    Tl x0;
    Tl SB = (bogtop - bogbot) / dpen;
    Tl s00 = bogbot / rho0j - D * wtwb;
    if (D * dpen < (Tl)1.e-8f) {
        if (s00 >= 0.0) x0 = dpen;
        else x0 = MX(0.0, MN(dpen, -0.5 * wtwb / s00));
    } else {
        if (s00 >= 0.0) x0 = dpen;
        else x0 = 0.0;
#pragma unroll 1
        for (int it = 0; it < 5; it++) {
            Tl f = uw_exp(-2.0 * D * x0) * (wtwb - (bogbot - SB / (2.0 * D)) / (D * rho0j)) +
                       (SB * x0 + bogbot - SB / (2.0 * D)) / (D * rho0j);
            Tl fs = -2.0 * D * uw_exp(-2.0 * D * x0) * (wtwb - (bogbot - SB / (2.0 * D)) / (D * rho0j)) +
                        (SB) / (D * rho0j);
            if (fs >= 0.0) fs = MX(fs, 1.e-10);
            else fs = MN(fs, -1.e-10);
            Tl x1 = x0 - f / fs;
            x0 = x1;
        }
    }
    return -MX(0.0, MN(dpen, x0));
}

// single_cin (uwshcu.F90:4704-4715) with the exner values of pbot/ptop supplied.
__device__ __forceinline__ Tl single_cin(Tl pbot, Tl exb, Tl thv0bot, Tl ptop, Tl ext,
                                             Tl thv0top, Tl thvubot, Tl thvutop)
{
    return ((1.0 - thvubot / thv0bot) + (1.0 - thvutop / thv0top)) * (pbot - ptop) /
           (pbot / (c.r * thv0bot * exb) + ptop / (c.r * thv0top * ext));
}

// getbuoy (uwshcu.F90:4672-4702) with the exner values supplied.
__device__ __forceinline__ void getbuoy(Tl pbot, Tl exb, Tl thv0bot, Tl ptop, Tl ext,
                                        Tl thv0top, Tl thvubot, Tl thvutop, Tl& plfc, Tl& cin)
{
    if (thvubot > thv0bot && thvutop > thv0top) {
        plfc = pbot;
    } else if (thvubot <= thv0bot && thvutop <= thv0top) {
        cin = cin - ((thvubot / thv0bot - 1.0) + (thvutop / thv0top - 1.0)) * (pbot - ptop) /
                        (pbot / (c.r * thv0bot * exb) + ptop / (c.r * thv0top * ext));
    } else if (thvubot > thv0bot && thvutop <= thv0top) {
        Tl frc = (thvutop / thv0top - 1.0) / ((thvutop / thv0top - 1.0) - (thvubot / thv0bot - 1.0));
        cin = cin - (thvutop / thv0top - 1.0) * ((ptop + frc * (pbot - ptop)) - ptop) /
                        (pbot / (c.r * thv0bot * exb) + ptop / (c.r * thv0top * ext));
    } else {
        Tl frc = (thvubot / thv0bot - 1.0) / ((thvubot / thv0bot - 1.0) - (thvutop / thv0top - 1.0));
        plfc = pbot - frc * (pbot - ptop);
        cin = cin - (thvubot / thv0bot - 1.0) * (pbot - plfc) /
                        (pbot / (c.r * thv0bot * exb) + ptop / (c.r * thv0top * ext));
    }
}

// fluxbelowinv (uwshcu.F90:5030-5094).  Writes xflx(0:kinv-1); the Fortran zeroes xflx(kinv:mkx)
// too, but the caller only reads 0..kinv-1.
__device__ __forceinline__ void fluxbelowinv(Tl cbmf, const Tl* ps0, int kinv, Tl dt, Tl xsrc,
                                             Tl xmean, Tl xtopin, Tl xbotin, Tl* xflx)
{
    Tl xtop, xbot;
    Tl dp = ps0[kinv - 1] - ps0[kinv];
    if (fabs(xbotin - xtopin) <= 1.e-13) {
        xbot = xbotin - 1.e-13;
        xtop = xtopin + 1.e-13;
    } else {
        xbot = xbotin;
        xtop = xtopin;
    }
    Tl xtop_ori = xtop, xbot_ori = xbot;
    Tl rcbmf = (cbmf * c.g * dt) / dp;
    Tl rpeff = (xmean - xtop) / (xbot - xtop);
    rpeff = MN(MX(0.0, rpeff), 1.0);
    if (rpeff == 0.0 || rpeff == 1.0) {
        xbot = xmean;
        xtop = xmean;
    }
    Tl rr = rpeff / rcbmf;
    Tl pinv = ps0[kinv - 1] - rpeff * dp;
#pragma unroll 1
    for (int k = 0; k <= kinv - 1; k++) xflx[k] = cbmf * (xsrc - xbot) * (ps0[0] - ps0[k]) / (ps0[0] - pinv);
    if (rr <= 1.0) xflx[kinv - 1] = xflx[kinv - 1] - (1.0 - rr) * cbmf * (xtop_ori - xbot_ori);
}

// findsp (uwshcu.F90:5164-5454) for one point; returns the wet-bulb qsp and ORs error bits.
__device__ Tl findsp_point(Tl q, Tl t, Tl p, unsigned int& errbits, const double* __restrict__ tbl)
{
    const Tl omeps = 1.0 - c.epsqs, trinv = 1.0 / c.ttrice, a1 = 7.5 * uw_log(10.0), rair = 287.04;
    const Tl c3 = rair * a1 / c.cpws, dttol = 1.e-4, dqtol = 1.e-4, tt0 = 273.15;
    Tl dtt = 0.0, dq = 0.0, enin, enout = 1.0, tsp, qsp, hltalt = 0.0;
    int doit = 0;
    Tl tlim = MN(MX(t, 173.0), 373.0);
    Tl es = estblf(tlim, tbl);
    Tl denom = p - omeps * es;
    Tl qs = c.epsqs * es / denom;
    if (p > 5.0 * es && qs > 0.0 && qs < 0.5) {
        qs = MN(c.epsqs * es / denom, 1.0);
        Tl tc = tlim - tt0;
        Tl weight = MN(-tc * trinv, 1.0);
        Tl hlatsb = c.hlatv + weight * c.hlatf;
        Tl hlatvp = c.hlatv - 2369.0 * tc;
        hltalt = (tlim < tt0) ? hlatsb : hlatvp;
        enin = c.cpws * tlim + hltalt * q;
        Tl tmp = q - qs;
        Tl c1 = hltalt * c3;
        Tl c2 = (tlim + 36.0) * (tlim + 36.0);
        Tl r1b = c2 / (c2 + c1 * qs);
        Tl qvd = r1b * tmp;
        tsp = tlim + ((hltalt / c.cpws) * qvd);
        es = estblf(tsp, tbl);
        qsp = MN(c.epsqs * es / (p - omeps * es), 1.0);
    } else {
        doit = 1;
        tsp = tlim;
        qsp = q;
        enin = 1.0;
    }
#pragma unroll 1
    for (int l = 1; l <= 8 && doit == 0; l++) {
        es = estblf(tsp, tbl);
        qs = MN(c.epsqs * es / (p - omeps * es), 1.0);
        Tl tc = tsp - tt0;
        bool lflg = (tc >= -c.ttrice && tc < 0.0);
        Tl weight = MN(-tc * trinv, 1.0);
        Tl hlatsb = c.hlatv + weight * c.hlatf;
        Tl hlatvp = c.hlatv - 2369.0 * tc;
        hltalt = (tsp < tt0) ? hlatsb : hlatvp;
        Tl tterm = lflg ? c.pcf[0] + tc * (c.pcf[1] + tc * (c.pcf[2] + tc * (c.pcf[3] + tc * c.pcf[4]))) : 0.0;
        Tl desdt = hltalt * es / (c.rgasv * tsp * tsp) + tterm * trinv;
        Tl dqsdt = (c.epsqs + omeps * qs) / (p - omeps * es) * desdt;
        Tl gg = enin - (c.cpws * tsp + hltalt * qsp);
        Tl dgdt = -(c.cpws + hltalt * dqsdt);
        Tl t1 = tsp - gg / dgdt;
        dtt = fabs(t1 - tsp) / t1;
        tsp = MX(t1, c.tmin);
        es = estblf(tsp, tbl);
        Tl q1 = MN(c.epsqs * es / (p - omeps * es), 1.0);
        dq = fabs(q1 - qsp) / MX(q1, 1.e-12);
        qsp = q1;
        if (dtt < dttol && dq < dqtol) doit = 2;
        enout = c.cpws * tsp + hltalt * qsp;
        if (tsp < 174.16) doit = 4;
    }
    if (doit == 0 && (dtt > dttol || dq > dqtol)) errbits |= UW_ERRBIT_FINDSP;
    if (doit == 2 && fabs((enin - enout) / (enin + enout)) > 1.e-4) errbits |= UW_ERRBIT_ENTHALPY;
    return qsp;
}

}  // namespace

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
#define UW_MODE_ALL 0
#define UW_MODE_TRIGGER 1
#define UW_MODE_LIST 2
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
__device__ __forceinline__ void uw_column(const UwArgs& A, const double* __restrict__ tbl, const int i_in,
                                          const bool active, int* __restrict__ wl, int* __restrict__ wl_count,
                                          const UwTangent& T)
{
    const int i = (MODE == UW_MODE_RESUME && active) ? A.hand->col[i_in] : i_in;
#define CONDEN(...) (FAST ? conden_fast(__VA_ARGS__) : conden(__VA_ARGS__))
    bool cand = false;
    // lanes of this warp that run a column; UW_SYNC() joins them where every one of them arrives
    const unsigned live = __ballot_sync(0xffffffffu, active);
#define UW_SYNC() __syncwarp(live)
    if (active) {

    const int mix = A.mix, mkx = A.mkx, ncnst = A.ncnst;
    const Tl dt = A.dt;
    const Tl xlv = c.xlv, xls = c.xls, cp = c.cp, zvir = c.zvir, r = c.r, g = c.g, p00 = c.p00,
                 rovcp = c.rovcp, rpen = Tl(c.rpen, T.drpen);
    const Tl rle = Tl(c.rle, T.drle), rkm = Tl(c.rkm, T.drkm), rkfre = 1.0, rmaxfrac = 0.10, mumin1 = 0.906, rbuoy = 1.0,
                 rdrag = 1.0, epsvarw = 5.e-4, PGFc = 0.7, criqc = Tl(c.criqc, T.dcriqc), frc_rasn = 1.0, kevp = 2.e-6;
    const int ixnumliq = c.ixnumliq, ixnumice = c.ixnumice;

    // Row of level k in the caller's arrays: bottom-up (compute_uwshcu) or CAM's top-down order
    // (compute_uwshcu_inv, uwshcu.F90:380-469, where interface k and layer k both sit at row mkx-k).
    const int inv = A.inv;
#define RI(k) (inv ? (mkx - (k)) : (k))
#define RL(k) (inv ? (mkx - (k)) : ((k) - 1))
#define GI(a, k) __ldg(&A.a[(size_t)RI(k) * mix + i])
#define GL(a, k) __ldg(&A.a[(size_t)RL(k) * mix + i])
#define GT(m, k) __ldg(&A.tr0[((size_t)((m) - 1) * mkx + RL(k)) * mix + i])
#define OI(a, k) A.a[(size_t)RI(k) * mix + i]
#define OL(a, k) A.a[(size_t)RL(k) * mix + i]
#define OT(m, k) A.trten[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]
#define TOI(a, k) T.a[(size_t)RI(k) * mix + i]
#define TOL(a, k) T.a[(size_t)RL(k) * mix + i]
#define TOT(m, k) T.trten[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]
#define SEEDL(a, da, k) Tl(GL(a, k), T.da ? __ldg(&T.da[(size_t)RL(k) * mix + i]) : 0.0)
#define SEEDI(a, da, k) Tl(GI(a, k), T.da ? __ldg(&T.da[(size_t)RI(k) * mix + i]) : 0.0)
#define CNT(x) (inv ? (Tl)(mkx + 1) - (x) : (x))
#define DLV(j, k) A.diag_level[((size_t)(j) * (mkx + 1) + (k)) * mix + i]
// per-level diagnostics of the current state, levels bottom-up in both level orders
// (uwshcu.F90:1945-1990 and :4383-4433)
#define PUT_DIAG_LEVEL()                                                                                  \
    if (A.diag_level) {                                                                                   \
        for (int k = 0; k <= mkx; k++) {                                                                  \
            DLV(UW_DL_UFRC, k) = tl_val(ufrc[k]);                                                                 \
            DLV(UW_DL_QTU, k) = tl_val(qtu[k]);                                                                   \
            DLV(UW_DL_THLU, k) = tl_val(thlu[k]);                                                                 \
            DLV(UW_DL_THVU, k) = tl_val(thvu[k]);                                                                 \
            DLV(UW_DL_UU, k) = tl_val(uu[k]);                                                                     \
            DLV(UW_DL_VU, k) = tl_val(vu[k]);                                                                     \
            DLV(UW_DL_UEMF, k) = tl_val(UEMF(k));                                                                 \
            DLV(UW_DL_FLXRAIN, k) = tl_val(flxrain[k]);                                                           \
            DLV(UW_DL_FLXSNOW, k) = tl_val(flxsnow[k]);                                                           \
        }                                                                                                 \
        for (int j = UW_DL_FER; j < UW_NDL; j++) DLV(j, 0) = tl_val(0.0);                                         \
        for (int k = 1; k <= mkx; k++) {                                                                  \
            DLV(UW_DL_FER, k) = tl_val(fer[k]);                                                                   \
            DLV(UW_DL_FDR, k) = tl_val(fdr[k]);                                                                   \
            DLV(UW_DL_DWTEN, k) = tl_val(dwten[k]);                                                               \
            DLV(UW_DL_DITEN, k) = tl_val(diten[k]);                                                               \
        }                                                                                                 \
    }

    // ---- thread-private profiles ---------------------------------------------------------------
    Tl ps0[KP], p0[KP], dp0[KP], zs0[KP], exn0[KP], exns0[KP];
    Tl qv0[KP], ql0[KP], qi0[KP], t0[KP], s0[KP], qt0[KP], thl0[KP];
    Tl ssthl0[KP], ssqt0[KP], ssu0[KP], ssv0[KP], sstr0[NC][KP];
    Tl thv0bot[KP], thv0top[KP], thvl0bot[KP], thvl0top[KP];
    Tl thv0bot_o[KP], thv0top_o[KP], thvl0bot_o[KP], thvl0top_o[KP];
    Tl umf[KP], emf[KP], thlu[KP], qtu[KP], uu[KP], vu[KP], thvu[KP], wu[KP], ufrc[KP], rei[KP];
    Tl fer[KP], fdr[KP], dwten[KP], diten[KP], tru[NC][KP];
    Tl thlu_emf[KP], qtu_emf[KP], uu_emf[KP], vu_emf[KP], tru_emf[NC][KP];
    Tl slflx[KP], qtflx[KP], uflx[KP], vflx[KP], trflx[NC][KP], xflx[KP];
    Tl qlten_sink[KP], qiten_sink[KP], nlten_sink[KP], niten_sink[KP];
    Tl uten[KP], vten[KP], uf[KP], vf[KP], qrten[KP], qsten[KP], slten[KP], qtten[KP];
    Tl qlten[KP], qiten[KP], qvten[KP], sten[KP], qc[KP], qc_l[KP], qc_i[KP], evapc[KP];
    Tl flxrain[KP], flxsnow[KP], cufrc[KP], qcu[KP], qlu[KP], qiu[KP], trten[NC][KP];
    Tl qw0[KP], trflx_d[KP], trflx_u[KP];
    Tl trsrc[NC], tre[NC];

    unsigned int errbits = 0;
    int xflags = 0, lflags = 0;
    bool id_exit = false;
    // stop: the column leaves the scheme (the Fortran's `go to 333`); every later section skips.
    bool stop = false;
    int kinv = 0, klcl = 0, klfc = 0, krel = 0, kbup = 0, kpen = 0;
    int kinv_s = 0, klcl_s = 0, klfc_s = 0, krel_s = 0, kbup_s = 0, kpen_s = 0;
    Tl cin = 0, cinlcl = 0, plcl = 0, plfc = 0, prel = 0, exlcl = 1.0, exprel = 1.0, tkeavg = 0,
           thvlmin = 0, qtsrc = 0, thlsrc = 0, thvlsrc = 0, usrc = 0, vsrc = 0, thv0lcl = 0, thv0rel = 0;
    Tl cin_i = 0, cinlcl_i = 0, ke = 0, kinv_o_d = 0;
    int kinv_o = 0, klcl_o = 0, klfc_o = 0;
    Tl plcl_o = 0, plfc_o = 0, tkeavg_o = 0, thvlmin_o = 0, qtsrc_o = 0, thvlsrc_o = 0, thlsrc_o = 0,
           usrc_o = 0, vsrc_o = 0, thv0lcl_o = 0, trsrc_o[NC];
    Tl cin_s = -1.0, cinlcl_s = -1.0, plcl_s = 0, plfc_s = 0, pinv_s = 0, pbup_s = 0, ppen_s = 0,
           tkeavg_s = 0;
    Tl cbmf = 0, wlcl = 0, ufrclcl = 0, ppen = 0, precip = 0, snow = 0, rliq = 0, cush, cnt, cnb;
    Tl thlu_top = 0, qtu_top = 0, exntop = 1.0, drage = 0, bogbot = 0, bogtop = 0, rho0j = 0,
           wtwb = 0, wtw = 0, xs1 = 0, xs2 = 0, xc1 = 0, xc2 = 0;
    Tl thj = 0, qvj = 0, qlj = 0, qij = 0;
    Tl rainflx = 0, snowflx = 0;
    (void)kinv_o_d;
    const Tl pblh = Tl(__ldg(&A.pblh[i]), T.dpblh ? __ldg(&T.dpblh[i]) : 0.0);
    Tl tscaleh_r = 0.0;   // UW_MODE_RESUME: tscaleh of the iteration handed over
    bool handed = false;      // UW_MODE_LIST1: the column continues in UW_MODE_RESUME

    if constexpr (MODE != UW_MODE_RESUME) {   // uniform

    // ---- output initialisation (uwshcu.F90:1087-1124) ------------------------------------------
    if (MODE != UW_MODE_TRIGGER) {
    for (int k = 0; k <= mkx; k++) {
        { const Tl v_ = (0.0); OI(umf, k) = tl_val(v_); TOI(umf, k) = tl_der(v_); }
        { const Tl v_ = (0.0); OI(slflx, k) = tl_val(v_); TOI(slflx, k) = tl_der(v_); }
        { const Tl v_ = (0.0); OI(qtflx, k) = tl_val(v_); TOI(qtflx, k) = tl_der(v_); }
        { const Tl v_ = (0.0); OI(flxprc1, k) = tl_val(v_); TOI(flxprc1, k) = tl_der(v_); }
        { const Tl v_ = (0.0); OI(flxsnow1, k) = tl_val(v_); TOI(flxsnow1, k) = tl_der(v_); }
        { const Tl v_ = (0.0); OI(wu, k) = tl_val(v_); TOI(wu, k) = tl_der(v_); }
    }
    for (int k = 1; k <= mkx; k++) {
        { const Tl v_ = (0.0); OL(qvten, k) = tl_val(v_); TOL(qvten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qlten, k) = tl_val(v_); TOL(qlten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qiten, k) = tl_val(v_); TOL(qiten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(sten, k) = tl_val(v_); TOL(sten, k) = tl_der(v_); }
        { const Tl v_ = (0.0); OL(uten, k) = tl_val(v_); TOL(uten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(vten, k) = tl_val(v_); TOL(vten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qrten, k) = tl_val(v_); TOL(qrten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qsten, k) = tl_val(v_); TOL(qsten, k) = tl_der(v_); }
        { const Tl v_ = (0.0); OL(evapc, k) = tl_val(v_); TOL(evapc, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(cufrc, k) = tl_val(v_); TOL(cufrc, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qcu, k) = tl_val(v_); TOL(qcu, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qlu, k) = tl_val(v_); TOL(qlu, k) = tl_der(v_); }
        { const Tl v_ = (0.0); OL(qiu, k) = tl_val(v_); TOL(qiu, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qc, k) = tl_val(v_); TOL(qc, k) = tl_der(v_); }
        for (int m = 1; m <= ncnst; m++) { const Tl v_ = (0.0); OT(m, k) = tl_val(v_); TOT(m, k) = tl_der(v_); }
    }
    { const Tl v_ = (0.0); A.precip[i] = tl_val(v_); T.precip[i] = tl_der(v_); }
    { const Tl v_ = (0.0); A.snow[i] = tl_val(v_); T.snow[i] = tl_der(v_); }
    { const Tl v_ = (0.0); A.cbmf[i] = tl_val(v_); T.cbmf[i] = tl_der(v_); }
    { const Tl v_ = (0.0); A.rliq[i] = tl_val(v_); T.rliq[i] = tl_der(v_); }
    A.cnt[i] = tl_val(CNT((Tl)mkx));
    A.cnb[i] = tl_val(CNT(0.0));
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
        exns0[k] = uw_pow(ps0[k] / p00, rovcp);
    }
    for (int k = 1; k <= mkx; k++) {
        p0[k] = GL(p0, k);
        dp0[k] = GL(dp0, k);
        qv0[k] = SEEDL(qv0, dqv0, k);
        ql0[k] = GL(ql0, k);
        qi0[k] = GL(qi0, k);
        t0[k] = SEEDL(t0, dt0, k);
        s0[k] = GL(s0, k);
        nonfinite |= !uw_isfinite(p0[k]) || !uw_isfinite(dp0[k]) || !uw_isfinite(qv0[k]) || !uw_isfinite(ql0[k]) ||
                     !uw_isfinite(qi0[k]) || !uw_isfinite(t0[k]) || !uw_isfinite(s0[k]) || !uw_isfinite(GL(z0, k));
        exn0[k] = uw_pow(p0[k] / p00, rovcp);
        qt0[k] = (qv0[k] + ql0[k] + qi0[k]);
        thl0[k] = (t0[k] - xlv * ql0[k] / cp - xls * qi0[k] / cp) / exn0[k];
        qw0[k] = nonfinite ? 0.0 : findsp_point(qv0[k], t0[k], p0[k], errbits, tbl);
    }
    cush = A.cush[i];
    {
        Tl tmpf[KP];
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
        Tl thl0bot = thl0[k] + ssthl0[k] * (ps0[k - 1] - p0[k]);
        Tl qt0bot = qt0[k] + ssqt0[k] * (ps0[k - 1] - p0[k]);
        if (CONDEN(ps0[k - 1], exns0[k - 1], thl0bot, qt0bot, thj, qvj, qlj, qij, tbl)) {
            xflags |= UW_X_CONDEN;
            id_exit = true;
            stop = true;
            break;
        }
        thv0bot[k] = thj * (1.0 + zvir * qvj - qlj - qij);
        thvl0bot[k] = thl0bot * (1.0 + zvir * qt0bot);
        Tl thl0top = thl0[k] + ssthl0[k] * (ps0[k] - p0[k]);
        Tl qt0top = qt0[k] + ssqt0[k] * (ps0[k] - p0[k]);
        if (CONDEN(ps0[k], exns0[k], thl0top, qt0top, thj, qvj, qlj, qij, tbl)) {
            xflags |= UW_X_CONDEN;
            id_exit = true;
            stop = true;
            break;
        }
        thv0top[k] = thj * (1.0 + zvir * qvj - qlj - qij);
        thvl0top[k] = thl0top * (1.0 + zvir * qt0top);
        thv0bot_o[k] = thv0bot[k];
        thv0top_o[k] = thv0top[k];
        thvl0bot_o[k] = thvl0bot[k];
        thvl0top_o[k] = thvl0top[k];
    }
    if (!stop) {
    // per-column initialisation (:1333-1408)
    for (int k = 0; k <= mkx; k++) {
        umf[k] = 0.0; emf[k] = 0.0; slflx[k] = 0.0; qtflx[k] = 0.0; uflx[k] = 0.0; vflx[k] = 0.0;
        ufrc[k] = 0.0; thlu[k] = 0.0; qtu[k] = 0.0; uu[k] = 0.0; vu[k] = 0.0; wu[k] = 0.0;
        thvu[k] = 0.0; thlu_emf[k] = 0.0; qtu_emf[k] = 0.0; uu_emf[k] = 0.0; vu_emf[k] = 0.0;
        for (int m = 0; m < ncnst; m++) {
            trflx[m][k] = 0.0;
            tru[m][k] = 0.0;
            tru_emf[m][k] = 0.0;
        }
    }
    for (int k = 1; k <= mkx; k++) {
        qvten[k] = 0.0; qlten[k] = 0.0; qiten[k] = 0.0; sten[k] = 0.0; uten[k] = 0.0; vten[k] = 0.0;
        qrten[k] = 0.0; qsten[k] = 0.0; dwten[k] = 0.0; diten[k] = 0.0; evapc[k] = 0.0;
        cufrc[k] = 0.0; qcu[k] = 0.0; qlu[k] = 0.0; qiu[k] = 0.0; fer[k] = 0.0; fdr[k] = 0.0;
        qc[k] = 0.0; qc_l[k] = 0.0; qc_i[k] = 0.0; qtten[k] = 0.0; slten[k] = 0.0;
        qlten_sink[k] = 0.0; qiten_sink[k] = 0.0; nlten_sink[k] = 0.0; niten_sink[k] = 0.0;
        rei[k] = 0.0; uf[k] = 0.0; vf[k] = 0.0;
        for (int m = 0; m < ncnst; m++) trten[m][k] = 0.0;
    }
    cnt = (Tl)mkx;
    cnb = 0.0;
    }
    } else {   // uniform
        // the state UW_MODE_LIST1 stored at the implicit-CIN branch of iteration 2 (uw_state.cuh),
        // and the arrays that the set-up and that branch's restore build from the inputs, rebuilt
        // with the same operations
        for (int k = 0; k <= mkx; k++) {
            ps0[k] = GI(ps0, k);
            zs0[k] = GI(zs0, k);
        }
        for (int k = 1; k <= mkx; k++) {
            p0[k] = GL(p0, k);
            dp0[k] = GL(dp0, k);
        }
        {
            Tl tmpf[KP];
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
            qv0[k] = SEEDL(qv0, dqv0, k);
            ql0[k] = GL(ql0, k);
            qi0[k] = GL(qi0, k);
            t0[k] = SEEDL(t0, dt0, k);
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
            umf[k] = 0.0; emf[k] = 0.0; slflx[k] = 0.0; qtflx[k] = 0.0; uflx[k] = 0.0;
            vflx[k] = 0.0; ufrc[k] = 0.0; thlu[k] = 0.0; qtu[k] = 0.0; uu[k] = 0.0;
            vu[k] = 0.0; wu[k] = 0.0; thvu[k] = 0.0; thlu_emf[k] = 0.0; qtu_emf[k] = 0.0;
            uu_emf[k] = 0.0; vu_emf[k] = 0.0;
            for (int m = 0; m < ncnst; m++) {
                trflx[m][k] = 0.0;
                tru[m][k] = 0.0;
                tru_emf[m][k] = 0.0;
            }
        }
        for (int k = 1; k <= mkx; k++) {
            qvten[k] = 0.0; qlten[k] = 0.0; qiten[k] = 0.0; sten[k] = 0.0; uten[k] = 0.0;
            vten[k] = 0.0; qrten[k] = 0.0; qsten[k] = 0.0; dwten[k] = 0.0; diten[k] = 0.0;
            evapc[k] = 0.0; cufrc[k] = 0.0; qcu[k] = 0.0; qlu[k] = 0.0; qiu[k] = 0.0;
            fer[k] = 0.0; fdr[k] = 0.0; qc[k] = 0.0; qc_l[k] = 0.0; qc_i[k] = 0.0;
            qtten[k] = 0.0; slten[k] = 0.0;
            for (int m = 0; m < ncnst; m++) trten[m][k] = 0.0;
        }
    }

    UW_SYNC();

    // ---- implicit-CIN loop (uwshcu.F90:1421-4331) --------------------------------------------
    // Lockstep skeleton.  Every lane of the warp runs the same iterations of this loop and of every
    // level loop inside it: a column's own level range and its exits are per-lane predicates.  Each
    // section is `if (!stop) do { ... } while (0);`, so an exit (`stop = true; break;`) skips the
    // rest of the section and every later one, and the lanes meet again at UW_SYNC() between
    // sections.  (Lanes that leave a loop at different iterations otherwise run apart for the rest
    // of the column: the worklist kernel ran with 1.9 of 32 lanes active.)  Loops marked `uniform`
    // have the same trip count on every live lane; UW_SYNC() appears only directly inside them.
    for (int iter = (MODE == UW_MODE_RESUME ? 2 : 1); iter <= (MODE == UW_MODE_TRIGGER ? 1 : 2); iter++) {   // uniform
        Tl tscaleh = tscaleh_r;
        if constexpr (MODE != UW_MODE_RESUME) {   // uniform
        if (!stop) do {
        tscaleh = cush;
        cush = -1.0;

        // kinv (:1455-1468): the first interface from the top whose layer brackets pblh + 5
        kinv = 1;
        {
            bool found = false;
            for (int k = mkx - 1; k >= 1; k--) {
                if (!found && (pblh + 5.0 - zs0[k]) * (pblh + 5.0 - zs0[k + 1]) < 0.0) {
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
            Tl dpsum = 0.0;
            tkeavg = 0.0;
            thvlmin = 1000.0;
            for (int k = 0; k <= mkx; k++) {
                if (k > kinv - 1) continue;
                Tl dpi;
                if (k == 0) dpi = ps0[0] - p0[1];
                else if (k == (kinv - 1)) dpi = p0[kinv - 1] - ps0[kinv - 1];
                else dpi = p0[k] - p0[k + 1];
                dpsum = dpsum + dpi;
                tkeavg = tkeavg + dpi * SEEDI(tke, dtke, k);
                if (k != 0) thvlmin = MN(thvlmin, MN(thvl0bot[k], thvl0top[k]));
            }
            tkeavg = tkeavg / dpsum;
        }
        // source air (:1509-1516)
        qtsrc = qt0[1];
        thvlsrc = thvlmin;
        thlsrc = thvlsrc / (1.0 + zvir * qtsrc);
        usrc = GL(u0, kinv - 1) + ssu0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        vsrc = GL(v0, kinv - 1) + ssv0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        for (int m = 1; m <= ncnst; m++) trsrc[m - 1] = GT(m, 1);
        } while (0);
        UW_SYNC();
        // LCL (:1533-1549)
        if (!stop) do {
        plcl = qsinvert(qtsrc, thlsrc, ps0[0], exns0[0], tbl);
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
        if (plcl < 30000.0) {
            xflags |= UW_X_KLCLMKX;
            id_exit = true;
            stop = true;
            break;
        }
        exlcl = exnf(plcl);
        {
            Tl thl0lcl = thl0[klcl] + ssthl0[klcl] * (plcl - p0[klcl]);
            Tl qt0lcl = qt0[klcl] + ssqt0[klcl] * (plcl - p0[klcl]);
            if (CONDEN(plcl, exlcl, thl0lcl, qt0lcl, thj, qvj, qlj, qij, tbl)) {
                xflags |= UW_X_CONDEN;
                id_exit = true;
                stop = true;
            break;
            }
            thv0lcl = thj * (1.0 + zvir * qvj - qlj - qij);
        }
        } while (0);
        UW_SYNC();
        // CIN (:1592-1685).  One loop over k = kinv .. mkx-1 serves both cases of the Fortran (LCL at
        // or above kinv, LCL below kinv), with one conden call at ps0(k) per level for every lane.
        // When the LCL is below kinv the Fortran also calls conden at ps0(k-1) with the same source
        // air; above the first level that repeats the previous level's call bit for bit, so only
        // the first level makes it here.
        if (!stop) {
            cin = 0.0;
            cinlcl = 0.0;
            plfc = 0.0;
            klfc = mkx;
        }
        {
            const bool lcl_above = (klcl >= kinv);
            Tl thvubot = 0.0, thvutop = 0.0;
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
                        if (CONDEN(ps0[k - 1], exns0[k - 1], thlsrc, qtsrc, thj, qvj, qlj, qij, tbl)) {
                            xflags |= UW_X_CONDEN;
                            id_exit = true;
                            stop = true;
                            break;
                        }
                        thvutop = thj * (1.0 + zvir * qvj - qlj - qij);
                    }
                    const bool atlcl = lcl_above && k == klcl;
                    if (atlcl) {
                        thvubot = thvlsrc;
                        thvutop = thvlsrc;
                        cin = cin + single_cin(ps0[k - 1], exns0[k - 1], thv0bot[k], plcl, exlcl, thv0lcl, thvubot, thvutop);
                        if (cin < 0.0) lflags |= UW_L_CINLCL;
                        cinlcl = MX(cin, 0.0);
                        cin = cinlcl;
                        thvubot = thvlsrc;
                    } else {
                        thvubot = thvutop;
                    }
                    if (CONDEN(ps0[k], exns0[k], thlsrc, qtsrc, thj, qvj, qlj, qij, tbl)) {
                        xflags |= UW_X_CONDEN;
                        id_exit = true;
                        stop = true;
                        break;
                    }
                    thvutop = thj * (1.0 + zvir * qvj - qlj - qij);
                    getbuoy(atlcl ? plcl : ps0[k - 1], atlcl ? exlcl : exns0[k - 1], atlcl ? thv0lcl : thv0bot[k],
                            ps0[k], exns0[k], thv0top[k], thvubot, thvutop, plfc, cin);
                    if (plfc > 0.0) {
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
        if (cin < 0.0) lflags |= UW_L_CIN;
        cin = MX(0.0, cin);
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
            Tl del_CIN = cin - cin_i;
            if (del_CIN > 0.0) {
                // implicit CIN: restore the iteration-1 state (:1759-1889)
                Tl alpha = compute_alpha(del_CIN, ke);
                cin = cin_i + alpha * del_CIN;
                cinlcl = cinlcl_i;
                kinv = kinv_o; klcl = klcl_o; klfc = klfc_o; plcl = plcl_o; plfc = plfc_o;
                tkeavg = tkeavg_o; thvlmin = thvlmin_o; qtsrc = qtsrc_o; thvlsrc = thvlsrc_o;
                thlsrc = thlsrc_o; usrc = usrc_o; vsrc = vsrc_o; thv0lcl = thv0lcl_o;
                for (int m = 0; m < ncnst; m++) trsrc[m] = trsrc_o[m];
                exlcl = exnf(plcl);
                for (int k = 1; k <= mkx; k++) {
                    qv0[k] = SEEDL(qv0, dqv0, k);
                    ql0[k] = GL(ql0, k);
                    qi0[k] = GL(qi0, k);
                    t0[k] = SEEDL(t0, dt0, k);
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
                    umf[k] = 0.0; emf[k] = 0.0; slflx[k] = 0.0; qtflx[k] = 0.0; uflx[k] = 0.0;
                    vflx[k] = 0.0; ufrc[k] = 0.0; thlu[k] = 0.0; qtu[k] = 0.0; uu[k] = 0.0;
                    vu[k] = 0.0; wu[k] = 0.0; thvu[k] = 0.0; thlu_emf[k] = 0.0; qtu_emf[k] = 0.0;
                    uu_emf[k] = 0.0; vu_emf[k] = 0.0;
                    for (int m = 0; m < ncnst; m++) {
                        trflx[m][k] = 0.0;
                        tru[m][k] = 0.0;
                        tru_emf[m][k] = 0.0;
                    }
                }
                for (int k = 1; k <= mkx; k++) {
                    qvten[k] = 0.0; qlten[k] = 0.0; qiten[k] = 0.0; sten[k] = 0.0; uten[k] = 0.0;
                    vten[k] = 0.0; qrten[k] = 0.0; qsten[k] = 0.0; dwten[k] = 0.0; diten[k] = 0.0;
                    evapc[k] = 0.0; cufrc[k] = 0.0; qcu[k] = 0.0; qlu[k] = 0.0; qiu[k] = 0.0;
                    fer[k] = 0.0; fdr[k] = 0.0; qc[k] = 0.0; qc_l[k] = 0.0; qc_i[k] = 0.0;
                    qtten[k] = 0.0; slten[k] = 0.0;
                    for (int m = 0; m < ncnst; m++) trten[m][k] = 0.0;
                }
                precip = 0.0; snow = 0.0; rliq = 0.0; cbmf = 0.0;
                cnt = (Tl)mkx; cnb = 0.0; ufrclcl = 0.0; wlcl = 0.0;
            } else {
                // explicit CIN: the iteration-1 outputs already sit in the output slots (:1891-2011);
                // flxprc1/flxsnow1 keep their initial zeros on this path, wu_out gets wu.
                lflags |= UW_L_DELCIN;
                for (int k = 0; k <= mkx; k++) { const Tl v_ = (wu[k]); OI(wu, k) = tl_val(v_); TOI(wu, k) = tl_der(v_); }
                if (A.diag_real) {
                    A.diag_real[UW_DR_CIN * (size_t)mix + i] = tl_val(cin_s);
                    A.diag_real[UW_DR_CINLCL * (size_t)mix + i] = tl_val(cinlcl_s);
                    A.diag_real[UW_DR_PLCL * (size_t)mix + i] = tl_val(plcl_s);
                    A.diag_real[UW_DR_PLFC * (size_t)mix + i] = tl_val(plfc_s);
                    A.diag_real[UW_DR_PINV * (size_t)mix + i] = tl_val(pinv_s);
                    A.diag_real[UW_DR_PBUP * (size_t)mix + i] = tl_val(pbup_s);
                    A.diag_real[UW_DR_PPEN * (size_t)mix + i] = tl_val(ppen_s);
                    A.diag_real[UW_DR_TKEAVG * (size_t)mix + i] = tl_val(tkeavg_s);
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
            Tl wcrit = sqrt(2.0 * cin * rbuoy);
            // compute_zwshcu computes rho0inv first and lowers wcrit by the large-scale ascent at
            // the PBL top (zwshcu.F90:2277, 2295-2303); the same value of rho0inv for both schemes
            Tl rho0inv = ps0[kinv - 1] / (r * thv0top[kinv - 1] * exns0[kinv - 1]);
            Tl sigmaw = sqrt(rkfre * tkeavg + epsvarw);
            if constexpr (ZW) {
                if (c.zw_lf) {
                    const Tl tmp1 = MN(MX(-GL(omega, kinv - 1), 0.0), 3.0);
                    wcrit = wcrit - tmp1 / rho0inv / 9.8;
                    wcrit = MX(wcrit, 0.0);
                }
                wcrit = wcrit * c.zw_fwcrit;
            }
            Tl mu = wcrit / sigmaw / 1.4142;
            if (mu >= 3.0) {
                id_exit = true;
                stop = true;
            break;
            }
            cbmf = (rho0inv * sigmaw / 2.5066) * uw_exp(-(mu * mu));
            Tl cbmflimit = 0.9 * dp0[kinv - 1] / g / dt;
            Tl mumin0 = 0.0;
            if (cbmf > cbmflimit) mumin0 = sqrt(-uw_log(2.5066 * cbmflimit / rho0inv / sigmaw));
            mu = MX(MX(mu, mumin0), mumin1);
            Tl mulcl = sqrt(2.0 * cinlcl * rbuoy) / 1.4142 / sigmaw;
            Tl ta = uw_exp(-(mu * mu)) / 2.5066, te = uw_erfc(mu);
            Tl mulclstar = sqrt(MX(0.0, 2.0 * (ta * ta) * (1.0 / (te * te) - 0.25 / (rmaxfrac * rmaxfrac))));
            if (mulcl > 1.e-8 && mulcl > mulclstar) {
                Tl mumin2 = compute_mumin2(mulcl, rmaxfrac, mu);
                if (mu > mumin2) errbits |= UW_ERRBIT_MU;
                mu = MX(mu, mumin2);
                if (mu == mumin2) lflags |= UW_L_UFRC;
            }
            if (mu == mumin0) lflags |= UW_L_CBMF;
            if (mu == mumin1) lflags |= UW_L_UFRC;
            cbmf = (rho0inv * sigmaw / 2.5066) * uw_exp(-(mu * mu));
            Tl winv = sigmaw * (2.0 / 2.5066) * uw_exp(-(mu * mu)) / uw_erfc(mu);
            wtw = winv * winv - 2.0 * cinlcl * rbuoy;
            if (wtw <= 0.0) {
                xflags |= UW_X_WTW;
                id_exit = true;
                stop = true;
            break;
            }
            wlcl = sqrt(wtw);
            ufrclcl = cbmf / wlcl / rho0inv;
            if (ufrclcl <= 0.0001) {
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
        emf[krel - 1] = 0.0;
        umf[krel - 1] = cbmf;
        wu[krel - 1] = wlcl;
        thlu[krel - 1] = thlsrc;
        qtu[krel - 1] = qtsrc;
        if (CONDEN(prel, exprel, thlsrc, qtsrc, thj, qvj, qlj, qij, tbl)) {
            xflags |= UW_X_CONDEN;
            id_exit = true;
            stop = true;
            break;
        }
        thvu[krel - 1] = thj * (1.0 + zvir * qvj - qlj - qij);
        {
            Tl uplus = 0.0, vplus = 0.0;
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
            Tl scaleh = tscaleh;
            if (tscaleh < 0.0) scaleh = 1000.0;
            // ---- buoyancy-sorting updraft, iter_scaleh loop (:2306-2952) ----------------------
            for (int iter_scaleh = 1; iter_scaleh <= 3; iter_scaleh++) {   // uniform
                Tl pe = 0.0, dpe = 0.0, exne = 1.0, thvebot = 0.0, thle = 0.0, qte = 0.0, ue = 0.0, ve = 0.0;
                if (!stop) {
                    kbup = krel;
                    kpen = krel;
                    wtw = wlcl * wlcl;
                    pe = 0.5 * (prel + ps0[krel]);
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
                    Tl thlue = thlu[km1];
                    Tl qtue = qtu[km1];
                    Tl wue = wu[km1];
                    wtwb = wtw;
                    bool xdone = false;
                    // environment at the layer midpoint: the same in both iter_xc passes, so the
                    // second pass reuses the first one's conden and qsat results (same bits)
                    Tl thv0j = 0.0, excess0 = 0.0;
                    for (int iter_xc = 1; iter_xc <= 2; iter_xc++) {
                        if (!xdone && !stop) do {
                        wtw = wu[km1] * wu[km1];
                        if (iter_xc == 1) {
                            if (CONDEN(pe, exne, thle, qte, thj, qvj, qlj, qij, tbl)) {
                                xflags |= UW_X_CONDEN;
                                id_exit = true;
                                stop = true;
                                break;
                            }
                            thv0j = thj * (1.0 + zvir * qvj - qlj - qij);
                            excess0 = qte - qsat_qs(thle * exne, pe, tbl);
                        }
                        rho0j = pe / (r * thv0j * exne);
                        if (CONDEN(pe, exne, thlue, qtue, thj, qvj, qlj, qij, tbl)) {
                            xflags |= UW_X_CONDEN;
                            id_exit = true;
                            stop = true;
            break;
                        }
                        // condensate above criqc leaves the updraft; without it the Fortran's
                        // second conden call repeats the first one's arguments and results
                        if ((qlj + qij) > criqc) {
                            Tl exql = ((qlj + qij) - criqc) * qlj / (qlj + qij);
                            Tl exqi = ((qlj + qij) - criqc) * qij / (qlj + qij);
                            qtue = qtue - exql - exqi;
                            thlue = thlue + (xlv / cp / exne) * exql + (xls / cp / exne) * exqi;
                            if (CONDEN(pe, exne, thlue, qtue, thj, qvj, qlj, qij, tbl)) {
                                xflags |= UW_X_CONDEN;
                                id_exit = true;
                                stop = true;
                                break;
                            }
                        }
                        Tl thvj = thj * (1.0 + zvir * qvj - qlj - qij);
                        Tl excessu = qtue - qsat_qs(thlue * exne, pe, tbl);
                        Tl cridis = rle * scaleh;
                        Tl xc;
                        if ((excessu <= 0.0 && excess0 <= 0.0) || (excessu >= 0.0 && excess0 >= 0.0)) {
                            xc = MN(1.0, MX(0.0, 1.0 - 2.0 * rbuoy * g * cridis / (wue * wue) * (1.0 - thvj / thv0j)));
                        } else {
                            Tl xsat = excessu / (excessu - excess0);
                            Tl thlxsat = thlue + xsat * (thle - thlue);
                            Tl qtxsat = qtue + xsat * (qte - qtue);
                            if (CONDEN(pe, exne, thlxsat, qtxsat, thj, qvj, qlj, qij, tbl)) {
                                xflags |= UW_X_CONDEN;
                                id_exit = true;
                                stop = true;
            break;
                            }
                            Tl thvxsat = thj * (1.0 + zvir * qvj - qlj - qij);
                            Tl x_cu = 0.0, x_en = 0.0;
                            for (int kk = 1; kk <= 2; kk++) {
                                Tl thv_x0, thv_x1;
                                if (kk == 1) {
                                    thv_x0 = thvj;
                                    thv_x1 = (1.0 - 1.0 / xsat) * thvj + (1.0 / xsat) * thvxsat;
                                } else {
                                    thv_x1 = thv0j;
                                    thv_x0 = (xsat / (xsat - 1.0)) * thv0j + (1.0 / (1.0 - xsat)) * thvxsat;
                                }
                                Tl aquad = wue * wue;
                                Tl bquad = 2.0 * rbuoy * g * cridis * (thv_x1 - thv_x0) / thv0j - 2.0 * (wue * wue);
                                Tl cquad = 2.0 * rbuoy * g * cridis * (thv_x0 - thv0j) / thv0j + (wue * wue);
                                if (kk == 1) {
                                    if ((bquad * bquad - 4.0 * aquad * cquad) >= 0.0) {
                                        roots(aquad, bquad, cquad, xs1, xs2);
                                        x_cu = MN(1.0, MX(0.0, MN(xsat, MN(xs1, xs2))));
                                    } else {
                                        x_cu = xsat;
                                    }
                                } else {
                                    if ((bquad * bquad - 4.0 * aquad * cquad) >= 0.0) {
                                        roots(aquad, bquad, cquad, xs1, xs2);
                                        x_en = MN(1.0, MX(0.0, MX(xsat, MN(xs1, xs2))));
                                    } else {
                                        x_en = 1.0;
                                    }
                                }
                            }
                            if (x_cu == xsat) xc = MX(x_cu, x_en);
                            else xc = x_cu;
                        }
                        Tl ee2 = xc * xc;
                        Tl ud2 = 1.0 - 2.0 * xc + xc * xc;
                        rei[k] = (0.5 * rkm / GL(z0, k) / g / rho0j);
                        if (xc > 0.5) rei[k] = MN(rei[k], 0.9 * uw_log(dp0[k] / g / dt / umf[km1] + 1.0) / dpe / (2.0 * xc - 1.0));
                        fer[k] = rei[k] * ee2;
                        fdr[k] = rei[k] * ud2;
                        // compute_zwshcu's entrainment option (zwshcu.F90:2818-2844)
                        if (ZW && c.zw_ent) {
                            bogbot = rbuoy * (thvu[km1] / thvebot - 1.0) * g;
                            fer[k] = c.zw_ent0 * bogbot / MX(wue * wue, 1.0e-4);
                            Tl fer_min = 0.0;
                            if (bogbot > 1.e-4) fer_min = 1.e-4;
                            fer[k] = MN(MX(fer[k], fer_min), 3.0e-2);
                        }
                        umf[k] = umf[km1] * uw_exp(dpe * (fer[k] - fdr[k]));
                        emf[k] = 0.0;
                        if (fer[k] * dpe < 1.e-4) {
                            thlu[k] = thlu[km1] + (thle + ssthl0[k] * dpe / 2.0 - thlu[km1]) * fer[k] * dpe;
                            qtu[k] = qtu[km1] + (qte + ssqt0[k] * dpe / 2.0 - qtu[km1]) * fer[k] * dpe;
                            uu[k] = uu[km1] + (ue + ssu0[k] * dpe / 2.0 - uu[km1]) * fer[k] * dpe - PGFc * ssu0[k] * dpe;
                            vu[k] = vu[km1] + (ve + ssv0[k] * dpe / 2.0 - vu[km1]) * fer[k] * dpe - PGFc * ssv0[k] * dpe;
                            for (int m = 0; m < ncnst; m++)
                                tru[m][k] = tru[m][km1] + (tre[m] + sstr0[m][k] * dpe / 2.0 - tru[m][km1]) * fer[k] * dpe;
                        } else {
                            const Tl ef = uw_exp(-fer[k] * dpe);
                            thlu[k] = (thle + ssthl0[k] / fer[k] - ssthl0[k] * dpe / 2.0) -
                                      (thle + ssthl0[k] * dpe / 2.0 - thlu[km1] + ssthl0[k] / fer[k]) * ef;
                            qtu[k] = (qte + ssqt0[k] / fer[k] - ssqt0[k] * dpe / 2.0) -
                                     (qte + ssqt0[k] * dpe / 2.0 - qtu[km1] + ssqt0[k] / fer[k]) * ef;
                            uu[k] = (ue + (1.0 - PGFc) * ssu0[k] / fer[k] - ssu0[k] * dpe / 2.0) -
                                    (ue + ssu0[k] * dpe / 2.0 - uu[km1] + (1.0 - PGFc) * ssu0[k] / fer[k]) * ef;
                            vu[k] = (ve + (1.0 - PGFc) * ssv0[k] / fer[k] - ssv0[k] * dpe / 2.0) -
                                    (ve + ssv0[k] * dpe / 2.0 - vu[km1] + (1.0 - PGFc) * ssv0[k] / fer[k]) * ef;
                            for (int m = 0; m < ncnst; m++)
                                tru[m][k] = (tre[m] + sstr0[m][k] / fer[k] - sstr0[m][k] * dpe / 2.0) -
                                            (tre[m] + sstr0[m][k] * dpe / 2.0 - tru[m][km1] + sstr0[m][k] / fer[k]) * ef;
                        }
                        if (CONDEN(ps0[k], exns0[k], thlu[k], qtu[k], thj, qvj, qlj, qij, tbl)) {
                            xflags |= UW_X_CONDEN;
                            id_exit = true;
                            stop = true;
            break;
                        }
                        if ((qlj + qij) > criqc) {
                            Tl exql = ((qlj + qij) - criqc) * qlj / (qlj + qij);
                            Tl exqi = ((qlj + qij) - criqc) * qij / (qlj + qij);
                            qtu[k] = qtu[k] - exql - exqi;
                            thlu[k] = thlu[k] + (xlv / cp / exns0[k]) * exql + (xls / cp / exns0[k]) * exqi;
                            dwten[k] = exql;
                            diten[k] = exqi;
                            if (CONDEN(ps0[k], exns0[k], thlu[k], qtu[k], thj, qvj, qlj, qij, tbl)) {
                                xflags |= UW_X_CONDEN;
                                id_exit = true;
                                stop = true;
                                break;
                            }
                        } else {
                            // nothing removed: the Fortran's second conden call repeats the first
                            dwten[k] = 0.0;
                            diten[k] = 0.0;
                        }
                        thvu[k] = thj * (1.0 + zvir * qvj - qlj - qij);
                        bogbot = rbuoy * (thvu[km1] / thvebot - 1.0);
                        bogtop = rbuoy * (thvu[k] / thv0top[k] - 1.0);
                        Tl delbog = bogtop - bogbot;
                        drage = fer[k] * (1.0 + rdrag);
                        Tl expfac = uw_exp(-2.0 * drage * dpe);
                        wtwb = wtw;
                        if (drage * dpe > 1.e-3)
                            wtw = wtw * expfac + (delbog + (1.0 - expfac) * (bogbot + delbog / (-2.0 * drage * dpe))) / (rho0j * drage);
                        else
                            wtw = wtw + dpe * (bogbot + bogtop) / rho0j;
                        if (wtw > 0.0) {
                            thlue = 0.5 * (thlu[km1] + thlu[k]);
                            qtue = 0.5 * (qtu[km1] + qtu[k]);
                            wue = 0.5 * sqrt(MX(wtwb + wtw, 0.0));
                        } else {
                            xdone = true;   // go to 111
                        }
                        } while (0);
                    }
                    if (stop) break;
                    // (label 111, :2726-2793)
                    if (umf[k] == 0.0) wtw = -1.0;
                    if (bogtop > 0.0 && wtw > 0.0) kbup = k;
                    if (wtw <= 0.0) {
                        kpen = k;
                        ldone = true;
                        break;   // go to 45
                    }
                    wu[k] = sqrt(wtw);
                    if (wu[k] > 100.0) {
                        xflags |= UW_X_WU;
                        id_exit = true;
                        stop = true;
            break;
                    }
                    {
                        Tl rhos0j = ps0[k] / (r * 0.5 * (thv0bot[k + 1] + thv0top[k]) * exns0[k]);
                        ufrc[k] = umf[k] / (rhos0j * wu[k]);
                        if (ufrc[k] > rmaxfrac) {
                            lflags |= UW_L_UFRC;
                            ufrc[k] = rmaxfrac;
                            umf[k] = rmaxfrac * rhos0j * wu[k];
                            fdr[k] = fer[k] - uw_log(umf[k] / umf[km1]) / dpe;
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
                if (drage == 0.0) {
                    Tl aquad = (bogtop - bogbot) / (ps0[kpen] - ps0[kpen - 1]);
                    Tl bquad = 2.0 * bogbot;
                    Tl cquad = -(wu[kpen - 1] * wu[kpen - 1]) * rho0j;
                    int status = roots(aquad, bquad, cquad, xc1, xc2);
                    if (status == 0) {
                        if (xc1 <= 0.0 && xc2 <= 0.0) {
                            ppen = MX(xc1, xc2);
                            ppen = MN(0.0, MX(-dp0[kpen], ppen));
                        } else if (xc1 > 0.0 && xc2 > 0.0) {
                            ppen = -dp0[kpen];
                        } else {
                            ppen = MN(xc1, xc2);
                            ppen = MN(0.0, MX(-dp0[kpen], ppen));
                        }
                    } else {
                        ppen = -dp0[kpen];
                    }
                } else {
                    ppen = compute_ppen(wtwb, drage, bogbot, bogtop, rho0j, dp0[kpen]);
                }
                if (ppen == -dp0[kpen] || ppen == 0.0) lflags |= UW_L_PPEN;
                // condensate at the cumulus top (:2917-2942)
                if (fer[kpen] * (-ppen) < 1.e-4) {
                    thlu_top = thlu[kpen - 1] + (thl0[kpen] + ssthl0[kpen] * (-ppen) / 2.0 - thlu[kpen - 1]) * fer[kpen] * (-ppen);
                    qtu_top = qtu[kpen - 1] + (qt0[kpen] + ssqt0[kpen] * (-ppen) / 2.0 - qtu[kpen - 1]) * fer[kpen] * (-ppen);
                } else {
                    const Tl ef = uw_exp(-fer[kpen] * (-ppen));
                    thlu_top = (thl0[kpen] + ssthl0[kpen] / fer[kpen] - ssthl0[kpen] * (-ppen) / 2.0) -
                               (thl0[kpen] + ssthl0[kpen] * (-ppen) / 2.0 - thlu[kpen - 1] + ssthl0[kpen] / fer[kpen]) * ef;
                    qtu_top = (qt0[kpen] + ssqt0[kpen] / fer[kpen] - ssqt0[kpen] * (-ppen) / 2.0) -
                              (qt0[kpen] + ssqt0[kpen] * (-ppen) / 2.0 - qtu[kpen - 1] + ssqt0[kpen] / fer[kpen]) * ef;
                }
                exntop = uw_pow((ps0[kpen - 1] + ppen) / p00, rovcp);
                if (CONDEN(ps0[kpen - 1] + ppen, exntop, thlu_top, qtu_top, thj, qvj, qlj, qij, tbl)) {
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
                    dwten[kpen] = 0.0;
                    diten[kpen] = 0.0;
                }
                {
                    Tl rhos0j = ps0[kpen - 1] / (r * 0.5 * (thv0bot[kpen] + thv0top[kpen - 1]) * exns0[kpen - 1]);
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
            umf[k] = 0.0;
            emf[k] = 0.0;
            ufrc[k] = 0.0;
        }
        for (int k = 0; k <= mkx; k++) {
            if (k < kpen + 1) continue;
            dwten[k] = 0.0;
            diten[k] = 0.0;
            fer[k] = 0.0;
            fdr[k] = 0.0;
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
            Tl rhos0j = ps0[k] / (r * 0.5 * (thv0bot[k + 1] + thv0top[k]) * exns0[k]);
            if (k == kpen - 1) {
                if ((umf[k] * ppen * rei[kpen] * rpen) < -0.1 * rhos0j) lflags |= UW_L_EMF;
                if ((umf[k] * ppen * rei[kpen] * rpen) < -0.9 * dp0[kpen] / g / dt) lflags |= UW_L_EMF;
                emf[k] = MX(MX(umf[k] * ppen * rei[kpen] * rpen, -0.1 * rhos0j), -0.9 * dp0[kpen] / g / dt);
                thlu_emf[k] = thl0[kpen] + ssthl0[kpen] * (ps0[k] - p0[kpen]);
                qtu_emf[k] = qt0[kpen] + ssqt0[kpen] * (ps0[k] - p0[kpen]);
                uu_emf[k] = GL(u0, kpen) + ssu0[kpen] * (ps0[k] - p0[kpen]);
                vu_emf[k] = GL(v0, kpen) + ssv0[kpen] * (ps0[k] - p0[kpen]);
                for (int m = 0; m < ncnst; m++) tru_emf[m][k] = GT(m + 1, kpen) + sstr0[m][kpen] * (ps0[k] - p0[kpen]);
            } else {
                if ((emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen) < -0.1 * rhos0j) lflags |= UW_L_EMF;
                if ((emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen) < -0.9 * dp0[k + 1] / g / dt) lflags |= UW_L_EMF;
                emf[k] = MX(MX(emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen, -0.1 * rhos0j), -0.9 * dp0[k + 1] / g / dt);
                if (fabs(emf[k]) > fabs(emf[k + 1])) {
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
        // 1. PBL fluxes (:3255-3290)
        {
            Tl xsrc = qtsrc, xmean = qt0[kinv];
            Tl xtop = qt0[kinv + 1] + ssqt0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
            Tl xbot = qt0[kinv - 1] + ssqt0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
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
        // 2. non-buoyancy-sorting fluxes (:3300-3313)
        {
            Tl uplus = 0.0, vplus = 0.0;
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
        // 3. buoyancy-sorting fluxes (:3322-3331)
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
        // 4. penetrative-entrainment fluxes (:3392-3401)
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
                      : ((kk) <= krel - 1 ? cbmf : ((kk) <= kbup - 1 ? umf[(kk)] : ((kk) <= kpen - 1 ? emf[(kk)] : 0.0))))
            bool ldone = stop;
            for (int k = 1; k <= mkx; k++) {   // uniform
                if (k > kpen) ldone = true;
                if (!ldone) do {
                Tl comsub = 0.5 * (UEMF(k) + UEMF(k - 1));
                Tl thlten_sub, qtten_sub, qlten_sub, qiten_sub, nlten_sub, niten_sub;
                if (comsub >= 0.0) {
                    if (k == mkx) {
                        thlten_sub = 0.0; qtten_sub = 0.0; qlten_sub = 0.0; qiten_sub = 0.0;
                        nlten_sub = 0.0; niten_sub = 0.0;
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
                        thlten_sub = 0.0; qtten_sub = 0.0; qlten_sub = 0.0; qiten_sub = 0.0;
                        nlten_sub = 0.0; niten_sub = 0.0;
                    } else {
                        thlten_sub = g * comsub * (thl0[k] - thl0[k - 1]) / (p0[k - 1] - p0[k]);
                        qtten_sub = g * comsub * (qt0[k] - qt0[k - 1]) / (p0[k - 1] - p0[k]);
                        qlten_sub = g * comsub * (ql0[k] - ql0[k - 1]) / (p0[k - 1] - p0[k]);
                        qiten_sub = g * comsub * (qi0[k] - qi0[k - 1]) / (p0[k - 1] - p0[k]);
                        nlten_sub = g * comsub * (GT(ixnumliq, k) - GT(ixnumliq, k - 1)) / (p0[k - 1] - p0[k]);
                        niten_sub = g * comsub * (GT(ixnumice, k) - GT(ixnumice, k - 1)) / (p0[k - 1] - p0[k]);
                    }
                }
                Tl thl_prog = thl0[k] + thlten_sub * dt;
                Tl qt_prog = MX(qt0[k] + qtten_sub * dt, 1.e-12);
                if (CONDEN(p0[k], exn0[k], thl_prog, qt_prog, thj, qvj, qlj, qij, tbl)) {
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
        rliq = 0.0;
        rainflx = 0.0;
        snowflx = 0.0;
        } while (0);
        UW_SYNC();
        {
            Tl qlubelow = 0.0, qiubelow = 0.0;
            bool ldone = stop;
            for (int k = 1; k <= mkx; k++) {   // uniform
                if (k > kpen) ldone = true;
                if (!ldone) do {
                const int km1 = k - 1;
                dwten[k] = dwten[k] * 0.5 * (umf[k - 1] + umf[k]) * g / dp0[k];
                diten[k] = diten[k] * 0.5 * (umf[k - 1] + umf[k]) * g / dp0[k];
                qrten[k] = frc_rasn * dwten[k];
                qsten[k] = frc_rasn * diten[k];
                rainflx = rainflx + qrten[k] * dp0[k] / g;
                snowflx = snowflx + qsten[k] * dp0[k] / g;
                slten[k] = (slflx[km1] - slflx[k]) * g / dp0[k];
                if (k == 1) {
                    const Tl u1 = GL(u0, k), u2 = GL(u0, k + 1), v1 = GL(v0, k), v2 = GL(v0, k + 1);
                    slten[k] = slten[k] - g / 4.0 / dp0[k] *
                                              (uflx[k] * (uf[k + 1] - uf[k] + u2 - u1) +
                                               vflx[k] * (vf[k + 1] - vf[k] + v2 - v1));
                } else if (k >= 2 && k <= kpen - 1) {
                    const Tl um = GL(u0, k - 1), u1 = GL(u0, k), u2 = GL(u0, k + 1);
                    const Tl vm = GL(v0, k - 1), v1 = GL(v0, k), v2 = GL(v0, k + 1);
                    slten[k] = slten[k] - g / 4.0 / dp0[k] *
                                              (uflx[k] * (uf[k + 1] - uf[k] + u2 - u1) +
                                               uflx[k - 1] * (uf[k] - uf[k - 1] + u1 - um) +
                                               vflx[k] * (vf[k + 1] - vf[k] + v2 - v1) +
                                               vflx[k - 1] * (vf[k] - vf[k - 1] + v1 - vm));
                } else if (k == kpen) {
                    const Tl um = GL(u0, k - 1), u1 = GL(u0, k), vm = GL(v0, k - 1), v1 = GL(v0, k);
                    slten[k] = slten[k] - g / 4.0 / dp0[k] *
                                              (uflx[k - 1] * (uf[k] - uf[k - 1] + u1 - um) +
                                               vflx[k - 1] * (vf[k] - vf[k - 1] + v1 - vm));
                }
                qtten[k] = (qtflx[km1] - qtflx[k]) * g / dp0[k];

                Tl qlu_mid, qiu_mid;
                if (k < krel || k > kpen) {
                    qlu_mid = 0.0;
                    qiu_mid = 0.0;
                    qlj = 0.0;
                    qij = 0.0;
                } else {
                    // one conden call site for the release level, the cloud top and the levels between
                    const bool atrel = (k == krel), attop = (k != krel && k == kpen);
                    if (atrel) {
                        if (CONDEN(prel, exprel, thlu[krel - 1], qtu[krel - 1], thj, qvj, qlj, qij, tbl)) {
                            xflags |= UW_X_CONDEN;
                            id_exit = true;
                            stop = true;
                            break;
                        }
                        qlubelow = qlj;
                        qiubelow = qij;
                    }
                    if (CONDEN(attop ? ps0[k - 1] + ppen : ps0[k], attop ? exntop : exns0[k], attop ? thlu_top : thlu[k],
                               attop ? qtu_top : qtu[k], thj, qvj, qlj, qij, tbl)) {
                        xflags |= UW_X_CONDEN;
                        id_exit = true;
                        stop = true;
                        break;
                    }
                    if (atrel) {
                        qlu_mid = 0.5 * (qlubelow + qlj) * (prel - ps0[k]) / (ps0[k - 1] - ps0[k]);
                        qiu_mid = 0.5 * (qiubelow + qij) * (prel - ps0[k]) / (ps0[k - 1] - ps0[k]);
                    } else if (attop) {
                        qlu_mid = 0.5 * (qlubelow + qlj) * (-ppen) / (ps0[k - 1] - ps0[k]);
                        qiu_mid = 0.5 * (qiubelow + qij) * (-ppen) / (ps0[k - 1] - ps0[k]);
                    } else {
                        qlu_mid = 0.5 * (qlubelow + qlj);
                        qiu_mid = 0.5 * (qiubelow + qij);
                    }
                }
                qlubelow = qlj;
                qiubelow = qij;

                Tl qc_lm, qc_im, nc_lm, nc_im;
                qc_l[k] = (1.0 - frc_rasn) * dwten[k];
                qc_i[k] = (1.0 - frc_rasn) * diten[k];
                const Tl trl = GT(ixnumliq, k), tri = GT(ixnumice, k);
                if (k <= kbup) {
                    qc_l[k] = qc_l[k] + g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * qlu_mid;
                    qc_i[k] = qc_i[k] + g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * qiu_mid;
                    qc_lm = -g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * ql0[k];
                    qc_im = -g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * qi0[k];
                    nc_lm = -g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * trl;
                    nc_im = -g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * tri;
                } else {
                    qc_lm = 0.0;
                    qc_im = 0.0;
                    nc_lm = 0.0;
                    nc_im = 0.0;
                }
                if (k == kbup) {
                    qc_l[k] = qc_l[k] + g * umf[k] * qlj / (ps0[k - 1] - ps0[k]);
                    qc_i[k] = qc_i[k] + g * umf[k] * qij / (ps0[k - 1] - ps0[k]);
                    qc_lm = qc_lm - g * umf[k] * ql0[k] / (ps0[k - 1] - ps0[k]);
                    qc_im = qc_im - g * umf[k] * qi0[k] / (ps0[k - 1] - ps0[k]);
                    nc_lm = nc_lm - g * umf[k] * trl / (ps0[k - 1] - ps0[k]);
                    nc_im = nc_im - g * umf[k] * tri / (ps0[k - 1] - ps0[k]);
                    Tl ql_emf_kbup, qi_emf_kbup, thjj, qvjj;
                    if (CONDEN(p0[k], exn0[k], thlu_emf[k], qtu_emf[k], thjj, qvjj, ql_emf_kbup, qi_emf_kbup, tbl)) {
                        id_exit = true;
                        stop = true;
            break;
                    }
                    Tl nl_emf_kbup = (ql_emf_kbup > 0.0) ? tru_emf[ixnumliq - 1][k] : 0.0;
                    Tl ni_emf_kbup = (qi_emf_kbup > 0.0) ? tru_emf[ixnumice - 1][k] : 0.0;
                    qc_lm = qc_lm - g * emf[k] * (ql_emf_kbup - ql0[k]) / (ps0[k - 1] - ps0[k]);
                    qc_im = qc_im - g * emf[k] * (qi_emf_kbup - qi0[k]) / (ps0[k - 1] - ps0[k]);
                    nc_lm = nc_lm - g * emf[k] * (nl_emf_kbup - trl) / (ps0[k - 1] - ps0[k]);
                    nc_im = nc_im - g * emf[k] * (ni_emf_kbup - tri) / (ps0[k - 1] - ps0[k]);
                }
                qlten[k] = qc_l[k] + frc_rasn * dwten[k] + (MX(0.0, ql0[k] + (qc_lm + qlten_sink[k]) * dt) - ql0[k]) / dt;
                qiten[k] = qc_i[k] + frc_rasn * diten[k] + (MX(0.0, qi0[k] + (qc_im + qiten_sink[k]) * dt) - qi0[k]) / dt;
                trten[ixnumliq - 1][k] = MX(nc_lm + nlten_sink[k], -trl / dt);
                trten[ixnumice - 1][k] = MX(nc_im + niten_sink[k], -tri / dt);
                qvten[k] = qtten[k] - qlten[k] - qiten[k];
                sten[k] = slten[k] + xlv * qlten[k] + xls * qiten[k];
                qc[k] = qc_l[k] + qc_i[k];
                rliq = rliq + qc[k] * dp0[k] / g / 1000.0;
                } while (0);
                if (stop) ldone = true;
            }
        }
        UW_SYNC();
        // evaporation and melting of precipitation (:3808-3934)
        if (!stop) do {
        {
            Tl evpint_rain = 0.0, evpint_snow = 0.0;
            for (int k = 0; k <= mkx; k++) {
                flxrain[k] = 0.0;
                flxsnow[k] = 0.0;
            }
            for (int k = mkx; k >= 1; k--) {
                Tl snowmlt;
                if (t0[k] > 273.16) snowmlt = MX(0.0, flxsnow[k] * g / dp0[k]);
                else snowmlt = 0.0;
                Tl qs1 = qsat_qs(t0[k], p0[k], tbl);
                Tl subsat = MX((1.0 - qv0[k] / qs1), 0.0);
                Tl evprain = kevp * subsat * sqrt(flxrain[k] + snowmlt * dp0[k] / g);
                Tl evpsnow = kevp * subsat * sqrt(MX(flxsnow[k] - snowmlt * dp0[k] / g, 0.0));
                Tl evplimit = MX(0.0, (qw0[k] - qv0[k]) / dt);
                Tl evplimit_rain = MN(evplimit, (flxrain[k] + snowmlt * dp0[k] / g) * g / dp0[k]);
                evplimit_rain = MN(evplimit_rain, (rainflx - evpint_rain) * g / dp0[k]);
                evprain = MX(0.0, MN(evplimit_rain, evprain));
                Tl evplimit_snow = MN(evplimit, MX(flxsnow[k] - snowmlt * dp0[k] / g, 0.0) * g / dp0[k]);
                evplimit_snow = MN(evplimit_snow, (snowflx - evpint_snow) * g / dp0[k]);
                evpsnow = MX(0.0, MN(evplimit_snow, evpsnow));
                if ((evprain + evpsnow) > evplimit) {
                    Tl tmp1 = evprain * evplimit / (evprain + evpsnow);
                    Tl tmp2 = evpsnow * evplimit / (evprain + evpsnow);
                    evprain = tmp1;
                    evpsnow = tmp2;
                }
                evapc[k] = evprain + evpsnow;
                evpint_rain = evpint_rain + evprain * dp0[k] / g;
                evpint_snow = evpint_snow + evpsnow * dp0[k] / g;
                Tl ntraprd = qrten[k] - evprain + snowmlt;
                Tl ntsnprd = qsten[k] - evpsnow - snowmlt;
                flxrain[k - 1] = flxrain[k] + ntraprd * dp0[k] / g;
                flxsnow[k - 1] = flxsnow[k] + ntsnprd * dp0[k] / g;
                flxrain[k - 1] = MX(flxrain[k - 1], 0.0);
                flxsnow[k - 1] = MX(flxsnow[k - 1], 0.0);
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
            precip = (flxrain[0] + flxsnow[0]) / 1000.0;
            snow = flxsnow[0] / 1000.0;
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
        // positive_moisture_single (uwshcu.F90:5096-5162 via :3995-4001); state after the tendencies
        {
            const Tl qvmin = c.qmin[0], qlmin = c.qmin[1], qimin = c.qmin[2];
            Tl qvs[KP];
            for (int k = 1; k <= mkx; k++) qvs[k] = qv0[k] + qvten[k] * dt;
            Tl dqv = 0.0;
            for (int k = mkx; k >= 1; k--) {
                Tl qlk = ql0[k] + qlten[k] * dt;
                Tl qik = qi0[k] + qiten[k] * dt;
                Tl dql = MX(0.0, 1.0 * qlmin - qlk);
                Tl dqi = MX(0.0, 1.0 * qimin - qik);
                qlten[k] = qlten[k] + dql / dt;
                qiten[k] = qiten[k] + dqi / dt;
                qvten[k] = qvten[k] - (dql + dqi) / dt;
                sten[k] = sten[k] + xlv * (dql / dt) + xls * (dqi / dt);
                qvs[k] = qvs[k] - dql - dqi;
                dqv = MX(0.0, 1.0 * qvmin - qvs[k]);
                qvten[k] = qvten[k] + dqv / dt;
                qvs[k] = qvs[k] + dqv;
                if (k != 1) {
                    qvs[k - 1] = qvs[k - 1] - dqv * dp0[k] / dp0[k - 1];
                    qvten[k - 1] = qvten[k - 1] - dqv * dp0[k] / dp0[k - 1] / dt;
                }
                qvs[k] = MX(qvs[k], qvmin);
            }
            if (dqv > 1.e-20) {
                Tl sum = 0.0;
                for (int k = 1; k <= mkx; k++)
                    if (qvs[k] > 2.0 * qvmin) sum = sum + qvs[k] * dp0[k];
                Tl aa = dqv * dp0[1] / MX(1.e-20, sum);
                if (aa < 0.5) {
                    for (int k = 1; k <= mkx; k++) {
                        if (qvs[k] > 2.0 * qvmin) {
                            Tl dum = aa * qvs[k];
                            qvs[k] = qvs[k] - dum;
                            qvten[k] = qvten[k] - dum / dt;
                        }
                    }
                }
            }
        }
        for (int k = 1; k <= mkx; k++) {
            qtten[k] = qvten[k] + qlten[k] + qiten[k];
            slten[k] = sten[k] - xlv * qlten[k] - xls * qiten[k];
        }
        // tracer tendencies (:4007-4076)
        for (int m = 4; m <= ncnst; m++) {
            if (m != ixnumliq && m != ixnumice) {
                const Tl trmin = c.qmin[m - 1];
                const bool wet = c.wet[m - 1] != 0;
                for (int k = 0; k <= mkx; k++) {
                    trflx_d[k] = 0.0;
                    trflx_u[k] = 0.0;
                }
                for (int k = 1; k <= mkx - 1; k++) {
                    Tl pdelx = wet ? dp0[k] : GL(dpdry0, k);
                    Tl dum = (GT(m, k) - trmin) * pdelx / g / dt + trflx[m - 1][k - 1] - trflx[m - 1][k] + trflx_d[k - 1];
                    trflx_d[k] = MN(0.0, dum);
                }
                for (int k = mkx; k >= 2; k--) {
                    Tl pdelx = wet ? dp0[k] : GL(dpdry0, k);
                    Tl dum = (GT(m, k) - trmin) * pdelx / g / dt + trflx[m - 1][k - 1] - trflx[m - 1][k] +
                                 trflx_d[k - 1] - trflx_d[k] - trflx_u[k];
                    trflx_u[k - 1] = MX(0.0, -dum);
                }
                for (int k = 1; k <= mkx; k++) {
                    Tl pdelx = wet ? dp0[k] : GL(dpdry0, k);
                    trten[m - 1][k] = (trflx[m - 1][k - 1] - trflx[m - 1][k] + trflx_d[k - 1] - trflx_d[k] +
                                       trflx_u[k - 1] - trflx_u[k]) * g / pdelx;
                }
            }
        }
        // in-cloud diagnostics (:4092-4158)
        if (CONDEN(prel, exprel, thlu[krel - 1], qtu[krel - 1], thj, qvj, qlj, qij, tbl)) {
            xflags |= UW_X_CONDEN;
            id_exit = true;
            stop = true;
            break;
        }
        } while (0);
        UW_SYNC();
        {
            Tl qcubelow = qlj + qij, qlubelow = qlj, qiubelow = qij;
            bool ldone = stop;
            for (int j = 0; j <= mkx; j++) {   // uniform
                const int k = krel + j;
                if (k > kpen) ldone = true;
                if (!ldone) do {
                const bool attop = (k == kpen);
                const int idc = CONDEN(attop ? ps0[k - 1] + ppen : ps0[k], attop ? exntop : exns0[k],
                                       attop ? thlu_top : thlu[k], attop ? qtu_top : qtu[k], thj, qvj, qlj, qij, tbl);
                if (idc) {
                    xflags |= UW_X_CONDEN;
                    id_exit = true;
                    stop = true;
                    break;
                }
                qcu[k] = 0.5 * (qcubelow + qlj + qij);
                qlu[k] = 0.5 * (qlubelow + qlj);
                qiu[k] = 0.5 * (qiubelow + qij);
                // compute_zwshcu's cloud-fraction option (zwshcu.F90:4413-4431, 4449)
                Tl zw_tmp2 = 0.0, zw_tmp3 = 1.0;
                if (ZW && c.zw_cloud_sh) {
                    zw_tmp3 = 0.5 * c.zw_ufrc0;
                    Tl tmp1 = (GL(z0, k) - GL(z0, krel)) / (GL(z0, kpen) - GL(z0, krel) + 10.0);
                    tmp1 = 1.0 + c.zw_ufrcz * tmp1;
                    zw_tmp3 = zw_tmp3 * tmp1;
                    zw_tmp2 = fdr[k] * umf[k] * (zs0[k] - zs0[k - 1]) * dt / dp0[k] * 9.8 * c.zw_ufrcd;
                    zw_tmp2 = MN(1.0 - rmaxfrac, zw_tmp2);
                }
                cufrc[k] = (ufrc[k - 1] + ufrc[k]);
                if (k == krel) {
                    cufrc[k] = (ufrclcl + ufrc[k]) * (prel - ps0[k]) / (ps0[k - 1] - ps0[k]);
                } else if (k == kpen) {
                    cufrc[k] = (ufrc[k - 1] + 0.0) * (-ppen) / (ps0[k - 1] - ps0[k]);
                    if ((qlj + qij) > criqc) {
                        qcu[k] = 0.5 * (qcubelow + criqc);
                        qlu[k] = 0.5 * (qlubelow + criqc * qlj / (qlj + qij));
                        qiu[k] = 0.5 * (qiubelow + criqc * qij / (qlj + qij));
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
        cnt = (Tl)kpen;
        cnb = (Tl)(krel - 1);

        if (iter == 1) {
            // Save the iteration-1 outputs into the output slots (the Fortran *_s copies, :4177-4277)
            for (int k = 0; k <= mkx; k++) {
                { const Tl v_ = (umf[k]); OI(umf, k) = tl_val(v_); TOI(umf, k) = tl_der(v_); }
                { const Tl v_ = (slflx[k]); OI(slflx, k) = tl_val(v_); TOI(slflx, k) = tl_der(v_); }
                { const Tl v_ = (qtflx[k]); OI(qtflx, k) = tl_val(v_); TOI(qtflx, k) = tl_der(v_); }
            }
            for (int k = 1; k <= mkx; k++) {
                { const Tl v_ = (qvten[k]); OL(qvten, k) = tl_val(v_); TOL(qvten, k) = tl_der(v_); } { const Tl v_ = (qlten[k]); OL(qlten, k) = tl_val(v_); TOL(qlten, k) = tl_der(v_); } { const Tl v_ = (qiten[k]); OL(qiten, k) = tl_val(v_); TOL(qiten, k) = tl_der(v_); }
                { const Tl v_ = (sten[k]); OL(sten, k) = tl_val(v_); TOL(sten, k) = tl_der(v_); } { const Tl v_ = (uten[k]); OL(uten, k) = tl_val(v_); TOL(uten, k) = tl_der(v_); } { const Tl v_ = (vten[k]); OL(vten, k) = tl_val(v_); TOL(vten, k) = tl_der(v_); }
                { const Tl v_ = (qrten[k]); OL(qrten, k) = tl_val(v_); TOL(qrten, k) = tl_der(v_); } { const Tl v_ = (qsten[k]); OL(qsten, k) = tl_val(v_); TOL(qsten, k) = tl_der(v_); } { const Tl v_ = (evapc[k]); OL(evapc, k) = tl_val(v_); TOL(evapc, k) = tl_der(v_); }
                { const Tl v_ = (cufrc[k]); OL(cufrc, k) = tl_val(v_); TOL(cufrc, k) = tl_der(v_); } { const Tl v_ = (qcu[k]); OL(qcu, k) = tl_val(v_); TOL(qcu, k) = tl_der(v_); } { const Tl v_ = (qlu[k]); OL(qlu, k) = tl_val(v_); TOL(qlu, k) = tl_der(v_); }
                { const Tl v_ = (qiu[k]); OL(qiu, k) = tl_val(v_); TOL(qiu, k) = tl_der(v_); } { const Tl v_ = (qc[k]); OL(qc, k) = tl_val(v_); TOL(qc, k) = tl_der(v_); }
                for (int m = 1; m <= ncnst; m++) { const Tl v_ = (trten[m - 1][k]); OT(m, k) = tl_val(v_); TOT(m, k) = tl_der(v_); }
            }
            { const Tl v_ = (precip); A.precip[i] = tl_val(v_); T.precip[i] = tl_der(v_); }
            { const Tl v_ = (snow); A.snow[i] = tl_val(v_); T.snow[i] = tl_der(v_); }
            { const Tl v_ = (cush); A.cush[i] = tl_val(v_); T.cush[i] = tl_der(v_); }
            { const Tl v_ = (cbmf); A.cbmf[i] = tl_val(v_); T.cbmf[i] = tl_der(v_); }
            { const Tl v_ = (rliq); A.rliq[i] = tl_val(v_); T.rliq[i] = tl_der(v_); }
            A.cnt[i] = tl_val(CNT(cnt));
            A.cnb[i] = tl_val(CNT(cnb));
            PUT_DIAG_LEVEL();
            cin_s = cin; cinlcl_s = cinlcl; plcl_s = plcl; pinv_s = ps0[kinv - 1]; plfc_s = plfc;
            pbup_s = ps0[kbup]; ppen_s = ps0[kpen - 1] + ppen; tkeavg_s = tkeavg;
            kinv_s = kinv; klcl_s = klcl; klfc_s = klfc; krel_s = krel; kbup_s = kbup; kpen_s = kpen;
            // advance the state for the second CIN estimate (:4177-4184, :4285-4327)
            for (int k = 1; k <= mkx; k++) {
                Tl qv0s = qv0[k] + qvten[k] * dt;
                Tl ql0s = ql0[k] + qlten[k] * dt;
                Tl qi0s = qi0[k] + qiten[k] * dt;
                Tl s0s = s0[k] + sten[k] * dt;
                Tl t0s = t0[k] + sten[k] * dt / cp;
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
                Tl thl0bot = thl0[k] + ssthl0[k] * (ps0[k - 1] - p0[k]);
                Tl qt0bot = qt0[k] + ssqt0[k] * (ps0[k - 1] - p0[k]);
                if (CONDEN(ps0[k - 1], exns0[k - 1], thl0bot, qt0bot, thj, qvj, qlj, qij, tbl)) {
                    xflags |= UW_X_CONDEN;
                    id_exit = true;
                    stop = true;
                    break;
                }
                thv0bot[k] = thj * (1.0 + zvir * qvj - qlj - qij);
                thvl0bot[k] = thl0bot * (1.0 + zvir * qt0bot);
                Tl thl0top = thl0[k] + ssthl0[k] * (ps0[k] - p0[k]);
                Tl qt0top = qt0[k] + ssqt0[k] * (ps0[k] - p0[k]);
                if (CONDEN(ps0[k], exns0[k], thl0top, qt0top, thj, qvj, qlj, qij, tbl)) {
                    xflags |= UW_X_CONDEN;
                    id_exit = true;
                    stop = true;
                    break;
                }
                thv0top[k] = thj * (1.0 + zvir * qvj - qlj - qij);
                thvl0top[k] = thl0top * (1.0 + zvir * qt0top);
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
        { const Tl v_ = (umf[k]); OI(umf, k) = tl_val(v_); TOI(umf, k) = tl_der(v_); }
        { const Tl v_ = (wu[k]); OI(wu, k) = tl_val(v_); TOI(wu, k) = tl_der(v_); }
        { const Tl v_ = (slflx[k]); OI(slflx, k) = tl_val(v_); TOI(slflx, k) = tl_der(v_); }
        { const Tl v_ = (qtflx[k]); OI(qtflx, k) = tl_val(v_); TOI(qtflx, k) = tl_der(v_); }
        { const Tl v_ = (flxrain[k] + flxsnow[k]); OI(flxprc1, k) = tl_val(v_); TOI(flxprc1, k) = tl_der(v_); }
        { const Tl v_ = (flxsnow[k]); OI(flxsnow1, k) = tl_val(v_); TOI(flxsnow1, k) = tl_der(v_); }
    }
    for (int k = 1; k <= mkx; k++) {
        { const Tl v_ = (qvten[k]); OL(qvten, k) = tl_val(v_); TOL(qvten, k) = tl_der(v_); } { const Tl v_ = (qlten[k]); OL(qlten, k) = tl_val(v_); TOL(qlten, k) = tl_der(v_); } { const Tl v_ = (qiten[k]); OL(qiten, k) = tl_val(v_); TOL(qiten, k) = tl_der(v_); }
        { const Tl v_ = (sten[k]); OL(sten, k) = tl_val(v_); TOL(sten, k) = tl_der(v_); } { const Tl v_ = (uten[k]); OL(uten, k) = tl_val(v_); TOL(uten, k) = tl_der(v_); } { const Tl v_ = (vten[k]); OL(vten, k) = tl_val(v_); TOL(vten, k) = tl_der(v_); }
        { const Tl v_ = (qrten[k]); OL(qrten, k) = tl_val(v_); TOL(qrten, k) = tl_der(v_); } { const Tl v_ = (qsten[k]); OL(qsten, k) = tl_val(v_); TOL(qsten, k) = tl_der(v_); } { const Tl v_ = (evapc[k]); OL(evapc, k) = tl_val(v_); TOL(evapc, k) = tl_der(v_); }
        { const Tl v_ = (cufrc[k]); OL(cufrc, k) = tl_val(v_); TOL(cufrc, k) = tl_der(v_); } { const Tl v_ = (qcu[k]); OL(qcu, k) = tl_val(v_); TOL(qcu, k) = tl_der(v_); } { const Tl v_ = (qlu[k]); OL(qlu, k) = tl_val(v_); TOL(qlu, k) = tl_der(v_); }
        { const Tl v_ = (qiu[k]); OL(qiu, k) = tl_val(v_); TOL(qiu, k) = tl_der(v_); } { const Tl v_ = (qc[k]); OL(qc, k) = tl_val(v_); TOL(qc, k) = tl_der(v_); }
        for (int m = 1; m <= ncnst; m++) { const Tl v_ = (trten[m - 1][k]); OT(m, k) = tl_val(v_); TOT(m, k) = tl_der(v_); }
    }
    { const Tl v_ = (precip); A.precip[i] = tl_val(v_); T.precip[i] = tl_der(v_); }
    { const Tl v_ = (snow); A.snow[i] = tl_val(v_); T.snow[i] = tl_der(v_); }
    { const Tl v_ = (cush); A.cush[i] = tl_val(v_); T.cush[i] = tl_der(v_); }
    { const Tl v_ = (cbmf); A.cbmf[i] = tl_val(v_); T.cbmf[i] = tl_der(v_); }
    { const Tl v_ = (rliq); A.rliq[i] = tl_val(v_); T.rliq[i] = tl_der(v_); }
    A.cnt[i] = tl_val(CNT(cnt));
    A.cnb[i] = tl_val(CNT(cnb));
    if (A.diag_real) {
        A.diag_real[UW_DR_CIN * (size_t)mix + i] = tl_val(cin);
        A.diag_real[UW_DR_CINLCL * (size_t)mix + i] = tl_val(cinlcl);
        A.diag_real[UW_DR_PLCL * (size_t)mix + i] = tl_val(plcl);
        A.diag_real[UW_DR_PLFC * (size_t)mix + i] = tl_val(plfc);
        A.diag_real[UW_DR_PINV * (size_t)mix + i] = tl_val(ps0[kinv - 1]);
        A.diag_real[UW_DR_PBUP * (size_t)mix + i] = tl_val(ps0[kbup]);
        A.diag_real[UW_DR_PPEN * (size_t)mix + i] = tl_val(ps0[kpen - 1] + ppen);
        A.diag_real[UW_DR_TKEAVG * (size_t)mix + i] = tl_val(tkeavg);
    }
    PUT_DIAG_LEVEL();
    }

    // (label 333, :4448-4549)
    if (!cand && !handed) {
    if (id_exit) {
        xflags |= UW_X_UWCU;
        for (int k = 0; k <= mkx; k++) {
            { const Tl v_ = (0.0); OI(umf, k) = tl_val(v_); TOI(umf, k) = tl_der(v_); }
            { const Tl v_ = (0.0); OI(wu, k) = tl_val(v_); TOI(wu, k) = tl_der(v_); }
            { const Tl v_ = (0.0); OI(slflx, k) = tl_val(v_); TOI(slflx, k) = tl_der(v_); }
            { const Tl v_ = (0.0); OI(qtflx, k) = tl_val(v_); TOI(qtflx, k) = tl_der(v_); }
            { const Tl v_ = (0.0); OI(flxprc1, k) = tl_val(v_); TOI(flxprc1, k) = tl_der(v_); }
            { const Tl v_ = (0.0); OI(flxsnow1, k) = tl_val(v_); TOI(flxsnow1, k) = tl_der(v_); }
        }
        for (int k = 1; k <= mkx; k++) {
            { const Tl v_ = (0.0); OL(qvten, k) = tl_val(v_); TOL(qvten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qlten, k) = tl_val(v_); TOL(qlten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qiten, k) = tl_val(v_); TOL(qiten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(sten, k) = tl_val(v_); TOL(sten, k) = tl_der(v_); }
            { const Tl v_ = (0.0); OL(uten, k) = tl_val(v_); TOL(uten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(vten, k) = tl_val(v_); TOL(vten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qrten, k) = tl_val(v_); TOL(qrten, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qsten, k) = tl_val(v_); TOL(qsten, k) = tl_der(v_); }
            { const Tl v_ = (0.0); OL(evapc, k) = tl_val(v_); TOL(evapc, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(cufrc, k) = tl_val(v_); TOL(cufrc, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qcu, k) = tl_val(v_); TOL(qcu, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qlu, k) = tl_val(v_); TOL(qlu, k) = tl_der(v_); }
            { const Tl v_ = (0.0); OL(qiu, k) = tl_val(v_); TOL(qiu, k) = tl_der(v_); } { const Tl v_ = (0.0); OL(qc, k) = tl_val(v_); TOL(qc, k) = tl_der(v_); }
            for (int m = 1; m <= ncnst; m++) { const Tl v_ = (0.0); OT(m, k) = tl_val(v_); TOT(m, k) = tl_der(v_); }
        }
        { const Tl v_ = (0.0); A.precip[i] = tl_val(v_); T.precip[i] = tl_der(v_); }
        { const Tl v_ = (0.0); A.snow[i] = tl_val(v_); T.snow[i] = tl_der(v_); }
        { const Tl v_ = (-1.0); A.cush[i] = tl_val(v_); T.cush[i] = tl_der(v_); }
        { const Tl v_ = (0.0); A.cbmf[i] = tl_val(v_); T.cbmf[i] = tl_der(v_); }
        { const Tl v_ = (0.0); A.rliq[i] = tl_val(v_); T.rliq[i] = tl_der(v_); }
        A.cnt[i] = tl_val(CNT(1.0));
        A.cnb[i] = tl_val(CNT((Tl)mkx));
        if (A.diag_real) {
            A.diag_real[UW_DR_CIN * (size_t)mix + i] = tl_val(-1.0);
            A.diag_real[UW_DR_CINLCL * (size_t)mix + i] = tl_val(-1.0);
            for (int j = UW_DR_PLCL; j < UW_NDR; j++) A.diag_real[j * (size_t)mix + i] = tl_val(0.0);
        }
        if (A.diag_level)
            for (int j = 0; j < UW_NDL; j++)
                for (int k = 0; k <= mkx; k++) DLV(j, k) = tl_val(0.0);
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
#undef SEEDI
#undef SEEDL
#undef TOT
#undef TOL
#undef TOI
#undef DLV
#undef PUT_DIAG_LEVEL
#undef UEMF
}

// ---- kernels ---------------------------------------------------------------------------------------

// Register caps (resident blocks of 128 per SM): the worklist launches at 128 registers (4 blocks
// instead of 3 at their natural 168; the extra warps hide more FP64 and local-memory latency than
// the added spills cost, -10 % time on the benchmark workload; 5 blocks cost +1.5 % for
// UW_MODE_LIST1), the UW_MODE_RESUME launch, which spills less, at 85 (6 blocks: 177.1-177.4 ms
// per 1,048,576-column step against 178.7-178.8 at 5 with the correctly rounded math routines),
// the trigger pass at 102 (6 blocks: no change), the single pass at 168.
#define UW_LIST_MINB(m) ((m) == UW_MODE_RESUME ? 6 : (UW_MODE_IS_LIST(m) ? 4 : ((m) == UW_MODE_TRIGGER ? 5 : 3)))
template <int KP, int NC, int MODE>
__global__ void __launch_bounds__(128)
uwshcu_tl_kernel(const __grid_constant__ UwArgs A, int* __restrict__ wl, int* __restrict__ wl_count,
                 const __grid_constant__ UwTangent T)
{
    __shared__ double tbl[UW_TBL];
    for (int t = threadIdx.x; t < UW_TBL; t += blockDim.x) tbl[t] = c_estbl[t];
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
    uw_column<KP, NC, MODE, 0>(A, tbl, i, active, wl, wl_count, T);
}

}  // namespace
