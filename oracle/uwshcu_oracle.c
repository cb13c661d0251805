/*
 * uwshcu_oracle.c -- CPU oracle for compute_uwshcu (TEST INFRASTRUCTURE ONLY; never the product path).
 *
 * A plain-C FP64 restatement, statement by statement and in the same evaluation order, of
 *   src/physics/uwshcu.F90        exnf 50-54, compute_uwshcu_inv 251-476, compute_uwshcu 478-4664,
 *                                 getbuoy 4672-4702, single_cin 4704-4715, conden 4718-4785,
 *                                 roots 4787-4829, slope 4831-4861, qsinvert 4863-4929,
 *                                 compute_alpha 4931-4950, compute_mumin2 4952-4979,
 *                                 compute_ppen 4981-5028, fluxbelowinv 5030-5094,
 *                                 positive_moisture_single 5096-5162, findsp 5164-5454
 *   src/physics/wv_saturation.F90 estblf 64-80, gestbl 82-204, vqsatd 482-609, fqsatd 734-751
 *   src/physics/gffgch.F90        gffgch 1-127
 *   src/physics/esinti.F90        esinti 38-51
 * Build with -O2 -ffp-contract=off (no FMA contraction, no fast-math) so every operation rounds as
 * written.  Fortran `x**2` is written x*x (what gfortran emits); `x**y` with real y is pow().
 * erfc is the C99 libm erfc: the reference's error_function module (CAM, not vendored) is not part of
 * the reference tree, so parity at that call is unpinned.
 *
 * Deterministic choices where the Fortran reads undefined values: `roots` leaves r1/r2 unwritten on
 * its failure branches exactly as the Fortran does, and the caller-side xs1/xs2/xc1/xc2 start each
 * column at 0 instead of holding stack garbage.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "uwshcu_oracle.h"
#ifdef UWO_FORTRAN_MATH
#define UW_ERFC_EXP exp
#endif
#include "uw_math.h"
#ifdef _OPENMP
#include <omp.h>
#define UWO_MAXTHREADS() omp_get_max_threads()
#else
#define UWO_MAXTHREADS() 1
#endif

#define MX(a, b) ((a) > (b) ? (a) : (b))
#define MN(a, b) ((a) < (b) ? (a) : (b))
#define NCMAX 64

typedef struct {
    /* uwshcu module constants (uwshcu.F90:25-37) */
    double xlv, xlf, xls, cp, zvir, r, g, ep2, p00, rovcp, rpen;
    /* compute_uwshcu parameters rle, rkm, criqc (uwshcu.F90:1036, 1038, 1065), settable for tuning */
    double rle, rkm, criqc;
    /* wv_saturation module data (wv_saturation.F90:43-59) */
    double estbl[250];
    double tmin, tmax, ttrice, pcf[6], epsqs, rgasv, hlatf, hlatv, cpws, tmelt;
    int icephs;
    /* constituents (constituents.F90:54, cnst_type) */
    int ncnst;
    double qmin[NCMAX];
    int wet[NCMAX];
    int ixnumliq, ixnumice;
    /* zwshcu options (zwshcu.F90:30-59, cloud_fraction.F90:52), in force when a call passes omega:
     * zmh_shallow_lf, zmh_shallow_fwcrit, zmh_shallow_ent, zmh_ent0, zmh_cloud_sh, zmh_ufrcd,
     * zmh_ufrc0, zmh_ufrcz */
    int zw_lf, zw_ent, zw_cloud_sh;
    double zw_fwcrit, zw_ent0, zw_ufrcd, zw_ufrc0, zw_ufrcz;
} uwo_state;

static uwo_state S;

/* ------------------------------------------------------------------ saturation thermodynamics */

/* gffgch.F90:1-127 (itype < 0: |itype| degree transition between water and ice) */
static double gffgch(double t, int itype)
{
    double tr, es, eswtr = 0.0, e1, e2, f, f1, f2, f3, f4, f5, ps, ts, t0, term1, term2, term3, weight;
    int itp = itype;
    if (itp < 0) {
        tr = fabs((double)itp);
        itp = 1;
    } else {
        tr = 0.0;
    }
    if (t < (S.tmelt - tr) && itp == 1) goto ice;
    ps = 1013.246;
    ts = 373.16;
    e1 = 11.344 * (1.0 - t / ts);
    e2 = -3.49149 * (ts / t - 1.0);
    f1 = -7.90298 * (ts / t - 1.0);
    f2 = 5.02808 * log10(ts / t);
    f3 = -1.3816 * (pow(10.0, e1) - 1.0) / 10000000.0;
    f4 = 8.1328 * (pow(10.0, e2) - 1.0) / 1000.0;
    f5 = log10(ps);
    f = f1 + f2 + f3 + f4 + f5;
    es = (pow(10.0, f)) * 100.0;
    eswtr = es;
    if (t >= S.tmelt || itp == 0) return es;
ice:
    t0 = S.tmelt;
    term1 = 2.01889049 / (t0 / t);
    term2 = 3.56654 * log(t0 / t);
    term3 = 20.947031 * (t0 / t);
    es = 575.185606e10 * exp(-(term1 + term2 + term3));
    if (t < (S.tmelt - tr)) return es;
    weight = MN((S.tmelt - t) / tr, 1.0);
    es = weight * es + (1.0 - weight) * eswtr;
    return es;
}

/* gestbl (wv_saturation.F90:82-204) */
static void gestbl(double tmn, double tmx, double trice, int ip, double epsil, double latvap,
                   double latice, double rh2o, double cpair, double tmeltx)
{
    int n, lentbl, itype;
    double t;
    S.tmin = tmn;
    S.tmax = tmx;
    S.ttrice = trice;
    S.icephs = ip;
    S.epsqs = epsil;
    S.hlatv = latvap;
    S.hlatf = latice;
    S.rgasv = rh2o;
    S.cpws = cpair;
    S.tmelt = tmeltx;
    lentbl = (int)(S.tmax - S.tmin + 2.000001);
    if (lentbl > 250) lentbl = 250;
    if (S.icephs) {
        if (S.ttrice != 0.0) itype = (int)(-S.ttrice);
        else itype = 1;
    } else {
        itype = 0;
    }
    t = S.tmin - 1.0;
    for (n = 1; n <= lentbl; n++) {
        t = t + 1.0;
        S.estbl[n - 1] = gffgch(t, itype);
    }
    for (n = lentbl + 1; n <= 250; n++) S.estbl[n - 1] = -99999.0;
    S.pcf[0] = 5.04469588506e-01;
    S.pcf[1] = -5.47288442819e+00;
    S.pcf[2] = -3.67471858735e-01;
    S.pcf[3] = -8.95963532403e-03;
    S.pcf[4] = -7.78053686625e-05;
    S.pcf[5] = 0.0;
}

/* The column physics below calls EXP/LOG/POW/ERFC:
 *  - default: glibc for all four, which is what the reference's C++ drop-in
 *    (bxcompute_uwshcu_inv.cpp) calls when built for the host; this build is pinned to it;
 *  - UWO_FORTRAN_MATH: glibc exp/log/pow and CALERF erfc (uw_math.h, calling glibc exp), the
 *    functions a Fortran build of uwshcu.F90 calls: the compiler's libm for exp, log and **, and
 *    CAM's error_function module (Cody's CALERF) for erfc (uwshcu.F90:5);
 *  - UWO_PORTABLE_MATH: the host/device-identical routines of uw_math.h
 *    (hpc-and-climate-model_b200/csrc), which is how the CUDA path evaluates them.
 * The saturation table above always uses glibc, as the library does. */
#if defined(UWO_PORTABLE_MATH)
#define EXP(x) uw_exp(x)
#define LOG(x) uw_log(x)
#define POW(x, y) uw_pow(x, y)
#define ERFC(x) uw_erfc(x)
#elif defined(UWO_FORTRAN_MATH)
#define EXP(x) exp(x)
#define LOG(x) log(x)
#define POW(x, y) pow(x, y)
#define ERFC(x) uw_erfc(x)
#else
#define EXP(x) exp(x)
#define LOG(x) log(x)
#define POW(x, y) pow(x, y)
#define ERFC(x) erfc(x)
#endif

/* estblf (wv_saturation.F90:64-80) */
static double estblf(double td)
{
    double e = MX(MN(td, S.tmax), S.tmin);
    int i = (int)(e - S.tmin) + 1;
    double ai = trunc(e - S.tmin);
    return (S.tmin + ai - e + 1.0) * S.estbl[i - 1] - (S.tmin + ai - e) * S.estbl[i];
}

/* vqsatd with len = 1 (wv_saturation.F90:482-609), reached through fqsatd (:734-751) */
static void qsat1(double t, double p, double *es_o, double *qs_o, double *gam_o)
{
    double omeps = 1.0 - S.epsqs, es, qs, gam, trinv, tc, weight, hlatsb, hlatvp, hltalt, tterm, desdt;
    int lflg;
    es = estblf(t);
    qs = S.epsqs * es / (p - omeps * es);
    qs = MN(1.0, qs);
    if (qs < 0.0) {
        qs = 1.0;
        es = p;
    }
    trinv = 0.0;
    if ((!S.icephs) || (S.ttrice == 0.0)) goto l10;
    trinv = 1.0 / S.ttrice;
    tc = t - S.tmelt;
    lflg = (tc >= -S.ttrice && tc < 0.0);
    weight = MN(-tc * trinv, 1.0);
    hlatsb = S.hlatv + weight * S.hlatf;
    hlatvp = S.hlatv - 2369.0 * tc;
    if (t < S.tmelt) hltalt = hlatsb;
    else hltalt = hlatvp;
    if (lflg) tterm = S.pcf[0] + tc * (S.pcf[1] + tc * (S.pcf[2] + tc * (S.pcf[3] + tc * S.pcf[4])));
    else tterm = 0.0;
    desdt = hltalt * es / (S.rgasv * t * t) + tterm * trinv;
    gam = hltalt * qs * p * desdt / (S.cpws * es * (p - omeps * es));
    if (qs == 1.0) gam = 0.0;
    goto done;
l10:
    hlatvp = S.hlatv - 2369.0 * (t - S.tmelt);
    if (S.icephs) hlatsb = S.hlatv + S.hlatf;
    else hlatsb = S.hlatv;
    if (t < S.tmelt) hltalt = hlatsb;
    else hltalt = hlatvp;
    desdt = hltalt * es / (S.rgasv * t * t);
    gam = hltalt * qs * p * desdt / (S.cpws * es * (p - omeps * es));
    if (qs == 1.0) gam = 0.0;
done:
    *es_o = es;
    *qs_o = qs;
    *gam_o = gam;
}

/* ---------------------------------------------------------------------------- uwshcu helpers */

/* exnf (uwshcu.F90:50-54) */
static double exnf(double p) { return POW(p / S.p00, S.rovcp); }

/* conden (uwshcu.F90:4718-4785) */
static void conden(double p, double thl, double qt, double *th, double *qv, double *ql, double *qi,
                   double *rvls, int *id_check)
{
    double tc, temps, leff, nu, qc, es, qs, gam;
    int iteration;
    tc = thl * exnf(p);
    nu = MX(MN((268.0 - tc) / 20.0, 1.0), 0.0);
    leff = (1.0 - nu) * S.xlv + nu * S.xls;
    temps = tc;
    qsat1(temps, p, &es, &qs, &gam);
    *rvls = qs;
    if (qs >= qt) {
        *id_check = 0;
        *qv = qt;
        qc = 0.0;
        *ql = 0.0;
        *qi = 0.0;
        *th = tc / exnf(p);
    } else {
        for (iteration = 1; iteration <= 10; iteration++) {
            temps = temps + ((tc - temps) * S.cp / leff + qt - *rvls) /
                                (S.cp / leff + S.ep2 * leff * *rvls / S.r / temps / temps);
            qsat1(temps, p, &es, &qs, &gam);
            *rvls = qs;
        }
        qc = MX(qt - qs, 0.0);
        *qv = qt - qc;
        *ql = qc * (1.0 - nu);
        *qi = nu * qc;
        *th = temps / exnf(p);
        if (fabs((temps - (leff / S.cp) * qc) - tc) >= 1.0) *id_check = 1;
        else *id_check = 0;
    }
}

/* roots (uwshcu.F90:4787-4829).  r1/r2 are left unwritten on the failure branches, as in Fortran. */
static void roots(double a, double b, double c, double *r1, double *r2, int *status)
{
    double q;
    *status = 0;
    if (a == 0.0) {
        if (b == 0.0) *status = 1;
        else *r1 = -c / b;
        *r2 = *r1;
    } else {
        if (b == 0.0) {
            if (a * c > 0.0) *status = 2;
            else *r1 = sqrt(-c / a);
            *r2 = -*r1;
        } else {
            if ((b * b - 4.0 * a * c) < 0.0) {
                *status = 3;
            } else {
                q = -0.5 * (b + copysign(1.0, b) * sqrt(b * b - 4.0 * a * c));
                *r1 = q / a;
                *r2 = c / q;
            }
        }
    }
}

/* slope (uwshcu.F90:4831-4861); 1-based field/p0, result in sl[1..mkx] */
static void slope(int mkx, const double *field, const double *p0, double *sl)
{
    double below, above;
    int k;
    below = (field[2] - field[1]) / (p0[2] - p0[1]);
    for (k = 2; k <= mkx; k++) {
        above = (field[k] - field[k - 1]) / (p0[k] - p0[k - 1]);
        if (above > 0.0) sl[k - 1] = MX(0.0, MN(above, below));
        else sl[k - 1] = MN(0.0, MX(above, below));
        below = above;
    }
    sl[mkx] = sl[mkx - 1];
}

/* qsinvert (uwshcu.F90:4863-4929) */
static double qsinvert(double qt, double thl, double psfc)
{
    double ps, Pis, Ts, err, dlnqsdT, dTdPis, dPisdps, dlnqsdps, derrdps, dps, Ti, rhi, TLCL, PiLCL,
        psmin, dpsmax, es, qs, gam, leff, nu;
    int i;
    psmin = 100.0 * 100.0;
    dpsmax = 1.0;
    Ti = thl * POW(psfc / S.p00, S.rovcp);
    qsat1(Ti, psfc, &es, &qs, &gam);
    rhi = qt / qs;
    if (rhi <= 0.01) return psmin;
    TLCL = 55.0 + 1.0 / (1.0 / (Ti - 55.0) - LOG(rhi) / 2840.0);
    PiLCL = TLCL / thl;
    ps = S.p00 * POW(PiLCL, 1.0 / S.rovcp);
    for (i = 1; i <= 10; i++) {
        Pis = POW(ps / S.p00, S.rovcp);
        Ts = thl * Pis;
        qsat1(Ts, ps, &es, &qs, &gam);
        err = qt - qs;
        nu = MX(MN((268.0 - Ts) / 20.0, 1.0), 0.0);
        leff = (1.0 - nu) * S.xlv + nu * S.xls;
        dlnqsdT = gam * (S.cp / leff) / qs;
        dTdPis = thl;
        dPisdps = S.rovcp * Pis / ps;
        dlnqsdps = -1.0 / (ps - (1.0 - S.ep2) * es);
        derrdps = -qs * (dlnqsdT * dTdPis * dPisdps + dlnqsdps);
        dps = -err / derrdps;
        ps = ps + dps;
        if (ps < 0.0) return psmin;
        if (fabs(dps) <= dpsmax) return ps;
    }
    return psmin;
}

/* compute_alpha (uwshcu.F90:4931-4950) */
static double compute_alpha(double del_CIN, double ke)
{
    double x0 = 0.0, x1;
    int it;
    for (it = 1; it <= 10; it++) {
        x1 = x0 - (EXP(-x0 * ke * del_CIN) - x0) / (-ke * del_CIN * EXP(-x0 * ke * del_CIN) - 1.0);
        x0 = x1;
    }
    return x0;
}

/* compute_mumin2 (uwshcu.F90:4952-4979) */
static double compute_mumin2(double mulcl, double rmaxfrac, double mulow)
{
    double x0, x1, ex, ef, exf, f, fs, t1, t2;
    int it;
    x0 = mulow;
    for (it = 1; it <= 10; it++) {
        ex = EXP(-(x0 * x0));
        ef = ERFC(x0);
        exf = ex / ef;
        t1 = ex / 2.0 / rmaxfrac;
        t2 = mulcl * 2.5066 / 2.0;
        f = 0.5 * (exf * exf) - 0.5 * (t1 * t1) - (t2 * t2);
        fs = (2.0 * (exf * exf)) * (exf / sqrt(3.141592) - x0) + (0.5 * x0 * (ex * ex)) / (rmaxfrac * rmaxfrac);
        x1 = x0 - f / fs;
        x0 = x1;
    }
    return x0;
}

/* compute_ppen (uwshcu.F90:4981-5028).  The `1.e-8` at :4998 is a default-real literal. */
static double compute_ppen(double wtwb, double D, double bogbot, double bogtop, double rho0j, double dpen)
{
    double x0, x1, f, fs, SB, s00;
    int it;
    SB = (bogtop - bogbot) / dpen;
    s00 = bogbot / rho0j - D * wtwb;
    if (D * dpen < (double)1.e-8f) {
        if (s00 >= 0.0) x0 = dpen;
        else x0 = MX(0.0, MN(dpen, -0.5 * wtwb / s00));
    } else {
        if (s00 >= 0.0) x0 = dpen;
        else x0 = 0.0;
        for (it = 1; it <= 5; it++) {
            f = EXP(-2.0 * D * x0) * (wtwb - (bogbot - SB / (2.0 * D)) / (D * rho0j)) +
                (SB * x0 + bogbot - SB / (2.0 * D)) / (D * rho0j);
            fs = -2.0 * D * EXP(-2.0 * D * x0) * (wtwb - (bogbot - SB / (2.0 * D)) / (D * rho0j)) +
                 (SB) / (D * rho0j);
            if (fs >= 0.0) fs = MX(fs, 1.e-10);
            else fs = MN(fs, -1.e-10);
            x1 = x0 - f / fs;
            x0 = x1;
        }
    }
    return -MX(0.0, MN(dpen, x0));
}

/* getbuoy (uwshcu.F90:4672-4702) */
static void getbuoy(double pbot, double thv0bot, double ptop, double thv0top, double thvubot,
                    double thvutop, double *plfc, double *cin)
{
    double frc;
    if (thvubot > thv0bot && thvutop > thv0top) {
        *plfc = pbot;
        return;
    } else if (thvubot <= thv0bot && thvutop <= thv0top) {
        *cin = *cin - ((thvubot / thv0bot - 1.0) + (thvutop / thv0top - 1.0)) * (pbot - ptop) /
                          (pbot / (S.r * thv0bot * exnf(pbot)) + ptop / (S.r * thv0top * exnf(ptop)));
    } else if (thvubot > thv0bot && thvutop <= thv0top) {
        frc = (thvutop / thv0top - 1.0) / ((thvutop / thv0top - 1.0) - (thvubot / thv0bot - 1.0));
        *cin = *cin - (thvutop / thv0top - 1.0) * ((ptop + frc * (pbot - ptop)) - ptop) /
                          (pbot / (S.r * thv0bot * exnf(pbot)) + ptop / (S.r * thv0top * exnf(ptop)));
    } else {
        frc = (thvubot / thv0bot - 1.0) / ((thvubot / thv0bot - 1.0) - (thvutop / thv0top - 1.0));
        *plfc = pbot - frc * (pbot - ptop);
        *cin = *cin - (thvubot / thv0bot - 1.0) * (pbot - *plfc) /
                          (pbot / (S.r * thv0bot * exnf(pbot)) + ptop / (S.r * thv0top * exnf(ptop)));
    }
}

/* single_cin (uwshcu.F90:4704-4715) */
static double single_cin(double pbot, double thv0bot, double ptop, double thv0top, double thvubot,
                         double thvutop)
{
    return ((1.0 - thvubot / thv0bot) + (1.0 - thvutop / thv0top)) * (pbot - ptop) /
           (pbot / (S.r * thv0bot * exnf(pbot)) + ptop / (S.r * thv0top * exnf(ptop)));
}

/* fluxbelowinv (uwshcu.F90:5030-5094); ps0 and xflx indexed 0..mkx */
static void fluxbelowinv(double cbmf, const double *ps0, int mkx, int kinv, double dt, double xsrc,
                         double xmean, double xtopin, double xbotin, double *xflx)
{
    int k;
    double rcbmf, rpeff, dp, rr, pinv_eff, xtop, xbot, pinv, xtop_ori, xbot_ori;
    for (k = 0; k <= mkx; k++) xflx[k] = 0.0;
    dp = ps0[kinv - 1] - ps0[kinv];
    if (fabs(xbotin - xtopin) <= 1.e-13) {
        xbot = xbotin - 1.e-13;
        xtop = xtopin + 1.e-13;
    } else {
        xbot = xbotin;
        xtop = xtopin;
    }
    xtop_ori = xtop;
    xbot_ori = xbot;
    rcbmf = (cbmf * S.g * dt) / dp;
    rpeff = (xmean - xtop) / (xbot - xtop);
    rpeff = MN(MX(0.0, rpeff), 1.0);
    if (rpeff == 0.0 || rpeff == 1.0) {
        xbot = xmean;
        xtop = xmean;
    }
    rr = rpeff / rcbmf;
    pinv = ps0[kinv - 1] - rpeff * dp;
    pinv_eff = ps0[kinv - 1] + (rcbmf - rpeff) * dp;
    (void)pinv_eff;
    for (k = 0; k <= kinv - 1; k++) xflx[k] = cbmf * (xsrc - xbot) * (ps0[0] - ps0[k]) / (ps0[0] - pinv);
    if (rr <= 1.0) xflx[kinv - 1] = xflx[kinv - 1] - (1.0 - rr) * cbmf * (xtop_ori - xbot_ori);
}

/* positive_moisture_single (uwshcu.F90:5096-5162); all arrays 1-based [1..mkx] */
static void positive_moisture_single(double xlv, double xls, int mkx, double dt, double qvmin,
                                     double qlmin, double qimin, const double *dp, double *qv,
                                     double *ql, double *qi, double *s, double *qvten, double *qlten,
                                     double *qiten, double *sten)
{
    int k;
    double dql, dqi, dqv = 0.0, sum, aa, dum;
    for (k = mkx; k >= 1; k--) {
        dql = MX(0.0, 1.0 * qlmin - ql[k]);
        dqi = MX(0.0, 1.0 * qimin - qi[k]);
        qlten[k] = qlten[k] + dql / dt;
        qiten[k] = qiten[k] + dqi / dt;
        qvten[k] = qvten[k] - (dql + dqi) / dt;
        sten[k] = sten[k] + xlv * (dql / dt) + xls * (dqi / dt);
        ql[k] = ql[k] + dql;
        qi[k] = qi[k] + dqi;
        qv[k] = qv[k] - dql - dqi;
        s[k] = s[k] + xlv * dql + xls * dqi;
        dqv = MX(0.0, 1.0 * qvmin - qv[k]);
        qvten[k] = qvten[k] + dqv / dt;
        qv[k] = qv[k] + dqv;
        if (k != 1) {
            qv[k - 1] = qv[k - 1] - dqv * dp[k] / dp[k - 1];
            qvten[k - 1] = qvten[k - 1] - dqv * dp[k] / dp[k - 1] / dt;
        }
        qv[k] = MX(qv[k], qvmin);
        ql[k] = MX(ql[k], qlmin);
        qi[k] = MX(qi[k], qimin);
    }
    if (dqv > 1.e-20) {
        sum = 0.0;
        for (k = 1; k <= mkx; k++)
            if (qv[k] > 2.0 * qvmin) sum = sum + qv[k] * dp[k];
        aa = dqv * dp[1] / MX(1.e-20, sum);
        if (aa < 0.5) {
            for (k = 1; k <= mkx; k++) {
                if (qv[k] > 2.0 * qvmin) {
                    dum = aa * qv[k];
                    qv[k] = qv[k] - dum;
                    qvten[k] = qvten[k] - dum / dt;
                }
            }
        }
    }
}

/* findsp (uwshcu.F90:5164-5454) for one (i,k) point.  Returns 0, 2 (no convergence in 8 Newton
 * steps) or 3 (enthalpy not conserved).  Columns are independent: a column leaves the Newton loop
 * when its own dt/dq pass the tolerances, which is what the per-level loop does for each column. */
static int findsp_point(double q, double t, double p, double *tsp_o, double *qsp_o)
{
    double omeps, trinv, es, desdt, dqsdt, dgdt, gg, weight, hlatsb, hlatvp, hltalt, tterm, qs, tc,
        tt0, t1, q1, dtt, dq, qvd, a1, tmp, rair, r1b, c1, c2, c3, denom, dttol, dqtol, enin, enout,
        tlim, tsp, qsp;
    int doit, l, lflg, iter;
    omeps = 1.0 - S.epsqs;
    trinv = 1.0 / S.ttrice;
    a1 = 7.5 * LOG(10.0);
    rair = 287.04;
    c3 = rair * a1 / S.cpws;
    dttol = 1.e-4;
    dqtol = 1.e-4;
    tt0 = 273.15;
    iter = 8;
    dtt = 0.0;
    dq = 0.0;

    tlim = MN(MX(t, 173.0), 373.0);
    es = estblf(tlim);
    denom = p - omeps * es;
    qs = S.epsqs * es / denom;
    doit = 0;
    enout = 1.0;
    if (p > 5.0 * es && qs > 0.0 && qs < 0.5) {
        qs = MN(S.epsqs * es / denom, 1.0);
        tc = tlim - tt0;
        weight = MN(-tc * trinv, 1.0);
        hlatsb = S.hlatv + weight * S.hlatf;
        hlatvp = S.hlatv - 2369.0 * tc;
        if (tlim < tt0) hltalt = hlatsb;
        else hltalt = hlatvp;
        enin = S.cpws * tlim + hltalt * q;
        tmp = q - qs;
        c1 = hltalt * c3;
        c2 = (tlim + 36.0) * (tlim + 36.0);
        r1b = c2 / (c2 + c1 * qs);
        qvd = r1b * tmp;
        tsp = tlim + ((hltalt / S.cpws) * qvd);
        es = estblf(tsp);
        qsp = MN(S.epsqs * es / (p - omeps * es), 1.0);
    } else {
        doit = 1;
        tsp = tlim;
        qsp = q;
        enin = 1.0;
        hltalt = 0.0;
    }
    for (l = 1; l <= iter; l++) {
        if (doit != 0) break;
        es = estblf(tsp);
        qs = MN(S.epsqs * es / (p - omeps * es), 1.0);
        tc = tsp - tt0;
        lflg = (tc >= -S.ttrice && tc < 0.0);
        weight = MN(-tc * trinv, 1.0);
        hlatsb = S.hlatv + weight * S.hlatf;
        hlatvp = S.hlatv - 2369.0 * tc;
        if (tsp < tt0) hltalt = hlatsb;
        else hltalt = hlatvp;
        if (lflg) tterm = S.pcf[0] + tc * (S.pcf[1] + tc * (S.pcf[2] + tc * (S.pcf[3] + tc * S.pcf[4])));
        else tterm = 0.0;
        desdt = hltalt * es / (S.rgasv * tsp * tsp) + tterm * trinv;
        dqsdt = (S.epsqs + omeps * qs) / (p - omeps * es) * desdt;
        gg = enin - (S.cpws * tsp + hltalt * qsp);
        dgdt = -(S.cpws + hltalt * dqsdt);
        t1 = tsp - gg / dgdt;
        dtt = fabs(t1 - tsp) / t1;
        tsp = MX(t1, S.tmin);
        es = estblf(tsp);
        q1 = MN(S.epsqs * es / (p - omeps * es), 1.0);
        dq = fabs(q1 - qsp) / MX(q1, 1.e-12);
        qsp = q1;
        if (dtt < dttol && dq < dqtol) doit = 2;
        enout = S.cpws * tsp + hltalt * qsp;
        if (tsp < 174.16) doit = 4;
    }
    *tsp_o = tsp;
    *qsp_o = qsp;
    if (doit == 0 && (dtt > dttol || dq > dqtol)) return 2;
    if (doit == 2 && fabs((enin - enout) / (enin + enout)) > 1.e-4) return 3;
    return 0;
}

/* ------------------------------------------------------------------------- compute_uwshcu */

typedef struct {
    int mix, mkx, iend, ncnst;
    double dt;
    const double *ps0, *zs0, *p0, *z0, *dp0, *u0, *v0, *qv0, *ql0, *qi0, *t0, *s0, *tr0, *tke, *pblh;
    double *cush;
    double *umf, *slflx, *qtflx, *flxprc1, *flxsnow1, *qvten, *qlten, *qiten, *sten, *uten, *vten,
        *trten, *qrten, *qsten, *precip, *snow, *evapc, *cufrc, *qcu, *qlu, *qiu, *cbmf, *qc, *rliq;
    double *cnt, *cnb;
    const double *dpdry0;
    double *wu;
    const double *qw0;
    int *diag_int;
    double *diag_real;
    double *diag_level;
    const double *omega;   /* (mix, mkx) pressure velocity of compute_zwshcu; NULL: compute_uwshcu */
} uwo_io;

/* Per-level diagnostics (the Fortran's history fields, uwshcu.F90:4383-4433), array
 * (UWO_NDL, mkx+1, mix), levels bottom-up (k = 0..mkx as in compute_uwshcu) for both entries;
 * layer fields use rows 1..mkx and leave row 0 at zero. */
enum { UWO_DL_UFRC, UWO_DL_QTU, UWO_DL_THLU, UWO_DL_THVU, UWO_DL_UU, UWO_DL_VU, UWO_DL_UEMF,
       UWO_DL_FLXRAIN, UWO_DL_FLXSNOW, UWO_DL_FER, UWO_DL_FDR, UWO_DL_DWTEN, UWO_DL_DITEN, UWO_NDL };

static void put_diag_level(const uwo_io *A, int i, int mkx, const double *const *f)
{
    int j, k;
    if (!A->diag_level) return;
    for (j = 0; j < UWO_NDL; j++)
        for (k = 0; k <= mkx; k++) {
            const int layer = j >= UWO_DL_FER;
            A->diag_level[((size_t)j * (mkx + 1) + k) * A->mix + (i - 1)] = (layer && k == 0) ? 0.0 : (f ? f[j][k] : 0.0);
        }
}

/* Fortran (mix,0:mkx), (mix,mkx) and (mix,mkx,ncnst) element addresses; i and k as in Fortran. */
#define AI(a, i, k) (a)[(size_t)(k) * (size_t)A->mix + (size_t)((i) - 1)]
#define AL(a, i, k) (a)[(size_t)((k) - 1) * (size_t)A->mix + (size_t)((i) - 1)]
#define AT(a, i, k, m) (a)[((size_t)((m) - 1) * (size_t)A->mkx + (size_t)((k) - 1)) * (size_t)A->mix + (size_t)((i) - 1)]

enum {
    X_UWCU = 1 << 0, X_CONDEN = 1 << 1, X_KLCLMKX = 1 << 2, X_KLFCMKX = 1 << 3, X_UFRC = 1 << 4,
    X_WTW = 1 << 5, X_DRYCORE = 1 << 6, X_WU = 1 << 7, X_CUFILTER = 1 << 8, X_KINV1 = 1 << 9,
    X_REI = 1 << 10
};
enum {
    L_SHCU = 1 << 0, L_NEGCON = 1 << 1, L_UFRC = 1 << 2, L_PPEN = 1 << 3, L_EMF = 1 << 4,
    L_CINLCL = 1 << 5, L_CIN = 1 << 6, L_CBMF = 1 << 7, L_REI = 1 << 8, L_DELCIN = 1 << 9
};

/* One column of compute_uwshcu: uwshcu.F90:1220-4549.  Returns 0 or 1 (mu inconsistency). */
static int uw_column(const uwo_io *A, int i)
{
    const int mkx = A->mkx, ncnst = A->ncnst;
    const double dt = A->dt;
    const double xlv = S.xlv, xls = S.xls, cp = S.cp, zvir = S.zvir, r = S.r, g = S.g, p00 = S.p00,
                 rovcp = S.rovcp, rpen = S.rpen;
    const int niter_xc = 2, iter_cin = 2;
    const double rle = S.rle, rkm = S.rkm, rkfre = 1.0, rmaxfrac = 0.10, mumin1 = 0.906, rbuoy = 1.0,
                 rdrag = 1.0, epsvarw = 5.e-4, PGFc = 0.7, criqc = S.criqc, frc_rasn = 1.0, kevp = 2.e-6;
    const int ixnumliq = S.ixnumliq, ixnumice = S.ixnumice;
    int status_ret = 0;

    /* 1. inputs (uwshcu.F90:603-621) */
    double ps0[mkx + 1], zs0[mkx + 1], p0[mkx + 1], z0[mkx + 1], dp0[mkx + 1], dpdry0[mkx + 1],
        u0[mkx + 1], v0[mkx + 1], tke[mkx + 1], qv0[mkx + 1], ql0[mkx + 1], qi0[mkx + 1], t0[mkx + 1],
        s0[mkx + 1], tr0[ncnst + 1][mkx + 1], pblh, cush;
    /* 2. environment (:625-646) */
    double qt0[mkx + 1], thl0[mkx + 1], thvl0[mkx + 1], ssqt0[mkx + 1], ssthl0[mkx + 1],
        ssu0[mkx + 1], ssv0[mkx + 1], thv0bot[mkx + 1], thv0top[mkx + 1], thvl0bot[mkx + 1],
        thvl0top[mkx + 1], exn0[mkx + 1], exns0[mkx + 1], sstr0[ncnst + 1][mkx + 1];
    double qv0_star[mkx + 1], ql0_star[mkx + 1], qi0_star[mkx + 1], s0_star[mkx + 1];
    /* 3. convection (:650-755) */
    double umf[mkx + 1], emf[mkx + 1], qvten[mkx + 1], qlten[mkx + 1], qiten[mkx + 1], sten[mkx + 1],
        uten[mkx + 1], vten[mkx + 1], qrten[mkx + 1], qsten[mkx + 1], precip, snow, evapc[mkx + 1],
        slflx[mkx + 1], qtflx[mkx + 1], uflx[mkx + 1], vflx[mkx + 1], cufrc[mkx + 1], qcu[mkx + 1],
        qlu[mkx + 1], qiu[mkx + 1], dwten[mkx + 1], diten[mkx + 1], fer[mkx + 1], fdr[mkx + 1],
        uf[mkx + 1], vf[mkx + 1], qc[mkx + 1], qc_l[mkx + 1], qc_i[mkx + 1], qc_lm, qc_im, nc_lm,
        nc_im, ql_emf_kbup, qi_emf_kbup, nl_emf_kbup, ni_emf_kbup, rliq, cnt, cnb, qtten[mkx + 1],
        slten[mkx + 1], ufrc[mkx + 1], trten[ncnst + 1][mkx + 1], trflx[ncnst + 1][mkx + 1],
        trflx_d[mkx + 1], trflx_u[mkx + 1], trmin, pdelx, dum;
    double uemf[mkx + 1], comsub[mkx + 1], qlten_sink[mkx + 1], qiten_sink[mkx + 1],
        nlten_sink[mkx + 1], niten_sink[mkx + 1], thlten_sub, qtten_sub, qlten_sub, qiten_sub,
        nlten_sub, niten_sub, thl_prog, qt_prog;
    double wu[mkx + 1], thlu[mkx + 1], qtu[mkx + 1], uu[mkx + 1], vu[mkx + 1], thvu[mkx + 1],
        rei[mkx + 1], tru[ncnst + 1][mkx + 1];
    double thlu_emf[mkx + 1], qtu_emf[mkx + 1], uu_emf[mkx + 1], vu_emf[mkx + 1],
        tru_emf[ncnst + 1][mkx + 1];
    double flxrain[mkx + 1], flxsnow[mkx + 1], ntraprd[mkx + 1], ntsnprd[mkx + 1], snowmlt, subsat,
        evprain, evpsnow, evplimit, evplimit_rain, evplimit_snow, evpint_rain, evpint_snow;
    int k, m, kk, km1, kp1, iter_scaleh, iter_xc, id_check, status, klcl = 0, kinv = 0, krel = 0,
                                                                   klfc = 0, kbup = 0, kpen = 0, id_exit;
    double thlsrc = 0, qtsrc = 0, usrc = 0, vsrc = 0, thvlsrc = 0, uplus, vplus, trsrc[ncnst + 1],
           tre[ncnst + 1];
    double plcl = 0, plfc = 0, prel = 0, wrel, ee2, ud2, wtw = 0, wtwb = 0, xc = 0, cridis,
           scaleh, tscaleh, sigmaw, tkeavg = 0, dpsum, dpi, thvlmin = 0, thlxsat, qtxsat, thvxsat,
           x_cu = 0, x_en = 0, thv_x0, thv_x1, thj, qvj, qlj, qij, thvj, tj, thv0j, rho0j = 0, rhos0j,
           qse, cin = 0, cinlcl = 0, pe, dpe, exne, thvebot, thle, qte, ue, ve, thlue, qtue, wue, mu,
           mumin0, mumin2, mulcl, mulclstar, cbmf = 0, wcrit, winv, wlcl = 0, ufrcinv, ufrclcl = 0,
           exql, exqi, ppen = 0, thl0top, thl0bot, qt0bot, qt0top, thvubot, thvutop = 0,
           thlu_top = 0, qtu_top = 0, qlu_top, qiu_top, qlu_mid, qiu_mid, exntop, thl0lcl, qt0lcl,
           thv0lcl = 0, thv0rel, rho0inv, aquad, bquad, cquad, xc1 = 0, xc2 = 0, excessu, excess0,
           xsat, xs1 = 0, xs2 = 0, bogbot = 0, bogtop = 0, delbog, drage = 0, expfac, qlubelow = 0,
           qiubelow = 0, rainflx, snowflx, es1, qs1, gam1, qsat_arg, xsrc, xmean, xtop, xbot,
           xflx[mkx + 1], tmp1, tmp2, cbmflimit;
    (void)tj;
    (void)qlu_top;
    (void)qiu_top;
    (void)qse;
    (void)cbmflimit;
    /* implicit-CIN saves (:919-931) and temporaries (:935-954) */
    double qv0_s[mkx + 1], ql0_s[mkx + 1], qi0_s[mkx + 1], s0_s[mkx + 1], t0_s[mkx + 1],
        qvten_s[mkx + 1], qlten_s[mkx + 1], qiten_s[mkx + 1], qrten_s[mkx + 1], qsten_s[mkx + 1],
        sten_s[mkx + 1], evapc_s[mkx + 1], uten_s[mkx + 1], vten_s[mkx + 1], cufrc_s[mkx + 1],
        qcu_s[mkx + 1], qlu_s[mkx + 1], qiu_s[mkx + 1], qc_s[mkx + 1], umf_s[mkx + 1],
        slflx_s[mkx + 1], qtflx_s[mkx + 1], trten_s[ncnst + 1][mkx + 1];
    /* iteration-1 copies of the per-level diagnostics (:919-931) */
    double ufrc_s[mkx + 1], qtu_s[mkx + 1], thlu_s[mkx + 1], thvu_s[mkx + 1], uu_s[mkx + 1], vu_s[mkx + 1],
        uemf_s[mkx + 1], flxrain_s[mkx + 1], flxsnow_s[mkx + 1], fer_s[mkx + 1], fdr_s[mkx + 1],
        dwten_s[mkx + 1], diten_s[mkx + 1];
    const double *const diag_s[UWO_NDL] = {ufrc_s, qtu_s, thlu_s, thvu_s, uu_s, vu_s, uemf_s, flxrain_s,
                                           flxsnow_s, fer_s, fdr_s, dwten_s, diten_s};
    double cush_s = 0, precip_s = 0, snow_s = 0, cin_s = 0, rliq_s = 0, cbmf_s = 0, cnt_s = 0,
           cnb_s = 0, cinlcl_s = 0, plcl_s = 0, plfc_s = 0, pinv_s = 0, pbup_s = 0, ppen_s = 0,
           tkeavg_s = 0;
    int kinv_s = 0, klcl_s = 0, klfc_s = 0, krel_s = 0, kbup_s = 0, kpen_s = 0;
    double cin_i = 0, cin_f, del_CIN, ke = 0, alpha, cinlcl_i = 0;
    int iter;
    double qv0_o[mkx + 1], ql0_o[mkx + 1], qi0_o[mkx + 1], t0_o[mkx + 1], s0_o[mkx + 1],
        u0_o[mkx + 1], v0_o[mkx + 1], qt0_o[mkx + 1], thl0_o[mkx + 1], thvl0_o[mkx + 1],
        thv0bot_o[mkx + 1], thv0top_o[mkx + 1], thvl0bot_o[mkx + 1], thvl0top_o[mkx + 1],
        ssthl0_o[mkx + 1], ssqt0_o[mkx + 1], ssu0_o[mkx + 1], ssv0_o[mkx + 1];
    double tkeavg_o = 0, thvlmin_o = 0, qtsrc_o = 0, thvlsrc_o = 0, thlsrc_o = 0, usrc_o = 0,
           vsrc_o = 0, plcl_o = 0, plfc_o = 0, thv0lcl_o = 0;
    int kinv_o = 0, klcl_o = 0, klfc_o = 0;
    double tr0_o[ncnst + 1][mkx + 1], sstr0_o[ncnst + 1][mkx + 1], trsrc_o[ncnst + 1];
    int xflags = 0, lflags = 0;

    /* Output initialisation for this column (uwshcu.F90:1087-1124). */
    for (k = 0; k <= mkx; k++) {
        AI(A->umf, i, k) = 0.0;
        AI(A->slflx, i, k) = 0.0;
        AI(A->qtflx, i, k) = 0.0;
        AI(A->flxprc1, i, k) = 0.0;
        AI(A->flxsnow1, i, k) = 0.0;
        AI(A->wu, i, k) = 0.0;
    }
    for (k = 1; k <= mkx; k++) {
        AL(A->qvten, i, k) = 0.0;
        AL(A->qlten, i, k) = 0.0;
        AL(A->qiten, i, k) = 0.0;
        AL(A->sten, i, k) = 0.0;
        AL(A->uten, i, k) = 0.0;
        AL(A->vten, i, k) = 0.0;
        AL(A->qrten, i, k) = 0.0;
        AL(A->qsten, i, k) = 0.0;
        AL(A->evapc, i, k) = 0.0;
        AL(A->cufrc, i, k) = 0.0;
        AL(A->qcu, i, k) = 0.0;
        AL(A->qlu, i, k) = 0.0;
        AL(A->qiu, i, k) = 0.0;
        AL(A->qc, i, k) = 0.0;
        for (m = 1; m <= ncnst; m++) AT(A->trten, i, k, m) = 0.0;
    }
    A->precip[i - 1] = 0.0;
    A->snow[i - 1] = 0.0;
    A->cbmf[i - 1] = 0.0;
    A->rliq[i - 1] = 0.0;
    A->cnt[i - 1] = (double)mkx;
    A->cnb[i - 1] = 0.0;

    id_exit = 0;

    /* Define 1D inputs (:1226-1246) */
    for (k = 0; k <= mkx; k++) {
        ps0[k] = AI(A->ps0, i, k);
        zs0[k] = AI(A->zs0, i, k);
        tke[k] = AI(A->tke, i, k);
    }
    for (k = 1; k <= mkx; k++) {
        p0[k] = AL(A->p0, i, k);
        z0[k] = AL(A->z0, i, k);
        dp0[k] = AL(A->dp0, i, k);
        dpdry0[k] = AL(A->dpdry0, i, k);
        u0[k] = AL(A->u0, i, k);
        v0[k] = AL(A->v0, i, k);
        qv0[k] = AL(A->qv0, i, k);
        ql0[k] = AL(A->ql0, i, k);
        qi0[k] = AL(A->qi0, i, k);
        t0[k] = AL(A->t0, i, k);
        s0[k] = AL(A->s0, i, k);
        for (m = 1; m <= ncnst; m++) tr0[m][k] = AT(A->tr0, i, k, m);
    }
    pblh = A->pblh[i - 1];
    cush = A->cush[i - 1];

    /* 1. environmental variables (:1255-1259) */
    for (k = 1; k <= mkx; k++) exn0[k] = POW(p0[k] / p00, rovcp);
    for (k = 0; k <= mkx; k++) exns0[k] = POW(ps0[k] / p00, rovcp);
    for (k = 1; k <= mkx; k++) {
        qt0[k] = (qv0[k] + ql0[k] + qi0[k]);
        thl0[k] = (t0[k] - xlv * ql0[k] / cp - xls * qi0[k] / cp) / exn0[k];
        thvl0[k] = (1.0 + zvir * qt0[k]) * thl0[k];
    }
    /* 2. slopes (:1264-1270) */
    slope(mkx, thl0, p0, ssthl0);
    slope(mkx, qt0, p0, ssqt0);
    slope(mkx, u0, p0, ssu0);
    slope(mkx, v0, p0, ssv0);
    for (m = 1; m <= ncnst; m++) slope(mkx, tr0[m], p0, sstr0[m]);
    /* 3. thv0 at layer bottom/top (:1275-1299) */
    for (k = 1; k <= mkx; k++) {
        thl0bot = thl0[k] + ssthl0[k] * (ps0[k - 1] - p0[k]);
        qt0bot = qt0[k] + ssqt0[k] * (ps0[k - 1] - p0[k]);
        conden(ps0[k - 1], thl0bot, qt0bot, &thj, &qvj, &qlj, &qij, &qse, &id_check);
        if (id_check == 1) {
            xflags |= X_CONDEN;
            id_exit = 1;
            goto l333;
        }
        thv0bot[k] = thj * (1.0 + zvir * qvj - qlj - qij);
        thvl0bot[k] = thl0bot * (1.0 + zvir * qt0bot);
        thl0top = thl0[k] + ssthl0[k] * (ps0[k] - p0[k]);
        qt0top = qt0[k] + ssqt0[k] * (ps0[k] - p0[k]);
        conden(ps0[k], thl0top, qt0top, &thj, &qvj, &qlj, &qij, &qse, &id_check);
        if (id_check == 1) {
            xflags |= X_CONDEN;
            id_exit = 1;
            goto l333;
        }
        thv0top[k] = thj * (1.0 + zvir * qvj - qlj - qij);
        thvl0top[k] = thl0top * (1.0 + zvir * qt0top);
    }
    /* Save for iter_cin = 2 (:1306-1327) */
    for (k = 1; k <= mkx; k++) {
        qv0_o[k] = qv0[k];
        ql0_o[k] = ql0[k];
        qi0_o[k] = qi0[k];
        t0_o[k] = t0[k];
        s0_o[k] = s0[k];
        u0_o[k] = u0[k];
        v0_o[k] = v0[k];
        qt0_o[k] = qt0[k];
        thl0_o[k] = thl0[k];
        thvl0_o[k] = thvl0[k];
        ssthl0_o[k] = ssthl0[k];
        ssqt0_o[k] = ssqt0[k];
        thv0bot_o[k] = thv0bot[k];
        thv0top_o[k] = thv0top[k];
        thvl0bot_o[k] = thvl0bot[k];
        thvl0top_o[k] = thvl0top[k];
        ssu0_o[k] = ssu0[k];
        ssv0_o[k] = ssv0[k];
        for (m = 1; m <= ncnst; m++) {
            tr0_o[m][k] = tr0[m][k];
            sstr0_o[m][k] = sstr0[m][k];
        }
    }
    /* Initialize per-column variables (:1333-1408) */
    for (k = 0; k <= mkx; k++) {
        umf[k] = 0.0;
        emf[k] = 0.0;
        slflx[k] = 0.0;
        qtflx[k] = 0.0;
        uflx[k] = 0.0;
        vflx[k] = 0.0;
        ufrc[k] = 0.0;
        thlu[k] = 0.0;
        qtu[k] = 0.0;
        uu[k] = 0.0;
        vu[k] = 0.0;
        wu[k] = 0.0;
        thvu[k] = 0.0;
        thlu_emf[k] = 0.0;
        qtu_emf[k] = 0.0;
        uu_emf[k] = 0.0;
        vu_emf[k] = 0.0;
        uemf[k] = 0.0;
        for (m = 1; m <= ncnst; m++) {
            trflx[m][k] = 0.0;
            tru[m][k] = 0.0;
            tru_emf[m][k] = 0.0;
        }
    }
    for (k = 1; k <= mkx; k++) {
        qvten[k] = 0.0;
        qlten[k] = 0.0;
        qiten[k] = 0.0;
        sten[k] = 0.0;
        uten[k] = 0.0;
        vten[k] = 0.0;
        qrten[k] = 0.0;
        qsten[k] = 0.0;
        dwten[k] = 0.0;
        diten[k] = 0.0;
        evapc[k] = 0.0;
        cufrc[k] = 0.0;
        qcu[k] = 0.0;
        qlu[k] = 0.0;
        qiu[k] = 0.0;
        fer[k] = 0.0;
        fdr[k] = 0.0;
        qc[k] = 0.0;
        qc_l[k] = 0.0;
        qc_i[k] = 0.0;
        qtten[k] = 0.0;
        slten[k] = 0.0;
        comsub[k] = 0.0;
        qlten_sink[k] = 0.0;
        qiten_sink[k] = 0.0;
        nlten_sink[k] = 0.0;
        niten_sink[k] = 0.0;
        rei[k] = 0.0;
        uf[k] = 0.0;
        vf[k] = 0.0;
        for (m = 1; m <= ncnst; m++) trten[m][k] = 0.0;
    }
    precip = 0.0;
    snow = 0.0;
    cin = 0.0;
    cbmf = 0.0;
    rliq = 0.0;
    cnt = (double)mkx;
    cnb = 0.0;
    ufrclcl = 0.0;
    wlcl = 0.0;

    for (iter = 1; iter <= iter_cin; iter++) {
        tscaleh = cush;
        cush = -1.0;

        /* kinv (:1455-1468) */
        kinv = 1;
        for (k = mkx - 1; k >= 1; k--) {
            if ((pblh + 5.0 - zs0[k]) * (pblh + 5.0 - zs0[k + 1]) < 0.0) {
                kinv = k + 1;
                break;
            }
        }
        if (kinv <= 1) {
            xflags |= X_KINV1;
            id_exit = 1;
            goto l333;
        }
        /* tkeavg, thvlmin (:1484-1499) */
        dpsum = 0.0;
        tkeavg = 0.0;
        thvlmin = 1000.0;
        for (k = 0; k <= kinv - 1; k++) {
            if (k == 0) dpi = ps0[0] - p0[1];
            else if (k == (kinv - 1)) dpi = p0[kinv - 1] - ps0[kinv - 1];
            else dpi = p0[k] - p0[k + 1];
            dpsum = dpsum + dpi;
            tkeavg = tkeavg + dpi * tke[k];
            if (k != 0) thvlmin = MN(thvlmin, MN(thvl0bot[k], thvl0top[k]));
        }
        tkeavg = tkeavg / dpsum;
        /* source air (:1509-1516) */
        qtsrc = qt0[1];
        thvlsrc = thvlmin;
        thlsrc = thvlsrc / (1.0 + zvir * qtsrc);
        usrc = u0[kinv - 1] + ssu0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        vsrc = v0[kinv - 1] + ssv0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        for (m = 1; m <= ncnst; m++) trsrc[m] = tr0[m][1];
        /* LCL (:1533-1549) */
        plcl = qsinvert(qtsrc, thlsrc, ps0[0]);
        klcl = mkx;
        for (k = 0; k <= mkx; k++) {
            if (ps0[k] < plcl) {
                klcl = k;
                break;
            }
        }
        klcl = MX(1, klcl);
        if (plcl < 30000.0) {
            xflags |= X_KLCLMKX;
            id_exit = 1;
            goto l333;
        }
        /* thv0lcl (:1559-1567) */
        thl0lcl = thl0[klcl] + ssthl0[klcl] * (plcl - p0[klcl]);
        qt0lcl = qt0[klcl] + ssqt0[klcl] * (plcl - p0[klcl]);
        conden(plcl, thl0lcl, qt0lcl, &thj, &qvj, &qlj, &qij, &qse, &id_check);
        if (id_check == 1) {
            xflags |= X_CONDEN;
            id_exit = 1;
            goto l333;
        }
        thv0lcl = thj * (1.0 + zvir * qvj - qlj - qij);

        /* CIN (:1592-1685) */
        cin = 0.0;
        cinlcl = 0.0;
        plfc = 0.0;
        klfc = mkx;
        if (klcl >= kinv) {
            for (k = kinv; k <= mkx - 1; k++) {
                if (k < klcl) {
                    thvubot = thvlsrc;
                    thvutop = thvlsrc;
                    cin = cin + single_cin(ps0[k - 1], thv0bot[k], ps0[k], thv0top[k], thvubot, thvutop);
                } else if (k == klcl) {
                    thvubot = thvlsrc;
                    thvutop = thvlsrc;
                    cin = cin + single_cin(ps0[k - 1], thv0bot[k], plcl, thv0lcl, thvubot, thvutop);
                    if (cin < 0.0) lflags |= L_CINLCL;
                    cinlcl = MX(cin, 0.0);
                    cin = cinlcl;
                    thvubot = thvlsrc;
                    conden(ps0[k], thlsrc, qtsrc, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                    if (id_check == 1) {
                        xflags |= X_CONDEN;
                        id_exit = 1;
                        goto l333;
                    }
                    thvutop = thj * (1.0 + zvir * qvj - qlj - qij);
                    getbuoy(plcl, thv0lcl, ps0[k], thv0top[k], thvubot, thvutop, &plfc, &cin);
                    if (plfc > 0.0) {
                        klfc = k;
                        goto l35;
                    }
                } else {
                    thvubot = thvutop;
                    conden(ps0[k], thlsrc, qtsrc, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                    if (id_check == 1) {
                        xflags |= X_CONDEN;
                        id_exit = 1;
                        goto l333;
                    }
                    thvutop = thj * (1.0 + zvir * qvj - qlj - qij);
                    getbuoy(ps0[k - 1], thv0bot[k], ps0[k], thv0top[k], thvubot, thvutop, &plfc, &cin);
                    if (plfc > 0.0) {
                        klfc = k;
                        goto l35;
                    }
                }
            }
        } else {
            cinlcl = 0.0;
            for (k = kinv; k <= mkx - 1; k++) {
                conden(ps0[k - 1], thlsrc, qtsrc, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                thvubot = thj * (1.0 + zvir * qvj - qlj - qij);
                conden(ps0[k], thlsrc, qtsrc, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                thvutop = thj * (1.0 + zvir * qvj - qlj - qij);
                getbuoy(ps0[k - 1], thv0bot[k], ps0[k], thv0top[k], thvubot, thvutop, &plfc, &cin);
                if (plfc > 0.0) {
                    klfc = k;
                    goto l35;
                }
            }
        }
    l35:
        if (cin < 0.0) lflags |= L_CIN;
        cin = MX(0.0, cin);
        if (klfc >= mkx) {
            klfc = mkx;
            xflags |= X_KLFCMKX;
            id_exit = 1;
            goto l333;
        }
        /* Save for implicit CIN (:1693-1713) */
        if (iter == 1) {
            cin_i = cin;
            cinlcl_i = cinlcl;
            ke = rbuoy / (rkfre * tkeavg + epsvarw);
            kinv_o = kinv;
            klcl_o = klcl;
            klfc_o = klfc;
            plcl_o = plcl;
            plfc_o = plfc;
            tkeavg_o = tkeavg;
            thvlmin_o = thvlmin;
            qtsrc_o = qtsrc;
            thvlsrc_o = thvlsrc;
            thlsrc_o = thlsrc;
            usrc_o = usrc;
            vsrc_o = vsrc;
            thv0lcl_o = thv0lcl;
            for (m = 1; m <= ncnst; m++) trsrc_o[m] = trsrc[m];
        }
        /* Implicit CIN (:1736-2014) */
        if (iter != 1) {
            cin_f = cin;
            del_CIN = cin_f - cin_i;
            if (del_CIN > 0.0) {
                alpha = compute_alpha(del_CIN, ke);
                cin = cin_i + alpha * del_CIN;
                cinlcl = cinlcl_i;
                kinv = kinv_o;
                klcl = klcl_o;
                klfc = klfc_o;
                plcl = plcl_o;
                plfc = plfc_o;
                tkeavg = tkeavg_o;
                thvlmin = thvlmin_o;
                qtsrc = qtsrc_o;
                thvlsrc = thvlsrc_o;
                thlsrc = thlsrc_o;
                usrc = usrc_o;
                vsrc = vsrc_o;
                thv0lcl = thv0lcl_o;
                for (m = 1; m <= ncnst; m++) trsrc[m] = trsrc_o[m];
                for (k = 1; k <= mkx; k++) {
                    qv0[k] = qv0_o[k];
                    ql0[k] = ql0_o[k];
                    qi0[k] = qi0_o[k];
                    t0[k] = t0_o[k];
                    s0[k] = s0_o[k];
                    u0[k] = u0_o[k];
                    v0[k] = v0_o[k];
                    qt0[k] = qt0_o[k];
                    thl0[k] = thl0_o[k];
                    thvl0[k] = thvl0_o[k];
                    ssthl0[k] = ssthl0_o[k];
                    ssqt0[k] = ssqt0_o[k];
                    thv0bot[k] = thv0bot_o[k];
                    thv0top[k] = thv0top_o[k];
                    thvl0bot[k] = thvl0bot_o[k];
                    thvl0top[k] = thvl0top_o[k];
                    ssu0[k] = ssu0_o[k];
                    ssv0[k] = ssv0_o[k];
                    for (m = 1; m <= ncnst; m++) {
                        tr0[m][k] = tr0_o[m][k];
                        sstr0[m][k] = sstr0_o[m][k];
                    }
                }
                for (k = 0; k <= mkx; k++) {
                    umf[k] = 0.0;
                    emf[k] = 0.0;
                    slflx[k] = 0.0;
                    qtflx[k] = 0.0;
                    uflx[k] = 0.0;
                    vflx[k] = 0.0;
                    ufrc[k] = 0.0;
                    thlu[k] = 0.0;
                    qtu[k] = 0.0;
                    uu[k] = 0.0;
                    vu[k] = 0.0;
                    wu[k] = 0.0;
                    thvu[k] = 0.0;
                    thlu_emf[k] = 0.0;
                    qtu_emf[k] = 0.0;
                    uu_emf[k] = 0.0;
                    vu_emf[k] = 0.0;
                    for (m = 1; m <= ncnst; m++) {
                        trflx[m][k] = 0.0;
                        tru[m][k] = 0.0;
                        tru_emf[m][k] = 0.0;
                    }
                }
                for (k = 1; k <= mkx; k++) {
                    qvten[k] = 0.0;
                    qlten[k] = 0.0;
                    qiten[k] = 0.0;
                    sten[k] = 0.0;
                    uten[k] = 0.0;
                    vten[k] = 0.0;
                    qrten[k] = 0.0;
                    qsten[k] = 0.0;
                    dwten[k] = 0.0;
                    diten[k] = 0.0;
                    evapc[k] = 0.0;
                    cufrc[k] = 0.0;
                    qcu[k] = 0.0;
                    qlu[k] = 0.0;
                    qiu[k] = 0.0;
                    fer[k] = 0.0;
                    fdr[k] = 0.0;
                    qc[k] = 0.0;
                    qc_l[k] = 0.0;
                    qc_i[k] = 0.0;
                    qtten[k] = 0.0;
                    slten[k] = 0.0;
                    for (m = 1; m <= ncnst; m++) trten[m][k] = 0.0;
                }
                precip = 0.0;
                snow = 0.0;
                rliq = 0.0;
                cbmf = 0.0;
                cnt = (double)mkx;
                cnb = 0.0;
                ufrclcl = 0.0;
                wlcl = 0.0;
            } else {
                /* del_CIN <= 0: write the iter_cin = 1 outputs and leave (:1891-2011).
                 * flxprc1/flxsnow1 keep their initial zeros on this path. */
                lflags |= L_DELCIN;
                for (k = 0; k <= mkx; k++) {
                    AI(A->umf, i, k) = umf_s[k];
                    AI(A->wu, i, k) = wu[k];
                    AI(A->slflx, i, k) = slflx_s[k];
                    AI(A->qtflx, i, k) = qtflx_s[k];
                }
                for (k = 1; k <= mkx; k++) {
                    AL(A->qvten, i, k) = qvten_s[k];
                    AL(A->qlten, i, k) = qlten_s[k];
                    AL(A->qiten, i, k) = qiten_s[k];
                    AL(A->sten, i, k) = sten_s[k];
                    AL(A->uten, i, k) = uten_s[k];
                    AL(A->vten, i, k) = vten_s[k];
                    AL(A->qrten, i, k) = qrten_s[k];
                    AL(A->qsten, i, k) = qsten_s[k];
                    AL(A->evapc, i, k) = evapc_s[k];
                    AL(A->cufrc, i, k) = cufrc_s[k];
                    AL(A->qcu, i, k) = qcu_s[k];
                    AL(A->qlu, i, k) = qlu_s[k];
                    AL(A->qiu, i, k) = qiu_s[k];
                    AL(A->qc, i, k) = qc_s[k];
                    for (m = 1; m <= ncnst; m++) AT(A->trten, i, k, m) = trten_s[m][k];
                }
                A->precip[i - 1] = precip_s;
                A->snow[i - 1] = snow_s;
                A->cush[i - 1] = cush_s;
                A->cbmf[i - 1] = cbmf_s;
                A->rliq[i - 1] = rliq_s;
                A->cnt[i - 1] = cnt_s;
                A->cnb[i - 1] = cnb_s;
                if (A->diag_real) {
                    double *dr = A->diag_real + (size_t)(i - 1); const size_t ds = (size_t)A->mix;
                    dr[UWO_DR_CIN * ds] = cin_s;
                    dr[UWO_DR_CINLCL * ds] = cinlcl_s;
                    dr[UWO_DR_PLCL * ds] = plcl_s;
                    dr[UWO_DR_PLFC * ds] = plfc_s;
                    dr[UWO_DR_PINV * ds] = pinv_s;
                    dr[UWO_DR_PBUP * ds] = pbup_s;
                    dr[UWO_DR_PPEN * ds] = ppen_s;
                    dr[UWO_DR_TKEAVG * ds] = tkeavg_s;
                }
                put_diag_level(A, i, mkx, diag_s);
                kinv = kinv_s;
                klcl = klcl_s;
                klfc = klfc_s;
                krel = krel_s;
                kbup = kbup_s;
                kpen = kpen_s;
                id_exit = 0;
                goto l333;
            }
        }

        /* Release level (:2035-2043) */
        if (klcl < kinv) {
            krel = kinv;
            prel = ps0[krel - 1];
            thv0rel = thv0bot[krel];
        } else {
            krel = klcl;
            prel = plcl;
            thv0rel = thv0lcl;
        }
        /* Closure (:2092-2184); compute_zwshcu computes rho0inv first (zwshcu.F90:2277) and lowers
         * wcrit by the large-scale ascent at the PBL top (zwshcu.F90:2295-2303) */
        wcrit = sqrt(2.0 * cin * rbuoy);
        rho0inv = ps0[kinv - 1] / (r * thv0top[kinv - 1] * exns0[kinv - 1]);
        sigmaw = sqrt(rkfre * tkeavg + epsvarw);
        if (A->omega) {
            if (S.zw_lf) {
                double tmp1 = MN(MX(-AL(A->omega, i, kinv - 1), 0.0), 3.0);
                wcrit = wcrit - tmp1 / rho0inv / 9.8;
                wcrit = MX(wcrit, 0.0);
            }
            wcrit = wcrit * S.zw_fwcrit;
        }
        mu = wcrit / sigmaw / 1.4142;
        if (mu >= 3.0) {
            id_exit = 1;
            goto l333;
        }
        cbmf = (rho0inv * sigmaw / 2.5066) * EXP(-(mu * mu));
        cbmflimit = 0.9 * dp0[kinv - 1] / g / dt;
        mumin0 = 0.0;
        if (cbmf > cbmflimit) mumin0 = sqrt(-LOG(2.5066 * cbmflimit / rho0inv / sigmaw));
        mu = MX(MX(mu, mumin0), mumin1);
        mulcl = sqrt(2.0 * cinlcl * rbuoy) / 1.4142 / sigmaw;
        {
            double ta = EXP(-(mu * mu)) / 2.5066, te = ERFC(mu);
            mulclstar = sqrt(MX(0.0, 2.0 * (ta * ta) * (1.0 / (te * te) - 0.25 / (rmaxfrac * rmaxfrac))));
        }
        if (mulcl > 1.e-8 && mulcl > mulclstar) {
            mumin2 = compute_mumin2(mulcl, rmaxfrac, mu);
            if (mu > mumin2) status_ret = 1;
            mu = MX(mu, mumin2);
            if (mu == mumin2) lflags |= L_UFRC;
        }
        if (mu == mumin0) lflags |= L_CBMF;
        if (mu == mumin1) lflags |= L_UFRC;
        cbmf = (rho0inv * sigmaw / 2.5066) * EXP(-(mu * mu));
        winv = sigmaw * (2.0 / 2.5066) * EXP(-(mu * mu)) / ERFC(mu);
        ufrcinv = cbmf / winv / rho0inv;
        (void)ufrcinv;
        wtw = winv * winv - 2.0 * cinlcl * rbuoy;
        if (wtw <= 0.0) {
            xflags |= X_WTW;
            id_exit = 1;
            goto l333;
        }
        wlcl = sqrt(wtw);
        ufrclcl = cbmf / wlcl / rho0inv;
        wrel = wlcl;
        if (ufrclcl <= 0.0001) {
            xflags |= X_UFRC;
            id_exit = 1;
            goto l333;
        }
        ufrc[krel - 1] = ufrclcl;
        for (k = kinv - 1; k <= krel - 1; k++) {
            umf[k] = cbmf;
            wu[k] = winv;
        }
        /* Updraft at the release level (:2205-2236) */
        emf[krel - 1] = 0.0;
        umf[krel - 1] = cbmf;
        wu[krel - 1] = wrel;
        thlu[krel - 1] = thlsrc;
        qtu[krel - 1] = qtsrc;
        conden(prel, thlsrc, qtsrc, &thj, &qvj, &qlj, &qij, &qse, &id_check);
        if (id_check == 1) {
            xflags |= X_CONDEN;
            id_exit = 1;
            goto l333;
        }
        thvu[krel - 1] = thj * (1.0 + zvir * qvj - qlj - qij);
        uplus = 0.0;
        vplus = 0.0;
        if (krel == kinv) {
            uplus = PGFc * ssu0[kinv] * (prel - ps0[kinv - 1]);
            vplus = PGFc * ssv0[kinv] * (prel - ps0[kinv - 1]);
        } else {
            for (k = kinv; k <= MX(krel - 1, kinv); k++) {
                uplus = uplus + PGFc * ssu0[k] * (ps0[k] - ps0[k - 1]);
                vplus = vplus + PGFc * ssv0[k] * (ps0[k] - ps0[k - 1]);
            }
            uplus = uplus + PGFc * ssu0[krel] * (prel - ps0[krel - 1]);
            vplus = vplus + PGFc * ssv0[krel] * (prel - ps0[krel - 1]);
        }
        uu[krel - 1] = usrc + uplus;
        vu[krel - 1] = vsrc + vplus;
        for (m = 1; m <= ncnst; m++) tru[m][krel - 1] = trsrc[m];

        scaleh = tscaleh;
        if (tscaleh < 0.0) scaleh = 1000.0;

        /* iter_scaleh loop (:2306-2952) */
        for (iter_scaleh = 1; iter_scaleh <= 3; iter_scaleh++) {
            kbup = krel;
            kpen = krel;
            wtw = wlcl * wlcl;
            pe = 0.5 * (prel + ps0[krel]);
            dpe = prel - ps0[krel];
            exne = exnf(pe);
            thvebot = thv0rel;
            thle = thl0[krel] + ssthl0[krel] * (pe - p0[krel]);
            qte = qt0[krel] + ssqt0[krel] * (pe - p0[krel]);
            ue = u0[krel] + ssu0[krel] * (pe - p0[krel]);
            ve = v0[krel] + ssv0[krel] * (pe - p0[krel]);
            for (m = 1; m <= ncnst; m++) tre[m] = tr0[m][krel] + sstr0[m][krel] * (pe - p0[krel]);

            for (k = krel; k <= mkx - 1; k++) {
                km1 = k - 1;
                thlue = thlu[km1];
                qtue = qtu[km1];
                wue = wu[km1];
                wtwb = wtw;
                for (iter_xc = 1; iter_xc <= niter_xc; iter_xc++) {
                    wtw = wu[km1] * wu[km1];
                    conden(pe, thle, qte, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                    if (id_check == 1) {
                        xflags |= X_CONDEN;
                        id_exit = 1;
                        goto l333;
                    }
                    thv0j = thj * (1.0 + zvir * qvj - qlj - qij);
                    rho0j = pe / (r * thv0j * exne);
                    qsat_arg = thle * exne;
                    qsat1(qsat_arg, pe, &es1, &qs1, &gam1);
                    excess0 = qte - qs1;
                    conden(pe, thlue, qtue, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                    if (id_check == 1) {
                        xflags |= X_CONDEN;
                        id_exit = 1;
                        goto l333;
                    }
                    if ((qlj + qij) > criqc) {
                        exql = ((qlj + qij) - criqc) * qlj / (qlj + qij);
                        exqi = ((qlj + qij) - criqc) * qij / (qlj + qij);
                        qtue = qtue - exql - exqi;
                        thlue = thlue + (xlv / cp / exne) * exql + (xls / cp / exne) * exqi;
                    }
                    conden(pe, thlue, qtue, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                    if (id_check == 1) {
                        xflags |= X_CONDEN;
                        id_exit = 1;
                        goto l333;
                    }
                    thvj = thj * (1.0 + zvir * qvj - qlj - qij);
                    tj = thj * exne;
                    qsat_arg = thlue * exne;
                    qsat1(qsat_arg, pe, &es1, &qs1, &gam1);
                    excessu = qtue - qs1;
                    cridis = rle * scaleh;
                    if ((excessu <= 0.0 && excess0 <= 0.0) || (excessu >= 0.0 && excess0 >= 0.0)) {
                        xc = MN(1.0, MX(0.0, 1.0 - 2.0 * rbuoy * g * cridis / (wue * wue) * (1.0 - thvj / thv0j)));
                        aquad = 0.0;
                        bquad = 0.0;
                        cquad = 0.0;
                    } else {
                        xsat = excessu / (excessu - excess0);
                        thlxsat = thlue + xsat * (thle - thlue);
                        qtxsat = qtue + xsat * (qte - qtue);
                        conden(pe, thlxsat, qtxsat, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                        if (id_check == 1) {
                            xflags |= X_CONDEN;
                            id_exit = 1;
                            goto l333;
                        }
                        thvxsat = thj * (1.0 + zvir * qvj - qlj - qij);
                        for (kk = 1; kk <= 2; kk++) {
                            if (kk == 1) {
                                thv_x0 = thvj;
                                thv_x1 = (1.0 - 1.0 / xsat) * thvj + (1.0 / xsat) * thvxsat;
                            } else {
                                thv_x1 = thv0j;
                                thv_x0 = (xsat / (xsat - 1.0)) * thv0j + (1.0 / (1.0 - xsat)) * thvxsat;
                            }
                            aquad = wue * wue;
                            bquad = 2.0 * rbuoy * g * cridis * (thv_x1 - thv_x0) / thv0j - 2.0 * (wue * wue);
                            cquad = 2.0 * rbuoy * g * cridis * (thv_x0 - thv0j) / thv0j + (wue * wue);
                            if (kk == 1) {
                                if ((bquad * bquad - 4.0 * aquad * cquad) >= 0.0) {
                                    roots(aquad, bquad, cquad, &xs1, &xs2, &status);
                                    x_cu = MN(1.0, MX(0.0, MN(xsat, MN(xs1, xs2))));
                                } else {
                                    x_cu = xsat;
                                }
                            } else {
                                if ((bquad * bquad - 4.0 * aquad * cquad) >= 0.0) {
                                    roots(aquad, bquad, cquad, &xs1, &xs2, &status);
                                    x_en = MN(1.0, MX(0.0, MX(xsat, MN(xs1, xs2))));
                                } else {
                                    x_en = 1.0;
                                }
                            }
                        }
                        if (x_cu == xsat) xc = MX(x_cu, x_en);
                        else xc = x_cu;
                    }
                    ee2 = xc * xc;
                    ud2 = 1.0 - 2.0 * xc + xc * xc;
                    rei[k] = (0.5 * rkm / z0[k] / g / rho0j);
                    if (xc > 0.5) rei[k] = MN(rei[k], 0.9 * LOG(dp0[k] / g / dt / umf[km1] + 1.0) / dpe / (2.0 * xc - 1.0));
                    fer[k] = rei[k] * ee2;
                    fdr[k] = rei[k] * ud2;
                    /* compute_zwshcu's entrainment option (zwshcu.F90:2818-2844) */
                    if (A->omega && S.zw_ent) {
                        double fer_min;
                        bogbot = rbuoy * (thvu[km1] / thvebot - 1.0) * g;
                        fer[k] = S.zw_ent0 * bogbot / MX(wue * wue, 1.0e-4);
                        fer_min = 0.0;
                        if (bogbot > 1.e-4) fer_min = 1.e-4;
                        fer[k] = MN(MX(fer[k], fer_min), 3.0e-2);
                    }
                    umf[k] = umf[km1] * EXP(dpe * (fer[k] - fdr[k]));
                    emf[k] = 0.0;
                    if (fer[k] * dpe < 1.e-4) {
                        thlu[k] = thlu[km1] + (thle + ssthl0[k] * dpe / 2.0 - thlu[km1]) * fer[k] * dpe;
                        qtu[k] = qtu[km1] + (qte + ssqt0[k] * dpe / 2.0 - qtu[km1]) * fer[k] * dpe;
                        uu[k] = uu[km1] + (ue + ssu0[k] * dpe / 2.0 - uu[km1]) * fer[k] * dpe - PGFc * ssu0[k] * dpe;
                        vu[k] = vu[km1] + (ve + ssv0[k] * dpe / 2.0 - vu[km1]) * fer[k] * dpe - PGFc * ssv0[k] * dpe;
                        for (m = 1; m <= ncnst; m++)
                            tru[m][k] = tru[m][km1] + (tre[m] + sstr0[m][k] * dpe / 2.0 - tru[m][km1]) * fer[k] * dpe;
                    } else {
                        thlu[k] = (thle + ssthl0[k] / fer[k] - ssthl0[k] * dpe / 2.0) -
                                  (thle + ssthl0[k] * dpe / 2.0 - thlu[km1] + ssthl0[k] / fer[k]) * EXP(-fer[k] * dpe);
                        qtu[k] = (qte + ssqt0[k] / fer[k] - ssqt0[k] * dpe / 2.0) -
                                 (qte + ssqt0[k] * dpe / 2.0 - qtu[km1] + ssqt0[k] / fer[k]) * EXP(-fer[k] * dpe);
                        uu[k] = (ue + (1.0 - PGFc) * ssu0[k] / fer[k] - ssu0[k] * dpe / 2.0) -
                                (ue + ssu0[k] * dpe / 2.0 - uu[km1] + (1.0 - PGFc) * ssu0[k] / fer[k]) * EXP(-fer[k] * dpe);
                        vu[k] = (ve + (1.0 - PGFc) * ssv0[k] / fer[k] - ssv0[k] * dpe / 2.0) -
                                (ve + ssv0[k] * dpe / 2.0 - vu[km1] + (1.0 - PGFc) * ssv0[k] / fer[k]) * EXP(-fer[k] * dpe);
                        for (m = 1; m <= ncnst; m++)
                            tru[m][k] = (tre[m] + sstr0[m][k] / fer[k] - sstr0[m][k] * dpe / 2.0) -
                                        (tre[m] + sstr0[m][k] * dpe / 2.0 - tru[m][km1] + sstr0[m][k] / fer[k]) * EXP(-fer[k] * dpe);
                    }
                    conden(ps0[k], thlu[k], qtu[k], &thj, &qvj, &qlj, &qij, &qse, &id_check);
                    if (id_check == 1) {
                        xflags |= X_CONDEN;
                        id_exit = 1;
                        goto l333;
                    }
                    if ((qlj + qij) > criqc) {
                        exql = ((qlj + qij) - criqc) * qlj / (qlj + qij);
                        exqi = ((qlj + qij) - criqc) * qij / (qlj + qij);
                        qtu[k] = qtu[k] - exql - exqi;
                        thlu[k] = thlu[k] + (xlv / cp / exns0[k]) * exql + (xls / cp / exns0[k]) * exqi;
                        dwten[k] = exql;
                        diten[k] = exqi;
                    } else {
                        dwten[k] = 0.0;
                        diten[k] = 0.0;
                    }
                    conden(ps0[k], thlu[k], qtu[k], &thj, &qvj, &qlj, &qij, &qse, &id_check);
                    if (id_check == 1) {
                        xflags |= X_CONDEN;
                        id_exit = 1;
                        goto l333;
                    }
                    thvu[k] = thj * (1.0 + zvir * qvj - qlj - qij);
                    bogbot = rbuoy * (thvu[km1] / thvebot - 1.0);
                    bogtop = rbuoy * (thvu[k] / thv0top[k] - 1.0);
                    delbog = bogtop - bogbot;
                    drage = fer[k] * (1.0 + rdrag);
                    expfac = EXP(-2.0 * drage * dpe);
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
                        goto l111;
                    }
                }
            l111:
                if (umf[k] == 0.0) wtw = -1.0;
                if (bogtop > 0.0 && wtw > 0.0) kbup = k;
                if (wtw <= 0.0) {
                    kpen = k;
                    goto l45;
                }
                wu[k] = sqrt(wtw);
                if (wu[k] > 100.0) {
                    xflags |= X_WU;
                    id_exit = 1;
                    goto l333;
                }
                rhos0j = ps0[k] / (r * 0.5 * (thv0bot[k + 1] + thv0top[k]) * exns0[k]);
                ufrc[k] = umf[k] / (rhos0j * wu[k]);
                if (ufrc[k] > rmaxfrac) {
                    lflags |= L_UFRC;
                    ufrc[k] = rmaxfrac;
                    umf[k] = rmaxfrac * rhos0j * wu[k];
                    fdr[k] = fer[k] - LOG(umf[k] / umf[km1]) / dpe;
                }
                pe = p0[k + 1];
                dpe = dp0[k + 1];
                exne = exn0[k + 1];
                thvebot = thv0bot[k + 1];
                thle = thl0[k + 1];
                qte = qt0[k + 1];
                ue = u0[k + 1];
                ve = v0[k + 1];
                for (m = 1; m <= ncnst; m++) tre[m] = tr0[m][k + 1];
            }
        l45:
            /* Penetration depth (:2884-2907) */
            if (drage == 0.0) {
                aquad = (bogtop - bogbot) / (ps0[kpen] - ps0[kpen - 1]);
                bquad = 2.0 * bogbot;
                cquad = -(wu[kpen - 1] * wu[kpen - 1]) * rho0j;
                roots(aquad, bquad, cquad, &xc1, &xc2, &status);
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
            if (ppen == -dp0[kpen] || ppen == 0.0) lflags |= L_PPEN;
            /* Condensate at the cumulus top (:2917-2942) */
            if (fer[kpen] * (-ppen) < 1.e-4) {
                thlu_top = thlu[kpen - 1] + (thl0[kpen] + ssthl0[kpen] * (-ppen) / 2.0 - thlu[kpen - 1]) * fer[kpen] * (-ppen);
                qtu_top = qtu[kpen - 1] + (qt0[kpen] + ssqt0[kpen] * (-ppen) / 2.0 - qtu[kpen - 1]) * fer[kpen] * (-ppen);
            } else {
                thlu_top = (thl0[kpen] + ssthl0[kpen] / fer[kpen] - ssthl0[kpen] * (-ppen) / 2.0) -
                           (thl0[kpen] + ssthl0[kpen] * (-ppen) / 2.0 - thlu[kpen - 1] + ssthl0[kpen] / fer[kpen]) * EXP(-fer[kpen] * (-ppen));
                qtu_top = (qt0[kpen] + ssqt0[kpen] / fer[kpen] - ssqt0[kpen] * (-ppen) / 2.0) -
                          (qt0[kpen] + ssqt0[kpen] * (-ppen) / 2.0 - qtu[kpen - 1] + ssqt0[kpen] / fer[kpen]) * EXP(-fer[kpen] * (-ppen));
            }
            conden(ps0[kpen - 1] + ppen, thlu_top, qtu_top, &thj, &qvj, &qlj, &qij, &qse, &id_check);
            if (id_check == 1) {
                xflags |= X_CONDEN;
                id_exit = 1;
                goto l333;
            }
            exntop = POW((ps0[kpen - 1] + ppen) / p00, rovcp);
            if ((qlj + qij) > criqc) {
                dwten[kpen] = ((qlj + qij) - criqc) * qlj / (qlj + qij);
                diten[kpen] = ((qlj + qij) - criqc) * qij / (qlj + qij);
                qtu_top = qtu_top - dwten[kpen] - diten[kpen];
                thlu_top = thlu_top + (xlv / cp / exntop) * dwten[kpen] + (xls / cp / exntop) * diten[kpen];
            } else {
                dwten[kpen] = 0.0;
                diten[kpen] = 0.0;
            }
            rhos0j = ps0[kpen - 1] / (r * 0.5 * (thv0bot[kpen] + thv0top[kpen - 1]) * exns0[kpen - 1]);
            cush = zs0[kpen - 1] - ppen / rhos0j / g;
            scaleh = cush;
        }

        /* forcedCu filter (:2964-2992) */
        if (kbup == krel) {
            lflags |= L_SHCU;
            xflags |= X_CUFILTER;
            id_exit = 1;
            goto l333;
        } else {
            lflags &= ~L_SHCU;
        }
        /* Clean above kpen (:3010-3016) */
        for (k = kpen; k <= mkx; k++) {
            umf[k] = 0.0;
            emf[k] = 0.0;
            ufrc[k] = 0.0;
        }
        for (k = kpen + 1; k <= mkx; k++) {
            dwten[k] = 0.0;
            diten[k] = 0.0;
            fer[k] = 0.0;
            fdr[k] = 0.0;
        }
        /* Penetrative entrainment (:3055-3183) */
        for (k = 0; k <= mkx; k++) {
            thlu_emf[k] = thlu[k];
            qtu_emf[k] = qtu[k];
            uu_emf[k] = uu[k];
            vu_emf[k] = vu[k];
            for (m = 1; m <= ncnst; m++) tru_emf[m][k] = tru[m][k];
        }
        for (k = kpen - 1; k >= kbup; k--) {
            rhos0j = ps0[k] / (r * 0.5 * (thv0bot[k + 1] + thv0top[k]) * exns0[k]);
            if (k == kpen - 1) {
                if ((umf[k] * ppen * rei[kpen] * rpen) < -0.1 * rhos0j) lflags |= L_EMF;
                if ((umf[k] * ppen * rei[kpen] * rpen) < -0.9 * dp0[kpen] / g / dt) lflags |= L_EMF;
                emf[k] = MX(MX(umf[k] * ppen * rei[kpen] * rpen, -0.1 * rhos0j), -0.9 * dp0[kpen] / g / dt);
                thlu_emf[k] = thl0[kpen] + ssthl0[kpen] * (ps0[k] - p0[kpen]);
                qtu_emf[k] = qt0[kpen] + ssqt0[kpen] * (ps0[k] - p0[kpen]);
                uu_emf[k] = u0[kpen] + ssu0[kpen] * (ps0[k] - p0[kpen]);
                vu_emf[k] = v0[kpen] + ssv0[kpen] * (ps0[k] - p0[kpen]);
                for (m = 1; m <= ncnst; m++) tru_emf[m][k] = tr0[m][kpen] + sstr0[m][kpen] * (ps0[k] - p0[kpen]);
            } else {
                if ((emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen) < -0.1 * rhos0j) lflags |= L_EMF;
                if ((emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen) < -0.9 * dp0[k + 1] / g / dt) lflags |= L_EMF;
                emf[k] = MX(MX(emf[k + 1] - umf[k] * dp0[k + 1] * rei[k + 1] * rpen, -0.1 * rhos0j), -0.9 * dp0[k + 1] / g / dt);
                if (fabs(emf[k]) > fabs(emf[k + 1])) {
                    thlu_emf[k] = (thlu_emf[k + 1] * emf[k + 1] + thl0[k + 1] * (emf[k] - emf[k + 1])) / emf[k];
                    qtu_emf[k] = (qtu_emf[k + 1] * emf[k + 1] + qt0[k + 1] * (emf[k] - emf[k + 1])) / emf[k];
                    uu_emf[k] = (uu_emf[k + 1] * emf[k + 1] + u0[k + 1] * (emf[k] - emf[k + 1])) / emf[k];
                    vu_emf[k] = (vu_emf[k + 1] * emf[k + 1] + v0[k + 1] * (emf[k] - emf[k + 1])) / emf[k];
                    for (m = 1; m <= ncnst; m++)
                        tru_emf[m][k] = (tru_emf[m][k + 1] * emf[k + 1] + tr0[m][k + 1] * (emf[k] - emf[k + 1])) / emf[k];
                } else {
                    thlu_emf[k] = thl0[k + 1];
                    qtu_emf[k] = qt0[k + 1];
                    uu_emf[k] = u0[k + 1];
                    vu_emf[k] = v0[k + 1];
                    for (m = 1; m <= ncnst; m++) tru_emf[m][k] = tr0[m][k + 1];
                }
            }
        }
        /* 1. PBL fluxes (:3255-3290) */
        xsrc = qtsrc;
        xmean = qt0[kinv];
        xtop = qt0[kinv + 1] + ssqt0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
        xbot = qt0[kinv - 1] + ssqt0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        fluxbelowinv(cbmf, ps0, mkx, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
        for (k = 0; k <= kinv - 1; k++) qtflx[k] = xflx[k];
        xsrc = thlsrc;
        xmean = thl0[kinv];
        xtop = thl0[kinv + 1] + ssthl0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
        xbot = thl0[kinv - 1] + ssthl0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        fluxbelowinv(cbmf, ps0, mkx, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
        for (k = 0; k <= kinv - 1; k++) slflx[k] = cp * exns0[k] * xflx[k];
        xsrc = usrc;
        xmean = u0[kinv];
        xtop = u0[kinv + 1] + ssu0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
        xbot = u0[kinv - 1] + ssu0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        fluxbelowinv(cbmf, ps0, mkx, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
        for (k = 0; k <= kinv - 1; k++) uflx[k] = xflx[k];
        xsrc = vsrc;
        xmean = v0[kinv];
        xtop = v0[kinv + 1] + ssv0[kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
        xbot = v0[kinv - 1] + ssv0[kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
        fluxbelowinv(cbmf, ps0, mkx, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
        for (k = 0; k <= kinv - 1; k++) vflx[k] = xflx[k];
        for (m = 1; m <= ncnst; m++) {
            xsrc = trsrc[m];
            xmean = tr0[m][kinv];
            xtop = tr0[m][kinv + 1] + sstr0[m][kinv + 1] * (ps0[kinv] - p0[kinv + 1]);
            xbot = tr0[m][kinv - 1] + sstr0[m][kinv - 1] * (ps0[kinv - 1] - p0[kinv - 1]);
            fluxbelowinv(cbmf, ps0, mkx, kinv, dt, xsrc, xmean, xtop, xbot, xflx);
            for (k = 0; k <= kinv - 1; k++) trflx[m][k] = xflx[k];
        }
        /* 2. Non-buoyancy sorting fluxes (:3300-3313) */
        uplus = 0.0;
        vplus = 0.0;
        for (k = kinv; k <= krel - 1; k++) {
            kp1 = k + 1;
            qtflx[k] = cbmf * (qtsrc - (qt0[kp1] + ssqt0[kp1] * (ps0[k] - p0[kp1])));
            slflx[k] = cbmf * (thlsrc - (thl0[kp1] + ssthl0[kp1] * (ps0[k] - p0[kp1]))) * cp * exns0[k];
            uplus = uplus + PGFc * ssu0[k] * (ps0[k] - ps0[k - 1]);
            vplus = vplus + PGFc * ssv0[k] * (ps0[k] - ps0[k - 1]);
            uflx[k] = cbmf * (usrc + uplus - (u0[kp1] + ssu0[kp1] * (ps0[k] - p0[kp1])));
            vflx[k] = cbmf * (vsrc + vplus - (v0[kp1] + ssv0[kp1] * (ps0[k] - p0[kp1])));
            for (m = 1; m <= ncnst; m++) trflx[m][k] = cbmf * (trsrc[m] - (tr0[m][kp1] + sstr0[m][kp1] * (ps0[k] - p0[kp1])));
        }
        /* 3. Buoyancy sorting fluxes (:3322-3331) */
        for (k = krel; k <= kbup - 1; k++) {
            kp1 = k + 1;
            slflx[k] = cp * exns0[k] * umf[k] * (thlu[k] - (thl0[kp1] + ssthl0[kp1] * (ps0[k] - p0[kp1])));
            qtflx[k] = umf[k] * (qtu[k] - (qt0[kp1] + ssqt0[kp1] * (ps0[k] - p0[kp1])));
            uflx[k] = umf[k] * (uu[k] - (u0[kp1] + ssu0[kp1] * (ps0[k] - p0[kp1])));
            vflx[k] = umf[k] * (vu[k] - (v0[kp1] + ssv0[kp1] * (ps0[k] - p0[kp1])));
            for (m = 1; m <= ncnst; m++) trflx[m][k] = umf[k] * (tru[m][k] - (tr0[m][kp1] + sstr0[m][kp1] * (ps0[k] - p0[kp1])));
        }
        /* 4. Penetrative entrainment fluxes (:3392-3401) */
        for (k = kbup; k <= kpen - 1; k++) {
            slflx[k] = cp * exns0[k] * emf[k] * (thlu_emf[k] - (thl0[k] + ssthl0[k] * (ps0[k] - p0[k])));
            qtflx[k] = emf[k] * (qtu_emf[k] - (qt0[k] + ssqt0[k] * (ps0[k] - p0[k])));
            uflx[k] = emf[k] * (uu_emf[k] - (u0[k] + ssu0[k] * (ps0[k] - p0[k])));
            vflx[k] = emf[k] * (vu_emf[k] - (v0[k] + ssv0[k] * (ps0[k] - p0[k])));
            for (m = 1; m <= ncnst; m++) trflx[m][k] = emf[k] * (tru_emf[m][k] - (tr0[m][k] + sstr0[m][k] * (ps0[k] - p0[k])));
        }
        /* Condensate tendency by compensating subsidence (:3416-3476) */
        for (k = 0; k <= mkx; k++) uemf[k] = 0.0;
        for (k = 0; k <= kinv - 2; k++) uemf[k] = cbmf * (ps0[0] - ps0[k]) / (ps0[0] - ps0[kinv - 1]);
        for (k = kinv - 1; k <= krel - 1; k++) uemf[k] = cbmf;
        for (k = krel; k <= kbup - 1; k++) uemf[k] = umf[k];
        for (k = kbup; k <= kpen - 1; k++) uemf[k] = emf[k];
        for (k = 1; k <= mkx; k++) comsub[k] = 0.0;
        for (k = 1; k <= kpen; k++) comsub[k] = 0.5 * (uemf[k] + uemf[k - 1]);
        for (k = 1; k <= kpen; k++) {
            if (comsub[k] >= 0.0) {
                if (k == mkx) {
                    thlten_sub = 0.0;
                    qtten_sub = 0.0;
                    qlten_sub = 0.0;
                    qiten_sub = 0.0;
                    nlten_sub = 0.0;
                    niten_sub = 0.0;
                } else {
                    thlten_sub = g * comsub[k] * (thl0[k + 1] - thl0[k]) / (p0[k] - p0[k + 1]);
                    qtten_sub = g * comsub[k] * (qt0[k + 1] - qt0[k]) / (p0[k] - p0[k + 1]);
                    qlten_sub = g * comsub[k] * (ql0[k + 1] - ql0[k]) / (p0[k] - p0[k + 1]);
                    qiten_sub = g * comsub[k] * (qi0[k + 1] - qi0[k]) / (p0[k] - p0[k + 1]);
                    nlten_sub = g * comsub[k] * (tr0[ixnumliq][k + 1] - tr0[ixnumliq][k]) / (p0[k] - p0[k + 1]);
                    niten_sub = g * comsub[k] * (tr0[ixnumice][k + 1] - tr0[ixnumice][k]) / (p0[k] - p0[k + 1]);
                }
            } else {
                if (k == 1) {
                    thlten_sub = 0.0;
                    qtten_sub = 0.0;
                    qlten_sub = 0.0;
                    qiten_sub = 0.0;
                    nlten_sub = 0.0;
                    niten_sub = 0.0;
                } else {
                    thlten_sub = g * comsub[k] * (thl0[k] - thl0[k - 1]) / (p0[k - 1] - p0[k]);
                    qtten_sub = g * comsub[k] * (qt0[k] - qt0[k - 1]) / (p0[k - 1] - p0[k]);
                    qlten_sub = g * comsub[k] * (ql0[k] - ql0[k - 1]) / (p0[k - 1] - p0[k]);
                    qiten_sub = g * comsub[k] * (qi0[k] - qi0[k - 1]) / (p0[k - 1] - p0[k]);
                    nlten_sub = g * comsub[k] * (tr0[ixnumliq][k] - tr0[ixnumliq][k - 1]) / (p0[k - 1] - p0[k]);
                    niten_sub = g * comsub[k] * (tr0[ixnumice][k] - tr0[ixnumice][k - 1]) / (p0[k - 1] - p0[k]);
                }
            }
            thl_prog = thl0[k] + thlten_sub * dt;
            qt_prog = MX(qt0[k] + qtten_sub * dt, 1.e-12);
            conden(p0[k], thl_prog, qt_prog, &thj, &qvj, &qlj, &qij, &qse, &id_check);
            if (id_check == 1) {
                id_exit = 1;
                goto l333;
            }
            qlten_sink[k] = MX(qlten_sub, -ql0[k] / dt);
            qiten_sink[k] = MX(qiten_sub, -qi0[k] / dt);
            nlten_sink[k] = MX(nlten_sub, -tr0[ixnumliq][k] / dt);
            niten_sink[k] = MX(niten_sub, -tr0[ixnumice][k] / dt);
        }
        /* Momentum tendency (:3488-3501) */
        for (k = 1; k <= kpen; k++) {
            km1 = k - 1;
            uten[k] = (uflx[km1] - uflx[k]) * g / dp0[k];
            vten[k] = (vflx[km1] - vflx[k]) * g / dp0[k];
            uf[k] = u0[k] + uten[k] * dt;
            vf[k] = v0[k] + vten[k] * dt;
        }
        /* Thermodynamic tendencies (:3511-3794) */
        rliq = 0.0;
        rainflx = 0.0;
        snowflx = 0.0;
        for (k = 1; k <= kpen; k++) {
            km1 = k - 1;
            dwten[k] = dwten[k] * 0.5 * (umf[k - 1] + umf[k]) * g / dp0[k];
            diten[k] = diten[k] * 0.5 * (umf[k - 1] + umf[k]) * g / dp0[k];
            qrten[k] = frc_rasn * dwten[k];
            qsten[k] = frc_rasn * diten[k];
            rainflx = rainflx + qrten[k] * dp0[k] / g;
            snowflx = snowflx + qsten[k] * dp0[k] / g;
            slten[k] = (slflx[km1] - slflx[k]) * g / dp0[k];
            if (k == 1) {
                slten[k] = slten[k] - g / 4.0 / dp0[k] *
                                          (uflx[k] * (uf[k + 1] - uf[k] + u0[k + 1] - u0[k]) +
                                           vflx[k] * (vf[k + 1] - vf[k] + v0[k + 1] - v0[k]));
            } else if (k >= 2 && k <= kpen - 1) {
                slten[k] = slten[k] - g / 4.0 / dp0[k] *
                                          (uflx[k] * (uf[k + 1] - uf[k] + u0[k + 1] - u0[k]) +
                                           uflx[k - 1] * (uf[k] - uf[k - 1] + u0[k] - u0[k - 1]) +
                                           vflx[k] * (vf[k + 1] - vf[k] + v0[k + 1] - v0[k]) +
                                           vflx[k - 1] * (vf[k] - vf[k - 1] + v0[k] - v0[k - 1]));
            } else if (k == kpen) {
                slten[k] = slten[k] - g / 4.0 / dp0[k] *
                                          (uflx[k - 1] * (uf[k] - uf[k - 1] + u0[k] - u0[k - 1]) +
                                           vflx[k - 1] * (vf[k] - vf[k - 1] + v0[k] - v0[k - 1]));
            }
            qtten[k] = (qtflx[km1] - qtflx[k]) * g / dp0[k];

            if (k < krel || k > kpen) {
                qlu_mid = 0.0;
                qiu_mid = 0.0;
                qlj = 0.0;
                qij = 0.0;
            } else if (k == krel) {
                conden(prel, thlu[krel - 1], qtu[krel - 1], &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                qlubelow = qlj;
                qiubelow = qij;
                conden(ps0[k], thlu[k], qtu[k], &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                qlu_mid = 0.5 * (qlubelow + qlj) * (prel - ps0[k]) / (ps0[k - 1] - ps0[k]);
                qiu_mid = 0.5 * (qiubelow + qij) * (prel - ps0[k]) / (ps0[k - 1] - ps0[k]);
            } else if (k == kpen) {
                conden(ps0[k - 1] + ppen, thlu_top, qtu_top, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                qlu_mid = 0.5 * (qlubelow + qlj) * (-ppen) / (ps0[k - 1] - ps0[k]);
                qiu_mid = 0.5 * (qiubelow + qij) * (-ppen) / (ps0[k - 1] - ps0[k]);
                qlu_top = qlj;
                qiu_top = qij;
            } else {
                conden(ps0[k], thlu[k], qtu[k], &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                qlu_mid = 0.5 * (qlubelow + qlj);
                qiu_mid = 0.5 * (qiubelow + qij);
            }
            qlubelow = qlj;
            qiubelow = qij;

            qc_l[k] = (1.0 - frc_rasn) * dwten[k];
            qc_i[k] = (1.0 - frc_rasn) * diten[k];
            if (k <= kbup) {
                qc_l[k] = qc_l[k] + g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * qlu_mid;
                qc_i[k] = qc_i[k] + g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * qiu_mid;
                qc_lm = -g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * ql0[k];
                qc_im = -g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * qi0[k];
                nc_lm = -g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * tr0[ixnumliq][k];
                nc_im = -g * 0.5 * (umf[k - 1] + umf[k]) * fdr[k] * tr0[ixnumice][k];
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
                nc_lm = nc_lm - g * umf[k] * tr0[ixnumliq][k] / (ps0[k - 1] - ps0[k]);
                nc_im = nc_im - g * umf[k] * tr0[ixnumice][k] / (ps0[k - 1] - ps0[k]);
            }
            if (k == kbup) {
                conden(p0[k], thlu_emf[k], qtu_emf[k], &thj, &qvj, &ql_emf_kbup, &qi_emf_kbup, &qse, &id_check);
                if (id_check == 1) {
                    id_exit = 1;
                    goto l333;
                }
                if (ql_emf_kbup > 0.0) nl_emf_kbup = tru_emf[ixnumliq][k];
                else nl_emf_kbup = 0.0;
                if (qi_emf_kbup > 0.0) ni_emf_kbup = tru_emf[ixnumice][k];
                else ni_emf_kbup = 0.0;
                qc_lm = qc_lm - g * emf[k] * (ql_emf_kbup - ql0[k]) / (ps0[k - 1] - ps0[k]);
                qc_im = qc_im - g * emf[k] * (qi_emf_kbup - qi0[k]) / (ps0[k - 1] - ps0[k]);
                nc_lm = nc_lm - g * emf[k] * (nl_emf_kbup - tr0[ixnumliq][k]) / (ps0[k - 1] - ps0[k]);
                nc_im = nc_im - g * emf[k] * (ni_emf_kbup - tr0[ixnumice][k]) / (ps0[k - 1] - ps0[k]);
            }
            /* use_expconten = .true., use_unicondet = .false. (:3748-3759) */
            qlten[k] = qc_l[k] + frc_rasn * dwten[k] + (MX(0.0, ql0[k] + (qc_lm + qlten_sink[k]) * dt) - ql0[k]) / dt;
            qiten[k] = qc_i[k] + frc_rasn * diten[k] + (MX(0.0, qi0[k] + (qc_im + qiten_sink[k]) * dt) - qi0[k]) / dt;
            trten[ixnumliq][k] = MX(nc_lm + nlten_sink[k], -tr0[ixnumliq][k] / dt);
            trten[ixnumice][k] = MX(nc_im + niten_sink[k], -tr0[ixnumice][k] / dt);
            qvten[k] = qtten[k] - qlten[k] - qiten[k];
            sten[k] = slten[k] + xlv * qlten[k] + xls * qiten[k];
            qc[k] = qc_l[k] + qc_i[k];
            rliq = rliq + qc[k] * dp0[k] / g / 1000.0;
        }
        precip = rainflx + snowflx;
        snow = snowflx;
        /* Evaporation and melting of precipitation (:3808-3926) */
        evpint_rain = 0.0;
        evpint_snow = 0.0;
        for (k = 0; k <= mkx; k++) {
            flxrain[k] = 0.0;
            flxsnow[k] = 0.0;
        }
        for (k = 1; k <= mkx; k++) {
            ntraprd[k] = 0.0;
            ntsnprd[k] = 0.0;
        }
        for (k = mkx; k >= 1; k--) {
            if (t0[k] > 273.16) snowmlt = MX(0.0, flxsnow[k] * g / dp0[k]);
            else snowmlt = 0.0;
            qsat1(t0[k], p0[k], &es1, &qs1, &gam1);
            subsat = MX((1.0 - qv0[k] / qs1), 0.0);
            evprain = kevp * subsat * sqrt(flxrain[k] + snowmlt * dp0[k] / g);
            evpsnow = kevp * subsat * sqrt(MX(flxsnow[k] - snowmlt * dp0[k] / g, 0.0));
            evplimit = MX(0.0, (A->qw0[k] - qv0[k]) / dt);
            evplimit_rain = MN(evplimit, (flxrain[k] + snowmlt * dp0[k] / g) * g / dp0[k]);
            evplimit_rain = MN(evplimit_rain, (rainflx - evpint_rain) * g / dp0[k]);
            evprain = MX(0.0, MN(evplimit_rain, evprain));
            evplimit_snow = MN(evplimit, MX(flxsnow[k] - snowmlt * dp0[k] / g, 0.0) * g / dp0[k]);
            evplimit_snow = MN(evplimit_snow, (snowflx - evpint_snow) * g / dp0[k]);
            evpsnow = MX(0.0, MN(evplimit_snow, evpsnow));
            if ((evprain + evpsnow) > evplimit) {
                tmp1 = evprain * evplimit / (evprain + evpsnow);
                tmp2 = evpsnow * evplimit / (evprain + evpsnow);
                evprain = tmp1;
                evpsnow = tmp2;
            }
            evapc[k] = evprain + evpsnow;
            evpint_rain = evpint_rain + evprain * dp0[k] / g;
            evpint_snow = evpint_snow + evpsnow * dp0[k] / g;
            ntraprd[k] = qrten[k] - evprain + snowmlt;
            ntsnprd[k] = qsten[k] - evpsnow - snowmlt;
            flxrain[k - 1] = flxrain[k] + ntraprd[k] * dp0[k] / g;
            flxsnow[k - 1] = flxsnow[k] + ntsnprd[k] * dp0[k] / g;
            flxrain[k - 1] = MX(flxrain[k - 1], 0.0);
            if (flxrain[k - 1] == 0.0) ntraprd[k] = -flxrain[k] * g / dp0[k];
            flxsnow[k - 1] = MX(flxsnow[k - 1], 0.0);
            if (flxsnow[k - 1] == 0.0) ntsnprd[k] = -flxsnow[k] * g / dp0[k];
            qlten[k] = qlten[k] - qrten[k];
            qiten[k] = qiten[k] - qsten[k];
            qvten[k] = qvten[k] + evprain + evpsnow;
            qtten[k] = qlten[k] + qiten[k] + qvten[k];
            if ((qv0[k] + qvten[k] * dt) < S.qmin[0] || (ql0[k] + qlten[k] * dt) < S.qmin[1] ||
                (qi0[k] + qiten[k] * dt) < S.qmin[2])
                lflags |= L_NEGCON;
            sten[k] = sten[k] - xlv * evprain - xls * evpsnow - (xls - xlv) * snowmlt;
            slten[k] = sten[k] - xlv * qlten[k] - xls * qiten[k];
        }
        precip = (flxrain[0] + flxsnow[0]) / 1000.0;
        snow = flxsnow[0] / 1000.0;
        /* Remove detrained condensate from the tendencies (:3966-3981) */
        for (k = 1; k <= kpen; k++) {
            qtten[k] = qtten[k] - qc[k];
            qlten[k] = qlten[k] - qc_l[k];
            qiten[k] = qiten[k] - qc_i[k];
            slten[k] = slten[k] + (xlv * qc_l[k] + xls * qc_i[k]);
            sten[k] = sten[k] - (xls - xlv) * qc_i[k];
        }
        /* Positive moisture (:3995-4001) */
        for (k = 1; k <= mkx; k++) {
            qv0_star[k] = qv0[k] + qvten[k] * dt;
            ql0_star[k] = ql0[k] + qlten[k] * dt;
            qi0_star[k] = qi0[k] + qiten[k] * dt;
            s0_star[k] = s0[k] + sten[k] * dt;
        }
        positive_moisture_single(xlv, xls, mkx, dt, S.qmin[0], S.qmin[1], S.qmin[2], dp0, qv0_star,
                                 ql0_star, qi0_star, s0_star, qvten, qlten, qiten, sten);
        for (k = 1; k <= mkx; k++) {
            qtten[k] = qvten[k] + qlten[k] + qiten[k];
            slten[k] = sten[k] - xlv * qlten[k] - xls * qiten[k];
        }
        /* Tracer tendencies (:4007-4076) */
        for (m = 4; m <= ncnst; m++) {
            if (m != ixnumliq && m != ixnumice) {
                trmin = S.qmin[m - 1];
                for (k = 0; k <= mkx; k++) {
                    trflx_d[k] = 0.0;
                    trflx_u[k] = 0.0;
                }
                for (k = 1; k <= mkx - 1; k++) {
                    pdelx = S.wet[m - 1] ? dp0[k] : dpdry0[k];
                    km1 = k - 1;
                    dum = (tr0[m][k] - trmin) * pdelx / g / dt + trflx[m][km1] - trflx[m][k] + trflx_d[km1];
                    trflx_d[k] = MN(0.0, dum);
                }
                for (k = mkx; k >= 2; k--) {
                    pdelx = S.wet[m - 1] ? dp0[k] : dpdry0[k];
                    km1 = k - 1;
                    dum = (tr0[m][k] - trmin) * pdelx / g / dt + trflx[m][km1] - trflx[m][k] +
                          trflx_d[km1] - trflx_d[k] - trflx_u[k];
                    trflx_u[km1] = MX(0.0, -dum);
                }
                for (k = 1; k <= mkx; k++) {
                    pdelx = S.wet[m - 1] ? dp0[k] : dpdry0[k];
                    km1 = k - 1;
                    trten[m][k] = (trflx[m][km1] - trflx[m][k] + trflx_d[km1] - trflx_d[k] +
                                   trflx_u[km1] - trflx_u[k]) * g / pdelx;
                }
            }
        }
        /* In-cloud diagnostics (:4092-4158) */
        conden(prel, thlu[krel - 1], qtu[krel - 1], &thj, &qvj, &qlj, &qij, &qse, &id_check);
        if (id_check == 1) {
            xflags |= X_CONDEN;
            id_exit = 1;
            goto l333;
        }
        {
            double qcubelow = qlj + qij, zw_tmp2, zw_tmp3;
            qlubelow = qlj;
            qiubelow = qij;
            for (k = krel; k <= kpen; k++) {
                if (k == kpen) conden(ps0[k - 1] + ppen, thlu_top, qtu_top, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                else conden(ps0[k], thlu[k], qtu[k], &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                qcu[k] = 0.5 * (qcubelow + qlj + qij);
                qlu[k] = 0.5 * (qlubelow + qlj);
                qiu[k] = 0.5 * (qiubelow + qij);
                /* compute_zwshcu's cloud-fraction option (zwshcu.F90:4413-4431) */
                zw_tmp2 = 0.0;
                zw_tmp3 = 1.0;
                if (A->omega && S.zw_cloud_sh) {
                    double tmp1;
                    zw_tmp3 = 0.5 * S.zw_ufrc0;
                    tmp1 = (z0[k] - z0[krel]) / (z0[kpen] - z0[krel] + 10.0);
                    tmp1 = 1.0 + S.zw_ufrcz * tmp1;
                    zw_tmp3 = zw_tmp3 * tmp1;
                    zw_tmp2 = fdr[k] * umf[k] * (zs0[k] - zs0[k - 1]) * dt / dp0[k] * 9.8 * S.zw_ufrcd;
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
                if (A->omega) cufrc[k] = zw_tmp3 * cufrc[k] + zw_tmp2;   /* zwshcu.F90:4449 */
                qcubelow = qlj + qij;
                qlubelow = qlj;
                qiubelow = qij;
            }
        }
        cnt = (double)kpen;
        cnb = (double)(krel - 1);

        /* Implicit-CIN state update (:4169-4329) */
        if (iter != iter_cin) {
            for (k = 1; k <= mkx; k++) {
                qv0_s[k] = qv0[k] + qvten[k] * dt;
                ql0_s[k] = ql0[k] + qlten[k] * dt;
                qi0_s[k] = qi0[k] + qiten[k] * dt;
                s0_s[k] = s0[k] + sten[k] * dt;
                t0_s[k] = t0[k] + sten[k] * dt / cp;
                qvten_s[k] = qvten[k];
                qlten_s[k] = qlten[k];
                qiten_s[k] = qiten[k];
                sten_s[k] = sten[k];
                uten_s[k] = uten[k];
                vten_s[k] = vten[k];
                qrten_s[k] = qrten[k];
                qsten_s[k] = qsten[k];
                evapc_s[k] = evapc[k];
                cufrc_s[k] = cufrc[k];
                qcu_s[k] = qcu[k];
                qlu_s[k] = qlu[k];
                qiu_s[k] = qiu[k];
                qc_s[k] = qc[k];
                for (m = 1; m <= ncnst; m++) trten_s[m][k] = trten[m][k];
            }
            for (k = 0; k <= mkx; k++) {
                umf_s[k] = umf[k];
                slflx_s[k] = slflx[k];
                qtflx_s[k] = qtflx[k];
                ufrc_s[k] = ufrc[k];
                qtu_s[k] = qtu[k];
                thlu_s[k] = thlu[k];
                thvu_s[k] = thvu[k];
                uu_s[k] = uu[k];
                vu_s[k] = vu[k];
                uemf_s[k] = uemf[k];
                flxrain_s[k] = flxrain[k];
                flxsnow_s[k] = flxsnow[k];
                fer_s[k] = fer[k];
                fdr_s[k] = fdr[k];
                dwten_s[k] = dwten[k];
                diten_s[k] = diten[k];
            }
            precip_s = precip;
            snow_s = snow;
            cush_s = cush;
            cin_s = cin;
            cinlcl_s = cinlcl;
            cbmf_s = cbmf;
            rliq_s = rliq;
            cnt_s = cnt;
            cnb_s = cnb;
            plcl_s = plcl;
            pinv_s = ps0[kinv - 1];
            plfc_s = plfc;
            pbup_s = ps0[kbup];
            ppen_s = ps0[kpen - 1] + ppen;
            tkeavg_s = tkeavg;
            kinv_s = kinv;
            klcl_s = klcl;
            klfc_s = klfc;
            krel_s = krel;
            kbup_s = kbup;
            kpen_s = kpen;

            for (k = 1; k <= mkx; k++) {
                qv0[k] = qv0_s[k];
                ql0[k] = ql0_s[k];
                qi0[k] = qi0_s[k];
                s0[k] = s0_s[k];
                t0[k] = t0_s[k];
                qt0[k] = (qv0[k] + ql0[k] + qi0[k]);
                thl0[k] = (t0[k] - xlv * ql0[k] / cp - xls * qi0[k] / cp) / exn0[k];
                thvl0[k] = (1.0 + zvir * qt0[k]) * thl0[k];
            }
            slope(mkx, thl0, p0, ssthl0);
            slope(mkx, qt0, p0, ssqt0);
            slope(mkx, u0, p0, ssu0);
            slope(mkx, v0, p0, ssv0);
            for (m = 1; m <= ncnst; m++) slope(mkx, tr0[m], p0, sstr0[m]);
            for (k = 1; k <= mkx; k++) {
                thl0bot = thl0[k] + ssthl0[k] * (ps0[k - 1] - p0[k]);
                qt0bot = qt0[k] + ssqt0[k] * (ps0[k - 1] - p0[k]);
                conden(ps0[k - 1], thl0bot, qt0bot, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                thv0bot[k] = thj * (1.0 + zvir * qvj - qlj - qij);
                thvl0bot[k] = thl0bot * (1.0 + zvir * qt0bot);
                thl0top = thl0[k] + ssthl0[k] * (ps0[k] - p0[k]);
                qt0top = qt0[k] + ssqt0[k] * (ps0[k] - p0[k]);
                conden(ps0[k], thl0top, qt0top, &thj, &qvj, &qlj, &qij, &qse, &id_check);
                if (id_check == 1) {
                    xflags |= X_CONDEN;
                    id_exit = 1;
                    goto l333;
                }
                thv0top[k] = thj * (1.0 + zvir * qvj - qlj - qij);
                thvl0top[k] = thl0top * (1.0 + zvir * qt0top);
            }
        }
    }

    /* Update output variables (:4337-4370) */
    for (k = 0; k <= mkx; k++) {
        AI(A->umf, i, k) = umf[k];
        AI(A->wu, i, k) = wu[k];
        AI(A->slflx, i, k) = slflx[k];
        AI(A->qtflx, i, k) = qtflx[k];
        AI(A->flxprc1, i, k) = flxrain[k] + flxsnow[k];
        AI(A->flxsnow1, i, k) = flxsnow[k];
    }
    for (k = 1; k <= mkx; k++) {
        AL(A->qvten, i, k) = qvten[k];
        AL(A->qlten, i, k) = qlten[k];
        AL(A->qiten, i, k) = qiten[k];
        AL(A->sten, i, k) = sten[k];
        AL(A->uten, i, k) = uten[k];
        AL(A->vten, i, k) = vten[k];
        AL(A->qrten, i, k) = qrten[k];
        AL(A->qsten, i, k) = qsten[k];
        AL(A->evapc, i, k) = evapc[k];
        AL(A->cufrc, i, k) = cufrc[k];
        AL(A->qcu, i, k) = qcu[k];
        AL(A->qlu, i, k) = qlu[k];
        AL(A->qiu, i, k) = qiu[k];
        AL(A->qc, i, k) = qc[k];
        for (m = 1; m <= ncnst; m++) AT(A->trten, i, k, m) = trten[m][k];
    }
    A->precip[i - 1] = precip;
    A->snow[i - 1] = snow;
    A->cush[i - 1] = cush;
    A->cbmf[i - 1] = cbmf;
    A->rliq[i - 1] = rliq;
    A->cnt[i - 1] = cnt;
    A->cnb[i - 1] = cnb;
    if (A->diag_real) {
        double *dr = A->diag_real + (size_t)(i - 1); const size_t ds = (size_t)A->mix;
        dr[UWO_DR_CIN * ds] = cin;
        dr[UWO_DR_CINLCL * ds] = cinlcl;
        dr[UWO_DR_PLCL * ds] = plcl;
        dr[UWO_DR_PLFC * ds] = plfc;
        dr[UWO_DR_PINV * ds] = ps0[kinv - 1];
        dr[UWO_DR_PBUP * ds] = ps0[kbup];
        dr[UWO_DR_PPEN * ds] = ps0[kpen - 1] + ppen;
        dr[UWO_DR_TKEAVG * ds] = tkeavg;
    }
    {
        const double *const fin[UWO_NDL] = {ufrc, qtu, thlu, thvu, uu, vu, uemf, flxrain, flxsnow, fer, fdr,
                                            dwten, diten};
        put_diag_level(A, i, mkx, fin);
    }

l333:
    if (id_exit) {
        xflags |= X_UWCU;
        for (k = 0; k <= mkx; k++) {
            AI(A->umf, i, k) = 0.0;
            AI(A->wu, i, k) = 0.0;
            AI(A->slflx, i, k) = 0.0;
            AI(A->qtflx, i, k) = 0.0;
        }
        for (k = 1; k <= mkx; k++) {
            AL(A->qvten, i, k) = 0.0;
            AL(A->qlten, i, k) = 0.0;
            AL(A->qiten, i, k) = 0.0;
            AL(A->sten, i, k) = 0.0;
            AL(A->uten, i, k) = 0.0;
            AL(A->vten, i, k) = 0.0;
            AL(A->qrten, i, k) = 0.0;
            AL(A->qsten, i, k) = 0.0;
            AL(A->evapc, i, k) = 0.0;
            AL(A->cufrc, i, k) = 0.0;
            AL(A->qcu, i, k) = 0.0;
            AL(A->qlu, i, k) = 0.0;
            AL(A->qiu, i, k) = 0.0;
            AL(A->qc, i, k) = 0.0;
            for (m = 1; m <= ncnst; m++) AT(A->trten, i, k, m) = 0.0;
        }
        A->precip[i - 1] = 0.0;
        A->snow[i - 1] = 0.0;
        A->cush[i - 1] = -1.0;
        A->cbmf[i - 1] = 0.0;
        A->rliq[i - 1] = 0.0;
        A->cnt[i - 1] = 1.0;
        A->cnb[i - 1] = (double)mkx;
        if (A->diag_real) {
            double *dr = A->diag_real + (size_t)(i - 1); const size_t ds = (size_t)A->mix;
            dr[UWO_DR_CIN * ds] = -1.0;
            dr[UWO_DR_CINLCL * ds] = -1.0;
            for (k = UWO_DR_PLCL; k < UWO_NDR; k++) dr[k * ds] = 0.0;
        }
        put_diag_level(A, i, mkx, 0);
        kinv = klcl = klfc = krel = kbup = kpen = 0;
    }
    if (A->diag_int) {
        int *di = A->diag_int + (size_t)(i - 1); const size_t ds = (size_t)A->mix;
        di[UWO_DI_EXIT * ds] = xflags;
        di[UWO_DI_LIMIT * ds] = lflags;
        di[UWO_DI_KINV * ds] = kinv;
        di[UWO_DI_KLCL * ds] = klcl;
        di[UWO_DI_KLFC * ds] = klfc;
        di[UWO_DI_KREL * ds] = krel;
        di[UWO_DI_KBUP * ds] = kbup;
        di[UWO_DI_KPEN * ds] = kpen;
    }
    return status_ret;
}

/* ---------------------------------------------------------------------------- public entry */

int uwo_init(double xlv, double cp, double xlf, double zvir, double r, double g, double ep2,
             double rpen, double tmn, double tmx, double trice, int icephs, double epsqs,
             double rgasv, double tmelt, int ncnst, const double *qmin, const int *cnst_wet,
             int ixnumliq, int ixnumice)
{
    int m;
    if (ncnst < 3 || ncnst > NCMAX || ixnumliq < 1 || ixnumliq > ncnst || ixnumice < 1 || ixnumice > ncnst)
        return -1;
    memset(&S, 0, sizeof(S));
    /* init_uwshcu (uwshcu.F90:230-239) */
    S.xlv = xlv;
    S.xlf = xlf;
    S.xls = S.xlv + S.xlf;
    S.cp = cp;
    S.zvir = zvir;
    S.r = r;
    S.g = g;
    S.ep2 = ep2;
    S.p00 = 1.e5;
    S.rovcp = S.r / S.cp;
    S.rpen = rpen;
    /* the Fortran parameter values (uwshcu.F90:1036, 1038, 1065) */
    S.rle = 0.1;
    S.rkm = 14.0;
    uwo_set_zw_options(1, 1.0, 0, 0.015, 0, 2.0, 2.0, 2.0);
    S.criqc = 0.7e-3;
    /* esinti -> gestbl (esinti.F90:44-51) */
    gestbl(tmn, tmx, trice, icephs, epsqs, xlv, xlf, rgasv, cp, tmelt);
    S.ncnst = ncnst;
    for (m = 0; m < ncnst; m++) {
        S.qmin[m] = qmin[m];
        S.wet[m] = cnst_wet[m] != 0;
    }
    S.ixnumliq = ixnumliq;
    S.ixnumice = ixnumice;
    return 0;
}

int uwo_set_params(double rpen, double rle, double rkm, double criqc)
{
    if (!(rpen > 0.0) || !(rle > 0.0) || !(rkm > 0.0) || !(criqc >= 0.0)) return -1;
    S.rpen = rpen;
    S.rle = rle;
    S.rkm = rkm;
    S.criqc = criqc;
    return 0;
}

int uwo_init_default(void)
{
    /* CESM shr_const values behind CAM's physconst: rair = R/mwdair, rh2o = R/mwwv,
     * zvir = rh2o/rair - 1, epsilo = mwwv/mwdair (the value init_uwshcu receives as mwh2o/mwdry). */
    const double boltz = 1.38065e-23, avogad = 6.02214e26, rgas = avogad * boltz;
    const double mwdair = 28.966, mwwv = 18.016;
    const double rdair = rgas / mwdair, rwv = rgas / mwwv, zv = (rwv / rdair) - 1.0;
    const double cpair = 1.00464e3, latvap = 2.501e6, latice = 3.337e5, gravit = 9.80616, tkfrz = 273.15;
    const double qmin[5] = {1.e-12, 0.0, 0.0, 0.0, 0.0};
    const int wet[5] = {1, 1, 1, 1, 1};
    return uwo_init(latvap, cpair, latice, zv, rdair, gravit, mwwv / mwdair, 10.0, 173.16, 375.16,
                    20.0, 1, mwwv / mwdair, rwv, tkfrz, 5, qmin, wet, 4, 5);
}

void uwo_get_estbl(double *out) { memcpy(out, S.estbl, sizeof(S.estbl)); }

void uwo_get_consts(double *o)
{
    o[0] = S.xlv; o[1] = S.xlf; o[2] = S.xls; o[3] = S.cp; o[4] = S.zvir; o[5] = S.r; o[6] = S.g;
    o[7] = S.ep2; o[8] = S.p00; o[9] = S.rovcp; o[10] = S.rpen; o[11] = S.tmin; o[12] = S.tmax;
    o[13] = S.ttrice; o[14] = S.epsqs; o[15] = S.rgasv; o[16] = S.tmelt;
    o[17] = S.pcf[0]; o[18] = S.pcf[1]; o[19] = S.pcf[2]; o[20] = S.pcf[3]; o[21] = S.pcf[4];
}

int uwo_findsp(int mix, int ncol, int pver, const double *q, const double *t, const double *p,
               double *tsp, double *qsp)
{
    int st = 0, i, k;
    for (k = 0; k < pver; k++)
        for (i = 0; i < ncol; i++) {
            size_t o = (size_t)k * mix + i;
            int s = findsp_point(q[o], t[o], p[o], &tsp[o], &qsp[o]);
            if (s > st) st = s;
        }
    return st;
}

/* compute_uwshcu (omega NULL) or compute_zwshcu (zwshcu.F90:630-4969, omega (mix, mkx)): the
 * driver of both, findsp over all (i,k) and the column loop. */
static int compute_core(int mix, int mkx, int iend, int ncnst, double dt,
                        const double *ps0, const double *zs0, const double *p0, const double *z0,
                        const double *dp0, const double *u0, const double *v0, const double *qv0,
                        const double *ql0, const double *qi0, const double *t0, const double *s0,
                        const double *tr0, const double *tke, const double *cldfrct,
                        const double *concldfrct, const double *pblh, double *cush,
                        double *umf, double *slflx, double *qtflx, double *flxprc1, double *flxsnow1,
                        double *qvten, double *qlten, double *qiten, double *sten, double *uten,
                        double *vten, double *trten, double *qrten, double *qsten, double *precip,
                        double *snow, double *evapc, double *cufrc, double *qcu, double *qlu,
                        double *qiu, double *cbmf, double *qc, double *rliq, const double *massflx_sh,
                        double *cnt, double *cnb, const double *dpdry0, double *wu,
                        int *diag_int, double *diag_real, double *diag_level, int nthreads,
                        const double *omega)
{
    int st = 0, i;
    int nthr = nthreads > 0 ? nthreads : UWO_MAXTHREADS();
    double *tw0, *qw0;
    (void)cldfrct;
    (void)concldfrct;
    (void)massflx_sh;
    if (mix < 1 || mkx < 3 || iend < 0 || iend > mix || ncnst != S.ncnst) return -1;
    tw0 = (double *)malloc(sizeof(double) * (size_t)mix * mkx);
    qw0 = (double *)malloc(sizeof(double) * (size_t)mix * mkx);
    if (!tw0 || !qw0) {
        free(tw0);
        free(qw0);
        return -2;
    }
    /* findsp over all (i,k) (uwshcu.F90:1216); each (i,k) is independent */
#pragma omp parallel for schedule(static) num_threads(nthr) reduction(max : st)
    for (i = 0; i < iend; i++) {
        int k;
        for (k = 0; k < mkx; k++) {
            size_t o = (size_t)k * mix + i;
            int s = findsp_point(qv0[o], t0[o], p0[o], &tw0[o], &qw0[o]);
            if (s > st) st = s;
        }
    }
    /* Fortran gives findsp errors status codes 2/3 and the mu error 1; report the largest code. */
#pragma omp parallel for schedule(dynamic, 8) num_threads(nthr) reduction(max : st)
    for (i = 1; i <= iend; i++) {
        uwo_io A;
        double qwcol[mkx + 1];
        int k, s;
        for (k = 1; k <= mkx; k++) qwcol[k] = qw0[(size_t)(k - 1) * mix + (i - 1)];
        A.mix = mix; A.mkx = mkx; A.iend = iend; A.ncnst = ncnst; A.dt = dt;
        A.ps0 = ps0; A.zs0 = zs0; A.p0 = p0; A.z0 = z0; A.dp0 = dp0; A.u0 = u0; A.v0 = v0;
        A.qv0 = qv0; A.ql0 = ql0; A.qi0 = qi0; A.t0 = t0; A.s0 = s0; A.tr0 = tr0; A.tke = tke;
        A.pblh = pblh; A.cush = cush; A.umf = umf; A.slflx = slflx; A.qtflx = qtflx;
        A.flxprc1 = flxprc1; A.flxsnow1 = flxsnow1; A.qvten = qvten; A.qlten = qlten;
        A.qiten = qiten; A.sten = sten; A.uten = uten; A.vten = vten; A.trten = trten;
        A.qrten = qrten; A.qsten = qsten; A.precip = precip; A.snow = snow; A.evapc = evapc;
        A.cufrc = cufrc; A.qcu = qcu; A.qlu = qlu; A.qiu = qiu; A.cbmf = cbmf; A.qc = qc;
        A.rliq = rliq; A.cnt = cnt; A.cnb = cnb; A.dpdry0 = dpdry0; A.wu = wu; A.qw0 = qwcol;
        A.diag_int = diag_int; A.diag_real = diag_real; A.diag_level = diag_level; A.omega = omega;
        s = uw_column(&A, i);
        if (s > st) st = s;
    }
    free(tw0);
    free(qw0);
    return st;
}

int uwo_compute_uwshcu(int mix, int mkx, int iend, int ncnst, double dt,
                       const double *ps0, const double *zs0, const double *p0, const double *z0,
                       const double *dp0, const double *u0, const double *v0, const double *qv0,
                       const double *ql0, const double *qi0, const double *t0, const double *s0,
                       const double *tr0, const double *tke, const double *cldfrct,
                       const double *concldfrct, const double *pblh, double *cush,
                       double *umf, double *slflx, double *qtflx, double *flxprc1, double *flxsnow1,
                       double *qvten, double *qlten, double *qiten, double *sten, double *uten,
                       double *vten, double *trten, double *qrten, double *qsten, double *precip,
                       double *snow, double *evapc, double *cufrc, double *qcu, double *qlu,
                       double *qiu, double *cbmf, double *qc, double *rliq, const double *massflx_sh,
                       double *cnt, double *cnb, const double *dpdry0, double *wu,
                       int *diag_int, double *diag_real, double *diag_level, int nthreads)
{
    return compute_core(mix, mkx, iend, ncnst, dt, ps0, zs0, p0, z0, dp0, u0, v0, qv0, ql0, qi0, t0, s0,
                        tr0, tke, cldfrct, concldfrct, pblh, cush, umf, slflx, qtflx, flxprc1, flxsnow1,
                        qvten, qlten, qiten, sten, uten, vten, trten, qrten, qsten, precip, snow, evapc,
                        cufrc, qcu, qlu, qiu, cbmf, qc, rliq, massflx_sh, cnt, cnb, dpdry0, wu, diag_int,
                        diag_real, diag_level, nthreads, NULL);
}

/* compute_zwshcu (zwshcu.F90:630-644): compute_uwshcu's arguments plus the pressure velocity omega
 * (mix, mkx) [Pa/s]; tpert2 is read only by the perturbation options, which are off here. */
int uwo_compute_zwshcu(int mix, int mkx, int iend, int ncnst, double dt,
                       const double *ps0, const double *zs0, const double *p0, const double *z0,
                       const double *dp0, const double *u0, const double *v0, const double *qv0,
                       const double *ql0, const double *qi0, const double *t0, const double *s0,
                       const double *tr0, const double *tke, const double *cldfrct,
                       const double *concldfrct, const double *pblh, double *cush,
                       double *umf, double *slflx, double *qtflx, double *flxprc1, double *flxsnow1,
                       double *qvten, double *qlten, double *qiten, double *sten, double *uten,
                       double *vten, double *trten, double *qrten, double *qsten, double *precip,
                       double *snow, double *evapc, double *cufrc, double *qcu, double *qlu,
                       double *qiu, double *cbmf, double *qc, double *rliq, const double *omega,
                       const double *massflx_sh, const double *tpert2, double *cnt, double *cnb,
                       const double *dpdry0, double *wu, int *diag_int, double *diag_real,
                       double *diag_level, int nthreads)
{
    (void)tpert2;
    if (!omega) return -1;
    return compute_core(mix, mkx, iend, ncnst, dt, ps0, zs0, p0, z0, dp0, u0, v0, qv0, ql0, qi0, t0, s0,
                        tr0, tke, cldfrct, concldfrct, pblh, cush, umf, slflx, qtflx, flxprc1, flxsnow1,
                        qvten, qlten, qiten, sten, uten, vten, trten, qrten, qsten, precip, snow, evapc,
                        cufrc, qcu, qlu, qiu, cbmf, qc, rliq, massflx_sh, cnt, cnb, dpdry0, wu, diag_int,
                        diag_real, diag_level, nthreads, omega);
}

/* The options of compute_zwshcu: zmh_shallow_lf, zmh_shallow_fwcrit, zmh_shallow_ent, zmh_ent0
 * (zwshcu.F90:30-32, 57) and zmh_cloud_sh, zmh_ufrcd, zmh_ufrc0, zmh_ufrcz (cloud_fraction.F90:52,
 * zwshcu.F90:36-38).  uwo_init sets the reference's defaults: 1, 1.0, 0, 0.015, 0, 2.0, 2.0, 2.0. */
int uwo_set_zw_options(int lf, double fwcrit, int ent, double ent0, int cloud_sh, double ufrcd,
                       double ufrc0, double ufrcz)
{
    S.zw_lf = lf != 0;
    S.zw_fwcrit = fwcrit;
    S.zw_ent = ent != 0;
    S.zw_ent0 = ent0;
    S.zw_cloud_sh = cloud_sh != 0;
    S.zw_ufrcd = ufrcd;
    S.zw_ufrc0 = ufrc0;
    S.zw_ufrcz = ufrcz;
    return 0;
}

int uwo_compute_uwshcu_inv(int mix, int mkx, int iend, int ncnst, double dt,
                           const double *ps0i, const double *zs0i, const double *p0i, const double *z0i,
                           const double *dp0i, const double *u0i, const double *v0i, const double *qv0i,
                           const double *ql0i, const double *qi0i, const double *t0i, const double *s0i,
                           const double *tr0i, const double *tkei, const double *cldfrcti,
                           const double *concldfrcti, const double *pblh, double *cush,
                           const double *tpert2, const double *qpert2, const double *massflx_sh,
                           double *umfi, double *slflxi, double *qtflxi, double *flxprc1i,
                           double *flxsnow1i, double *qvteni, double *qlteni, double *qiteni,
                           double *steni, double *uteni, double *vteni, double *trteni, double *qrteni,
                           double *qsteni, double *precip, double *snow, double *evapci,
                           double *cufrci, double *qcui, double *qlui, double *qiui, double *cbmf,
                           double *qci, double *rliq, double *cnti, double *cnbi,
                           const double *dpdry0i, double *wui, int nthreads)
{
    /* uwshcu.F90:380-469: reverse levels, run the core, reverse back. */
    size_t nl = (size_t)mix * mkx, ni = (size_t)mix * (mkx + 1), nt = nl * ncnst;
    int k, m, i, st;
    double *buf, *p;
    double *ps0, *zs0, *p0, *z0, *dp0, *u0, *v0, *qv0, *ql0, *qi0, *t0, *s0, *tr0, *tke, *cf, *ccf,
        *dpdry0, *umf, *slflx, *qtflx, *fp1, *fs1, *qvten, *qlten, *qiten, *sten, *uten, *vten,
        *trten, *qrten, *qsten, *evapc, *cufrc, *qcu, *qlu, *qiu, *qc, *cnt, *cnb, *wu;
    (void)tpert2;
    (void)qpert2;
    buf = (double *)calloc(4 * nt + 40 * ni + 2 * (size_t)mix, sizeof(double));
    if (!buf) return -2;
    p = buf;
#define TAKE(v, n) (v = p, p += (n))
    TAKE(ps0, ni); TAKE(zs0, ni); TAKE(tke, ni); TAKE(umf, ni); TAKE(slflx, ni); TAKE(qtflx, ni);
    TAKE(fp1, ni); TAKE(fs1, ni); TAKE(wu, ni);
    TAKE(p0, nl); TAKE(z0, nl); TAKE(dp0, nl); TAKE(u0, nl); TAKE(v0, nl); TAKE(qv0, nl);
    TAKE(ql0, nl); TAKE(qi0, nl); TAKE(t0, nl); TAKE(s0, nl); TAKE(cf, nl); TAKE(ccf, nl);
    TAKE(dpdry0, nl); TAKE(qvten, nl); TAKE(qlten, nl); TAKE(qiten, nl); TAKE(sten, nl);
    TAKE(uten, nl); TAKE(vten, nl); TAKE(qrten, nl); TAKE(qsten, nl); TAKE(evapc, nl);
    TAKE(cufrc, nl); TAKE(qcu, nl); TAKE(qlu, nl); TAKE(qiu, nl); TAKE(qc, nl);
    TAKE(tr0, nt); TAKE(trten, nt); TAKE(cnt, mix); TAKE(cnb, mix);
#undef TAKE
    for (k = 1; k <= mkx; k++) {
        int kv = mkx + 1 - k;
        for (i = 0; i < iend; i++) {
            size_t d = (size_t)(k - 1) * mix + i, s = (size_t)(kv - 1) * mix + i;
            p0[d] = p0i[s]; u0[d] = u0i[s]; v0[d] = v0i[s]; z0[d] = z0i[s]; dp0[d] = dp0i[s];
            dpdry0[d] = dpdry0i[s]; qv0[d] = qv0i[s]; ql0[d] = ql0i[s]; qi0[d] = qi0i[s];
            t0[d] = t0i[s]; s0[d] = s0i[s]; cf[d] = cldfrcti[s]; ccf[d] = concldfrcti[s];
            for (m = 0; m < ncnst; m++) tr0[d + nl * m] = tr0i[s + nl * m];
        }
    }
    for (k = 0; k <= mkx; k++) {
        int kv = mkx + 1 - k;
        for (i = 0; i < iend; i++) {
            size_t d = (size_t)k * mix + i, s = (size_t)(kv - 1) * mix + i;
            ps0[d] = ps0i[s]; zs0[d] = zs0i[s]; tke[d] = tkei[s];
        }
    }
    st = uwo_compute_uwshcu(mix, mkx, iend, ncnst, dt, ps0, zs0, p0, z0, dp0, u0, v0, qv0, ql0, qi0,
                            t0, s0, tr0, tke, cf, ccf, pblh, cush, umf, slflx, qtflx, fp1, fs1,
                            qvten, qlten, qiten, sten, uten, vten, trten, qrten, qsten, precip, snow,
                            evapc, cufrc, qcu, qlu, qiu, cbmf, qc, rliq, massflx_sh, cnt, cnb, dpdry0,
                            wu, NULL, NULL, NULL, nthreads);
    for (i = 0; i < iend; i++) {
        cnti[i] = mkx + 1 - cnt[i];
        cnbi[i] = mkx + 1 - cnb[i];
    }
    for (k = 0; k <= mkx; k++) {
        int kv = mkx + 1 - k;
        for (i = 0; i < iend; i++) {
            size_t s = (size_t)k * mix + i, d = (size_t)(kv - 1) * mix + i;
            umfi[d] = umf[s]; wui[d] = wu[s]; slflxi[d] = slflx[s]; qtflxi[d] = qtflx[s];
            flxprc1i[d] = fp1[s]; flxsnow1i[d] = fs1[s];
        }
    }
    for (k = 1; k <= mkx; k++) {
        int kv = mkx + 1 - k;
        for (i = 0; i < iend; i++) {
            size_t s = (size_t)(k - 1) * mix + i, d = (size_t)(kv - 1) * mix + i;
            qvteni[d] = qvten[s]; qlteni[d] = qlten[s]; qiteni[d] = qiten[s]; steni[d] = sten[s];
            uteni[d] = uten[s]; vteni[d] = vten[s]; qrteni[d] = qrten[s]; qsteni[d] = qsten[s];
            evapci[d] = evapc[s]; cufrci[d] = cufrc[s]; qcui[d] = qcu[s]; qlui[d] = qlu[s];
            qiui[d] = qiu[s]; qci[d] = qc[s];
            for (m = 0; m < ncnst; m++) trteni[d + nl * m] = trten[s + nl * m];
        }
    }
    free(buf);
    return st;
}

/* ---------------------------------------------------------------------- exported helpers */

double uwo_exnf(double p) { return exnf(p); }
double uwo_estblf(double t) { return estblf(t); }
void uwo_qsat(double t, double p, double *es, double *qs, double *gam) { qsat1(t, p, es, qs, gam); }
void uwo_conden(double p, double thl, double qt, double *th, double *qv, double *ql, double *qi,
                double *rvls, int *id_check)
{
    conden(p, thl, qt, th, qv, ql, qi, rvls, id_check);
}
void uwo_roots(double a, double b, double c, double *r1, double *r2, int *status) { roots(a, b, c, r1, r2, status); }
void uwo_slope(int mkx, const double *field, const double *p0, double *out)
{
    double f[mkx + 1], pp[mkx + 1], sl[mkx + 1];
    int k;
    for (k = 1; k <= mkx; k++) {
        f[k] = field[k - 1];
        pp[k] = p0[k - 1];
    }
    slope(mkx, f, pp, sl);
    for (k = 1; k <= mkx; k++) out[k - 1] = sl[k];
}
double uwo_qsinvert(double qt, double thl, double psfc) { return qsinvert(qt, thl, psfc); }
double uwo_compute_alpha(double d, double ke) { return compute_alpha(d, ke); }
double uwo_compute_mumin2(double a, double b, double c) { return compute_mumin2(a, b, c); }
double uwo_compute_ppen(double wtwb, double d, double bb, double bt, double rho, double dpen)
{
    return compute_ppen(wtwb, d, bb, bt, rho, dpen);
}
void uwo_getbuoy(double pbot, double thv0bot, double ptop, double thv0top, double thvubot,
                 double thvutop, double *plfc, double *cin)
{
    getbuoy(pbot, thv0bot, ptop, thv0top, thvubot, thvutop, plfc, cin);
}
double uwo_single_cin(double pbot, double thv0bot, double ptop, double thv0top, double thvubot, double thvutop)
{
    return single_cin(pbot, thv0bot, ptop, thv0top, thvubot, thvutop);
}
void uwo_fluxbelowinv(double cbmf, const double *ps0, int mkx, int kinv, double dt, double xsrc,
                      double xmean, double xtopin, double xbotin, double *xflx)
{
    fluxbelowinv(cbmf, ps0, mkx, kinv, dt, xsrc, xmean, xtopin, xbotin, xflx);
}
void uwo_positive_moisture_single(double xlv, double xls, int mkx, double dt, double qvmin,
                                  double qlmin, double qimin, const double *dp, double *qv,
                                  double *ql, double *qi, double *s, double *qvten, double *qlten,
                                  double *qiten, double *sten)
{
    /* 0-based arrays from the caller; shift to the 1-based internal form */
    positive_moisture_single(xlv, xls, mkx, dt, qvmin, qlmin, qimin, dp - 1, qv - 1, ql - 1, qi - 1,
                             s - 1, qvten - 1, qlten - 1, qiten - 1, sten - 1);
}

/* Evaluate the uw_math.h routines on the host (fn: 0 exp, 1 log, 2 pow, 3 erfc). */
void uwo_uwmath(int fn, const double *x, const double *y, double *out, int n)
{
    int i;
    for (i = 0; i < n; i++) {
        switch (fn) {
        case 0: out[i] = uw_exp(x[i]); break;
        case 1: out[i] = uw_log(x[i]); break;
        case 2: out[i] = uw_pow(x[i], y[i]); break;
        default: out[i] = uw_erfc(x[i]); break;
        }
    }
}
