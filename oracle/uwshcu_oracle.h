/*
 * uwshcu_oracle.h -- CPU oracle for the UW shallow-cumulus scheme (TEST INFRASTRUCTURE ONLY).
 *
 * This header declares a plain-C, FP64, statement-by-statement restatement of
 *   src/physics/uwshcu.F90        compute_uwshcu (478-4664) and its helpers (4672-5454)
 *   src/physics/wv_saturation.F90 estblf (64-80), gestbl (82-204), vqsatd (482-609), fqsatd (734-751)
 *   src/physics/gffgch.F90        gffgch (1-127)
 *   src/physics/esinti.F90        esinti (38-51)
 * of guirenbenxin/HPC-and-climate-model.  Only tests, the smoke check and the CPU-baseline leg of the
 * benchmark may link it: it is the checker, never the product path.
 *
 * Arrays follow the Fortran layout: column index fastest, leading dimension `mix`, k = 1 at the surface
 * (interface arrays run k = 0..mkx).  All routines are single-threaded per column; the driver splits
 * columns across OpenMP threads.
 */
#ifndef UWSHCU_ORACLE_H
#define UWSHCU_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Per-column integer diagnostics written when `diag_int` is non-null: array (8, mix), entry j of
 * column i at diag_int[j*mix + i-1]. */
enum {
    UWO_DI_EXIT = 0,   /* bitmask of exit_* flags (uwshcu.F90:889-899); 0 = convection performed */
    UWO_DI_LIMIT = 1,  /* bitmask of limit_* flags and ind_delcin (uwshcu.F90:901-910)           */
    UWO_DI_KINV = 2, UWO_DI_KLCL = 3, UWO_DI_KLFC = 4, UWO_DI_KREL = 5, UWO_DI_KBUP = 6, UWO_DI_KPEN = 7,
    UWO_NDI = 8
};
/* Per-column real diagnostics written when `diag_real` is non-null: array (8, mix) as above. */
enum {
    UWO_DR_CIN = 0, UWO_DR_CINLCL = 1, UWO_DR_PLCL = 2, UWO_DR_PLFC = 3, UWO_DR_PINV = 4,
    UWO_DR_PBUP = 5, UWO_DR_PPEN = 6, UWO_DR_TKEAVG = 7,
    UWO_NDR = 8
};

/* Set the physical constants (init_uwshcu, uwshcu.F90:102-249; uwshcu_readnl rpen, :58-98) and build
 * the saturation table (esinti.F90:38-51 -> gestbl).  `qmin` and `cnst_wet` have ncnst entries
 * (cnst_wet[m] != 0 for 'wet' constituents).  ixnumliq/ixnumice are 1-based tracer indices. */
int uwo_init(double xlv, double cp, double xlf, double zvir, double r, double g, double ep2,
             double rpen, double tmn, double tmx, double trice, int icephs, double epsqs,
             double rgasv, double tmelt, int ncnst, const double *qmin, const int *cnst_wet,
             int ixnumliq, int ixnumice);

/* Same with the CESM shr_const values CAM passes at init (rpen = 10, 5 tracers qv ql qi nl ni,
 * qmin = {1e-12, 0, 0, 0, 0}, all wet, ixnumliq = 4, ixnumice = 5). */
int uwo_init_default(void);

/* Tuning parameters: rpen (namelist, uwshcu.F90:58-98) and the compute_uwshcu parameters rle, rkm,
 * criqc (uwshcu.F90:1036, 1038, 1065; uwo_init sets the Fortran values 0.1, 14, 0.7e-3).
 * Returns -1 for non-positive values (criqc may be 0). */
int uwo_set_params(double rpen, double rle, double rkm, double criqc);

/* Copy of the 250-entry saturation-vapour-pressure table built by uwo_init. */
void uwo_get_estbl(double *out250);
/* Constants in the order: xlv xlf xls cp zvir r g ep2 p00 rovcp rpen tmin tmax ttrice epsqs rgasv
 * tmelt pcf1..pcf5 (22 values). */
void uwo_get_consts(double *out22);

/* Per-level diagnostics (the Fortran's history fields ufrc, qtu, thlu, thvu, uu, vu, uemf, flxrain,
 * flxsnow on interfaces and fer, fdr, dwten, diten on layers; uwshcu.F90:4383-4433 and the explicit-CIN
 * copies :1945-1989): optional diag_level array (13, mkx+1, mix), levels bottom-up k = 0..mkx, layer
 * fields in rows 1..mkx. */
/* compute_uwshcu (uwshcu.F90:478-492) with the Fortran argument list; qsat/lchnk are not needed
 * (the built-in fqsatd semantics are used).  Optional diagnostics may be null.  nthreads <= 0 uses
 * the OpenMP default.  Returns 0, or a positive status for the reference's endrun cases
 * (1 = mu inconsistency uwshcu.F90:2119-2122, 2 = findsp non-convergence :5423-5431,
 *  3 = findsp enthalpy error :5435-5447). */
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
                       int *diag_int, double *diag_real, double *diag_level, int nthreads);

/* compute_zwshcu (zwshcu.F90:630-4969), the CAS-ESM variant of the scheme: compute_uwshcu's
 * arguments plus the pressure velocity omega (mix, mkx) [Pa/s] (and tpert2, read only by the
 * perturbation options, which are not restated); the options of uwo_set_zw_options apply. */
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
                       double *diag_level, int nthreads);

/* Options of compute_zwshcu (zwshcu.F90:30-59, cloud_fraction.F90:52): large-scale forcing of the
 * closure (zmh_shallow_lf), wcrit factor (zmh_shallow_fwcrit), buoyancy-based entrainment
 * (zmh_shallow_ent, zmh_ent0), cloud-fraction enhancement (zmh_cloud_sh, zmh_ufrcd, zmh_ufrc0,
 * zmh_ufrcz).  Defaults: 1, 1.0, 0, 0.015, 0, 2.0, 2.0, 2.0. */
int uwo_set_zw_options(int lf, double fwcrit, int ent, double ent0, int cloud_sh, double ufrcd,
                       double ufrc0, double ufrcz);

/* compute_uwshcu_inv (uwshcu.F90:251-476): CAM top-down level order in and out. */
int uwo_compute_uwshcu_inv(int mix, int mkx, int iend, int ncnst, double dt,
                           const double *ps0, const double *zs0, const double *p0, const double *z0,
                           const double *dp0, const double *u0, const double *v0, const double *qv0,
                           const double *ql0, const double *qi0, const double *t0, const double *s0,
                           const double *tr0, const double *tke, const double *cldfrct,
                           const double *concldfrct, const double *pblh, double *cush,
                           const double *tpert2, const double *qpert2, const double *massflx_sh,
                           double *umf, double *slflx, double *qtflx, double *flxprc1,
                           double *flxsnow1, double *qvten, double *qlten, double *qiten,
                           double *sten, double *uten, double *vten, double *trten, double *qrten,
                           double *qsten, double *precip, double *snow, double *evapc,
                           double *cufrc, double *qcu, double *qlu, double *qiu, double *cbmf,
                           double *qc, double *rliq, double *cnt, double *cnb,
                           const double *dpdry0, double *wu, int nthreads);

/* ---- helpers exported for unit tests (scalar forms of the Fortran routines) ---- */
double uwo_exnf(double p);
double uwo_estblf(double t);
void   uwo_qsat(double t, double p, double *es, double *qs, double *gam);
void   uwo_conden(double p, double thl, double qt, double *th, double *qv, double *ql, double *qi,
                  double *rvls, int *id_check);
void   uwo_roots(double a, double b, double c, double *r1, double *r2, int *status);
void   uwo_slope(int mkx, const double *field, const double *p0, double *out);   /* 1-based k -> out[k-1] */
double uwo_qsinvert(double qt, double thl, double psfc);
double uwo_compute_alpha(double del_cin, double ke);
double uwo_compute_mumin2(double mulcl, double rmaxfrac, double mulow);
double uwo_compute_ppen(double wtwb, double d, double bogbot, double bogtop, double rho0j, double dpen);
void   uwo_getbuoy(double pbot, double thv0bot, double ptop, double thv0top, double thvubot,
                   double thvutop, double *plfc, double *cin);
double uwo_single_cin(double pbot, double thv0bot, double ptop, double thv0top, double thvubot,
                      double thvutop);
void   uwo_fluxbelowinv(double cbmf, const double *ps0, int mkx, int kinv, double dt, double xsrc,
                        double xmean, double xtopin, double xbotin, double *xflx);
void   uwo_positive_moisture_single(double xlv, double xls, int mkx, double dt, double qvmin,
                                    double qlmin, double qimin, const double *dp, double *qv,
                                    double *ql, double *qi, double *s, double *qvten,
                                    double *qlten, double *qiten, double *sten);
/* The host-side evaluation of the portable math routines (uw_math.h): fn 0 exp, 1 log, 2 pow, 3 erfc. */
void   uwo_uwmath(int fn, const double *x, const double *y, double *out, int n);
/* findsp (uwshcu.F90:5164-5454) over columns 1..ncol of (mix, pver) arrays; returns the status. */
int    uwo_findsp(int mix, int ncol, int pver, const double *q, const double *t, const double *p,
                  double *tsp, double *qsp);

#ifdef __cplusplus
}
#endif
#endif
