/*
 * uwshcu.h -- C ABI of the B200 UW shallow-cumulus library (libuwshcu_b200.so).
 *
 * Drop-in for the per-column driver of the UW shallow convection scheme of CAM / CAS-ESM
 * (guirenbenxin/HPC-and-climate-model, src/physics/uwshcu.F90).  Every entry point takes plain
 * pointers and sizes.  Host entry points follow Fortran calling conventions (all arguments by
 * reference, trailing underscore) so a Fortran caller binds them with an iso_c_binding interface
 * block; arrays are column-major with the column index fastest and leading dimension `mix`, exactly
 * as the Fortran routines declare them.
 *
 * All entry points return an int status: 0 on success, > 0 for the conditions on which the
 * reference stops the model with endrun (the outputs are still produced), < 0 for errors that
 * prevented the computation.  Nothing in the library prints or aborts.
 */
#ifndef UWSHCU_B200_H
#define UWSHCU_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define UWSHCU_OK 0
#define UWSHCU_ERR_MU_INCONSISTENT 1     /* uwshcu.F90:2119-2122 'Critical error in mu calculation' */
#define UWSHCU_ERR_FINDSP_NONCONVERGED 2 /* uwshcu.F90:5423-5431 'findsp not converging'           */
#define UWSHCU_ERR_FINDSP_ENTHALPY 3     /* uwshcu.F90:5435-5447 'enthalpy is not conserved'       */
#define UWSHCU_WARN_NONFINITE_INPUT 4    /* no counterpart in the reference: a column had a NaN or Inf
                                            input; it took the exit path (zero tendencies, cush = -1,
                                            exit bit UWSHCU_EXIT_NONFINITE in diag_int row 0) and
                                            every other column is computed as usual.  Reported
                                            when none of 1..3 occurred.                          */
#define UWSHCU_EXIT_NONFINITE (1 << 11)  /* diag_int row 0 (exit flags): the non-finite-input exit */
#define UWSHCU_ERR_BAD_ARGS (-1)         /* null pointer or dimension out of range                 */
#define UWSHCU_ERR_NOT_INITIALIZED (-2)  /* uwshcu_init was not called                             */
#define UWSHCU_ERR_CUDA (-3)             /* CUDA runtime error (uwshcu_last_cuda_error names it)   */
#define UWSHCU_ERR_NO_DEVICE (-4)        /* no CUDA device visible                                 */
#define UWSHCU_ERR_ALLOC (-5)            /* device or pinned host allocation failed                */
#define UWSHCU_ERR_TOO_LARGE (-6)        /* size beyond a fixed limit (UWSHCU_NOALLOC_MAX_COLUMNS) */

#define UWSHCU_MAX_LEVELS 63             /* mkx limit of the compiled kernels                      */
#define UWSHCU_MAX_TRACERS 32            /* ncnst limit of the compiled kernels                    */

/* Precision modes of the device path (uwshcu_set_precision). */
#define UWSHCU_PREC_FP64 0               /* FP64 throughout, Fortran evaluation order, no FMA      */
#define UWSHCU_PREC_MIXED 1              /* FP32 bulk, FP64 conden/roots/qsinvert/implicit CIN/
                                            positive_moisture, Kahan vertical sums (ncnst <= 5).
                                            1.7x the FP64 path; column heating/moistening/precip
                                            ~0.9 % relative RMS (cloud tops of ~0.6 % of the
                                            convecting columns move)                            */
#define UWSHCU_PREC_FAST 2               /* FP64 throughout with a Newton conden that stops each
                                            lane after its first step below 1e-10 T and divides
                                            twice per step; FMA contraction allowed.  Not
                                            bit-exact (~1e-12 relative per conden call); about
                                            the FP64 path's speed                              */

/* ---- set-up -------------------------------------------------------------------------------- */

/* Replaces init_uwshcu (uwshcu.F90:102-249) + esinti/gestbl (esinti.F90:38-51,
 * wv_saturation.F90:82-204) + the constituent metadata compute_uwshcu reads (qmin,
 * constituents.F90:54; cnst_get_type_byind; cnst_get_ind NUMLIQ/NUMICE, uwshcu.F90:1076-1077).
 * Host-only: builds the saturation table and stores the constants; the device copy is made on the
 * first compute call.  ixnumliq/ixnumice are 1-based; cnst_wet[m] != 0 marks a 'wet' tracer. */
int uwshcu_init(double xlv, double cp, double xlf, double zvir, double r, double g, double ep2,
                double tmin, double tmax, double ttrice, int icephs, double epsqs, double rgasv,
                double tmelt, int ncnst, const double *qmin, const int *cnst_wet, int ixnumliq,
                int ixnumice);

/* Replaces uwshcu_readnl (uwshcu.F90:58-98): the penetrative-entrainment efficiency rpen. */
int uwshcu_set_rpen(double rpen);

/* Tuning parameters: rpen (as uwshcu_set_rpen) and the compute_uwshcu parameters rle (critical
 * stopping distance for lateral entrainment), rkm (air involved in buoyancy sorting) and criqc
 * (maximum updraft condensate), Fortran parameters at uwshcu.F90:1036, 1038, 1065 with the values
 * 0.1, 14 and 0.7e-3 that uwshcu_init_default sets.  Must follow uwshcu_init; non-positive values
 * (negative criqc) are rejected. */
int uwshcu_set_params(double rpen, double rle, double rkm, double criqc);

/* uwshcu_init + uwshcu_set_params with the CESM shr_const values CAM passes (convect_shallow.F90:280,
 * physpkg.F90:638), rpen = 10, rle = 0.1, rkm = 14, criqc = 0.7e-3, five tracers (Q, CLDLIQ, CLDICE, NUMLIQ, NUMICE) with
 * qmin = {1e-12, 0, 0, 0, 0}. */
int uwshcu_init_default(void);

/* Precision of the device path: UWSHCU_PREC_FP64 (default), UWSHCU_PREC_MIXED or UWSHCU_PREC_FAST. */
int uwshcu_set_precision(int mode);

/* Kernel schedules (uwshcu_set_schedule). */
#define UWSHCU_SCHED_SINGLE_PASS 0       /* one launch, every column runs the whole scheme          */
#define UWSHCU_SCHED_TWO_PHASE 1         /* trigger pass over all columns, then the convecting
                                            columns from a device worklist                        */
#define UWSHCU_SCHED_SORTED 2            /* default: two-phase with the worklist pass split at the CIN
                                            decision of iteration 2: the implicit-CIN columns
                                            finish in a second launch, in warps sorted by their
                                            iteration-1 updraft depth (every precision mode).
                                            Holds up to 4 GiB of device memory per stream for the
                                            column state.                                        */

/* Select the kernel schedule; all give identical results. */
int uwshcu_set_schedule(int schedule);

/* Cap on the columns one call of the sorted schedule hands to its second launch (per stream;
 * 0 = default, bounded by 4 GiB of state, about 160,000 columns at 30 levels and 5 tracers;
 * values below 32 count as 32).  Columns beyond the cap finish in the first launch: the results are
 * the same, the memory smaller, the sorting partial.  No counterpart in the reference. */
int uwshcu_set_hand_slots(int slots);

/* Opt-in timing of the two-phase schedule: when on, every call records CUDA events on its stream
 * around the trigger launch and the worklist launch (up to 256 calls between reads). */
int uwshcu_set_profiling(int on);

/* Wait for the recorded calls and return their number, the summed device time of the trigger and
 * worklist launches in milliseconds and (optional) the worklist length of the last call; resets. */
int uwshcu_profile_read(int *calls, double *trigger_ms, double *list_ms, int *list_columns);

/* Host-array entries (compute_uwshcu_, compute_uwshcu_inv_, bxcompute_uwshcu_inv_): split a call
 * into chunks of chunk_columns columns (0: one chunk) pipelined over `streams` CUDA streams (1..8)
 * of decreasing priority, so that copies in and out and the host-side packing overlap the
 * computation.  Results do not depend on it.  Default (and chunk_columns = -1, streams ignored):
 * the shape follows each call's size, chunks of iend/8 columns rounded up to 1,024 and clamped to
 * 32,768 .. 262,144, over 4 streams up to 65,536-column chunks and 2 streams above; where the call
 * holds enough columns the first two and the last two chunks are a quarter and a half of that size
 * (32,768 at least), so that the computation starts sooner and the last copy out is shorter
 * (page-locked arrays: 259,200 columns in ~75 ms, 1,048,576 in ~210 ms against 217 ms with uniform
 * 131,072-column chunks and 272 ms with 32,768 x 4).  chunk_columns < -1: chunks of -chunk_columns
 * columns over `streams` streams with those ramped ends. */
int uwshcu_set_pipeline(int chunk_columns, int streams);

/* No counterpart in the reference.  on = 1: every worklist pass (device-array calls per caller
 * stream, host-array calls per device) orders its convecting columns by the updraft the same
 * column index had in the previous call (explicit-CIN columns first, then by cloud-top depth above
 * the release level), so that the lanes of a warp climb about as far.  A model that calls with the
 * same column layout every time step (CAM's chunks) gets warps of like columns, as the weather
 * changes slowly from step to step; results do not depend on it.  Measured on 1,048,576 columns
 * whose state evolves by the computed tendencies each step: 2-6 % less time per step; on repeated
 * identical inputs (the upper bound) 8 %.  Costs one sort of the worklist per pass and an int per
 * column (uwshcu_compute_device_noalloc, which allocates nothing, keeps trigger order).  on = 0
 * (default): trigger order. */
int uwshcu_set_depth_order(int on);

/* Threads per block of the column kernel (0 = built-in default). */
int uwshcu_set_block(int threads);

/* Copy of the 250-entry saturation-vapour-pressure table (wv_saturation.F90 estbl). */
int uwshcu_get_estbl(double *out250);

/* Release the device arena and pinned staging buffers. */
int uwshcu_finalize(void);

/* Text of the last CUDA error seen by the library ("" if none). */
const char *uwshcu_last_cuda_error(void);

/* ---- host entry points (Fortran conventions) --------------------------------------------------- */

/* compute_uwshcu (uwshcu.F90:478-492), argument list unchanged.  Arrays (mix, 0:mkx), (mix, mkx),
 * (mix, mkx, ncnst) with k = 1 the surface layer; columns 1..iend are computed.  `qsat` (the
 * fqsatd function pointer) and `lchnk` are accepted and ignored: the library evaluates the
 * saturation functions of wv_saturation itself.  cldfrct/concldfrct/massflx_sh are accepted and
 * unused, as in the Fortran with shallow_closure_scheme = 'cam'. */
int compute_uwshcu_(const int *mix, const int *mkx, const int *iend, const int *ncnst,
                    const double *dt, const double *ps0_in, const double *zs0_in,
                    const double *p0_in, const double *z0_in, const double *dp0_in,
                    const double *u0_in, const double *v0_in, const double *qv0_in,
                    const double *ql0_in, const double *qi0_in, const double *t0_in,
                    const double *s0_in, const double *tr0_in, const double *tke_in,
                    const double *cldfrct_in, const double *concldfrct_in, const double *pblh_in,
                    double *cush_inout, double *umf_out, double *slflx_out, double *qtflx_out,
                    double *flxprc1_out, double *flxsnow1_out, double *qvten_out,
                    double *qlten_out, double *qiten_out, double *sten_out, double *uten_out,
                    double *vten_out, double *trten_out, double *qrten_out, double *qsten_out,
                    double *precip_out, double *snow_out, double *evapc_out, double *cufrc_out,
                    double *qcu_out, double *qlu_out, double *qiu_out, double *cbmf_out,
                    double *qc_out, double *rliq_out, const double *massflx_sh, double *cnt_out,
                    double *cnb_out, void *qsat, const int *lchnk, const double *dpdry0_in,
                    double *wu_out);

/* compute_uwshcu_inv (uwshcu.F90:251-265, called from convect_shallow.F90:585-600): the same
 * computation on CAM's top-down level order.  The level reversal is folded into the kernel's
 * loads and stores instead of being copied.  tpert2/qpert2 are unused (shallow_zmh_pert =
 * .false., uwshcu.F90:40). */
int compute_uwshcu_inv_(const int *mix, const int *mkx, const int *iend, const int *ncnst,
                        const double *dt, const double *ps0_inv, const double *zs0_inv,
                        const double *p0_inv, const double *z0_inv, const double *dp0_inv,
                        const double *u0_inv, const double *v0_inv, const double *qv0_inv,
                        const double *ql0_inv, const double *qi0_inv, const double *t0_inv,
                        const double *s0_inv, const double *tr0_inv, const double *tke_inv,
                        const double *cldfrct_inv, const double *concldfrct_inv,
                        const double *pblh, double *cush, const double *tpert2,
                        const double *qpert2, const double *massflx_sh, double *umf_inv,
                        double *slflx_inv, double *qtflx_inv, double *flxprc1_inv,
                        double *flxsnow1_inv, double *qvten_inv, double *qlten_inv,
                        double *qiten_inv, double *sten_inv, double *uten_inv, double *vten_inv,
                        double *trten_inv, double *qrten_inv, double *qsten_inv, double *precip,
                        double *snow, double *evapc_inv, double *cufrc_inv, double *qcu_inv,
                        double *qlu_inv, double *qiu_inv, double *cbmf, double *qc_inv,
                        double *rliq, double *cnt_inv, double *cnb_inv, void *qsat,
                        const int *lchnk, const double *dpdry0_inv, double *wu_inv);

/* bxcompute_uwshcu_inv_ (src/physics/bxcompute_uwshcu_inv.cpp:6172-6184): the entry of the
 * reference's own GPU drop-in, same argument list (pcols, pver, ncol, pcnst, ztodt, ..., lchnk,
 * dpdry0_inv, wu_inv).  Runs compute_uwshcu_inv_; unlike the reference it honours pcols as the
 * leading dimension when ncol < pcols and computes every column (no ncol/32 tail drop). */
int bxcompute_uwshcu_inv_(const int *pcols, const int *pver, const int *ncol, const int *pcnst,
                          const double *ztodt, const double *ps0_inv, const double *zs0_inv,
                          const double *p0_inv, const double *z0_inv, const double *dp0_inv,
                          const double *u0_inv, const double *v0_inv, const double *qv0_inv,
                          const double *ql0_inv, const double *qi0_inv, const double *t0_inv,
                          const double *s0_inv, const double *tr0_inv, const double *tke_inv,
                          const double *cldfrct_inv, const double *concldfrct_inv,
                          const double *pblh, double *cush, double *umf_inv, double *slflx_inv,
                          double *qtflx_inv, double *flxprc1_inv, double *flxsnow1_inv,
                          double *qvten_inv, double *qlten_inv, double *qiten_inv,
                          double *sten_inv, double *uten_inv, double *vten_inv, double *trten_inv,
                          double *qrten_inv, double *qsten_inv, double *precip, double *snow,
                          double *evapc_inv, double *cufrc_inv, double *qcu_inv, double *qlu_inv,
                          double *qiu_inv, double *cbmf, double *qc_inv, double *rliq,
                          double *cnt_inv, double *cnb_inv, const int *lchnk,
                          const double *dpdry0_inv, double *wu_inv);

/* ---- compute_zwshcu: the CAS-ESM variant of the scheme (zwshcu.F90) ----------------------------- */

/* compute_zwshcu (zwshcu.F90:630-644), argument list unchanged: compute_uwshcu's arguments with the
 * pressure velocity omega (mix, mkx) [Pa/s, negative upwards], massflx_sh and tpert2 between rliq_out
 * and cnt_out.  Same column code as compute_uwshcu_ plus the variant's options (uwshcu_set_zw_options):
 * with zmh_shallow_lf the closure lowers wcrit by min(max(-omega, 0), 3) / rho0inv / 9.8 at the
 * PBL-top layer (zwshcu.F90:2295-2303), and the optional buoyancy-based entrainment
 * (zwshcu.F90:2818-2844) and cloud-fraction enhancement (zwshcu.F90:4413-4449).  tpert2 is read by the
 * perturbation options only, which are not built (off in the reference).  rpen and rkm keep the values
 * of uwshcu_set_params (the variant's namelist defaults are rpen = 15, rkm = 10,
 * zwshcu.F90:43-44).  omega = 0 everywhere gives compute_uwshcu_'s results bit for bit.  FP64
 * precision setting only (UWSHCU_ERR_BAD_ARGS otherwise). */
int compute_zwshcu_(const int *mix, const int *mkx, const int *iend, const int *ncnst,
                    const double *dt, const double *ps0_in, const double *zs0_in,
                    const double *p0_in, const double *z0_in, const double *dp0_in,
                    const double *u0_in, const double *v0_in, const double *qv0_in,
                    const double *ql0_in, const double *qi0_in, const double *t0_in,
                    const double *s0_in, const double *tr0_in, const double *tke_in,
                    const double *cldfrct_in, const double *concldfrct_in, const double *pblh_in,
                    double *cush_inout, double *umf_out, double *slflx_out, double *qtflx_out,
                    double *flxprc1_out, double *flxsnow1_out, double *qvten_out,
                    double *qlten_out, double *qiten_out, double *sten_out, double *uten_out,
                    double *vten_out, double *trten_out, double *qrten_out, double *qsten_out,
                    double *precip_out, double *snow_out, double *evapc_out, double *cufrc_out,
                    double *qcu_out, double *qlu_out, double *qiu_out, double *cbmf_out,
                    double *qc_out, double *rliq_out, const double *omega, const double *massflx_sh,
                    const double *tpert2, double *cnt_out, double *cnb_out, void *qsat,
                    const int *lchnk, const double *dpdry0_in, double *wu_out);

/* compute_zwshcu_inv (zwshcu.F90:336-628, called from convect_shallow.F90:717-731), argument list
 * unchanged: CAM's top-down level order, with omega_inv, tpert2, qpert2, gradt, gradq, landfrac, lat,
 * lon and massflx_sh after cush.  gradt, gradq, landfrac, lat, lon, tpert2 and qpert2 feed the
 * perturbation options only (zwshcu.F90:511-566, all off in the reference) and are unused. */
int compute_zwshcu_inv_(const int *mix, const int *mkx, const int *iend, const int *ncnst,
                        const double *dt, const double *ps0_inv, const double *zs0_inv,
                        const double *p0_inv, const double *z0_inv, const double *dp0_inv,
                        const double *u0_inv, const double *v0_inv, const double *qv0_inv,
                        const double *ql0_inv, const double *qi0_inv, const double *t0_inv,
                        const double *s0_inv, const double *tr0_inv, const double *tke_inv,
                        const double *cldfrct_inv, const double *concldfrct_inv,
                        const double *pblh, double *cush, const double *omega_inv,
                        const double *tpert2, const double *qpert2, const double *gradt,
                        const double *gradq, const double *landfrac, const double *lat,
                        const double *lon, const double *massflx_sh, double *umf_inv,
                        double *slflx_inv, double *qtflx_inv, double *flxprc1_inv,
                        double *flxsnow1_inv, double *qvten_inv, double *qlten_inv,
                        double *qiten_inv, double *sten_inv, double *uten_inv, double *vten_inv,
                        double *trten_inv, double *qrten_inv, double *qsten_inv, double *precip,
                        double *snow, double *evapc_inv, double *cufrc_inv, double *qcu_inv,
                        double *qlu_inv, double *qiu_inv, double *cbmf, double *qc_inv,
                        double *rliq, double *cnt_inv, double *cnb_inv, void *qsat,
                        const int *lchnk, const double *dpdry0_inv, double *wu_inv);

/* Options of the compute_zwshcu entries (zwshcu.F90:30-59 namelist uwshcu_nl, cloud_fraction.F90:52):
 * zmh_shallow_lf, zmh_shallow_fwcrit, zmh_shallow_ent, zmh_ent0, zmh_cloud_sh, zmh_ufrcd, zmh_ufrc0,
 * zmh_ufrcz.  uwshcu_init sets the reference's defaults 1, 1.0, 0, 0.015, 0, 2.0, 2.0, 2.0; they do not
 * affect the compute_uwshcu entries. */
int uwshcu_set_zw_options(int lf, double fwcrit, int ent, double ent0, int cloud_sh, double ufrcd,
                          double ufrc0, double ufrcz);

/* ---- device-resident entry point -------------------------------------------------------------- */

/* The computation of compute_uwshcu (inv = 0) or compute_uwshcu_inv (inv = 1) on arrays that
 * already live in device memory, in the same layouts with leading dimension mix.  Enqueued on
 * `stream` (a cudaStream_t, 0 = legacy default stream) and returns without synchronising;
 * diag_int (8, mix) and diag_real (8, mix) are optional per-column diagnostics (exit/limit flags,
 * kinv, klcl, klfc, krel, kbup, kpen; cin, cinlcl, plcl, plfc, pinv, pbup, ppen, tkeavg).
 * The endrun conditions of the call are collected on the device; uwshcu_device_status(stream)
 * waits for the stream and returns them.
 * Streams: the library keeps a worklist, a hand-off region and an endrun word per caller stream
 * (up to 32 streams per device; a call on a 33rd stream synchronises the device and takes over the
 * least recently used stream's set, whose uncollected endrun bits are lost), so calls on different
 * streams may overlap on the GPU (one stream per host thread).  Calls on one stream run in stream
 * order.  cudaStreamPerThread is one handle for all host threads: order such calls yourself.
 * The same holds for uwshcu_compute_member, uwshcu_tangent_device and uwshcu_adjoint_device. */
int uwshcu_compute_device(int mix, int mkx, int iend, int ncnst, double dt, int inv,
                          const double *ps0, const double *zs0, const double *p0,
                          const double *z0, const double *dp0, const double *u0, const double *v0,
                          const double *qv0, const double *ql0, const double *qi0,
                          const double *t0, const double *s0, const double *tr0,
                          const double *tke, const double *pblh, double *cush, double *umf,
                          double *slflx, double *qtflx, double *flxprc1, double *flxsnow1,
                          double *qvten, double *qlten, double *qiten, double *sten, double *uten,
                          double *vten, double *trten, double *qrten, double *qsten,
                          double *precip, double *snow, double *evapc, double *cufrc, double *qcu,
                          double *qlu, double *qiu, double *cbmf, double *qc, double *rliq,
                          double *cnt, double *cnb, const double *dpdry0, double *wu,
                          int *diag_int, double *diag_real, void *stream);

/* compute_zwshcu on device-resident arrays: uwshcu_compute_device's arguments plus omega (mix, mkx),
 * in the level order of the call (inv). */
int compute_zwshcu_device(int mix, int mkx, int iend, int ncnst, double dt, int inv,
                          const double *ps0, const double *zs0, const double *p0,
                          const double *z0, const double *dp0, const double *u0, const double *v0,
                          const double *qv0, const double *ql0, const double *qi0,
                          const double *t0, const double *s0, const double *tr0,
                          const double *tke, const double *pblh, const double *omega, double *cush,
                          double *umf, double *slflx, double *qtflx, double *flxprc1,
                          double *flxsnow1, double *qvten, double *qlten, double *qiten, double *sten,
                          double *uten, double *vten, double *trten, double *qrten, double *qsten,
                          double *precip, double *snow, double *evapc, double *cufrc, double *qcu,
                          double *qlu, double *qiu, double *cbmf, double *qc, double *rliq,
                          double *cnt, double *cnb, const double *dpdry0, double *wu,
                          int *diag_int, double *diag_real, void *stream);

/* Wait for `stream` and return the status collected by the device-array calls enqueued on that
 * stream (uwshcu_compute_device, uwshcu_compute_member, uwshcu_tangent_device) since the previous
 * uwshcu_device_status call on it; calls on other streams are not reported and not reset.
 * (uwshcu_compute_device_noalloc reports through its own status_bits instead.) */
int uwshcu_device_status(void *stream);

/* ---- batched uneven launches ----------------------------------------------------------------- */

/* One ensemble member / grid of a batch: the arguments of uwshcu_compute_device for one set of
 * device-resident arrays (ncnst is the one given to uwshcu_init).  Members may differ in mkx, mix,
 * iend and level order. */
typedef struct uwshcu_member {
    int mix, mkx, iend, inv;
    double dt;
    const double *ps0, *zs0, *p0, *z0, *dp0, *u0, *v0, *qv0, *ql0, *qi0, *t0, *s0, *tr0, *tke, *pblh;
    double *cush, *umf, *slflx, *qtflx, *flxprc1, *flxsnow1, *qvten, *qlten, *qiten, *sten, *uten,
        *vten, *trten, *qrten, *qsten, *precip, *snow, *evapc, *cufrc, *qcu, *qlu, *qiu, *cbmf, *qc,
        *rliq, *cnt, *cnb;
    const double *dpdry0;
    double *wu;
    int *diag_int;      /* optional, as in uwshcu_compute_device */
    double *diag_real;  /* optional */
    double *diag_level; /* optional per-level diagnostics (UWSHCU_NDL, mkx + 1, mix), see below */
} uwshcu_member;

/* Per-level diagnostics: the history fields compute_uwshcu writes for every column
 * (uwshcu.F90:1945-1990 after the explicit-CIN fallback, :4383-4433 otherwise, zeros at the exit
 * :4484-4529).  Array (UWSHCU_NDL, mkx + 1, mix), element (j, k, i) at (j * (mkx + 1) + k) * mix + i,
 * levels bottom-up (k = 0 at the surface) for both level orders.  Rows 0..8 are interface fields
 * (k = 0..mkx), rows 9..12 layer fields (k = 1..mkx; k = 0 holds 0).  The Fortran stores them
 * top-down in its *_out arrays (ufrc_out(i, mkx:0:-1) = ufrc(0:mkx)); reverse k to get that order. */
#define UWSHCU_DL_UFRC 0     /* updraft fractional area */
#define UWSHCU_DL_QTU 1      /* updraft total water */
#define UWSHCU_DL_THLU 2     /* updraft liquid-water potential temperature */
#define UWSHCU_DL_THVU 3     /* updraft virtual potential temperature */
#define UWSHCU_DL_UU 4       /* updraft zonal wind */
#define UWSHCU_DL_VU 5       /* updraft meridional wind */
#define UWSHCU_DL_UEMF 6     /* net updraft mass flux including penetrative entrainment */
#define UWSHCU_DL_FLXRAIN 7  /* rain flux */
#define UWSHCU_DL_FLXSNOW 8  /* snow flux */
#define UWSHCU_DL_FER 9      /* lateral fractional entrainment rate */
#define UWSHCU_DL_FDR 10     /* lateral fractional detrainment rate */
#define UWSHCU_DL_DWTEN 11   /* detrained liquid water tendency */
#define UWSHCU_DL_DITEN 12   /* detrained ice tendency */
#define UWSHCU_NDL 13

/* uwshcu_compute_device with its arguments in a member struct (ncnst from uwshcu_init), which also
 * carries the optional per-level diagnostics.  No counterpart in the reference: compute_uwshcu
 * writes these fields to module arrays for CAM's history output (outfld), which a C caller cannot
 * reach.  Same status codes, stream semantics and results as uwshcu_compute_device. */
int uwshcu_compute_member(const uwshcu_member *m, void *stream);

#define UWSHCU_MAX_MEMBERS 8

/* No counterpart in the reference (CAM calls compute_uwshcu once per chunk; the reference's
 * load-balanced ports, mpiuwshcu.cpp / bxcompute_uwshcu_inv.cpp, launch one grid per call).
 * A batch plan for up to UWSHCU_MAX_MEMBERS members on the current device: the library allocates
 * the plan's worklists and counters here, once.  A run makes one trigger launch and one persistent
 * worklist launch per level class (mkx + 1 <= 32 or <= 64): the worklist kernel pulls warps of
 * one member's convecting columns from a device counter until every member's queue is drained.
 * The plan runs in the precision mode set when it is created (uwshcu_set_precision: FP64, FAST, or
 * MIXED with ncnst <= 5).  Results are the same bits as uwshcu_compute_device on each member in
 * that mode. */
int uwshcu_batch_create(int nmembers, const uwshcu_member *members, void **plan);

/* Enqueue one run of the plan on `stream` (the captured CUDA graph when there is one). */
int uwshcu_batch_run(void *plan, void *stream);

/* Capture one run into a CUDA graph held by the plan; later uwshcu_batch_run calls replay it.
 * The capture itself launches nothing. */
int uwshcu_batch_capture(void *plan, void *stream);

/* Time the compiled launch shapes of the worklist pass (block of 64 or 128 threads, register cap
 * 168/128/80 = 3/4/6 blocks of 128 per SM in FP64, 128 in the other modes, 32 or 64 columns per
 * warp task) on this plan's data and keep the fastest in the plan (it drops a captured graph).  Runs the scheme several times:
 * the outputs are overwritten and cush is restored to its value on entry.  Reports the choice. */
int uwshcu_batch_autotune(void *plan, void *stream, int *block, int *regcap_blocks, int *chunk);

/* Wait for `stream` and return the endrun status collected by the plan's runs since the last call. */
int uwshcu_batch_status(void *plan, void *stream);

/* Release the plan (its graph, worklists and counters). */
int uwshcu_batch_destroy(void *plan);

/* ---- tangent-linear model ---------------------------------------------------------------------- */

/* Directions and tangent outputs of a tangent-linear call.  The direction arrays have the layout of
 * the call's inputs (t0, qv0: (mix, mkx); tke: (mix, mkx+1); pblh: (mix)); NULL means zero.  The
 * tangent outputs have the layout of the outputs of the same name. */
typedef struct uwshcu_tangent {
    const double *dt0, *dqv0, *dtke, *dpblh;
    double drpen, drle, drkm, dcriqc;     /* directions in the tuning parameters */
    double *cush, *umf, *slflx, *qtflx, *flxprc1, *flxsnow1, *qvten, *qlten, *qiten, *sten, *uten,
        *vten, *trten, *qrten, *qsten, *precip, *snow, *evapc, *cufrc, *qcu, *qlu, *qiu, *cbmf, *qc,
        *rliq, *wu;
} uwshcu_tangent;

/* No counterpart in the reference.  Tangent-linear model of compute_uwshcu: the outputs of `m`
 * (bit for bit those of uwshcu_compute_device) and their derivatives along the direction in `t`
 * (forward mode through every statement of the scheme, the Newton iterations included; the
 * derivative is that of the branch the FP64 path takes).  Device arrays, enqueued on `stream`;
 * FP64 precision setting only; mkx + 1 <= 64, ncnst <= 5. */
int uwshcu_tangent_device(const uwshcu_member *m, const uwshcu_tangent *t, void *stream);

/* ---- adjoint model ------------------------------------------------------------------------------ */

/* Cotangents and gradients of an adjoint call (device arrays).  The cotangents ("output weights")
 * have the layouts of the outputs of the same name; NULL means zero.  The gradients have the layouts
 * of the inputs (t0, qv0: (mix, mkx); tke: (mix, mkx+1); pblh: (mix)); the tuning-parameter
 * gradients are per column (mix): the gradient of the whole call is their sum over the columns.
 * A NULL gradient is not computed. */
typedef struct uwshcu_adjoint {
    const double *cush, *umf, *slflx, *qtflx, *flxprc1, *flxsnow1, *qvten, *qlten, *qiten, *sten,
        *uten, *vten, *trten, *qrten, *qsten, *precip, *snow, *evapc, *cufrc, *qcu, *qlu, *qiu, *cbmf,
        *qc, *rliq, *wu;
    double *t0, *qv0, *tke, *pblh;
    double *rpen, *rle, *rkm, *criqc;
} uwshcu_adjoint;

/* No counterpart in the reference.  Adjoint (reverse mode) of compute_uwshcu: for the member `m` it
 * computes the outputs (bit for bit those of uwshcu_compute_device) and the gradient of
 * J = sum over outputs of (cotangent x output) with respect to t0, qv0, tke, pblh and, per column,
 * rpen, rle, rkm and criqc -- the transpose of uwshcu_tangent_device (the derivative is that of the
 * branch the FP64 path takes; a saturation adjustment's derivative is taken at its converged
 * state).  The columns that leave the scheme in the trigger pass have constant outputs and zero
 * gradients; the others run a taped forward sweep (a tape per warp of 32 columns) and a reverse
 * sweep, in batches that fit 85 % of the device memory that is free or already held by the adjoint
 * buffer.  The library keeps that buffer between calls (release it with uwshcu_adjoint_release) and
 * sizes the tapes from the previous call's largest tape.  Waits for `stream` before it returns.
 * FP64 precision setting; mkx + 1 <= 64, ncnst <= 5.  UWSHCU_ERR_TOO_LARGE if a warp's tape exceeds
 * 2^18 rows (mkx + 1 <= 32) or 2^19 rows (33 .. 64 levels). */
int uwshcu_adjoint_device(const uwshcu_member *m, const uwshcu_adjoint *a, void *stream);

/* No counterpart in the reference.  uwshcu_adjoint_device (same outputs and gradients, bit for bit)
 * that also writes, per column, how far rounding in the reverse sweep moved that column's gradients:
 * the reverse sweep runs again on the same tape for the two parts w1, w2 of a split of the
 * cotangents (w1 + w2 = w exactly, a fixed fraction in [1/2, 7/8) per cotangent), and
 * defect[i] = the largest, over the gradients asked for (non-NULL in `a`), of
 * max |g(w) - g(w1) - g(w2)| / max (|g(w1)| + |g(w2)|) over that gradient's entries of column i.
 * The sweep is linear in w, so only rounding makes it non-zero: ~1e-16 .. 1e-14 on a well-
 * conditioned column; a column whose intermediate adjoints cancel over many orders of magnitude
 * shows its lost digits here (a gradient with defect 1e-6 has about 6 correct digits fewer than
 * FP64's 16).  0 for the columns that leave the scheme in the trigger pass.  `defect`: device array
 * (mix), not NULL.  Costs three reverse sweeps instead of one. */
int uwshcu_adjoint_device_checked(const uwshcu_member *m, const uwshcu_adjoint *a, double *defect,
                                  void *stream);

/* Largest tape of the last uwshcu_adjoint_device call, in rows per warp of 32 columns (a sizing
 * aid). */
int uwshcu_adjoint_last_records(void);

/* No counterpart in the reference.  Tape capacity of the next uwshcu_adjoint_device call, in rows per
 * warp (1 .. 2^19, at most the full capacity of the call's level count; 0: the library's choice).  A
 * batch that overflows it makes that call start again at the full capacity; later calls size the
 * tapes from the largest tape seen. */
int uwshcu_set_adjoint_rows(int rows);

/* No counterpart in the reference.  Frees the adjoint buffer on every device (uwshcu_finalize
 * frees it too); the next adjoint call allocates it again. */
int uwshcu_adjoint_release(void);

/* Column limit of uwshcu_compute_device_noalloc: its worklist is one fixed device array of
 * 64 + UWSHCU_NOALLOC_MAX_COLUMNS ints (4 MiB + 256 B) that every GPU which loads the library holds
 * until the process exits. */
#define UWSHCU_NOALLOC_MAX_COLUMNS 1048576

/* No counterpart in the reference.  uwshcu_compute_device with the two-phase schedule (trigger
 * pass, then the convecting columns' pass) that allocates nothing: for callers that cannot
 * allocate device memory when they call the scheme -- a host model whose memory manager claims
 * the GPU's memory at start-up and hands out only its own pool, where a cudaMalloc of this library
 * would fail or fragment that pool, and time-step code that must not call cudaMalloc/cudaFree
 * because they can synchronize the whole device.  The caller passes the inputs and outputs as for
 * uwshcu_compute_device (device pointers, enqueued on `stream`, same precision and block settings);
 * the worklist of convecting columns lives in a file-scope device array of the library instead of
 * a cudaMalloc'd buffer, and the call makes no cudaMalloc, cudaFree or other allocating call.
 *   - iend > UWSHCU_NOALLOC_MAX_COLUMNS is rejected with UWSHCU_ERR_TOO_LARGE
 *     (uwshcu_last_cuda_error names the limit); split larger calls.
 *   - The first call on each device does the set-up: it looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current and, unless another entry point already
 *     did, copies the constants to the device (cudaMemcpyToSymbol); the first call after each
 *     uwshcu_init / uwshcu_set_rpen copies them again.  Make that first call before any stream
 *     capture.
 *   - Every call on a device shares the one array, which keeps the last call's contents; each
 *     call clears the parts that must start at zero on its stream.  Calls whose GPU work overlaps
 *     (two streams, two host threads, or a call running beside another) race on the array and
 *     give wrong results: order them on one stream or with events.
 *   - status_bits: NULL, or a device pointer to one unsigned int that the call zeroes on `stream`
 *     and into which the kernels OR the endrun conditions of this call (1 mu inconsistency,
 *     2 findsp non-convergence, 4 findsp enthalpy, 8 non-finite input).  uwshcu_device_status
 *     does not see them.
 *   - The first call on a device can still make the CUDA driver allocate device memory: with lazy
 *     module loading (CUDA_MODULE_LOADING=LAZY, the default since CUDA 12.2) the library's kernels
 *     and the array itself are loaded when a call first uses them, and the first launches can
 *     enlarge the context's local-memory reservation for the kernels' stack frames.  Make one call
 *     per device during set-up, before the host's memory pool claims the GPU (or run with
 *     CUDA_MODULE_LOADING=EAGER); later calls allocate nothing. */
int uwshcu_compute_device_noalloc(int mix, int mkx, int iend, int ncnst, double dt, int inv,
                                  const double *ps0, const double *zs0, const double *p0,
                                  const double *z0, const double *dp0, const double *u0,
                                  const double *v0, const double *qv0, const double *ql0,
                                  const double *qi0, const double *t0, const double *s0,
                                  const double *tr0, const double *tke, const double *pblh,
                                  double *cush, double *umf, double *slflx, double *qtflx,
                                  double *flxprc1, double *flxsnow1, double *qvten, double *qlten,
                                  double *qiten, double *sten, double *uten, double *vten,
                                  double *trten, double *qrten, double *qsten, double *precip,
                                  double *snow, double *evapc, double *cufrc, double *qcu,
                                  double *qlu, double *qiu, double *cbmf, double *qc, double *rliq,
                                  double *cnt, double *cnb, const double *dpdry0, double *wu,
                                  int *diag_int, double *diag_real, unsigned int *status_bits,
                                  void *stream);

/* No counterpart in the reference.  Measures the FP64 throughput of the current device in TFLOP/s:
 * independent chains of fused multiply-adds over two full waves of blocks, best of three timed
 * launches on `stream` (after a warm-up).  The denominator of the FP64 roofline fractions of the
 * benchmark; allocates and frees 8 bytes of device memory. */
int uwshcu_fp64_peak(double *tflops, void *stream);

/* Column energy and water budgets of a call, on device arrays: check_energy_chng
 * (check_energy.F90:321-395) as CAM applies it after the shallow scheme (tphysbc.F90:446-447),
 * for the state before the call (s0, qv0, ql0, qi0, u0, v0, dp0: the call's inputs) and the
 * state advanced by dt with the call's tendencies.  Writes CAM's relative errors te_rer and
 * tw_rer (iend values; CAM flags |te_rer| > 1e-14 and |tw_rer| > 1e-10).  Level order as the call
 * (inv).  Enqueued on `stream`. */
int uwshcu_budget_device(int mix, int mkx, int iend, int inv, double dt, const double *s0,
                         const double *qv0, const double *ql0, const double *qi0, const double *u0,
                         const double *v0, const double *dp0, const double *sten,
                         const double *qvten, const double *qlten, const double *qiten,
                         const double *uten, const double *vten, const double *precip,
                         const double *snow, const double *rliq, double *te_rer, double *tw_rer,
                         void *stream);

/* Evaluate the library's exp (fn 0), log (1), pow (2, with y) or erfc (3) on n device values, on
 * the GPU, with the routines the kernels use.  They give the same bits as the host build of the
 * same routines, which is what makes the FP64 path reproducible on the CPU. */
int uwshcu_eval_math(int fn, const double *x, const double *y, double *out, int n, void *stream);

#ifdef __cplusplus
}
#endif
#endif
