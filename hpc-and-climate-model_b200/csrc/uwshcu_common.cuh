// uwshcu_common.cuh -- data shared by the UW shallow-cumulus kernels and the host library.
//
// Layout conventions (the Fortran compute_uwshcu argument layout, uwshcu.F90:529-580):
//   interface fields (mix, 0:mkx) -> a[k*mix + i],            k = 0 .. mkx, k = 0 at the surface
//   layer fields     (mix, mkx)   -> a[(k-1)*mix + i],        k = 1 .. mkx
//   tracer fields    (mix, mkx, ncnst) -> a[((m-1)*mkx + k-1)*mix + i]
// with i the 0-based column index.  Column index fastest means a warp of consecutive columns reads
// and writes 32 consecutive doubles for every (k, m): level-major structure of arrays.
#pragma once
#include <cstdint>

#define UW_NCMAX 32      // largest tracer count the kernels accept
#define UW_TBL 250       // saturation-vapour-pressure table length (wv_saturation.F90:43)

// Per-column integer diagnostics, array (UW_NDI, mix).
#define UW_DI_EXIT 0     // bitmask of the exit_* flags (uwshcu.F90:889-899); 0 = convection ran
#define UW_DI_LIMIT 1    // bitmask of the limit_* flags and ind_delcin (uwshcu.F90:901-910)
#define UW_DI_KINV 2
#define UW_DI_KLCL 3
#define UW_DI_KLFC 4
#define UW_DI_KREL 5
#define UW_DI_KBUP 6
#define UW_DI_KPEN 7
#define UW_NDI 8
// Per-column real diagnostics, array (UW_NDR, mix).
#define UW_DR_CIN 0
#define UW_DR_CINLCL 1
#define UW_DR_PLCL 2
#define UW_DR_PLFC 3
#define UW_DR_PINV 4
#define UW_DR_PBUP 5
#define UW_DR_PPEN 6
#define UW_DR_TKEAVG 7
#define UW_NDR 8
// Per-level diagnostics, array (UW_NDL, mkx + 1, mix): the history fields of compute_uwshcu
// (uwshcu.F90:1945-1990, :4383-4433), levels bottom-up k = 0 .. mkx for both level orders.  Interface
// fields fill k = 0 .. mkx; layer fields (UW_DL_FER and after) fill k = 1 .. mkx and hold 0 at k = 0.
#define UW_DL_UFRC 0
#define UW_DL_QTU 1
#define UW_DL_THLU 2
#define UW_DL_THVU 3
#define UW_DL_UU 4
#define UW_DL_VU 5
#define UW_DL_UEMF 6
#define UW_DL_FLXRAIN 7
#define UW_DL_FLXSNOW 8
#define UW_DL_FER 9
#define UW_DL_FDR 10
#define UW_DL_DWTEN 11
#define UW_DL_DITEN 12
#define UW_NDL 13

// exit_* bits
#define UW_X_UWCU (1 << 0)
#define UW_X_CONDEN (1 << 1)
#define UW_X_KLCLMKX (1 << 2)
#define UW_X_KLFCMKX (1 << 3)
#define UW_X_UFRC (1 << 4)
#define UW_X_WTW (1 << 5)
#define UW_X_DRYCORE (1 << 6)
#define UW_X_WU (1 << 7)
#define UW_X_CUFILTER (1 << 8)
#define UW_X_KINV1 (1 << 9)
#define UW_X_REI (1 << 10)
#define UW_X_NONFINITE (1 << 11)   // a non-finite input (no counterpart in the Fortran)
// limit_* bits
#define UW_L_SHCU (1 << 0)
#define UW_L_NEGCON (1 << 1)
#define UW_L_UFRC (1 << 2)
#define UW_L_PPEN (1 << 3)
#define UW_L_EMF (1 << 4)
#define UW_L_CINLCL (1 << 5)
#define UW_L_CIN (1 << 6)
#define UW_L_CBMF (1 << 7)
#define UW_L_REI (1 << 8)
#define UW_L_DELCIN (1 << 9)

// isfinite for the value types of the column code (double, float; the tangent-linear and adjoint
// value types add their own overloads).
#if defined(__CUDACC__)
__host__ __device__ inline bool uw_isfinite(double x) { return isfinite(x); }
__host__ __device__ inline bool uw_isfinite(float x) { return isfinite(x); }
#endif

// Device error word bits (set with atomicOr, read back by the host and mapped to status codes).
#define UW_ERRBIT_MU 1        // 'Critical error in mu calculation' (uwshcu.F90:2119-2122)
#define UW_ERRBIT_FINDSP 2    // findsp did not converge (uwshcu.F90:5423-5431)
#define UW_ERRBIT_ENTHALPY 4  // findsp enthalpy not conserved (uwshcu.F90:5435-5447)
#define UW_ERRBIT_NONFINITE 8 // a column had a non-finite input and took the exit path

// Physical constants and tables, set once by uwshcu_init and copied to __constant__ memory.
struct UwConst {
    // uwshcu module (uwshcu.F90:25-37)
    double xlv, xlf, xls, cp, zvir, r, g, ep2, p00, rovcp, rpen;
    double rle, rkm, criqc;   // compute_uwshcu parameters (uwshcu.F90:1036, 1038, 1065)
    double rinv;              // 1 / r, correctly rounded (divisions by r in conden)
    // compute_zwshcu options (zwshcu.F90:30-59, cloud_fraction.F90:52), in force for calls that pass
    // omega: zmh_shallow_lf, zmh_shallow_ent, zmh_cloud_sh, zmh_shallow_fwcrit, zmh_ent0, zmh_ufrcd,
    // zmh_ufrc0, zmh_ufrcz
    int zw_lf, zw_ent, zw_cloud_sh;
    double zw_fwcrit, zw_ent0, zw_ufrcd, zw_ufrc0, zw_ufrcz;
    // wv_saturation module (wv_saturation.F90:48-59)
    double tmin, tmax, ttrice, epsqs, rgasv, hlatf, hlatv, cpws, tmelt;
    double pcf[6];
    double omeps, trinv;   // 1 - epsqs and 1/ttrice, as vqsatd computes them on every call
    int icephs;
    // constituents
    int ncnst, ixnumliq, ixnumice;
    double qmin[UW_NCMAX];
    int wet[UW_NCMAX];
};

// Hand-off between the two launches of the split worklist pass (UW_MODE_LIST1 -> UW_MODE_RESUME),
// one region of device memory per stream that runs the pass.  Slots beyond cap are not handed off:
// those columns finish in the first launch.
#define UW_HAND_KEYS 64   // sort keys: 63 - iteration-1 updraft depth (deepest first)
struct UwHand {
    double* state;   // (uw_state_words, cap): word w of slot s at state[w * cap + s]
    int cap;         // slots
    int* count;      // slots requested by the first launch (may exceed cap)
    int* col;        // column of each slot
    int* key;        // sort key of each slot
    int* order;      // slots in key order (counting sort)
    int* hist;       // UW_HAND_KEYS counters of the sort
};

// One batch of the adjoint model (device addresses): slot t is worklist entry wl[b0 + t], t < nb, and
// warp w holds slots 32w .. 32w+31.  Warp w's tape (uw_adj.h) has rcap rows, its adjoints
// (index x of lane l at x * 32 + l) start at adj + w * astride; slot t's output-index table entry
// (f, k) is ids[(f * KP + k) * cap + t].
struct UwAdjHost {
    const int* wl;
    int b0, nb;
    void* ab;            // int2 operand indices, warp w at w * rcap * 32
    void* d;             // double2 partials, same layout
    int rcap;            // tape rows per warp
    int* ids;
    int cap;
    int* nrow;           // rows taken per warp
    int* ovf;            // tape overflow per warp
    double* adj;
    size_t astride;      // doubles of adjoints per warp
    unsigned int* status;
    int split;           // reverse sweep: 0 the cotangents, 1 and 2 the two parts of their split
    double* gsave;       // the split sweeps' gradients, 2 x (3 mkx + 6) x cap
    double* defect;      // per column: defect of linearity under the split (NULL: not computed)
};

// Pointers of one compute_uwshcu call (device addresses), in the Fortran argument order.
struct UwArgs {
    int mix, mkx, iend, ncnst;
    int inv;             // 1: level order of compute_uwshcu_inv (top-down), 0: bottom-up
    double dt;
    const double *ps0, *zs0, *p0, *z0, *dp0, *u0, *v0, *qv0, *ql0, *qi0, *t0, *s0, *tr0, *tke;
    const double *pblh;
    double *cush;
    double *umf, *slflx, *qtflx, *flxprc1, *flxsnow1, *qvten, *qlten, *qiten, *sten, *uten, *vten,
        *trten, *qrten, *qsten, *precip, *snow, *evapc, *cufrc, *qcu, *qlu, *qiu, *cbmf, *qc, *rliq;
    double *cnt, *cnb;
    const double *dpdry0;
    double *wu;
    int *diag_int;       // optional (UW_NDI, mix)
    double *diag_real;   // optional (UW_NDR, mix)
    double *diag_level;  // optional (UW_NDL, mkx + 1, mix)
    const double *omega; // (mix, mkx) pressure velocity: compute_zwshcu; nullptr: compute_uwshcu
    unsigned int *err;   // device error word
    const UwHand *hand;  // UW_MODE_LIST1 / UW_MODE_RESUME only: device copy of the hand-off region
    int *depth_key;      // optional (mix): each computed column's ordering key for the next call
};

// ---- batched launches --------------------------------------------------------------------------
// Members of one batch that share a level/tracer class run in one trigger launch and one persistent
// worklist launch.  Passed by value as a __grid_constant__ kernel parameter.
#define UW_MAXM 8
struct UwBatch {
    int nm;                          // members in this launch (<= UW_MAXM)
    int chunk;                       // worklist entries per task = 32 * chunk
    int block_start[UW_MAXM + 1];    // trigger launch: first block of each member
    int *count;                      // per-member worklist counts (device, nm ints)
    int *task_head;                  // device task counter of the persistent worklist launch
    int *task_head2;                 // the same for the resume launch of the sorted schedule
    int *wl[UW_MAXM];                // per-member worklists (device)
    UwArgs m[UW_MAXM];
};
