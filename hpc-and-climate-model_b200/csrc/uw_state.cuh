// uw_state.cuh -- the thread-private state of one column in the FP64 column code at the implicit-CIN
// branch of iteration 2, as lists, and its copy to and from a hand-off buffer.
//
// The worklist pass runs in two launches: UW_MODE_LIST1 computes iteration 1 of the implicit-CIN
// loop and iteration 2 up to the CIN decision; a column taking the implicit branch restores its
// iteration-1 state there (uwshcu.F90:1759-1889), stores it here, and UW_MODE_RESUME continues it
// in warps sorted by updraft depth.  Right after that restore the column's state is:
//   - the arrays of UW_ST_FULL, which hold values the rest of the column may read (the iteration-1
//     environment, the Exner functions, the wet-bulb humidity, and arrays the Fortran does not reset
//     between the iterations, such as the condensate sinks above the new cloud top): stored whole;
//   - every other array, which the restore or the set-up rebuilt from the inputs or zeroed over
//     k = 1..mkx (or 0..mkx): UW_MODE_RESUME rebuilds it with the same operations, and only its
//     k = 0 element, which neither touches, is stored;
//   - the tracer vectors and every scalar: stored.
// So the second launch computes exactly what a single launch would.
//
// Buffer layout: word w of slot s at state[w * cap + s] (consecutive slots of a warp are
// consecutive doubles).  Integers are exact in a double.
#pragma once
#include <cstddef>

#define UW_ST_FULL(X)                                                                                     \
    X(exn0) X(exns0) X(qw0) X(thv0bot_o) X(thv0top_o) X(thvl0bot_o) X(thvl0top_o) X(rei) X(uf)          \
    X(vf) X(xflx) X(qlten_sink) X(qiten_sink) X(nlten_sink) X(niten_sink) X(flxrain) X(flxsnow)         \
    X(trflx_d) X(trflx_u)
#define UW_ST_LEV0(X)                                                                                     \
    X(ps0) X(p0) X(dp0) X(zs0) X(qv0) X(ql0) X(qi0) X(t0) X(s0) X(qt0) X(thl0) X(ssthl0) X(ssqt0)      \
    X(ssu0) X(ssv0) X(thv0bot) X(thv0top) X(thvl0bot) X(thvl0top) X(umf) X(emf) X(thlu) X(qtu)         \
    X(uu) X(vu) X(thvu) X(wu) X(ufrc) X(fer) X(fdr) X(dwten) X(diten) X(thlu_emf) X(qtu_emf)           \
    X(uu_emf) X(vu_emf) X(slflx) X(qtflx) X(uflx) X(vflx) X(uten) X(vten) X(qrten) X(qsten)            \
    X(slten) X(qtten) X(qlten) X(qiten) X(qvten) X(sten) X(qc) X(qc_l) X(qc_i) X(evapc) X(cufrc)       \
    X(qcu) X(qlu) X(qiu)
#define UW_ST_TRA(X) X(sstr0) X(tru) X(tru_emf) X(trflx) X(trten)
#define UW_ST_VEC(X) X(trsrc) X(tre) X(trsrc_o)
#define UW_ST_DBL(X)                                                                                      \
    X(cin) X(cinlcl) X(plcl) X(plfc) X(prel) X(exlcl) X(exprel) X(tkeavg) X(thvlmin) X(qtsrc) X(thlsrc)  \
    X(thvlsrc) X(usrc) X(vsrc) X(thv0lcl) X(thv0rel) X(cin_i) X(cinlcl_i) X(ke) X(plcl_o) X(plfc_o)     \
    X(tkeavg_o) X(thvlmin_o) X(qtsrc_o) X(thvlsrc_o) X(thlsrc_o) X(usrc_o) X(vsrc_o) X(thv0lcl_o)       \
    X(cin_s) X(cinlcl_s) X(plcl_s) X(plfc_s) X(pinv_s) X(pbup_s) X(ppen_s) X(tkeavg_s) X(cbmf) X(wlcl) \
    X(ufrclcl) X(ppen) X(precip) X(snow) X(rliq) X(cush) X(cnt) X(cnb) X(thlu_top) X(qtu_top)          \
    X(exntop) X(drage) X(bogbot) X(bogtop) X(rho0j) X(wtwb) X(wtw) X(xs1) X(xs2) X(xc1) X(xc2) X(thj)  \
    X(qvj) X(qlj) X(qij) X(rainflx) X(snowflx)
#define UW_ST_INT(X)                                                                                      \
    X(xflags) X(lflags) X(kinv) X(klcl) X(klfc) X(krel) X(kbup) X(kpen) X(kinv_s) X(klcl_s) X(klfc_s)   \
    X(krel_s) X(kbup_s) X(kpen_s) X(kinv_o) X(klcl_o) X(klfc_o)

#define UW_ST_ONE(x) +1
// Extra words for scalars that take two (the compensated sums rliq, rainflx, snowflx of the
// mixed-precision column code).
#define UW_ST_WIDE 3
// words of one slot: the lists above, plus tscaleh and errbits
__host__ __device__ inline size_t uw_state_words(int mkx, int ncnst)
{
    const size_t lv = (size_t)mkx + 1;
    return (0 UW_ST_FULL(UW_ST_ONE)) * lv + (0 UW_ST_LEV0(UW_ST_ONE)) + (0 UW_ST_TRA(UW_ST_ONE)) * (size_t)ncnst +
           (0 UW_ST_VEC(UW_ST_ONE)) * (size_t)ncnst + (0 UW_ST_DBL(UW_ST_ONE)) + (0 UW_ST_INT(UW_ST_ONE)) + 2 +
           UW_ST_WIDE;
}

// One scalar to / from the buffer, whatever its type (every integer and float is exact in a
// double).  A type of two words provides its own overloads next to its definition.
#if defined(__CUDACC__)
__device__ __forceinline__ void uw_st_put(double* st, size_t& w, size_t cs, double x) { st[w++ * cs] = x; }
__device__ __forceinline__ void uw_st_put(double* st, size_t& w, size_t cs, float x) { st[w++ * cs] = (double)x; }
__device__ __forceinline__ void uw_st_put(double* st, size_t& w, size_t cs, int x) { st[w++ * cs] = (double)x; }
__device__ __forceinline__ void uw_st_put(double* st, size_t& w, size_t cs, unsigned int x) { st[w++ * cs] = (double)x; }
__device__ __forceinline__ void uw_st_get(const double* st, size_t& w, size_t cs, double& x) { x = st[w++ * cs]; }
__device__ __forceinline__ void uw_st_get(const double* st, size_t& w, size_t cs, float& x) { x = (float)st[w++ * cs]; }
__device__ __forceinline__ void uw_st_get(const double* st, size_t& w, size_t cs, int& x) { x = (int)st[w++ * cs]; }
__device__ __forceinline__ void uw_st_get(const double* st, size_t& w, size_t cs, unsigned int& x)
{
    x = (unsigned int)st[w++ * cs];
}
#endif

// Column code only (names mkx, ncnst, errbits and the listed variables in scope).
#define UW_SV_FULL(a) for (int k_ = 0; k_ <= mkx; k_++) st_[(w_ + k_) * cs_] = a[k_]; w_ += mkx + 1;
#define UW_SV_LEV0(a) st_[w_ * cs_] = a[0]; w_++;
#define UW_SV_TRA(a) for (int m_ = 0; m_ < ncnst; m_++) st_[(w_ + m_) * cs_] = a[m_][0]; w_ += ncnst;
#define UW_SV_VEC(a) for (int m_ = 0; m_ < ncnst; m_++) st_[(w_ + m_) * cs_] = a[m_]; w_ += ncnst;
#define UW_SV_ONE(x) uw_st_put(st_, w_, cs_, x);
#define UW_SAVE_STATE(ST, CS, TSCALEH)                                                                    \
    do {                                                                                                  \
        double* const st_ = (ST);                                                                         \
        const size_t cs_ = (CS);                                                                          \
        size_t w_ = 0;                                                                                    \
        UW_ST_FULL(UW_SV_FULL) UW_ST_LEV0(UW_SV_LEV0) UW_ST_TRA(UW_SV_TRA) UW_ST_VEC(UW_SV_VEC)          \
        UW_ST_DBL(UW_SV_ONE) UW_ST_INT(UW_SV_ONE) UW_SV_ONE(TSCALEH) UW_SV_ONE(errbits)                  \
    } while (0)

#define UW_LD_FULL(a) for (int k_ = 0; k_ <= mkx; k_++) a[k_] = st_[(w_ + k_) * cs_]; w_ += mkx + 1;
#define UW_LD_LEV0(a) a[0] = st_[w_ * cs_]; w_++;
#define UW_LD_TRA(a) for (int m_ = 0; m_ < ncnst; m_++) a[m_][0] = st_[(w_ + m_) * cs_]; w_ += ncnst;
#define UW_LD_VEC(a) for (int m_ = 0; m_ < ncnst; m_++) a[m_] = st_[(w_ + m_) * cs_]; w_ += ncnst;
#define UW_LD_ONE(x) uw_st_get(st_, w_, cs_, x);
#define UW_LOAD_STATE(ST, CS, TSCALEH)                                                                    \
    do {                                                                                                  \
        const double* const st_ = (ST);                                                                   \
        const size_t cs_ = (CS);                                                                          \
        size_t w_ = 0;                                                                                    \
        UW_ST_FULL(UW_LD_FULL) UW_ST_LEV0(UW_LD_LEV0) UW_ST_TRA(UW_LD_TRA) UW_ST_VEC(UW_LD_VEC)          \
        UW_ST_DBL(UW_LD_ONE) UW_ST_INT(UW_LD_ONE) UW_LD_ONE(TSCALEH) UW_LD_ONE(errbits)                  \
    } while (0)
