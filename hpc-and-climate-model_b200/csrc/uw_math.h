// uw_math.h -- exp, log, pow and erfc that give the same bits on the host and on the GPU.
//
// The scheme amplifies last-bit differences of the transcendental functions strongly (for example
// wu = sqrt(wtw) with wtw near 0, or 1 - thvj/thv0j multiplied by 2 g cridis / wue^2 ~ 1e4): two
// libms that differ by one ulp give column differences of up to 1e-5.  These routines use only
// operations that IEEE 754 rounds exactly the same way everywhere (+ - * /, sqrt, fma, rint,
// floor, frexp, ldexp, comparisons), so a host build (-ffp-contract=off) and a device build
// (-fmad=false, or explicit __dmul_rn/__dadd_rn where contraction is on) of the same expression
// produce identical results.
//
// Methods:
//   exp, log, pow -- correctly rounded (Ziv's fast path, rounding test and accurate double-double
//           path; description and references below), so that they return what every correctly
//           rounding libm returns, and glibc's exp/log/pow (the functions a Fortran build of the
//           scheme calls on Linux) in all but the few cases in 10^3 that glibc rounds the other way.
//   erfc -- W. J. Cody, "Rational Chebyshev approximations for the error function", Math. Comp.
//           23 (1969) 631-637: the three-interval rational approximations of CALERF (SPECFUN), the
//           algorithm of CAM's error_function module that uwshcu.F90:5 uses, with the exp above.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define UW_HD __host__ __device__ __forceinline__
#else
#define UW_HD static inline
#endif

// Multiplications and additions that no compiler contracts into an fma: __dmul_rn/__dadd_rn on
// the device, plain operators on the host (built with -ffp-contract=off).
#if defined(__CUDA_ARCH__)
#define UW_MUL(a, b) __dmul_rn((a), (b))
#define UW_ADD(a, b) __dadd_rn((a), (b))
#define UW_SUB(a, b) __dsub_rn((a), (b))
#else
#define UW_MUL(a, b) ((a) * (b))
#define UW_ADD(a, b) ((a) + (b))
#define UW_SUB(a, b) ((a) - (b))
#endif

// a / b from the correctly rounded reciprocal y = RN(1/b): q = RN(a y), e = a - b q (exact with an
// FMA), RN(q + e y) = RN(a / b) for operands and quotient in the normal range (P. Markstein, IBM J.
// Res. Dev. 34 (1990) 111-119; J.-M. Muller et al., Handbook of Floating-Point Arithmetic, the
// division theorems of ch. 5): the IEEE quotient from one multiply and two FMAs once 1/b is known.
// Used where one divisor serves several divisions.
UW_HD double uw_div_by(double a, double b, double y)
{
    const double q = UW_MUL(a, y);
    const double e = fma(-b, q, a);
    return fma(e, y, q);
}

// ---------------------------------------------------------------------------------------------
// Correctly rounded exp, log and pow (round to nearest), after Ziv's strategy (A. Ziv, "Fast
// evaluation of elementary mathematical functions with correctly rounded last bit", ACM TOMS 17
// (1991) 410-423): a fast evaluation to about 2^-64 relative as an unevaluated sum hi + lo, a
// rounding test that proves RN(hi + lo) is the rounding of the exact value, and otherwise an
// accurate double-double evaluation to about 2^-100 whose rounding is wrong only if the exact
// value lies within 2^-100 of a midpoint between two doubles.  Double-double arithmetic uses the
// error-free transformations TwoSum (Knuth), Fast2Sum (Dekker) and TwoProd with an FMA.  Table
// reduction (J.-M. Muller, Elementary Functions, 3rd ed., ch. 6): exp(x) = 2^m 2^(j/64) e^r with
// |r| <= ln2/128 and a 64-entry double-double table of 2^(j/64); log(x) = e ln2 - log(INVC) +
// log1p(m INVC - 1) with m in [sqrt(1/2), sqrt(2)), a 7-bit reciprocal INVC per 1/128-wide bin
// (so the reduced argument is exact), and Taylor series of e^r and log1p.  The constants are
// computed from their definitions by gen_crmath_tables.py.  Subnormal results of exp and pow are
// scaled after rounding (one extra rounding; the scheme never produces them).
//
// Agreement with other correctly rounding libraries is what these routines are for: a libm whose
// results are correctly rounded in all but a few cases in 10^3 (glibc's exp, log and pow) then
// gives the same bits in all but those cases.
#include "uw_crmath_tables.h"

// On the device the tables are read through the read-only data path (__ldg).  (Staged in shared
// memory, 3.2 KB per block, they changed the FP64 kernels' time by under 1 % and slowed the adjoint's
// one-warp blocks by 14 %, whose shared-memory carveout then leaves less L1 for their stacks.)
#if defined(__CUDACC__)
#define UW_HD_SLOW static __host__ __device__ __noinline__
static __device__ const double uw_cr_expt_d[128] = UW_CR_EXPT_INIT;
static __device__ const double uw_cr_logt_d[276] = UW_CR_LOGT_INIT;
#else
#define UW_HD_SLOW static
#endif
static const double uw_cr_expt_h[128] = UW_CR_EXPT_INIT;
static const double uw_cr_logt_h[276] = UW_CR_LOGT_INIT;
#if defined(__CUDA_ARCH__)
#define UW_CR_EXPT(i) __ldg(&uw_cr_expt_d[(i)])
#define UW_CR_LOGT(i) __ldg(&uw_cr_logt_d[(i)])
#else
#define UW_CR_EXPT(i) (uw_cr_expt_h[(i)])
#define UW_CR_LOGT(i) (uw_cr_logt_h[(i)])
#endif

// s + e = a + b exactly (TwoSum).
UW_HD void uw_two_sum(double a, double b, double* s, double* e)
{
    const double ss = UW_ADD(a, b);
    const double v = UW_SUB(ss, a);
    *e = UW_ADD(UW_SUB(a, UW_SUB(ss, v)), UW_SUB(b, v));
    *s = ss;
}

// s + e = a + b exactly when |a| >= |b| or a = 0 (Fast2Sum).
UW_HD void uw_fast_two_sum(double a, double b, double* s, double* e)
{
    const double ss = UW_ADD(a, b);
    *e = UW_SUB(b, UW_SUB(ss, a));
    *s = ss;
}

// (h, l) = (h, l) (bh, bl) + (ch, cl) in double-double, for |(h, l) (bh, bl)| well below |c|.
UW_HD void uw_dd_mul_add(double* h, double* l, double bh, double bl, double ch, double cl)
{
    const double p = UW_MUL(*h, bh);
    const double q = UW_ADD(fma(*h, bh, -p), UW_ADD(UW_MUL(*h, bl), UW_MUL(*l, bh)));
    double s, e;
    uw_two_sum(ch, p, &s, &e);
    e = UW_ADD(e, UW_ADD(q, cl));
    uw_fast_two_sum(s, e, h, l);
}

// Ziv's rounding test: RN(h + l) is the correctly rounded value of every number within err of
// h + l when both ends of that interval round to the same double.
UW_HD int uw_cr_rounds(double h, double l, double err)
{
    return UW_ADD(h, UW_ADD(l, err)) == UW_ADD(h, UW_SUB(l, err));
}

// rh + rl = xh + xl - kd ln2/64 (error below 2^-100 absolute for |k| < 2^17), with
// kd = RN(xh * 64/ln2) rounded to an integer.  xh - kd*C1 is exact (kd*C1 is exact and the
// operands are within a factor 2), the rest is collected by TwoSum.
UW_HD void uw_exp_reduce(double xh, double xl, double* kd, double* rh, double* rl)
{
    const double k = rint(UW_MUL(xh, UW_CR_INVL));
    const double t = fma(-k, UW_CR_C1, xh);
    double h, e;
    uw_two_sum(t, UW_MUL(-k, UW_CR_C2), &h, &e);
    e = UW_ADD(e, UW_SUB(xl, UW_MUL(k, UW_CR_C3)));
    uw_two_sum(h, e, rh, rl);
    *kd = k;
}

// Bit patterns of doubles (exact on both sides).
#if defined(__CUDA_ARCH__)
#define UW_D2LL(x) __double_as_longlong(x)
#define UW_LL2D(x) __longlong_as_double(x)
#else
#include <string.h>
UW_HD long long UW_D2LL(double x)
{
    long long i;
    memcpy(&i, &x, sizeof i);
    return i;
}
UW_HD double UW_LL2D(long long i)
{
    double x;
    memcpy(&x, &i, sizeof x);
    return x;
}
#endif

// 2^m y for y in [0.98, 2.03] (|m| <= 1076): one exact multiplication by 2^m where 2^m and the
// result are normal, ldexp otherwise (subnormal results, overflow).
UW_HD double uw_cr_scale(double y, int m)
{
    if (m >= -1021 && m <= 1022) return UW_MUL(y, UW_LL2D((long long)(m + 1023) << 52));
    return ldexp(y, m);
}

// Accurate exp(xh + xl), |xh + xl| <= 746: e^r by its Taylor series to degree 11 (truncation
// below 2^-119 for |r| <= ln2/128), degrees 6..11 in double, 0..5 by double-double Horner steps,
// times the double-double table entry; relative error about 2^-100.
UW_HD double uw_exp_accurate_core(double xh, double xl)
{
    double kd, rh, rl;
    uw_exp_reduce(xh, xl, &kd, &rh, &rl);
    const int k = (int)kd;
    const int j = k & 63;
    const int m = (k - j) / 64;
    double q = UW_CR_F11_H;
    q = fma(q, rh, UW_CR_F10_H);
    q = fma(q, rh, UW_CR_F9_H);
    q = fma(q, rh, UW_CR_F8_H);
    q = fma(q, rh, UW_CR_F7_H);
    q = fma(q, rh, UW_CR_F6_H);
    double h = q, l = 0.0;
    uw_dd_mul_add(&h, &l, rh, rl, UW_CR_F5_H, UW_CR_F5_L);
    uw_dd_mul_add(&h, &l, rh, rl, UW_CR_F4_H, UW_CR_F4_L);
    uw_dd_mul_add(&h, &l, rh, rl, UW_CR_F3_H, UW_CR_F3_L);
    uw_dd_mul_add(&h, &l, rh, rl, 0.5, 0.0);
    uw_dd_mul_add(&h, &l, rh, rl, 1.0, 0.0);
    uw_dd_mul_add(&h, &l, rh, rl, 1.0, 0.0);
    const double th = UW_CR_EXPT(2 * j), tl = UW_CR_EXPT(2 * j + 1);
    double H, L;
    {
        const double p = UW_MUL(th, h);
        const double e = UW_ADD(fma(th, h, -p), UW_ADD(UW_MUL(th, l), UW_MUL(tl, h)));
        uw_fast_two_sum(p, e, &H, &L);
    }
    return uw_cr_scale(UW_ADD(H, L), m);
}

UW_HD_SLOW double uw_exp_accurate(double x) { return uw_exp_accurate_core(x, 0.0); }

// Fast exp(xh + xl): e^r = 1 + r + r^2 P(r) with P to degree 5 in double (absolute error below
// 2^-66), times the table entry.  Returns 1 and sets *y when the rounding test passes with the
// relative error bound err_rel (at least 2^-63).
UW_HD int uw_exp_fast(double xh, double xl, double err_rel, double* y)
{
    double kd, rh, rl;
    uw_exp_reduce(xh, xl, &kd, &rh, &rl);
    const int k = (int)kd;
    const int j = k & 63;
    const int m = (k - j) / 64;
    double p = UW_CR_F7_H;
    p = fma(p, rh, UW_CR_F6_H);
    p = fma(p, rh, UW_CR_F5_H);
    p = fma(p, rh, UW_CR_F4_H);
    p = fma(p, rh, UW_CR_F3_H);
    p = fma(p, rh, 0.5);
    const double q = UW_MUL(UW_MUL(rh, rh), p);
    double h, l;
    uw_fast_two_sum(1.0, rh, &h, &l);
    l = UW_ADD(l, UW_ADD(rl, q));
    const double th = UW_CR_EXPT(2 * j), tl = UW_CR_EXPT(2 * j + 1);
    const double H = UW_MUL(th, h);
    const double L = UW_ADD(fma(th, h, -H), UW_ADD(UW_MUL(th, l), UW_MUL(tl, h)));
    if (!uw_cr_rounds(H, L, UW_MUL(err_rel, H))) return 0;
    *y = uw_cr_scale(UW_ADD(H, L), m);
    return 1;
}

UW_HD double uw_exp(double x)
{
    if (x != x) return x;
    if (x > 709.8) return HUGE_VAL;
    if (x < -745.2) return 0.0;
    double y;
    if (uw_exp_fast(x, 0.0, 0x1p-63, &y)) return y;
    return uw_exp_accurate(x);
}

// Reduction of log: x = 2^e m, m in [sqrt(1/2), sqrt(2)), bin i = floor(128 m) - 90, t = m INVC - 1
// (exact, |t| < 2^-6).  x must be positive and finite.
UW_HD void uw_log_reduce(double x, int* e, int* i, double* t)
{
    int ea = 0;
    if (x < 0x1p-1022) {
        x = UW_MUL(x, 0x1p54);
        ea = -54;
    }
    // x = 2^e m with m in [1/2, 1) (x positive and normal here): frexp by its bits
    const long long b = UW_D2LL(x);
    *e = (int)((b >> 52) & 0x7ff) - 1022;
    double m = UW_LL2D((b & 0x000fffffffffffffLL) | 0x3fe0000000000000LL);
    if (m < UW_CR_SQRTH) {
        m = UW_MUL(m, 2.0);
        *e = *e - 1;
    }
    *e = *e + ea;
    *i = (int)UW_MUL(m, 128.0) - 90;
    *t = fma(m, UW_CR_LOGT(3 * *i), -1.0);
}

// Accurate log as a double-double (relative error about 2^-100): log1p(t) = t S(t) with the
// Taylor coefficients of degrees 9..17 of S in double and 1..8 by double-double Horner steps.
UW_HD void uw_log_accurate_dd(double x, double* H, double* L)
{
    int e, i;
    double t;
    uw_log_reduce(x, &e, &i, &t);
    double q = UW_CR_L17_H;
    q = fma(q, t, UW_CR_L16_H);
    q = fma(q, t, UW_CR_L15_H);
    q = fma(q, t, UW_CR_L14_H);
    q = fma(q, t, UW_CR_L13_H);
    q = fma(q, t, UW_CR_L12_H);
    q = fma(q, t, UW_CR_L11_H);
    q = fma(q, t, UW_CR_L10_H);
    q = fma(q, t, UW_CR_L9_H);
    double h = q, l = 0.0;
    uw_dd_mul_add(&h, &l, t, 0.0, UW_CR_L8_H, UW_CR_L8_L);
    uw_dd_mul_add(&h, &l, t, 0.0, UW_CR_L7_H, UW_CR_L7_L);
    uw_dd_mul_add(&h, &l, t, 0.0, UW_CR_L6_H, UW_CR_L6_L);
    uw_dd_mul_add(&h, &l, t, 0.0, UW_CR_L5_H, UW_CR_L5_L);
    uw_dd_mul_add(&h, &l, t, 0.0, UW_CR_L4_H, UW_CR_L4_L);
    uw_dd_mul_add(&h, &l, t, 0.0, UW_CR_L3_H, UW_CR_L3_L);
    uw_dd_mul_add(&h, &l, t, 0.0, UW_CR_L2_H, UW_CR_L2_L);
    uw_dd_mul_add(&h, &l, t, 0.0, 1.0, 0.0);
    // log1p(t) = t (h + l)
    double ph = UW_MUL(t, h);
    double pl = UW_ADD(fma(t, h, -ph), UW_MUL(t, l));
    // e ln2 - log(INVC): e*LN2H is exact (42-bit constant, |e| < 2^11)
    const double ed = (double)e;
    double sh, sl;
    uw_two_sum(UW_MUL(ed, UW_CR_LN2H), UW_CR_LOGT(3 * i + 1), &sh, &sl);
    sl = UW_ADD(sl, UW_ADD(UW_MUL(ed, UW_CR_LN2L), UW_CR_LOGT(3 * i + 2)));
    uw_fast_two_sum(sh, sl, &sh, &sl);
    double rh, rl;
    uw_two_sum(sh, ph, &rh, &rl);
    rl = UW_ADD(rl, UW_ADD(sl, pl));
    uw_fast_two_sum(rh, rl, H, L);
}

UW_HD_SLOW double uw_log_accurate(double x)
{
    double H, L;
    uw_log_accurate_dd(x, &H, &L);
    return UW_ADD(H, L);
}

// Fast log as a double-double, relative error below 2^-64: t - t^2/2 exactly (TwoProd), t^3 P(t)
// in double with P to degree 9 (truncation below 2^-75 relative).
UW_HD void uw_log_fast(double x, double* H, double* L)
{
    int e, i;
    double t;
    uw_log_reduce(x, &e, &i, &t);
    double p = UW_CR_L12_H;
    p = fma(p, t, UW_CR_L11_H);
    p = fma(p, t, UW_CR_L10_H);
    p = fma(p, t, UW_CR_L9_H);
    p = fma(p, t, UW_CR_L8_H);
    p = fma(p, t, UW_CR_L7_H);
    p = fma(p, t, UW_CR_L6_H);
    p = fma(p, t, UW_CR_L5_H);
    p = fma(p, t, UW_CR_L4_H);
    p = fma(p, t, UW_CR_L3_H);
    const double t3p = UW_MUL(UW_MUL(t, t), UW_MUL(t, p));
    const double t2h = UW_MUL(t, t);
    const double t2l = fma(t, t, -t2h);
    const double ed = (double)e;
    double s1, e1, s2, e2, s3, e3;
    uw_two_sum(UW_MUL(ed, UW_CR_LN2H), UW_CR_LOGT(3 * i + 1), &s1, &e1);
    uw_two_sum(s1, t, &s2, &e2);
    uw_two_sum(s2, UW_MUL(-0.5, t2h), &s3, &e3);
    double lo = UW_ADD(UW_ADD(e1, e2), e3);
    lo = UW_ADD(lo, UW_ADD(UW_MUL(ed, UW_CR_LN2L), UW_CR_LOGT(3 * i + 2)));
    lo = UW_ADD(lo, UW_SUB(t3p, UW_MUL(0.5, t2l)));
    uw_fast_two_sum(s3, lo, H, L);
}

UW_HD double uw_log(double x)
{
    if (!(x > 0.0)) {
        if (x == 0.0) return -HUGE_VAL;
        return (x != x) ? x : (x - x) / (x - x);   // NaN for x < 0
    }
    if (x == HUGE_VAL) return x;
    double H, L;
    uw_log_fast(x, &H, &L);
    if (uw_cr_rounds(H, L, UW_MUL(0x1p-62, fabs(H)))) return UW_ADD(H, L);
    return uw_log_accurate(x);
}

UW_HD_SLOW double uw_pow_accurate(double x, double y)
{
    double Lh, Ll;
    uw_log_accurate_dd(x, &Lh, &Ll);
    const double zh = UW_MUL(y, Lh);
    const double zl = UW_ADD(fma(y, Lh, -zh), UW_MUL(y, Ll));
    return uw_exp_accurate_core(zh, zl);
}

// pow(x, y) for x >= 0: exp(y log x) with log and the product in double-double.
UW_HD double uw_pow(double x, double y)
{
    if (x != x || y != y) return x + y;
    if (y == 0.0) return 1.0;
    if (x == 0.0) return (y > 0.0) ? 0.0 : HUGE_VAL;
    if (x < 0.0) return (x - x) / (x - x);
    if (x == HUGE_VAL) return (y > 0.0) ? HUGE_VAL : 0.0;
    double Lh, Ll;
    uw_log_fast(x, &Lh, &Ll);
    const double zh = UW_MUL(y, Lh);
    if (zh > 709.8) return HUGE_VAL;
    if (zh < -745.2) return 0.0;
    const double zl = UW_ADD(fma(y, Lh, -zh), UW_MUL(y, Ll));
    // |z| 2^-64 from the logarithm plus 2^-66 from the exponential, with a factor 4 to spare
    double r;
    if (uw_exp_fast(zh, zl, UW_MUL(0x1p-62, UW_ADD(1.0, fabs(zh))), &r)) return r;
    return uw_pow_accurate(x, y);
}

// The exponential CALERF calls: this file's correctly rounded exp unless the includer names another
// (the oracle's Fortran-math build names the C library's exp, as a Fortran build of CALERF calls it).
#ifndef UW_ERFC_EXP
#define UW_ERFC_EXP uw_exp
#endif

// erfc(x), Cody's CALERF with jint = 1.
UW_HD double uw_erfc(double x)
{
    const double A[5] = {3.16112374387056560e00, 1.13864154151050156e02, 3.77485237685302021e02,
                         3.20937758913846947e03, 1.85777706184603153e-1};
    const double B[4] = {2.36012909523441209e01, 2.44024637934444173e02, 1.28261652607737228e03,
                         2.84423683343917062e03};
    const double C[9] = {5.64188496988670089e-1, 8.88314979438837594e00, 6.61191906371416295e01,
                         2.98635138197400131e02, 8.81952221241769090e02, 1.71204761263407058e03,
                         2.05107837782607147e03, 1.23033935479799725e03, 2.15311535474403846e-8};
    const double D[8] = {1.57449261107098347e01, 1.17693950891312499e02, 5.37181101862009858e02,
                         1.62138957456669019e03, 3.29079923573345963e03, 4.36261909014324716e03,
                         3.43936767414372164e03, 1.23033935480374942e03};
    const double P[6] = {3.05326634961232344e-1, 3.60344899949804439e-1, 1.25781726111229246e-1,
                         1.60837851487422766e-2, 6.58749161529837803e-4, 1.63153871373020978e-2};
    const double Q[5] = {2.56852019228982242e00, 1.87295284992346047e00, 5.27905102951428412e-1,
                         6.05183413124413191e-2, 2.33520497626869185e-3};
    const double sqrpi = 5.6418958354775628695e-1, thresh = 0.46875, xsmall = 1.11e-16, xbig = 26.543;
    if (x != x) return x;
    const double y = fabs(x);
    double result;
    if (y <= thresh) {
        const double ysq = (y > xsmall) ? UW_MUL(y, y) : 0.0;
        double xnum = UW_MUL(A[4], ysq), xden = ysq;
        for (int i = 0; i < 3; i++) {
            xnum = UW_MUL(UW_ADD(xnum, A[i]), ysq);
            xden = UW_MUL(UW_ADD(xden, B[i]), ysq);
        }
        return UW_SUB(1.0, UW_MUL(x, UW_ADD(xnum, A[3])) / UW_ADD(xden, B[3]));
    } else if (y <= 4.0) {
        double xnum = UW_MUL(C[8], y), xden = y;
        for (int i = 0; i < 7; i++) {
            xnum = UW_MUL(UW_ADD(xnum, C[i]), y);
            xden = UW_MUL(UW_ADD(xden, D[i]), y);
        }
        result = UW_ADD(xnum, C[7]) / UW_ADD(xden, D[7]);
        const double ysq = floor(UW_MUL(y, 16.0)) / 16.0;
        const double del = UW_MUL(UW_SUB(y, ysq), UW_ADD(y, ysq));
        result = UW_MUL(UW_MUL(UW_ERFC_EXP(-UW_MUL(ysq, ysq)), UW_ERFC_EXP(-del)), result);
    } else if (y >= xbig) {
        result = 0.0;
    } else {
        const double ysq = 1.0 / UW_MUL(y, y);
        double xnum = UW_MUL(P[5], ysq), xden = ysq;
        for (int i = 0; i < 4; i++) {
            xnum = UW_MUL(UW_ADD(xnum, P[i]), ysq);
            xden = UW_MUL(UW_ADD(xden, Q[i]), ysq);
        }
        result = UW_MUL(ysq, UW_ADD(xnum, P[4])) / UW_ADD(xden, Q[4]);
        result = UW_SUB(sqrpi, result) / y;
        const double ysq2 = floor(UW_MUL(y, 16.0)) / 16.0;
        const double del = UW_MUL(UW_SUB(y, ysq2), UW_ADD(y, ysq2));
        result = UW_MUL(UW_MUL(UW_ERFC_EXP(-UW_MUL(ysq2, ysq2)), UW_ERFC_EXP(-del)), result);
    }
    if (x < 0.0) result = UW_SUB(2.0, result);
    return result;
}
