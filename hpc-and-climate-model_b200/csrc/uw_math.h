// uw_math.h -- exp, log, pow and erfc that give the same bits on the host and on the GPU.
//
// The scheme amplifies last-bit differences of the transcendental functions strongly (for example
// wu = sqrt(wtw) with wtw near 0, or 1 - thvj/thv0j multiplied by 2 g cridis / wue^2 ~ 1e4): two
// libms that differ by one ulp give column differences of up to 1e-5.  These routines use only
// operations that IEEE 754 rounds exactly the same way everywhere (+ - * /, sqrt, fma, floor,
// frexp, ldexp, comparisons), so a host build (-ffp-contract=off) and a device build
// (-fmad=false) of the same expression produce identical results.  Accuracy is about 1 ulp
// (exp, log), a few ulp (pow with |y log x| < 1) and about 1e-16 relative (erfc).
//
// Methods:
//   exp  -- Cody-Waite argument reduction x = k ln2 + r with a two-part ln2, Taylor polynomial of
//           degree 13 for e^r on |r| <= ln2/2 (Horner with fma), scaling by 2^k.
//   log  -- x = m 2^e with m in [sqrt(1/2), sqrt(2)), f = m - 1, s = f / (2 + f),
//           log(1+f) = f - (f^2/2 - s (f^2/2 + R)), R = z (2/3 + 2/5 z + ... + 2/25 z^11), z = s^2
//           (the atanh series), plus e ln2 in two parts.
//   pow  -- exp(y log x) for x > 0.
//   erfc -- W. J. Cody, "Rational Chebyshev approximations for the error function", Math. Comp.
//           23 (1969) 631-637: the three-interval rational approximations of CALERF (SPECFUN), the
//           algorithm of CAM's error_function module that uwshcu.F90:5 uses.
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

UW_HD double uw_exp(double x)
{
    if (x != x) return x;
    if (x > 709.782712893384) return HUGE_VAL;
    if (x < -745.1332191019412) return 0.0;
    const double LOG2E = 1.4426950408889634074;
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    const double kd = floor(fma(x, LOG2E, 0.5));
    double r = fma(-kd, LN2_HI, x);
    r = fma(-kd, LN2_LO, r);
    double p = 1.0 / 6227020800.0;          // 1/13!
    p = fma(p, r, 1.0 / 479001600.0);       // 1/12!
    p = fma(p, r, 1.0 / 39916800.0);        // 1/11!
    p = fma(p, r, 1.0 / 3628800.0);         // 1/10!
    p = fma(p, r, 1.0 / 362880.0);          // 1/9!
    p = fma(p, r, 1.0 / 40320.0);           // 1/8!
    p = fma(p, r, 1.0 / 5040.0);            // 1/7!
    p = fma(p, r, 1.0 / 720.0);             // 1/6!
    p = fma(p, r, 1.0 / 120.0);             // 1/5!
    p = fma(p, r, 1.0 / 24.0);              // 1/4!
    p = fma(p, r, 1.0 / 6.0);               // 1/3!
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    int k = (int)kd;
    if (k < -1020) return ldexp(ldexp(p, k + 60), -60);
    return ldexp(p, k);
}

UW_HD double uw_log(double x)
{
    if (!(x > 0.0)) {
        if (x == 0.0) return -HUGE_VAL;
        return (x != x) ? x : (x - x) / (x - x);   // NaN for x < 0
    }
    if (x == HUGE_VAL) return x;
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    int e;
    double m = frexp(x, &e);                 // m in [0.5, 1)
    if (m < 0.70710678118654752440) {
        m = m * 2.0;
        e = e - 1;
    }
    const double f = m - 1.0;                // exact
    const double s = f / (2.0 + f);
    const double z = UW_MUL(s, s);
    double q = 2.0 / 25.0;
    q = fma(q, z, 2.0 / 23.0);
    q = fma(q, z, 2.0 / 21.0);
    q = fma(q, z, 2.0 / 19.0);
    q = fma(q, z, 2.0 / 17.0);
    q = fma(q, z, 2.0 / 15.0);
    q = fma(q, z, 2.0 / 13.0);
    q = fma(q, z, 2.0 / 11.0);
    q = fma(q, z, 2.0 / 9.0);
    q = fma(q, z, 2.0 / 7.0);
    q = fma(q, z, 2.0 / 5.0);
    q = fma(q, z, 2.0 / 3.0);
    const double R = UW_MUL(z, q);
    const double hfsq = UW_MUL(UW_MUL(0.5, f), f);
    const double dk = (double)e;
    const double t = UW_ADD(UW_MUL(s, UW_ADD(hfsq, R)), UW_MUL(dk, LN2_LO));
    return UW_SUB(UW_MUL(dk, LN2_HI), UW_SUB(UW_SUB(hfsq, t), f));
}

UW_HD double uw_pow(double x, double y)
{
    if (x != x || y != y) return x + y;
    if (y == 0.0) return 1.0;
    if (x == 0.0) return (y > 0.0) ? 0.0 : HUGE_VAL;
    if (x < 0.0) return (x - x) / (x - x);
    return uw_exp(UW_MUL(y, uw_log(x)));
}

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
        result = UW_MUL(UW_MUL(uw_exp(-UW_MUL(ysq, ysq)), uw_exp(-del)), result);
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
        result = UW_MUL(UW_MUL(uw_exp(-UW_MUL(ysq2, ysq2)), uw_exp(-del)), result);
    }
    if (x < 0.0) result = UW_SUB(2.0, result);
    return result;
}
