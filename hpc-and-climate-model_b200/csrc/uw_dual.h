// uw_dual.h -- forward-mode (tangent-linear) arithmetic for the column code.
//
// Tl carries a value and its derivative along one direction.  Every operation applies the chain
// rule to the derivative and computes the value exactly as the FP64 code does (same operation,
// same rounding), so the values of a tangent run are the FP64 path's.  Branches follow the values:
// the tangent is that of the branch the FP64 path takes (the derivative is undefined only exactly
// at a branch switch).  Transcendentals use the library's own routines (uw_math.h).
#pragma once
#include <math.h>
#include "uw_math.h"

#if defined(__CUDACC__)
#define TL_HD __host__ __device__ __forceinline__
#else
#define TL_HD static inline
#endif

struct Tl {
    double v, d;
    Tl() = default;
    TL_HD constexpr Tl(double x) : v(x), d(0.0) {}
    TL_HD constexpr Tl(double x, double dx) : v(x), d(dx) {}
    TL_HD explicit operator double() const { return v; }
    TL_HD explicit operator int() const { return (int)v; }
    TL_HD Tl& operator+=(Tl o) { v = v + o.v; d = d + o.d; return *this; }
    TL_HD Tl& operator-=(Tl o) { v = v - o.v; d = d - o.d; return *this; }
};

TL_HD Tl operator+(Tl a, Tl b) { return Tl(a.v + b.v, a.d + b.d); }
TL_HD Tl operator-(Tl a, Tl b) { return Tl(a.v - b.v, a.d - b.d); }
TL_HD Tl operator*(Tl a, Tl b) { return Tl(a.v * b.v, a.d * b.v + a.v * b.d); }
TL_HD Tl operator/(Tl a, Tl b)
{
    const double q = a.v / b.v;
    return Tl(q, (a.d - q * b.d) / b.v);
}
TL_HD Tl operator-(Tl a) { return Tl(-a.v, -a.d); }
TL_HD Tl operator+(Tl a) { return a; }
TL_HD bool operator<(Tl a, Tl b) { return a.v < b.v; }
TL_HD bool operator>(Tl a, Tl b) { return a.v > b.v; }
TL_HD bool operator<=(Tl a, Tl b) { return a.v <= b.v; }
TL_HD bool operator>=(Tl a, Tl b) { return a.v >= b.v; }
TL_HD bool operator==(Tl a, Tl b) { return a.v == b.v; }
TL_HD bool operator!=(Tl a, Tl b) { return a.v != b.v; }

TL_HD double tl_val(Tl x) { return x.v; }
TL_HD double tl_val(double x) { return x; }
TL_HD double tl_der(Tl x) { return x.d; }
TL_HD double tl_der(double) { return 0.0; }

TL_HD Tl uw_div_by(Tl a, Tl b, Tl y)
{
    const double q = uw_div_by(a.v, b.v, y.v);
    return Tl(q, (a.d - q * b.d) / b.v);
}
TL_HD bool uw_isfinite(const Tl& x) { return isfinite(x.v); }
TL_HD Tl uw_exp(Tl x)
{
    const double e = uw_exp(x.v);
    return Tl(e, e * x.d);
}
TL_HD Tl uw_log(Tl x) { return Tl(uw_log(x.v), x.d / x.v); }
TL_HD Tl uw_pow(Tl x, Tl y)
{
    const double p = uw_pow(x.v, y.v);
    double d = 0.0;
    if (x.d != 0.0) d = p * y.v * x.d / x.v;
    if (y.d != 0.0) d = d + p * uw_log(x.v) * y.d;
    return Tl(p, d);
}
TL_HD Tl uw_erfc(Tl x)
{
    // d/dx erfc(x) = -2/sqrt(pi) exp(-x^2)
    const double e = uw_erfc(x.v);
    return Tl(e, x.d == 0.0 ? 0.0 : -1.1283791670955126 * uw_exp(-(x.v * x.v)) * x.d);
}
TL_HD Tl sqrt(Tl x)
{
    const double s = sqrt(x.v);
    return Tl(s, x.d == 0.0 ? 0.0 : x.d / (2.0 * s));
}
TL_HD Tl fabs(Tl x) { return Tl(fabs(x.v), x.v < 0.0 ? -x.d : x.d); }
TL_HD Tl trunc(Tl x) { return Tl(trunc(x.v), 0.0); }
TL_HD Tl floor(Tl x) { return Tl(floor(x.v), 0.0); }
TL_HD Tl copysign(Tl a, Tl b)
{
    const double r = copysign(a.v, b.v);
    return Tl(r, (r == a.v) ? a.d : -a.d);
}
