// opcount.hpp -- operation-counting build of the oracle (TEST AND MEASUREMENT INFRASTRUCTURE ONLY).
//
// Force-included ahead of uwshcu_oracle.c compiled as C++ with `double` defined to `cdouble`: every
// floating-point value of the restatement becomes a cdouble, which computes exactly what a double
// computes and counts each operation it performs.  The counts are the algorithmic operations of the
// Fortran scheme (uwshcu.F90) as the oracle states it, statement by statement:
//   add  : + and - (binary)          mul : *          div : /          sqrt : sqrt
//   tr   : exp, log, pow, erfc, log10 (one operation each)
// Comparisons, min/max, fabs, trunc/floor/rint and conversions are not counted.  One thread only: the
// counters are thread-local and the driver runs the oracle with nthreads = 1.
#pragma once
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <cmath>

struct OpCounts {
    unsigned long long add, mul, div, sqrt, tr;
};
extern thread_local OpCounts g_ops;

struct cdouble {
    double v;
    cdouble() = default;
    constexpr cdouble(double x) : v(x) {}
    explicit operator double() const { return v; }
    explicit operator int() const { return (int)v; }
    cdouble& operator+=(cdouble o) { g_ops.add++; v += o.v; return *this; }
    cdouble& operator-=(cdouble o) { g_ops.add++; v -= o.v; return *this; }
    cdouble& operator*=(cdouble o) { g_ops.mul++; v *= o.v; return *this; }
    cdouble& operator/=(cdouble o) { g_ops.div++; v /= o.v; return *this; }
};
static_assert(sizeof(cdouble) == sizeof(double), "layout of the counted type must match double");

inline cdouble operator+(cdouble a, cdouble b) { g_ops.add++; return cdouble(a.v + b.v); }
inline cdouble operator-(cdouble a, cdouble b) { g_ops.add++; return cdouble(a.v - b.v); }
inline cdouble operator*(cdouble a, cdouble b) { g_ops.mul++; return cdouble(a.v * b.v); }
inline cdouble operator/(cdouble a, cdouble b) { g_ops.div++; return cdouble(a.v / b.v); }
inline cdouble operator-(cdouble a) { return cdouble(-a.v); }
inline cdouble operator+(cdouble a) { return a; }
inline bool operator<(cdouble a, cdouble b) { return a.v < b.v; }
inline bool operator>(cdouble a, cdouble b) { return a.v > b.v; }
inline bool operator<=(cdouble a, cdouble b) { return a.v <= b.v; }
inline bool operator>=(cdouble a, cdouble b) { return a.v >= b.v; }
inline bool operator==(cdouble a, cdouble b) { return a.v == b.v; }
inline bool operator!=(cdouble a, cdouble b) { return a.v != b.v; }

inline cdouble exp(cdouble x) { g_ops.tr++; return cdouble(std::exp(x.v)); }
inline cdouble log(cdouble x) { g_ops.tr++; return cdouble(std::log(x.v)); }
inline cdouble log10(cdouble x) { g_ops.tr++; return cdouble(std::log10(x.v)); }
inline cdouble pow(cdouble x, cdouble y) { g_ops.tr++; return cdouble(std::pow(x.v, y.v)); }
inline cdouble erfc(cdouble x) { g_ops.tr++; return cdouble(std::erfc(x.v)); }
inline cdouble sqrt(cdouble x) { g_ops.sqrt++; return cdouble(std::sqrt(x.v)); }
inline cdouble fabs(cdouble x) { return cdouble(std::fabs(x.v)); }
inline cdouble trunc(cdouble x) { return cdouble(std::trunc(x.v)); }
inline cdouble floor(cdouble x) { return cdouble(std::floor(x.v)); }
inline cdouble rint(cdouble x) { return cdouble(std::rint(x.v)); }
inline cdouble copysign(cdouble x, cdouble y) { return cdouble(std::copysign(x.v, y.v)); }
inline cdouble fma(cdouble a, cdouble b, cdouble c) { g_ops.mul++; g_ops.add++; return cdouble(std::fma(a.v, b.v, c.v)); }
inline cdouble frexp(cdouble x, int* e) { return cdouble(std::frexp(x.v, e)); }
inline cdouble ldexp(cdouble x, int e) { return cdouble(std::ldexp(x.v, e)); }

#define double cdouble
