// uw_adj.h -- reverse-mode (adjoint) arithmetic for the column code: a taped value type on a tape
// shared by the lanes of a warp.
//
// Ad carries a value and its index on the tape (-1: passive, a constant or a value that does not
// depend on the differentiated inputs).  Every operation computes its value exactly as the FP64 code
// does (same operation, same rounding; the unit is built without FMA contraction) and, when an
// operand is active, records {a, b, da, db}: the operands' indices and the partial derivatives of the
// result with respect to them.  The partials are the ones the tangent-linear type (uw_dual.h) applies,
// so the adjoint is the transpose of the tangent-linear model.
//
// The tape belongs to a warp.  One lane computes one column, and the lanes run the column code
// together, so the lanes that execute an operation at once record it in one ROW: record (row, lane)
// at row * 32 + lane.  A lane's indices are its own (row numbers of its column).  Each lane counts
// its rows; at the column code's warp synchronisations (ad_align, the points where every live lane
// arrives) the live lanes continue from the largest count, so lanes that then run the same
// operations record them in the same rows.  Between those points a lane's rows follow its own
// branches only, so the rows, and with them the reverse sweep's order of additions, depend on the
// columns alone (not on how the hardware happens to group diverged lanes).  A row a lane skipped holds
// no record of that lane: no value of the lane has that index, so its adjoint stays zero and the
// reverse sweep never uses the entry.  The rows of a warp are read back as 32 contiguous records, and
// the adjoint of row r of every lane is one contiguous 256-byte line, so the reverse sweep reads and
// writes whole lines.
//
// Index space of a warp: 0 .. base-1 are the differentiated inputs, base + r is row r.  A row beyond
// the tape's capacity is not written and sets the overflow flag: the caller reports it as an error
// instead of using the gradients.
#pragma once
#include <math.h>
#include "uw_math.h"

#define UW_ADJ_BLOCK 32    // threads per block of the forward sweep: one warp, spread over every SM
#define UW_ADJ_WIN 64      // rows of the reverse sweep's shared-memory window (a power of two)
#define UW_ADJ_PF 16       // rows per block of the reverse sweep's prefetch (records and far adjoints)

// the tape of one warp
struct AdWarpTape {
    int2* ab;          // operand indices of (row, lane) at ab[row * 32 + lane] (-1: none)
    double2* d;        // their partials, same layout
    int cap;           // rows available
    int base;          // index of row 0
    int overflow;
    int n[32];         // rows counted by each lane
};

__device__ __forceinline__ AdWarpTape& uw_adj_tape()
{
    __shared__ AdWarpTape t[UW_ADJ_BLOCK / 32];
    return t[threadIdx.x >> 5];
}

struct Ad {
    double v;
    int i;
    // passive by default: an index is either a row's, an input's or -1, never uninitialised
    __device__ __forceinline__ Ad() : v(0.0), i(-1) {}
    __device__ __forceinline__ constexpr Ad(double x) : v(x), i(-1) {}
    __device__ __forceinline__ constexpr Ad(double x, int id) : v(x), i(id) {}
    __device__ __forceinline__ explicit operator double() const { return v; }
    __device__ __forceinline__ explicit operator int() const { return (int)v; }
};

// The row of a record with operands (a, da) and (b, db): the lane's next row.  Called, not inlined:
// the column code records from ~10^4 sites, and one shared copy keeps the kernel's code inside the
// instruction cache.
static __device__ __noinline__ int ad_row(int a, double da, int b, double db)
{
    AdWarpTape& t = uw_adj_tape();
    const int lane = threadIdx.x & 31;
    const int r = t.n[lane];
    t.n[lane] = r + 1;
    if (r < t.cap) {
        t.ab[(size_t)r * 32 + lane] = make_int2(a, b);
        t.d[(size_t)r * 32 + lane] = make_double2(da, db);
    } else {
        t.overflow = 1;
    }
    return t.base + r;
}

// The column code's warp synchronisation over the live lanes, which also aligns their row counts.
__device__ __forceinline__ void ad_align(unsigned live)
{
    __syncwarp(live);
    AdWarpTape& t = uw_adj_tape();
    const int lane = threadIdx.x & 31;
    t.n[lane] = __reduce_max_sync(live, t.n[lane]);
}

// Bit 30 of an index marks a value that is minus the one the index names (negations record
// nothing); a record takes the sign into its partial.  Indices stay below 2^20.
#define AD_NEG (1 << 30)

__device__ __forceinline__ Ad ad_rec(double v, int a, double da, int b, double db)
{
    if (a < 0 && b < 0) return Ad(v);
    if (a >= 0 && (a & AD_NEG)) {
        a ^= AD_NEG;
        da = -da;
    }
    if (b >= 0 && (b & AD_NEG)) {
        b ^= AD_NEG;
        db = -db;
    }
    return Ad(v, ad_row(a, da, b, db));
}

// the index of -x
__device__ __forceinline__ int ad_neg(int i) { return i < 0 ? i : i ^ AD_NEG; }

// A result whose derivative is exactly 1 or -1 in its only active operand (x + c, c + x, x - c, c - x,
// -x, |x|) takes that operand's index, with the sign, instead of a record: an adjoint added to the
// index is the chain rule with factor +-1.
__device__ __forceinline__ Ad operator+(Ad a, Ad b)
{
    if (b.i < 0) return Ad(a.v + b.v, a.i);
    if (a.i < 0) return Ad(a.v + b.v, b.i);
    return ad_rec(a.v + b.v, a.i, 1.0, b.i, 1.0);
}
__device__ __forceinline__ Ad operator-(Ad a, Ad b)
{
    if (b.i < 0) return Ad(a.v - b.v, a.i);
    if (a.i < 0) return Ad(a.v - b.v, ad_neg(b.i));
    return ad_rec(a.v - b.v, a.i, 1.0, b.i, -1.0);
}
__device__ __forceinline__ Ad operator*(Ad a, Ad b) { return ad_rec(a.v * b.v, a.i, b.v, b.i, a.v); }
__device__ __forceinline__ Ad operator/(Ad a, Ad b)
{
    const double q = a.v / b.v;
    return ad_rec(q, a.i, 1.0 / b.v, b.i, -q / b.v);
}
__device__ __forceinline__ Ad operator-(Ad a) { return Ad(-a.v, ad_neg(a.i)); }
__device__ __forceinline__ Ad operator+(Ad a) { return a; }
__device__ __forceinline__ Ad& operator+=(Ad& a, Ad b) { return a = a + b; }
__device__ __forceinline__ Ad& operator-=(Ad& a, Ad b) { return a = a - b; }
__device__ __forceinline__ bool operator<(Ad a, Ad b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(Ad a, Ad b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(Ad a, Ad b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(Ad a, Ad b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(Ad a, Ad b) { return a.v == b.v; }
__device__ __forceinline__ bool operator!=(Ad a, Ad b) { return a.v != b.v; }

__device__ __forceinline__ double tl_val(Ad x) { return x.v; }
__device__ __forceinline__ double tl_val(double x) { return x; }

__device__ __forceinline__ Ad uw_div_by(Ad a, Ad b, Ad y)
{
    const double q = uw_div_by(a.v, b.v, y.v);
    return ad_rec(q, a.i, 1.0 / b.v, b.i, -q / b.v);
}
__device__ __forceinline__ bool uw_isfinite(const Ad& x) { return isfinite(x.v); }
__device__ __forceinline__ Ad uw_exp(Ad x)
{
    const double e = uw_exp(x.v);
    return ad_rec(e, x.i, e, -1, 0.0);
}
__device__ __forceinline__ Ad uw_log(Ad x) { return ad_rec(uw_log(x.v), x.i, 1.0 / x.v, -1, 0.0); }
__device__ __forceinline__ Ad uw_pow(Ad x, Ad y)
{
    const double p = uw_pow(x.v, y.v);
    return ad_rec(p, x.i, x.i >= 0 ? p * y.v / x.v : 0.0, y.i, y.i >= 0 ? p * uw_log(x.v) : 0.0);
}
__device__ __forceinline__ Ad uw_erfc(Ad x)
{
    const double e = uw_erfc(x.v);
    return ad_rec(e, x.i, x.i >= 0 ? -1.1283791670955126 * uw_exp(-(x.v * x.v)) : 0.0, -1, 0.0);
}
__device__ __forceinline__ Ad sqrt(Ad x)
{
    const double s = sqrt(x.v);
    return ad_rec(s, x.i, x.i >= 0 ? 1.0 / (2.0 * s) : 0.0, -1, 0.0);
}
__device__ __forceinline__ Ad fabs(Ad x) { return Ad(fabs(x.v), x.v < 0.0 ? ad_neg(x.i) : x.i); }
__device__ __forceinline__ Ad trunc(Ad x) { return Ad(trunc(x.v)); }
__device__ __forceinline__ Ad floor(Ad x) { return Ad(floor(x.v)); }
__device__ __forceinline__ Ad copysign(Ad a, Ad b)
{
    const double r = copysign(a.v, b.v);
    return Ad(r, r == a.v ? a.i : ad_neg(a.i));
}

// A value with its derivatives along 4 directions (forward mode, no tape), for the inner iterations of
// one function call: the saturation adjustment's 10 Newton steps carry the derivatives with respect
// to its 4 inputs, and the converged temperature's record takes them (3 records instead of ~200).
// The value is computed by the operation of the FP64 code, the derivatives by the tangent-linear
// rules of uw_dual.h.
struct Fd4 {
    double v, d[4];
    __device__ __forceinline__ Fd4() : v(0.0), d{0.0, 0.0, 0.0, 0.0} {}
    __device__ __forceinline__ Fd4(double x) : v(x), d{0.0, 0.0, 0.0, 0.0} {}
    __device__ __forceinline__ Fd4(double x, int dir) : v(x), d{dir == 0 ? 1.0 : 0.0, dir == 1 ? 1.0 : 0.0, dir == 2 ? 1.0 : 0.0, dir == 3 ? 1.0 : 0.0} {}
    __device__ __forceinline__ explicit operator int() const { return (int)v; }
};
__device__ __forceinline__ Fd4 fd4_lin(double v, const Fd4& a, double da, const Fd4& b, double db)
{
    Fd4 r(v);
#pragma unroll
    for (int j = 0; j < 4; j++) r.d[j] = a.d[j] * da + b.d[j] * db;
    return r;
}
__device__ __forceinline__ Fd4 fd4_lin(double v, const Fd4& a, double da)
{
    Fd4 r(v);
#pragma unroll
    for (int j = 0; j < 4; j++) r.d[j] = a.d[j] * da;
    return r;
}
__device__ __forceinline__ Fd4 operator+(const Fd4& a, const Fd4& b) { return fd4_lin(a.v + b.v, a, 1.0, b, 1.0); }
__device__ __forceinline__ Fd4 operator-(const Fd4& a, const Fd4& b) { return fd4_lin(a.v - b.v, a, 1.0, b, -1.0); }
__device__ __forceinline__ Fd4 operator*(const Fd4& a, const Fd4& b) { return fd4_lin(a.v * b.v, a, b.v, b, a.v); }
__device__ __forceinline__ Fd4 operator/(const Fd4& a, const Fd4& b)
{
    const double q = a.v / b.v;
    return fd4_lin(q, a, 1.0 / b.v, b, -q / b.v);
}
__device__ __forceinline__ Fd4 operator-(const Fd4& a) { return fd4_lin(-a.v, a, -1.0); }
__device__ __forceinline__ bool operator<(const Fd4& a, const Fd4& b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(const Fd4& a, const Fd4& b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(const Fd4& a, const Fd4& b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(const Fd4& a, const Fd4& b) { return a.v >= b.v; }
__device__ __forceinline__ Fd4 uw_div_by(const Fd4& a, const Fd4& b, const Fd4& y)
{
    const double q = uw_div_by(a.v, b.v, y.v);
    return fd4_lin(q, a, 1.0 / b.v, b, -q / b.v);
}
__device__ __forceinline__ Fd4 fabs(const Fd4& x) { return fd4_lin(fabs(x.v), x, x.v < 0.0 ? -1.0 : 1.0); }
__device__ __forceinline__ Fd4 trunc(const Fd4& x) { return Fd4(trunc(x.v)); }

// Records of UW_ADJ_PF rows of a warp in shared memory, staged by asynchronous copies.
struct AdStage {
    int2 ab[UW_ADJ_PF][32];
    double2 d[UW_ADJ_PF][32];
};

// Copies the records of row r of this lane into stage slot s (one commit group per row; a row below
// zero commits an empty group, so that every row has one).
__device__ __forceinline__ void ad_stage_row(AdStage& st, int s, const int2* ab, const double2* dd, int r)
{
    const int lane = threadIdx.x & 31;
    if (r >= 0) {
        const unsigned sa = (unsigned)__cvta_generic_to_shared(&st.ab[s][lane]);
        const unsigned sd = (unsigned)__cvta_generic_to_shared(&st.d[s][lane]);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(ab + (size_t)r * 32 + lane) : "memory");
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sd), "l"(dd + (size_t)r * 32 + lane) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// Reverse sweep of one warp's tape, run by the 32 lanes together (every lane of the warp calls it
// with the same rows and base).  af holds the adjoints of the warp's index space, index x of lane l
// at af[x * 32 + l]; it carries the seeds on entry and, on return, the inputs' gradients in indices
// 0 .. base-1.  near is the warp's window of UW_ADJ_WIN x 32 doubles in shared memory, zero on entry;
// st the warp's staging slots.
//
// A contribution of row x to an index y with x - y < UW_ADJ_WIN is added in the window (slot
// y mod UW_ADJ_WIN, which row y + UW_ADJ_WIN leaves free before it); one to an older index is added
// in af by a reduction that returns nothing.  Row y's value in af is final once rows y + UW_ADJ_WIN
// and above are done.  The rows go in blocks of UW_ADJ_PF: at the start of a block the far values of
// the next block are loaded (2 UW_ADJ_PF <= UW_ADJ_WIN, so their reductions are all done, and a
// lane's loads follow its own reductions to the same address in program order), and each row's
// records arrive by an asynchronous copy issued UW_ADJ_PF rows ahead.  An entry a lane did not record
// has a zero adjoint and is skipped; its operands are checked to lie below the row all the same, so
// no entry can address outside the index space.
__device__ __forceinline__ void uw_adj_sweep(const int2* __restrict__ ab, const double2* __restrict__ dd,
                                             int rows, int base, double* af, double (*near)[32], AdStage& st)
{
    static_assert(2 * UW_ADJ_PF <= UW_ADJ_WIN && (UW_ADJ_WIN & (UW_ADJ_WIN - 1)) == 0, "window");
    static_assert((UW_ADJ_PF & (UW_ADJ_PF - 1)) == 0, "stage");
    const int lane = threadIdx.x & 31;
    const int top = base + rows - 1;
    double fa[UW_ADJ_PF], fb[UW_ADJ_PF];
#pragma unroll
    for (int j = 0; j < UW_ADJ_PF; j++) {
        const int x = top - j;
        ad_stage_row(st, x & (UW_ADJ_PF - 1), ab, dd, x - base);
        fa[j] = x >= 0 ? __ldcg(&af[(size_t)x * 32 + lane]) : 0.0;
    }
    for (int x0 = top; x0 >= 0; x0 -= UW_ADJ_PF) {   // uniform
#pragma unroll
        for (int j = 0; j < UW_ADJ_PF; j++) {
            const int x = x0 - UW_ADJ_PF - j;
            fb[j] = x >= 0 ? __ldcg(&af[(size_t)x * 32 + lane]) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < UW_ADJ_PF; j++) {
            const int x = x0 - j;
            if (x < 0) break;
            asm volatile("cp.async.wait_group %0;\n" ::"n"(UW_ADJ_PF - 1) : "memory");
            const int s = x & (UW_ADJ_PF - 1);
            const int2 q = st.ab[s][lane];
            const double2 p = st.d[s][lane];
            double* const slot = &near[x & (UW_ADJ_WIN - 1)][lane];
            const double g = *slot + fa[j];
            *slot = 0.0;
            if (x < base) {
                af[(size_t)x * 32 + lane] = g;
            } else if (g != 0.0) {
                double va = p.x * g, vb = p.y * g;
                int ya = q.x, yb = q.y;
                if (ya == yb) {   // both operands the same value (x * x): one contribution
                    va += vb;
                    yb = -1;
                }
                if ((unsigned)ya < (unsigned)x) {
                    if (x - ya < UW_ADJ_WIN) near[ya & (UW_ADJ_WIN - 1)][lane] += va;
                    else atomicAdd(&af[(size_t)ya * 32 + lane], va);
                }
                if ((unsigned)yb < (unsigned)x) {
                    if (x - yb < UW_ADJ_WIN) near[yb & (UW_ADJ_WIN - 1)][lane] += vb;
                    else atomicAdd(&af[(size_t)yb * 32 + lane], vb);
                }
            }
            // the slot's records are in registers and used: refill it with row x - UW_ADJ_PF
            ad_stage_row(st, s, ab, dd, x - UW_ADJ_PF - base);
        }
#pragma unroll
        for (int j = 0; j < UW_ADJ_PF; j++) fa[j] = fb[j];
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
