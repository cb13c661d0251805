"""Generate uwshcu_adj_kernel.cuh, the adjoint (reverse-mode) column kernels, from the FP64 column code
in uwshcu_fp64_kernel.cuh.  Run after changing the FP64 column code:

    python hpc-and-climate-model_b200/csrc/gen_adjoint.py

Every FP64 variable becomes an Ad (uw_adj.h: value and tape index); the saturation table and the
constant bank stay double.  The differentiated inputs get fixed indices at their loads: t0 and qv0
(every load of level k, the set-up's and the implicit-CIN restore's, gets the same index), tke (the
PBL average), pblh, and the tuning parameters rpen, rle, rkm, criqc.  Every output store writes the
value to the FP64 output and the value's tape index to the column's output-index table (the last
store of an element wins, as the value does).

The saturation adjustment (conden, uwshcu.F90:4718-4785) iterates a Newton step 10 times.  Its taped
version runs the FP64 function on values that carry their derivatives with respect to the 4 inputs
(Fd4, forward mode in registers: conden_f) and records only the converged temperature, with those 4
partials; the outputs follow from it as in the FP64 function.  The derivative is the tangent-linear
model's (the 10 steps differentiated) without ~200 records per call.

The values are computed by the same operations as the FP64 path (the unit is built without FMA
contraction), so the forward kernel also reproduces the FP64 outputs bit for bit.
"""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "uwshcu_fp64_kernel.cuh")
DST = os.path.join(HERE, "uwshcu_adj_kernel.cuh")
# outputs with a cotangent, in the order of the output-index table (trten after them)
ADJ_OUT = ("cush umf slflx qtflx flxprc1 flxsnow1 qvten qlten qiten sten uten vten qrten qsten precip snow "
           "evapc cufrc qcu qlu qiu cbmf qc rliq wu").split()


def rep(s, old, new, count=1):
    n = s.count(old)
    assert n == count, (old[:80], n)
    return s.replace(old, new)


def function(s, head):
    """The text of the function whose definition starts with head, through its closing brace."""
    start = s.index(head)
    return s[start: s.index("\n}\n", start) + 3]


KERNELS = r'''
// ---- adjoint kernels ---------------------------------------------------------------------------

// Forward sweep: thread t runs worklist entry b0 + t as the FP64 path does (same values, written to
// the outputs) and records its column on the tape of its warp and in its output-index table.
template <int KP, int NC>
__global__ void __launch_bounds__(UW_ADJ_BLOCK) uwshcu_adj_forward(const __grid_constant__ UwArgs A,
                                                                   const __grid_constant__ UwAdj G)
{
    __shared__ double tbl[UW_TBL];
    for (int t = threadIdx.x; t < UW_TBL; t += blockDim.x) tbl[t] = c_estbl[t];
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const int w = slot >> 5, lane = threadIdx.x & 31;
    const bool active = slot < G.nb;
    const int i = active ? G.wl[G.b0 + slot] : 0;
    AdWarpTape& tp = uw_adj_tape();
    tp.n[lane] = 0;
    if (lane == 0) {
        tp.ab = G.ab + (size_t)w * G.rcap * 32;
        tp.d = G.d + (size_t)w * G.rcap * 32;
        tp.cap = G.rcap;
        tp.base = 3 * A.mkx + 6;
        tp.overflow = 0;
    }
    __syncthreads();
    uw_column<KP, NC, UW_MODE_LIST, 0>(A, tbl, i, active, nullptr, nullptr, G, slot);
    __syncwarp();
    const int rows = __reduce_max_sync(0xffffffffu, tp.n[lane]);
    if (lane == 0) {
        G.nrow[w] = rows;
        G.ovf[w] = tp.overflow;
    }
}

// Fraction r in [1/2, 7/8) for the n-th seed of column i (a hash of both): the split sweeps seed
// RN(r w) and w - RN(r w), whose sum is w exactly (Sterbenz: RN(r w) lies in [w/2, w]).
__device__ __forceinline__ double uw_adj_split_frac(unsigned i, unsigned n)
{
    unsigned h = i * 0x9E3779B1u ^ (n + 0x7F4A7C15u) * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    h *= 0x297A2D39u;
    h ^= h >> 15;
    return 0.5 + 0.375 * (double)(h >> 8) * 0x1p-24;
}

// Reverse sweep: warp w seeds the indices of its lanes' output-index tables with the cotangents of C,
// sweeps its tape (uw_adj_sweep) and writes the gradients of its columns.  The adjoints of warp w are
// zero on entry.  G.split 1 and 2 seed the two parts of a split of every cotangent (uw_adj_split_frac)
// and store the gradients in G.gsave instead of C; a G.split 0 sweep after them writes, with the
// gradients, the column's defect of linearity under that split to G.defect.
template <int KP, int NC>
__global__ void __launch_bounds__(UW_ADJ_RBLOCK) uwshcu_adj_reverse(const __grid_constant__ UwArgs A,
                                                                    const __grid_constant__ UwAdj G,
                                                                    const __grid_constant__ uwshcu_adjoint C)
{
    __shared__ double near[UW_ADJ_RBLOCK / 32][UW_ADJ_WIN][32];
    __shared__ AdStage stage[UW_ADJ_RBLOCK / 32];
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const int w = slot >> 5, lane = threadIdx.x & 31;
    if ((w << 5) >= G.nb) return;   // uniform over the warp: no slot of the warp is in use
    const bool active = slot < G.nb;
    const int i = active ? G.wl[G.b0 + slot] : 0;
    const int mix = A.mix, mkx = A.mkx, ncnst = A.ncnst, inv = A.inv, nin = 3 * mkx + 6;
    const int rows = G.nrow[w];
    if (G.ovf[w] || rows > G.rcap) {
        if (lane == 0) atomicOr(G.status, 1u);
        return;
    }
    double* const af = G.adj + (size_t)w * G.astride;
    double (*const nr)[32] = near[threadIdx.x >> 5];
    for (int r = 0; r < UW_ADJ_WIN; r++) nr[r][lane] = 0.0;
#define RI(k) (inv ? (mkx - (k)) : (k))
#define RL(k) (inv ? (mkx - (k)) : ((k) - 1))
#define AID(f, k) G.ids[((size_t)(f) * KP + (k)) * G.cap + slot]
// a seed at an index with the sign bit goes to the index, negated
#define SEED_AT(id, w)                                                                                    \
    {                                                                                                     \
        const int id_ = (id), ix_ = id_ & ~AD_NEG;                                                        \
        double w_ = (w);                                                                                  \
        if (G.split) {                                                                                    \
            const double p_ = uw_adj_split_frac((unsigned)i, nseed++) * w_;                               \
            w_ = G.split == 1 ? p_ : w_ - p_;                                                             \
        }                                                                                                 \
        if (id_ >= 0 && ix_ < nin + rows) atomicAdd(&af[(size_t)ix_ * 32 + lane], (id_ & AD_NEG) ? -w_ : w_); \
    }
#define SEED(f, k, row)                                                                                   \
    if (C.f) SEED_AT(AID(UW_AO_##f, k), C.f[(size_t)(row) * mix + i])
    unsigned nseed = 0;
    if (active) {
        for (int k = 0; k <= mkx; k++) {
            SEED(umf, k, RI(k)) SEED(slflx, k, RI(k)) SEED(qtflx, k, RI(k)) SEED(flxprc1, k, RI(k))
            SEED(flxsnow1, k, RI(k)) SEED(wu, k, RI(k))
        }
        for (int k = 1; k <= mkx; k++) {
            SEED(qvten, k, RL(k)) SEED(qlten, k, RL(k)) SEED(qiten, k, RL(k)) SEED(sten, k, RL(k))
            SEED(uten, k, RL(k)) SEED(vten, k, RL(k)) SEED(qrten, k, RL(k)) SEED(qsten, k, RL(k))
            SEED(evapc, k, RL(k)) SEED(cufrc, k, RL(k)) SEED(qcu, k, RL(k)) SEED(qlu, k, RL(k))
            SEED(qiu, k, RL(k)) SEED(qc, k, RL(k))
        }
        SEED(cush, 0, 0) SEED(precip, 0, 0) SEED(snow, 0, 0) SEED(cbmf, 0, 0) SEED(rliq, 0, 0)
        if (C.trten)
            for (int m = 1; m <= ncnst; m++)
                for (int k = 1; k <= mkx; k++) SEED_AT(AID(UW_AO_N + m - 1, k), C.trten[((size_t)(m - 1) * mkx + RL(k)) * mix + i])
    }
    __syncwarp();
    uw_adj_sweep(G.ab + (size_t)w * G.rcap * 32, G.d + (size_t)w * G.rcap * 32, rows, nin, af, nr,
                 stage[threadIdx.x >> 5]);
    if (!active) return;
#define GR(x) __ldcg(&af[(size_t)(x) * 32 + lane])
#define GS(s, x) G.gsave[((size_t)(s) * nin + (x)) * G.cap + slot]
    if (G.split) {
        for (int x = 0; x < nin; x++) GS(G.split - 1, x) = GR(x);
        return;
    }
    if (G.defect) {
        // per gradient asked for (t0, qv0, tke, pblh, rpen, rle, rkm, criqc): max |g - g1 - g2| over
        // max (|g1| + |g2|); the column's defect is the largest of them
        const double* const want[8] = {C.t0, C.qv0, C.tke, C.pblh, C.rpen, C.rle, C.rkm, C.criqc};
        double worst = 0.0;
        for (int f = 0; f < 8; f++) {
            if (!want[f]) continue;
            const int x0 = f < 3 ? f * mkx : 3 * mkx + f - 2, x1 = f < 2 ? x0 + mkx : (f == 2 ? x0 + mkx + 1 : x0 + 1);
            double num = 0.0, den = 0.0;
            for (int x = x0; x < x1; x++) {
                const double g1 = GS(0, x), g2 = GS(1, x);
                num = MX(num, fabs(GR(x) - g1 - g2));
                den = MX(den, fabs(g1) + fabs(g2));
            }
            if (den > 0.0) worst = MX(worst, num / den);
        }
        G.defect[i] = worst;
    }
    for (int k = 1; k <= mkx; k++) {
        if (C.t0) C.t0[(size_t)RL(k) * mix + i] = GR(k - 1);
        if (C.qv0) C.qv0[(size_t)RL(k) * mix + i] = GR(mkx + k - 1);
    }
    if (C.tke)
        for (int k = 0; k <= mkx; k++) C.tke[(size_t)RI(k) * mix + i] = GR(2 * mkx + k);
    if (C.pblh) C.pblh[i] = GR(3 * mkx + 1);
    if (C.rpen) C.rpen[i] = GR(3 * mkx + 2);
    if (C.rle) C.rle[i] = GR(3 * mkx + 3);
    if (C.rkm) C.rkm[i] = GR(3 * mkx + 4);
    if (C.criqc) C.criqc[i] = GR(3 * mkx + 5);
#undef GS
#undef GR
#undef SEED
#undef SEED_AT
#undef AID
#undef RI
#undef RL
}

}  // namespace
'''

CONDEN = r'''
// The saturation adjustment: conden_f runs the FP64 function with the derivatives along its 4 inputs
// (p, ex, thl, qt) through the 10 Newton steps; the converged temperature is recorded with them
// (3 records) and the outputs follow from it as in the FP64 function.
__device__ __noinline__ int conden(Ad p, Ad ex, Ad thl, Ad qt, Ad& th, Ad& qv, Ad& ql, Ad& qi,
                                   const double* __restrict__ tbl)
{
    Fd4 th_, qv_, ql_, qi_, ts(0.0);
    const int id = conden_f(Fd4(p.v, 0), Fd4(ex.v, 1), Fd4(thl.v, 2), Fd4(qt.v, 3), th_, qv_, ql_, qi_, tbl, ts);
    const Ad tc = thl * ex;
    if (ts.v == 0.0) {   // unsaturated
        qv = qt;
        ql = Ad(0.0);
        qi = Ad(0.0);
        th = tc / ex;
        return id;
    }
    const Ad nu = MX(MN((268.0 - tc) / 20.0, 1.0), 0.0);
    const Ad t1 = ad_rec(ts.v, p.i, ts.d[0], ex.i, ts.d[1]);
    const Ad t2 = ad_rec(ts.v, thl.i, ts.d[2], qt.i, ts.d[3]);
    const Ad temps = ad_rec(ts.v, t1.i, 1.0, t2.i, 1.0);
    const Ad qs = qsat_qs(temps, p, tbl);
    const Ad qc = MX(qt - qs, 0.0);
    qv = qt - qc;
    ql = qc * (1.0 - nu);
    qi = nu * qc;
    th = temps / ex;
    return id;
}
'''


def forward_helpers(src):
    """estblf_f, qsat_qs_f and conden_f: the FP64 functions on Fd4 values; conden_f also returns the
    converged temperature of a saturated adjustment in t_sat (left alone when unsaturated)."""
    est = function(src, "__device__ __forceinline__ double estblf(double td,")
    est = rep(est, "double estblf(", "double estblf_f(")
    qs = function(src, "__device__ __forceinline__ double qsat_qs(double t, double p,")
    qs = rep(qs, "double qsat_qs(", "double qsat_qs_f(")
    qs = rep(qs, "estblf(", "estblf_f(")
    cd = function(src, "__device__ __noinline__ int conden(double p,")
    cd = rep(cd, "int conden(", "int conden_f(")
    cd = rep(cd, "const double* __restrict__ tbl)\n{", "const double* __restrict__ tbl, double& t_sat)\n{")
    cd = rep(cd, "qsat_qs(", "qsat_qs_f(", 2)
    cd = rep(cd, "        th = temps / ex;\n", "        th = temps / ex;\n        t_sat = temps;\n")
    out = est + "\n" + qs + "\n" + cd
    out = re.sub(r"\bdouble\b", "Fd4", out).replace("const Fd4* __restrict__ tbl", "const double* __restrict__ tbl")
    return "\n// the FP64 functions on values with 4 derivatives, for the taped saturation adjustment\n" + out


def main():
    src = open(SRC).read()
    s = src[src.index("#pragma once"):]
    # the column code only: the FP64 kernels are replaced by the adjoint kernels
    s = s[: s.index("// ---- kernels ------")].rstrip() + "\n"
    s = rep(s, '#include "uw_math.h"', '#include "uw_math.h"\n#include "uw_adj.h"')
    s = rep(s, '#include "uwshcu_common.cuh"', '#include "uwshcu_common.cuh"\n#include "uwshcu.h"')
    s = re.sub(r"\bdouble\b", "Ad", s)
    # tables and constants stay double
    s = s.replace("__constant__ Ad c_estbl[UW_TBL];", "__constant__ double c_estbl[UW_TBL];")
    s = s.replace("const Ad* __restrict__ tbl", "const double* __restrict__ tbl")
    s = s.replace("__shared__ Ad tbl[UW_TBL];", "__shared__ double tbl[UW_TBL];")
    # conden: the taped version with the implicit derivative, after the FP64 helpers
    old = function(s, "__device__ __noinline__ int conden(Ad p,")
    s = rep(s, old, forward_helpers(src) + CONDEN)
    # launch arguments of the adjoint kernels and the output-index table
    fields = "\n".join("#define UW_AO_%s %d" % (f, j) for j, f in enumerate(ADJ_OUT))
    s = s.replace("namespace {\n", "namespace {\n\n"
                  "// Output-index table: entry (f, k) of a slot for output field f (UW_AO_*) at level k, trten\n"
                  "// tracer m at f = UW_AO_N + m - 1; a column field at k = 0.\n" + fields +
                  "\n#define UW_AO_N %d\n#define UW_ADJ_RBLOCK 32   // threads per block of the reverse sweep (one warp)\n\n"
                  "// One adjoint launch: slot t is worklist entry wl[b0 + t], t < nb; warp w holds slots 32w .. 32w+31.\n"
                  "struct UwAdj {\n"
                  "    const int* wl;\n"
                  "    int b0, nb;\n"
                  "    int2* ab;            // warp w's tape: ab + w * rcap * 32, d + w * rcap * 32\n"
                  "    double2* d;\n"
                  "    int rcap;            // rows per warp\n"
                  "    int* ids;            // output-index table, entry (f, k) of slot t at (f * KP + k) * cap + t\n"
                  "    int cap;             // slots of the table (>= nb)\n"
                  "    int* nrow;           // rows taken per warp\n"
                  "    int* ovf;            // tape overflow per warp\n"
                  "    double* adj;         // warp w's adjoints at adj + w * astride (index x of lane l at x * 32 + l)\n"
                  "    size_t astride;\n"
                  "    unsigned int* status;\n"
                  "    int split;           // reverse sweep: 0 the cotangents, 1 and 2 the two parts of their split\n"
                  "    double* gsave;       // gradients of split s at ((s - 1) * (3 mkx + 6) + x) * cap + slot\n"
                  "    double* defect;      // per column (mix), written by a split-0 sweep; NULL: not computed\n"
                  "};\n" % len(ADJ_OUT), 1)
    s = rep(s, "const bool active, int* __restrict__ wl, int* __restrict__ wl_count)",
            "const bool active, int* __restrict__ wl, int* __restrict__ wl_count,\n"
            "                                          const UwAdj& G, const int slot)")
    # differentiated inputs: fixed tape indices 0 .. 3 mkx + 5
    s = rep(s, "#define OT(m, k) A.trten[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]",
            "#define OT(m, k) A.trten[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]\n"
            "#define AOI(f, k) G.ids[((size_t)UW_AO_##f * KP + (k)) * G.cap + slot]\n"
            "#define AOT(m, k) G.ids[((size_t)(UW_AO_N + (m) - 1) * KP + (k)) * G.cap + slot]")
    s = rep(s, "t0[k] = GL(t0, k);", "t0[k] = Ad(GL(t0, k), (k) - 1);", 3)
    s = rep(s, "qv0[k] = GL(qv0, k);", "qv0[k] = Ad(GL(qv0, k), mkx + (k) - 1);", 3)
    s = rep(s, "tkeavg = tkeavg + dpi * GI(tke, k);", "tkeavg = tkeavg + dpi * Ad(GI(tke, k), 2 * mkx + (k));")
    s = rep(s, "const Ad pblh = __ldg(&A.pblh[i]);", "const Ad pblh = Ad(__ldg(&A.pblh[i]), 3 * mkx + 1);")
    s = rep(s, "rpen = c.rpen;", "rpen = Ad(c.rpen, 3 * mkx + 2);")
    s = rep(s, "const Ad rle = c.rle, rkm = c.rkm,", "const Ad rle = Ad(c.rle, 3 * mkx + 3), rkm = Ad(c.rkm, 3 * mkx + 4),")
    s = rep(s, "criqc = c.criqc,", "criqc = Ad(c.criqc, 3 * mkx + 5),")
    # stores: the value to the output, its tape index to the output-index table
    s = re.sub(r"\b(OI|OL)\((\w+), ([^()]*?)\) = ([^;]+);",
               lambda m: "{ const Ad v_ = (%s); %s(%s, %s) = v_.v; AOI(%s, %s) = v_.i; }" % (
                   m.group(4), m.group(1), m.group(2), m.group(3), m.group(2), m.group(3)), s)
    s = re.sub(r"\bOT\((\w+), (\w+)\) = ([^;]+);",
               lambda m: "{ const Ad v_ = (%s); OT(%s, %s) = v_.v; AOT(%s, %s) = v_.i; }" % (
                   m.group(3), m.group(1), m.group(2), m.group(1), m.group(2)), s)

    def col_store(m):
        f, x = m.group(1), m.group(2)
        if f in ADJ_OUT:
            return "{ const Ad v_ = (%s); A.%s[i] = v_.v; AOI(%s, 0) = v_.i; }" % (x, f, f)
        return "A.%s[i] = tl_val(%s);" % (f, x)
    s = re.sub(r"\bA\.(precip|snow|cush|cbmf|rliq|cnt|cnb)\[i\] = ([^;]+);", col_store, s)
    s = re.sub(r"(A\.diag_real\[[^\]]+\]) = ([^;]+);", lambda m: "%s = tl_val(%s);" % (m.group(1), m.group(2)), s)
    s = re.sub(r"\bDLV\(([^()]*)\) = ([^;]+);", lambda m: "DLV(%s) = tl_val(%s);" % (m.group(1), m.group(2)), s)
    # the warp synchronisations also align the lanes' tape rows
    s = rep(s, "#define UW_SYNC() __syncwarp(live)", "#define UW_SYNC() ad_align(live)")
    # the split worklist pass is not used here: no state copies
    s = re.sub(r"\n[ ]*UW_T?(SAVE|LOAD)_STATE\([^;]*\);", "", s)
    for u in ("AOI", "AOT"):
        s = s.replace("#undef OT\n", "#undef OT\n#undef %s\n" % u, 1)
    # close the column code's namespace block, then the kernels in a new one
    assert s.rstrip().endswith("}"), s[-200:]
    s = s + "\n}  // namespace\n\nnamespace {\n" + KERNELS
    header = ("// uwshcu_adj_kernel.cuh -- adjoint (reverse-mode) kernels of compute_uwshcu\n"
              "// (uwshcu.F90:478-4664).  GENERATED by gen_adjoint.py from uwshcu_fp64_kernel.cuh: do not edit;\n"
              "// change the FP64 column code and regenerate.  See gen_adjoint.py for what the generator does.\n")
    open(DST, "w").write(header + s)
    print("wrote", DST)


if __name__ == "__main__":
    main()
