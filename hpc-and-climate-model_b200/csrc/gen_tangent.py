"""Generate uwshcu_tl_kernel.cuh, the tangent-linear (forward-mode) column kernel, from the FP64
column code in uwshcu_fp64_kernel.cuh.  Run after changing the FP64 column code:

    python hpc-and-climate-model_b200/csrc/gen_tangent.py

Every FP64 variable becomes a Tl (uw_dual.h: value and derivative along one direction); the
saturation table and the constant bank stay double.  The directions enter at the loads of t0, qv0,
tke and pblh and at the tuning parameters rpen, rle, rkm, criqc (UwTangent); every output store
writes the value to the FP64 outputs and the derivative to the matching tangent output.  The values
are computed by the same operations as the FP64 path (the unit is built without FMA contraction),
so a tangent run also reproduces the FP64 outputs bit for bit.
"""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "uwshcu_fp64_kernel.cuh")
DST = os.path.join(HERE, "uwshcu_tl_kernel.cuh")
TANGENT_OUT = ("cush umf slflx qtflx flxprc1 flxsnow1 qvten qlten qiten sten uten vten trten qrten "
               "qsten precip snow evapc cufrc qcu qlu qiu cbmf qc rliq wu").split()


def rep(s, old, new, count=1):
    n = s.count(old)
    assert n == count, (old[:80], n)
    return s.replace(old, new)


def main():
    s = open(SRC).read()
    head_end = s.index("#pragma once")
    s = s[head_end:]
    # drop the batched and fast-mode kernels: the tangent kernel has its own launches
    s = s[: s.index("// Batched trigger pass: every column of every member of B")].rstrip() + "\n\n}  // namespace\n"
    s = rep(s, '#include "uw_math.h"', '#include "uw_math.h"\n#include "uw_dual.h"')
    s = re.sub(r"\bdouble\b", "Tl", s)
    # tables stay double
    s = s.replace("__constant__ Tl c_estbl[UW_TBL];", "__constant__ double c_estbl[UW_TBL];")
    s = s.replace("const Tl* __restrict__ tbl", "const double* __restrict__ tbl")
    s = s.replace("__shared__ Tl tbl[UW_TBL];", "__shared__ double tbl[UW_TBL];")
    # the tangent argument block
    s = rep(s, '#include "uwshcu_common.cuh"', '#include "uwshcu_common.cuh"\n#include "uwshcu.h"')
    # directions and tangent outputs of one launch: the ABI's uwshcu_tangent
    assert s.count("namespace {\n") >= 1
    s = s.replace("namespace {\n", "namespace {\n\ntypedef uwshcu_tangent UwTangent;\n", 1)
    s = rep(s, "const bool active, int* __restrict__ wl, int* __restrict__ wl_count)",
            "const bool active, int* __restrict__ wl, int* __restrict__ wl_count,\n"
            "                                          const UwTangent& T)")
    # seeded loads
    s = rep(s, "#define OT(m, k) A.trten[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]",
            "#define OT(m, k) A.trten[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]\n"
            "#define TOI(a, k) T.a[(size_t)RI(k) * mix + i]\n"
            "#define TOL(a, k) T.a[(size_t)RL(k) * mix + i]\n"
            "#define TOT(m, k) T.trten[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]\n"
            "#define SEEDL(a, da, k) Tl(GL(a, k), T.da ? __ldg(&T.da[(size_t)RL(k) * mix + i]) : 0.0)\n"
            "#define SEEDI(a, da, k) Tl(GI(a, k), T.da ? __ldg(&T.da[(size_t)RI(k) * mix + i]) : 0.0)")
    s = rep(s, "t0[k] = GL(t0, k);", "t0[k] = SEEDL(t0, dt0, k);", 3)
    s = rep(s, "qv0[k] = GL(qv0, k);", "qv0[k] = SEEDL(qv0, dqv0, k);", 3)
    s = rep(s, "tkeavg = tkeavg + dpi * GI(tke, k);", "tkeavg = tkeavg + dpi * SEEDI(tke, dtke, k);")
    s = rep(s, "const Tl pblh = __ldg(&A.pblh[i]);",
            "const Tl pblh = Tl(__ldg(&A.pblh[i]), T.dpblh ? __ldg(&T.dpblh[i]) : 0.0);")
    s = rep(s, "rpen = c.rpen;", "rpen = Tl(c.rpen, T.drpen);")
    s = rep(s, "const Tl rle = c.rle, rkm = c.rkm,", "const Tl rle = Tl(c.rle, T.drle), rkm = Tl(c.rkm, T.drkm),")
    s = rep(s, "criqc = c.criqc,", "criqc = Tl(c.criqc, T.dcriqc),")
    # stores: value to the output, derivative to the tangent output
    s = re.sub(r"\b(OI|OL)\((\w+), ([^()]*?)\) = ([^;]+);",
               lambda m: "{ const Tl v_ = (%s); %s(%s, %s) = tl_val(v_); T%s(%s, %s) = tl_der(v_); }" % (
                   m.group(4), m.group(1), m.group(2), m.group(3), m.group(1), m.group(2), m.group(3)), s)
    s = re.sub(r"\bOT\((\w+), (\w+)\) = ([^;]+);",
               lambda m: "{ const Tl v_ = (%s); OT(%s, %s) = tl_val(v_); TOT(%s, %s) = tl_der(v_); }" % (
                   m.group(3), m.group(1), m.group(2), m.group(1), m.group(2)), s)

    def col_store(m):
        f, x = m.group(1), m.group(2)
        if f in TANGENT_OUT:
            return "{ const Tl v_ = (%s); A.%s[i] = tl_val(v_); T.%s[i] = tl_der(v_); }" % (x, f, f)
        return "A.%s[i] = tl_val(%s);" % (f, x)
    s = re.sub(r"\bA\.(precip|snow|cush|cbmf|rliq|cnt|cnb)\[i\] = ([^;]+);", col_store, s)
    s = re.sub(r"(A\.diag_real\[[^\]]+\]) = ([^;]+);", lambda m: "%s = tl_val(%s);" % (m.group(1), m.group(2)), s)
    s = re.sub(r"\bDLV\(([^()]*)\) = ([^;]+);", lambda m: "DLV(%s) = tl_val(%s);" % (m.group(1), m.group(2)), s)
    # the kernel
    s = s.replace("uwshcu_fp64_kernel", "uwshcu_tl_kernel")
    s = rep(s, "uwshcu_tl_kernel(const __grid_constant__ UwArgs A, int* __restrict__ wl, int* __restrict__ wl_count)",
            "uwshcu_tl_kernel(const __grid_constant__ UwArgs A, int* __restrict__ wl, int* __restrict__ wl_count,\n"
            "                 const __grid_constant__ UwTangent T)")
    # the compute_zwshcu instantiation (ZW) is FP64 only: the tangent kernel is compute_uwshcu's
    s = s.replace("uw_column<KP, NC, MODE, 0, ZW>(A, tbl, i, active, wl, wl_count);",
                  "uw_column<KP, NC, MODE, 0>(A, tbl, i, active, wl, wl_count);")
    s = s.replace("template <int KP, int NC, int MODE, int ZW = 0>\n__global__", "template <int KP, int NC, int MODE>\n__global__")
    s = rep(s, "uw_column<KP, NC, MODE, 0>(A, tbl, i, active, wl, wl_count);",
            "uw_column<KP, NC, MODE, 0>(A, tbl, i, active, wl, wl_count, T);")
    s = rep(s, "__launch_bounds__(128, UW_LIST_MINB(MODE))", "__launch_bounds__(128)")
    # the split worklist pass (UW_MODE_LIST1 / UW_MODE_RESUME) is FP64 and FAST only: no state copies here
    s = re.sub(r"\n[ ]*UW_(SAVE|LOAD)_STATE\([^;]*\);", "", s)
    for u in ("TOI", "TOL", "TOT", "SEEDL", "SEEDI"):
        s = s.replace("#undef OT\n", "#undef OT\n#undef %s\n" % u, 1)
    header = ("// uwshcu_tl_kernel.cuh -- tangent-linear (forward-mode) kernel of compute_uwshcu\n"
              "// (uwshcu.F90:478-4664).  GENERATED by gen_tangent.py from uwshcu_fp64_kernel.cuh: do not edit;\n"
              "// change the FP64 column code and regenerate.  See gen_tangent.py for what the generator does.\n")
    open(DST, "w").write(header + s)
    print("wrote", DST)


if __name__ == "__main__":
    main()
