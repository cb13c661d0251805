"""Regenerate uwshcu_mixed_kernel.cuh from the FP64 column code in uwshcu_fp64_kernel.cuh.  Run after
changing the FP64 column code:

    python hpc-and-climate-model_b200/csrc/gen_mixed.py

The hand-written helper head of the mixed kernel (its FP32 helpers and FP64 islands: conden, roots,
qsinvert, compute_alpha, Kahan sums) is kept from the current file; the column code is the FP64
one with `double` -> R (float), float literals and float math, then the FP64 islands re-applied:
the CIN sums and compute_alpha, the roots of the mixing-fraction and penetration solves, Kahan sums
for tkeavg, the precipitation fluxes and rliq, and the positive_moisture fixer in FP64
(mixed_positive_moisture.inc).
"""
import os
import re
D = os.path.dirname(os.path.abspath(__file__)) + '/'
marker = '// ------------------------------------------------------------------------------------------------\n// The column kernel.'
cur = open(D + 'uwshcu_mixed_kernel.cuh').read()
head = cur[:cur.index(marker)]
# helper head fixes: warp-uniform early stop in the mixed conden, not inlined
old = '''        if (fabs(dT) < 1.e-9) break;'''
if old in head:
    head = head.replace(old, '''        if (__all_sync(__activemask(), fabs(dT) < 1.e-9)) break;''')
head = head.replace('__device__ __forceinline__ int conden(R p, R ex, R thl, R qt, R& th, R& qv, R& ql, R& qi,',
                    '__device__ __noinline__ int conden(R p, R ex, R thl, R qt, R& th, R& qv, R& ql, R& qi,')

src = open(D + 'uwshcu_fp64_kernel.cuh').read()
b = src[src.index(marker):]
# keep uw_column and the plain kernel only
cut = b.index('// The fast-FP64 precision mode: same launch shapes as uwshcu_fp64_kernel.')
b = b[:cut].rstrip() + '\n\n}  // namespace\n'
b = b.replace('uwshcu_fp64_kernel', 'uwshcu_mixed_kernel')
# the compute_zwshcu instantiation (ZW) is FP64 only: the mixed kernel is compute_uwshcu's
b = b.replace('uw_column<KP, NC, MODE, 0, ZW>(A, tbl, i, active, wl, wl_count);',
              'uw_column<KP, NC, MODE, 0>(A, tbl, i, active, wl, wl_count);')
b = b.replace('template <int KP, int NC, int MODE, int ZW = 0>\n__global__', 'template <int KP, int NC, int MODE>\n__global__')
b = b.replace('#define CONDEN(...) (FAST ? conden_fast(__VA_ARGS__) : conden(__VA_ARGS__))', '#define CONDEN(...) conden(__VA_ARGS__)')
b = re.sub(r'\bdouble\b', 'R', b)
lit = re.compile(r'(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)(?![\w.f])')
b = lit.sub(lambda m: m.group(1) + 'f', b)
b = re.sub(r'(?<![\w.])uw_(exp|log|pow|erfc)\(', lambda m: m.group(1) + '(', b)
for fn in ('exp', 'log', 'sqrt', 'pow', 'fabs', 'erfc', 'trunc'):
    b = re.sub(r'(?<![\w.])%s\(' % fn, fn + 'f(', b)
def rep(old, new, count=1):
    global b
    n = b.count(old)
    assert n == count, (old[:90], n)
    b = b.replace(old, new)
rep('#define GI(a, k) __ldg(&A.a[(size_t)RI(k) * mix + i])', '#define GI(a, k) ((R)__ldg(&A.a[(size_t)RI(k) * mix + i]))')
rep('#define GL(a, k) __ldg(&A.a[(size_t)RL(k) * mix + i])', '#define GL(a, k) ((R)__ldg(&A.a[(size_t)RL(k) * mix + i]))')
rep('#define GT(m, k) __ldg(&A.tr0[((size_t)((m) - 1) * mkx + RL(k)) * mix + i])', '#define GT(m, k) ((R)__ldg(&A.tr0[((size_t)((m) - 1) * mkx + RL(k)) * mix + i]))')
rep('#define CNT(x) (inv ? (R)(mkx + 1) - (x) : (x))', '#define CNT(x) (inv ? (double)(mkx + 1) - (double)(x) : (double)(x))')
rep('const R* __restrict__ tbl, const int i_in,', 'const double* __restrict__ tbld, const float* __restrict__ tblf, const int i_in,')

rep('''    __shared__ R tbl[UW_TBL];
    for (int t = threadIdx.x; t < UW_TBL; t += blockDim.x) tbl[t] = c_estbl[t];''',
'''    __shared__ double tbld[UW_TBL];
    __shared__ float tblf[UW_TBL];
    for (int t = threadIdx.x; t < UW_TBL; t += blockDim.x) {
        tbld[t] = c_estbl[t];
        tblf[t] = (float)c_estbl[t];
    }''', 4)
rep('uw_column<KP, NC, MODE, 0>(A, tbl, i, active, wl, wl_count);', 'uw_column<KP, NC, MODE, 0>(A, tbld, tblf, i, active, wl, wl_count);')
rep('(B.m[m], tbl, tid, active, B.wl[m], B.count + m);', '(B.m[m], tbld, tblf, tid, active, B.wl[m], B.count + m);')
rep('(B.m[m], tbl, i, active, nullptr, nullptr);', '(B.m[m], tbld, tblf, i, active, nullptr, nullptr);')
rep('(B.m[m], tbl, slot, active, nullptr, nullptr);', '(B.m[m], tbld, tblf, slot, active, nullptr, nullptr);')
b = b.replace(', tbl)', ', tbld, tblf)')
rep("""    R cin = 0, cinlcl = 0, plcl = 0,""", """    double cin = 0, cinlcl = 0;
    R plcl = 0,""")
rep("""    R cin_i = 0, cinlcl_i = 0, ke = 0, kinv_o_d = 0;""", """    double cin_i = 0, cinlcl_i = 0, ke = 0;
    R kinv_o_d = 0;""")
rep("""    R cbmf = 0, wlcl = 0, ufrclcl = 0, ppen = 0, precip = 0, snow = 0, rliq = 0, cush, cnt, cnb;""",
    """    R cbmf = 0, wlcl = 0, ufrclcl = 0, ppen = 0, precip = 0, snow = 0, cush, cnt, cnb;
    Kahan rliq;""")
rep("""           wtwb = 0, wtw = 0, xs1 = 0, xs2 = 0, xc1 = 0, xc2 = 0;""", """           wtwb = 0, wtw = 0;
    double xs1 = 0, xs2 = 0, xc1 = 0, xc2 = 0;""")
rep("""    R rainflx = 0, snowflx = 0;""", """    Kahan rainflx, snowflx;""")
rep("""            R del_CIN = cin - cin_i;""", """            double del_CIN = cin - cin_i;""")
rep("""                R alpha = compute_alpha(del_CIN, ke);""", """                double alpha = compute_alpha(del_CIN, ke);""")
rep("""            R dpsum = 0.0f;
            tkeavg = 0.0f;""", """            Kahan dpsum, tksum;""")
rep("""                dpsum = dpsum + dpi;
                tkeavg = tkeavg + dpi * GI(tke, k);""", """                dpsum.add(dpi);
                tksum.add(dpi * GI(tke, k));""")
rep("""            tkeavg = tkeavg / dpsum;""", """            tkeavg = tksum.s / dpsum.s;""")
rep("""                precip = 0.0f; snow = 0.0f; rliq = 0.0f; cbmf = 0.0f;""", """                precip = 0.0f; snow = 0.0f; rliq.reset(); cbmf = 0.0f;""")
rep("""        rliq = 0.0f;
        rainflx = 0.0f;
        snowflx = 0.0f;""", """        rliq.reset();
        rainflx.reset();
        snowflx.reset();""")
rep("""                rainflx = rainflx + qrten[k] * dp0[k] / g;
                snowflx = snowflx + qsten[k] * dp0[k] / g;""", """                rainflx.add(qrten[k] * dp0[k] / g);
                snowflx.add(qsten[k] * dp0[k] / g);""")
rep("""                rliq = rliq + qc[k] * dp0[k] / g / 1000.0f;""", """                rliq.add(qc[k] * dp0[k] / g / 1000.0f);""")
rep("""            R evpint_rain = 0.0f, evpint_snow = 0.0f;""", """            Kahan evpint_rain, evpint_snow;""")
rep("""                evplimit_rain = MN(evplimit_rain, (rainflx - evpint_rain) * g / dp0[k]);""", """                evplimit_rain = MN(evplimit_rain, (rainflx.s - evpint_rain.s) * g / dp0[k]);""")
rep("""                evplimit_snow = MN(evplimit_snow, (snowflx - evpint_snow) * g / dp0[k]);""", """                evplimit_snow = MN(evplimit_snow, (snowflx.s - evpint_snow.s) * g / dp0[k]);""")
rep("""                evpint_rain = evpint_rain + evprain * dp0[k] / g;
                evpint_snow = evpint_snow + evpsnow * dp0[k] / g;""", """                evpint_rain.add(evprain * dp0[k] / g);
                evpint_snow.add(evpsnow * dp0[k] / g);""")
rep("""            A.rliq[i] = rliq;""", """            A.rliq[i] = rliq.s;""")
rep("""    A.rliq[i] = rliq;""", """    A.rliq[i] = rliq.s;""")
# occupancy of the worklist launches: FP32 profiles need fewer registers (the same results at any)
i0 = b.index("// Register caps (resident blocks of 128 per SM)")
i1 = b.index("\n", b.index("#define UW_LIST_MINB(m)", i0))
b = b[:i0] + """// Register caps (resident blocks of 128 per SM): the worklist launches at 72 registers (7 blocks;
// 1,048,576 x 30 columns: 103.9 ms against 115.6 ms at the FP64 kernel's 4 and 5 blocks, 109.8 ms
// at 6, 104.5 ms at 8), the trigger pass at 72 too (7 blocks: 103.1-103.4 ms against 104.8 ms at 5),
// the single pass at 168.
#define UW_LIST_MINB(m) ((m) == UW_MODE_RESUME ? 7 : (UW_MODE_IS_LIST(m) ? 7 : ((m) == UW_MODE_TRIGGER ? 7 : 3)))""" + b[i1:]
start = b.index("        // positive_moisture_single (uwshcu.F90:5096-5162 via :3995-4001); state after the tendencies")
end = b.index("        for (int k = 1; k <= mkx; k++) {\n            qtten[k] = qvten[k] + qlten[k] + qiten[k];", start)
pm = open(D + 'mixed_positive_moisture.inc').read()
b = b[:start] + pm + b[end:]
b = b.replace("""#define UW_MODE_ALL 0
#define UW_MODE_TRIGGER 1
#define UW_MODE_LIST 2
""", "")
open(D + 'uwshcu_mixed_kernel.cuh', 'w').write(head + b)
print("ok")
