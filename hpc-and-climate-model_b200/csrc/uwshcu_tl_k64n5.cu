// uwshcu_tl_k64n5.cu -- the tangent-linear kernel for mkx + 1 <= 64 levels and ncnst <= 5 tracers,
// with this unit's constant bank and launch hook.  Built without FMA contraction (values = FP64 path).
#include "uwshcu_tl_kernel.cuh"

extern "C" cudaError_t uw_tl_set_constants_k64n5(const UwConst* h, const double* tbl)
{
    cudaError_t e = cudaMemcpyToSymbol(c, h, sizeof(UwConst));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_estbl, tbl, sizeof(double) * UW_TBL);
}

// mode: UW_MODE_ALL, UW_MODE_TRIGGER or UW_MODE_LIST (worklist wl / *wl_count), as the FP64 kernel.
extern "C" cudaError_t uw_tl_launch_k64n5(const UwArgs* a, const uwshcu_tangent* t, int mode, int* wl,
                                            int* wl_count, int nthreads, int block, cudaStream_t stream)
{
    if (nthreads <= 0) return cudaSuccess;
    dim3 grid((unsigned)((nthreads + block - 1) / block));
    if (mode == UW_MODE_ALL) uwshcu_tl_kernel<64, 5, UW_MODE_ALL><<<grid, block, 0, stream>>>(*a, wl, wl_count, *t);
    else if (mode == UW_MODE_TRIGGER) uwshcu_tl_kernel<64, 5, UW_MODE_TRIGGER><<<grid, block, 0, stream>>>(*a, wl, wl_count, *t);
    else uwshcu_tl_kernel<64, 5, UW_MODE_LIST><<<grid, block, 0, stream>>>(*a, wl, wl_count, *t);
    return cudaGetLastError();
}
