// uwshcu_fast_k64n32.cu -- the fast-FP64 precision mode (conden_fast in place of conden) for
// mkx + 1 <= 64 levels and ncnst <= 32 tracers, with this unit's constant bank and launch hook.
#include "uwshcu_fp64_kernel.cuh"

extern "C" cudaError_t uw_fast_set_constants_k64n32(const UwConst* h, const double* tbl)
{
    cudaError_t e = cudaMemcpyToSymbol(c, h, sizeof(UwConst));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_estbl, tbl, sizeof(double) * UW_TBL);
}

extern "C" cudaError_t uw_fast_launch_k64n32(const UwArgs* a, int mode, int* wl, int* wl_count, int nthreads,
                                              int block, cudaStream_t stream)
{
    if (nthreads <= 0) return cudaSuccess;
    dim3 grid((unsigned)((nthreads + block - 1) / block));
    if (mode == UW_MODE_ALL) uwshcu_fast_kernel<64, 32, UW_MODE_ALL><<<grid, block, 0, stream>>>(*a, wl, wl_count);
    else if (mode == UW_MODE_TRIGGER) uwshcu_fast_kernel<64, 32, UW_MODE_TRIGGER><<<grid, block, 0, stream>>>(*a, wl, wl_count);
    else uwshcu_fast_kernel<64, 32, UW_MODE_LIST><<<grid, block, 0, stream>>>(*a, wl, wl_count);
    return cudaGetLastError();
}
