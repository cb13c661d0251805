// uwshcu_fp64_k64n32.cu -- instantiations of the FP64 column kernel for mkx + 1 <= 64 levels and
// ncnst <= 32 tracers, with this unit's constant bank and launch hook.
#include "uwshcu_fp64_kernel.cuh"

extern "C" cudaError_t uw_fp64_set_constants_k64n32(const UwConst* h, const double* tbl)
{
    cudaError_t e = cudaMemcpyToSymbol(c, h, sizeof(UwConst));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_estbl, tbl, sizeof(double) * UW_TBL);
}

// a->omega: compute_zwshcu's instantiations.  mode: UW_MODE_ALL, UW_MODE_TRIGGER, UW_MODE_LIST, UW_MODE_LIST1 or UW_MODE_RESUME; nthreads: columns (ALL/TRIGGER) or the
// worklist capacity (LIST).
extern "C" cudaError_t uw_fp64_launch_k64n32(const UwArgs* a, int mode, int* wl, int* wl_count,
                                                     int nthreads, int block, cudaStream_t stream)
{
    if (nthreads <= 0) return cudaSuccess;
    dim3 grid((unsigned)((nthreads + block - 1) / block));
    if (a->omega) {   // compute_zwshcu
        if (mode == UW_MODE_ALL) uwshcu_fp64_kernel<64, 32, UW_MODE_ALL, 1><<<grid, block, 0, stream>>>(*a, wl, wl_count);
        else if (mode == UW_MODE_TRIGGER) uwshcu_fp64_kernel<64, 32, UW_MODE_TRIGGER, 1><<<grid, block, 0, stream>>>(*a, wl, wl_count);
        else if (mode == UW_MODE_LIST1) uwshcu_fp64_kernel<64, 32, UW_MODE_LIST1, 1><<<grid, block, 0, stream>>>(*a, wl, wl_count);
        else if (mode == UW_MODE_RESUME) uwshcu_fp64_kernel<64, 32, UW_MODE_RESUME, 1><<<grid, block, 0, stream>>>(*a, wl, wl_count);
        else uwshcu_fp64_kernel<64, 32, UW_MODE_LIST, 1><<<grid, block, 0, stream>>>(*a, wl, wl_count);
    } else {
        if (mode == UW_MODE_ALL) uwshcu_fp64_kernel<64, 32, UW_MODE_ALL><<<grid, block, 0, stream>>>(*a, wl, wl_count);
        else if (mode == UW_MODE_TRIGGER) uwshcu_fp64_kernel<64, 32, UW_MODE_TRIGGER><<<grid, block, 0, stream>>>(*a, wl, wl_count);
        else if (mode == UW_MODE_LIST1) uwshcu_fp64_kernel<64, 32, UW_MODE_LIST1><<<grid, block, 0, stream>>>(*a, wl, wl_count);
        else if (mode == UW_MODE_RESUME) uwshcu_fp64_kernel<64, 32, UW_MODE_RESUME><<<grid, block, 0, stream>>>(*a, wl, wl_count);
        else uwshcu_fp64_kernel<64, 32, UW_MODE_LIST><<<grid, block, 0, stream>>>(*a, wl, wl_count);
    }
    return cudaGetLastError();
}

// Batched trigger (phase 0), persistent worklist (phase 1), and for the sorted schedule the
// persistent first worklist (phase 2) and resume (phase 3) launches; minb selects the
// worklist instantiation (register cap = 65536 / (128 * minb)).  Returns cudaErrorInvalidValue
// for a minb that is not compiled here.
extern "C" cudaError_t uw_fp64_batch_k64n32(const UwBatch* b, int phase, int grid, int block, int minb,
                                          cudaStream_t stream)
{
    if (grid <= 0) return cudaSuccess;
    if (phase == 0) {
        uwshcu_batch_trigger<64, 32, 0><<<grid, block, 0, stream>>>(*b);
        return cudaGetLastError();
    }
    if (phase == 2) {   // sorted schedule: first worklist launch (register cap of minb 4)
        uwshcu_batch_list<64, 32, 4, 0, UW_MODE_LIST1><<<grid, block, 0, stream>>>(*b);
        return cudaGetLastError();
    }
    if (phase == 3) {   // sorted schedule: resume launch
        uwshcu_batch_resume<64, 32, 0><<<grid, block, 0, stream>>>(*b);
        return cudaGetLastError();
    }
    if (minb == 4) {
        uwshcu_batch_list<64, 32, 4, 0><<<grid, block, 0, stream>>>(*b);
        return cudaGetLastError();
    }
    return cudaErrorInvalidValue;
}

// Resident blocks per SM of the worklist instantiation minb at this block size (0 if absent).
extern "C" cudaError_t uw_fp64_batch_occupancy_k64n32(int minb, int block, int* blocks_per_sm)
{
    *blocks_per_sm = 0;
    if (minb == 4)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, uwshcu_batch_list<64, 32, 4, 0>, block, 0);
    return cudaSuccess;
}
