// uwshcu_probe.cu -- measured FP64 throughput of the device: the denominator of the FP64 roofline
// fractions that the benchmark reports for the column kernels (a copy loop and a library GEMM are
// the HBM and tensor-core denominators; the column kernels run on the FP64 pipe).
#include <cuda_runtime.h>
#include "uwshcu.h"

namespace {

constexpr int kChains = 8;     // independent FMA chains per thread: enough to cover the FMA latency
constexpr int kBlock = 256;
constexpr int kIters = 1024;

// Each thread runs kChains independent chains of kIters fused multiply-adds (2 flops each).  The
// result is written only if it equals a value it cannot take, so the loop is not removed and the
// kernel writes nothing.
__global__ void __launch_bounds__(kBlock) fp64_fma_loop(double* sink, double b, double c)
{
    double a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; j++) a[j] = 1.0 + 1e-9 * (threadIdx.x + j);
#pragma unroll 4
    for (int it = 0; it < kIters; it++) {
#pragma unroll
        for (int j = 0; j < kChains; j++) a[j] = fma(a[j], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kChains; j++) s += a[j];
    if (s == -1.0) *sink = s;
}

}  // namespace

extern "C" int uwshcu_fp64_peak(double* tflops, void* stream)
{
    if (!tflops) return UWSHCU_ERR_BAD_ARGS;
    *tflops = 0.0;
    int dev = 0, nsm = 0, per_sm = 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaGetDevice(&dev) != cudaSuccess) return UWSHCU_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fp64_fma_loop, kBlock, 0) != cudaSuccess)
        return UWSHCU_ERR_CUDA;
    double* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return UWSHCU_ERR_ALLOC;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = UWSHCU_OK;
    const unsigned grid = (unsigned)(nsm * per_sm * 2);   // two full waves
    float best = 0.f;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = UWSHCU_ERR_CUDA;
    } else {
        for (int rep = 0; rep < 4 && rc == UWSHCU_OK; rep++) {   // the first is a warm-up
            cudaEventRecord(e0, st);
            fp64_fma_loop<<<grid, kBlock, 0, st>>>(sink, 0.999999999, 1e-12);
            cudaEventRecord(e1, st);
            float ms = 0.f;
            if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
                rc = UWSHCU_ERR_CUDA;
            else if (rep > 0 && (best == 0.f || ms < best))
                best = ms;
        }
    }
    if (rc == UWSHCU_OK && best > 0.f)
        *tflops = 2.0 * kChains * (double)kIters * grid * kBlock / (best * 1e-3) / 1e12;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    return rc;
}
