/* Host shim of the few HIP runtime calls used by the reference drop-in
 * src/physics/bxcompute_uwshcu_inv.cpp, so that file compiles unchanged with g++ and its
 * kernel runs on the CPU, one simulated thread at a time (TEST INFRASTRUCTURE ONLY).
 * Device memory is host memory; copies are memcpy; a launch loops over blocks and threads. */
#ifndef UWREF_HIP_SHIM_H
#define UWREF_HIP_SHIM_H
#include <stdlib.h>
#include <string.h>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ static

typedef int hipError_t;
#define hipSuccess 0
enum hipMemcpyKind { hipMemcpyHostToHost = 0, hipMemcpyHostToDevice = 1, hipMemcpyDeviceToHost = 2,
                     hipMemcpyDeviceToDevice = 3, hipMemcpyDefault = 4 };
struct dim3 {
    unsigned x, y, z;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
extern dim3 threadIdx, blockIdx, blockDim, gridDim;

template <class T> static inline hipError_t hipMalloc(T **p, size_t n) { *p = (T *)calloc(n ? n : 1, 1); return 0; }
template <class T> static inline hipError_t hipHostMalloc(T **p, size_t n, unsigned f = 0) { (void)f; *p = (T *)calloc(n ? n : 1, 1); return 0; }
static inline hipError_t hipFree(void *p) { free(p); return 0; }
static inline hipError_t hipHostFree(void *p) { free(p); return 0; }
static inline hipError_t hipMemcpy(void *d, const void *s, size_t n, hipMemcpyKind k) { (void)k; memmove(d, s, n); return 0; }
template <class T> static inline hipError_t hipMemcpyToSymbol(T &sym, const void *s, size_t n, size_t off = 0,
                                                              hipMemcpyKind k = hipMemcpyHostToDevice)
{ (void)k; memcpy((char *)&sym + off, s, n); return 0; }
static inline hipError_t hipDeviceSynchronize(void) { return 0; }
static inline hipError_t hipGetLastError(void) { return 0; }
static inline const char *hipGetErrorString(hipError_t e) { (void)e; return "no error"; }

#define hipLaunchKernelGGL(F, G, B, SHM, STREAM, ...)                                     \
    do {                                                                                  \
        dim3 g_ = dim3(G), b_ = dim3(B);                                                  \
        gridDim = g_;                                                                     \
        blockDim = b_;                                                                    \
        for (unsigned bx_ = 0; bx_ < g_.x; bx_++)                                         \
            for (unsigned tx_ = 0; tx_ < b_.x; tx_++) {                                   \
                blockIdx = dim3(bx_);                                                     \
                threadIdx = dim3(tx_);                                                    \
                F(__VA_ARGS__);                                                           \
            }                                                                             \
    } while (0)
#endif
