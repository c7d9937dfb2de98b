/*
 * cuda_runtime.h -- host stand-in for the CUDA runtime, used only to compile
 * the reference solver (src/cuda/street_solve.cu) as plain C++ so that its own
 * kernel bodies run on the CPU as the reference oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Device memory is host memory; a kernel launch is
 * a loop over (block, thread) in order.  The reference kernels use no shared
 * memory, barriers or warp operations, so each (block, thread) call is
 * independent and the loop reproduces their results.
 */
#ifndef ORACLE_REF_SHIM_CUDA_RUNTIME_H
#define ORACLE_REF_SHIM_CUDA_RUNTIME_H

#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <stddef.h>

#define __global__
#define __device__
#define __host__

struct shim_dim3 { unsigned x, y, z; };
extern thread_local shim_dim3 threadIdx;
extern thread_local shim_dim3 blockIdx;

typedef int cudaError_t;
#define cudaSuccess 0
enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3
};

template <class T> static inline cudaError_t cudaMalloc(T **p, size_t n)
{
    *p = (T *)malloc(n ? n : 1);
    return *p ? 0 : 2;
}
static inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind)
{
    memmove(d, s, n);
    return 0;
}
static inline cudaError_t cudaMemset(void *d, int v, size_t n)
{
    memset(d, v, n);
    return 0;
}
static inline cudaError_t cudaFree(void *p)
{
    free(p);
    return 0;
}
static inline cudaError_t cudaDeviceSynchronize(void) { return 0; }
static inline const char *cudaGetErrorString(cudaError_t) { return "host shim error"; }

#define SHIM_LAUNCH(kernel, grid, block, ...)                                  \
    do {                                                                       \
        int shim_g_ = (int)(grid), shim_b_ = (int)(block);                     \
        for (int shim_bx_ = 0; shim_bx_ < shim_g_; shim_bx_++)                 \
            for (int shim_tx_ = 0; shim_tx_ < shim_b_; shim_tx_++) {           \
                blockIdx.x = (unsigned)shim_bx_;                               \
                threadIdx.x = (unsigned)shim_tx_;                              \
                kernel(__VA_ARGS__);                                           \
            }                                                                  \
    } while (0)

#endif
