// ss_rank_kernels.cu -- the 7-card ranker on the GPU, standalone.
//
// ss_rank7_batch ranks caller-supplied hands; ss_rank7_checksum enumerates
// every 7-card set on the device and reduces them to one order-independent
// checksum (sum over sets of mix64(card mask) * strength, mod 2^64) and the
// per-category counts, which pins the ranker bit for bit against the
// reference evaluator src/hand_eval.h over all 133,784,560 sets.
#include "ss_engine.h"
#include "ss_rank.cuh"

#include <cuda_runtime.h>

#include <string>

namespace ssb {

namespace {

__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void k_rank_batch(const int *__restrict__ cards, int n, unsigned *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c[7];
    for (int k = 0; k < 7; ++k) c[k] = cards[7 * i + k];
    out[i] = rank7(c);
}

// one block per (c0 < c1 < c2); threads split the (c3, c4) pairs above c2
__global__ void __launch_bounds__(256) k_rank_all(unsigned long long *sum, unsigned long long *hist) {
    const int c0 = blockIdx.z, c1 = blockIdx.y, c2 = blockIdx.x;
    if (!(c0 < c1 && c1 < c2 && c2 < 48)) return;
    __shared__ unsigned long long s_sum;
    __shared__ unsigned long long s_hist[10];
    if (threadIdx.x == 0) s_sum = 0ull;
    if (threadIdx.x < 10) s_hist[threadIdx.x] = 0ull;
    __syncthreads();
    unsigned long long local = 0ull;
    unsigned cnt[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int m = 51 - c2;  // cards above c2
    const int pairs = m * (m - 1) / 2;
    for (int p = threadIdx.x; p < pairs; p += blockDim.x) {
        // decode pair index p into (i < j) over the m cards above c2
        int i = 0, rem = p;
        while (rem >= m - 1 - i) {
            rem -= m - 1 - i;
            ++i;
        }
        const int c3 = c2 + 1 + i, c4 = c3 + 1 + rem;
        int c[7] = {c0, c1, c2, c3, c4, 0, 0};
        const unsigned long long base =
            (1ull << c0) | (1ull << c1) | (1ull << c2) | (1ull << c3) | (1ull << c4);
        for (int c5 = c4 + 1; c5 < 52; ++c5)
            for (int c6 = c5 + 1; c6 < 52; ++c6) {
                c[5] = c5;
                c[6] = c6;
                const unsigned s = rank7(c);
                local += mix64(base | (1ull << c5) | (1ull << c6)) * static_cast<unsigned long long>(s);
                cnt[s >> 20]++;
            }
    }
    atomicAdd(&s_sum, local);
    for (int k = 0; k < 10; ++k)
        if (cnt[k]) atomicAdd(&s_hist[k], static_cast<unsigned long long>(cnt[k]));
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(sum, s_sum);
    if (threadIdx.x < 10 && s_hist[threadIdx.x]) atomicAdd(&hist[threadIdx.x], s_hist[threadIdx.x]);
}

}  // namespace

int rank7_checksum(unsigned long long *checksum, unsigned long long *hist10) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device");
        return SS_ERR_NO_DEVICE;
    }
    unsigned long long *d = nullptr;
    cudaError_t e = cudaMalloc(&d, 11 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(d, 0, 11 * sizeof(unsigned long long));
    if (e == cudaSuccess) {
        k_rank_all<<<dim3(48, 48, 48), 256>>>(d, d + 1);
        e = cudaGetLastError();
    }
    unsigned long long h[11] = {};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) {
        set_error(std::string("CUDA: ") + cudaGetErrorString(e));
        return SS_ERR_CUDA;
    }
    *checksum = h[0];
    if (hist10)
        for (int k = 0; k < 10; ++k) hist10[k] = h[1 + k];
    return SS_OK;
}

int rank7_batch(const int *cards7, int n, unsigned *out) {
    if (n < 0 || (n > 0 && (!cards7 || !out))) {
        set_error("rank7_batch: bad arguments");
        return SS_ERR_INVALID;
    }
    for (long i = 0; i < 7L * n; ++i)
        if (cards7[i] < 0 || cards7[i] > 51) {
            set_error("rank7_batch: card out of range");
            return SS_ERR_INVALID;
        }
    if (n == 0) return SS_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device");
        return SS_ERR_NO_DEVICE;
    }
    int *dc = nullptr;
    unsigned *dout = nullptr;
    cudaError_t e = cudaMalloc(&dc, sizeof(int) * 7 * static_cast<size_t>(n));
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(unsigned) * static_cast<size_t>(n));
    if (e == cudaSuccess) e = cudaMemcpy(dc, cards7, sizeof(int) * 7 * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_rank_batch<<<(n + 255) / 256, 256>>>(dc, n, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(unsigned) * static_cast<size_t>(n), cudaMemcpyDeviceToHost);
    if (dc) cudaFree(dc);
    if (dout) cudaFree(dout);
    if (e != cudaSuccess) {
        set_error(std::string("CUDA: ") + cudaGetErrorString(e));
        return SS_ERR_CUDA;
    }
    return SS_OK;
}

}  // namespace ssb
