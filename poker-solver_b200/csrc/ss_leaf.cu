// ss_leaf.cu -- continuation-value producer on the GPU (ss_leaf_values_gpu).
//
// The reference computes a depth-limited subgame's leaf values in Python
// before every turn or flop solve (python/leaf_values.py:408-571, 694-816):
// O(runouts x players x hands x tuples) interpreted comparisons, the bulk of
// its flop wall time.  Here the host plan (ss_leaf_plan.cpp) fixes the
// runouts, live hands and opponent tuples; five grid-stride kernels over the
// per-element functions of ss_leaf.cuh do the rest:
//   k_leaf_strength  ranks every live hand on every runout (device ranker)
//   k_leaf_digest    reduces each opponent tuple to (card mask, best, count)
//   k_leaf_ratio     one thread per (runout, player, hand) walks its tuples
//                    in order; a warp shares (runout, player), so the 16-byte
//                    digests it reads are broadcasts from L1
//   k_leaf_equity    averages the ratios over the runouts in order
//   k_leaf_value     writes the bias-adjusted rows, in chunks of at most
//                    256 MiB that are copied to the caller's buffer in turn
// Every kernel is bound by latency or by the ratio walk's issue rate, not by
// HBM: the only large array is the output (4 bytes per value, written once).
#include "ss_engine.h"
#include "ss_leaf.cuh"
#include "ss_leaf.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

namespace ssb {
namespace leaf {

namespace {

constexpr int kThreads = 256;
constexpr size_t kValueChunkBytes = size_t(256) << 20;

#define SSB_LEAF_STRIDE_LOOP(i, n) \
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < (n); i += static_cast<long>(gridDim.x) * blockDim.x)

__global__ void __launch_bounds__(kThreads) k_leaf_strength(Ctx c, long n) {
    SSB_LEAF_STRIDE_LOOP(i, n) strength_at(i, c);
}
__global__ void __launch_bounds__(kThreads) k_leaf_digest(Ctx c, long n) {
    SSB_LEAF_STRIDE_LOOP(i, n) digest_at(i, c);
}
__global__ void __launch_bounds__(kThreads) k_leaf_ratio(Ctx c, long n) {
    SSB_LEAF_STRIDE_LOOP(i, n) ratio_at(i, c);
}
__global__ void __launch_bounds__(kThreads) k_leaf_equity(Ctx c, long n) {
    SSB_LEAF_STRIDE_LOOP(i, n) equity_at(i, c);
}
__global__ void __launch_bounds__(kThreads) k_leaf_value(Ctx c, long row0, long n) {
    SSB_LEAF_STRIDE_LOOP(i, n) value_at(i, row0, c);
}

#undef SSB_LEAF_STRIDE_LOOP

// blocks for n elements: one per kThreads elements, at most 8 per SM (the
// loops stride over the rest)
unsigned blocks_for(long n, int sms) {
    const long b = (n + kThreads - 1) / kThreads;
    return static_cast<unsigned>(std::max(1L, std::min(b, 8L * sms)));
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

int leaf_values_gpu(const SSLeafValueInput *in, float *out) {
    Plan P;
    std::string err;
    int rc = make_plan(in, &P, &err);
    if (rc != SS_OK) {
        set_error(err);
        return rc;
    }
    const size_t nvals = P.num_values();
    if (nvals == 0) return SS_OK;
    if (!out) {
        set_error("ss_leaf_values_gpu: null output");
        return SS_ERR_INVALID;
    }
    int ndev = 0, dev = 0, sms = 148;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device");
        return SS_ERR_NO_DEVICE;
    }
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

    const size_t per_row = static_cast<size_t>(P.np) * P.mh;
    const size_t rows = P.num_rows();
    const size_t rows_chunk = std::max<size_t>(1, std::min(rows, kValueChunkBytes / (per_row * sizeof(float))));
    const size_t nsh = static_cast<size_t>(P.nr) * per_row;   // (runout, player, hand) elements
    const size_t T = P.num_tuples();

    // one device block: inputs, intermediates and one chunk of output rows
    struct Part {
        size_t off, bytes;
        const void *src;   // host data to upload, or nullptr
    };
    size_t top = 0;
    auto part = [&top](size_t bytes, const void *src) {
        Part p{top, bytes, src};
        top += align256(bytes);
        return p;
    };
    const Part p_nh = part(P.nh.size() * sizeof(int), P.nh.data());
    const Part p_cards = part(P.hand_cards.size() * sizeof(int), P.hand_cards.data());
    const Part p_board = part(P.board5.size() * sizeof(int), P.board5.data());
    const Part p_off = part(P.tuple_off.size() * sizeof(int), P.tuple_off.data());
    const Part p_owner = part(P.tuple_owner.size() * sizeof(int), P.tuple_owner.data());
    const Part p_thand = part(P.tuple_hand.size() * sizeof(uint16_t), P.tuple_hand.data());
    const Part p_pot = part(P.row_pot.size() * sizeof(double), P.row_pot.data());
    const Part p_set = part(P.row_set.size(), P.row_set.data());
    const Part p_str = part(nsh * sizeof(unsigned), nullptr);
    const Part p_dig = part(T * sizeof(Digest), nullptr);
    const Part p_ratio = part(nsh * sizeof(double), nullptr);
    const Part p_eq = part(per_row * sizeof(double), nullptr);
    const Part p_val = part(rows_chunk * per_row * sizeof(float), nullptr);

    unsigned char *base = nullptr;
    cudaStream_t stream = nullptr;
    cudaError_t e = cudaMalloc(&base, top);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        set_error("ss_leaf_values_gpu: device allocation of " + std::to_string(top) + " bytes failed");
        return SS_ERR_NOMEM;
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        for (const Part *p : {&p_nh, &p_cards, &p_board, &p_off, &p_owner, &p_thand, &p_pot, &p_set})
            if (e == cudaSuccess && p->bytes > 0)
                e = cudaMemcpyAsync(base + p->off, p->src, p->bytes, cudaMemcpyHostToDevice, stream);
    }
    if (e == cudaSuccess) {
        Ctx c;
        c.np = P.np;
        c.mh = P.mh;
        c.nr = P.nr;
        c.per = P.per;
        c.num_leaves = P.num_leaves;
        c.nh = reinterpret_cast<const int *>(base + p_nh.off);
        c.hand_cards = reinterpret_cast<const int *>(base + p_cards.off);
        c.board5 = reinterpret_cast<const int *>(base + p_board.off);
        c.tuple_off = reinterpret_cast<const int *>(base + p_off.off);
        c.tuple_owner = reinterpret_cast<const int *>(base + p_owner.off);
        c.tuple_hand = reinterpret_cast<const uint16_t *>(base + p_thand.off);
        c.row_pot = reinterpret_cast<const double *>(base + p_pot.off);
        c.row_set = reinterpret_cast<const unsigned char *>(base + p_set.off);
        c.strength = reinterpret_cast<unsigned *>(base + p_str.off);
        c.digest = reinterpret_cast<Digest *>(base + p_dig.off);
        c.ratio = reinterpret_cast<double *>(base + p_ratio.off);
        c.equity = reinterpret_cast<double *>(base + p_eq.off);
        c.values = reinterpret_cast<float *>(base + p_val.off);

        const long n_sh = static_cast<long>(nsh), n_t = static_cast<long>(T), n_eq = static_cast<long>(per_row);
        if (n_sh > 0) k_leaf_strength<<<blocks_for(n_sh, sms), kThreads, 0, stream>>>(c, n_sh);
        if (n_t > 0) k_leaf_digest<<<blocks_for(n_t, sms), kThreads, 0, stream>>>(c, n_t);
        if (n_sh > 0) k_leaf_ratio<<<blocks_for(n_sh, sms), kThreads, 0, stream>>>(c, n_sh);
        k_leaf_equity<<<blocks_for(n_eq, sms), kThreads, 0, stream>>>(c, n_eq);
        e = cudaGetLastError();
        for (size_t row0 = 0; e == cudaSuccess && row0 < rows; row0 += rows_chunk) {
            const size_t nrows = std::min(rows_chunk, rows - row0);
            const long n = static_cast<long>(nrows * per_row);
            k_leaf_value<<<blocks_for(n, sms), kThreads, 0, stream>>>(c, static_cast<long>(row0), n);
            e = cudaGetLastError();
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(out + row0 * per_row, c.values, nrows * per_row * sizeof(float),
                                    cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        }
    }
    if (stream) {
        const cudaError_t s = cudaStreamSynchronize(stream);
        if (e == cudaSuccess) e = s;
        cudaStreamDestroy(stream);
    }
    if (base) cudaFree(base);
    if (e != cudaSuccess) {
        set_error(std::string("ss_leaf_values_gpu: CUDA: ") + cudaGetErrorString(e));
        return SS_ERR_CUDA;
    }
    return SS_OK;
}

}  // namespace leaf
}  // namespace ssb
