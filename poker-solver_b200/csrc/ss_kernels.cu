// ss_kernels.cu -- sm_100a kernels of the single-street Linear-CFR solver.
//
// Per-hand kernels (reach, cfv): one block per (work item, 256-hand chunk),
// each thread owns 4 consecutive hands and moves them with 128-bit loads and
// stores; rows are HS floats (HS a multiple of 32), so every warp touches
// 512 contiguous bytes per row.
//
// Per-terminal kernels: one block per terminal node.  The block stages the
// counted opponents' reach at that node in shared memory as 52x52 combo
// matrices (or as a strength-sorted vector for showdowns), reduces them to
// per-card aggregates, and then evaluates the exact card-removal formula for
// every traverser hand in O(1) (plus one small matrix product for two
// opponents).  The reference enumerates opponent tuples per traverser hand
// instead (street_solve.cu:704-1130), which is O(H^k).
#include "ss_kernels.h"

#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include "ss_cr3.cuh"

namespace ssb {

// Device fault word: a kernel that gives up a bounded wait on the tensor
// cores, or gets a block it was not built for, records it here instead of
// trapping; the host reads and clears it after a solve (read_device_fault).
__device__ unsigned g_ss_fault = 0;

namespace {

constexpr unsigned kFaultTcInput = 1u;   // k_term_cr2_tc: a subgame outside its path
constexpr unsigned kFaultTcWait = 2u;    // k_term_cr2_tc: the MMA completion wait ran out

constexpr int MS = 52;  // shared-memory row stride of a 52x52 combo matrix (16-byte rows)

// Programmatic dependent launch: the kernels of an iteration are launched
// with it (pdl_launch), so a kernel's blocks are scheduled while the kernel
// before it in the stream drains.  Every kernel starts here:
// griddepcontrol.wait returns once the preceding kernel has completed and its
// writes are visible (at once when there is no programmatic predecessor).
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... P, typename... A>
cudaError_t pdl_launch(void (*kernel)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                       A &&...args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}
// pdl_launch(kernel, grid, block, shared bytes, stream, kernel arguments...),
// returning its error from the enclosing function
#define SSB_LAUNCH(...)                                      \
    do {                                                     \
        const cudaError_t le_ = pdl_launch(__VA_ARGS__);     \
        if (le_ != cudaSuccess) return le_;                  \
    } while (0)

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float get(const float4 &v, int i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Regret matching for 4 hands at one node (street_solve.cu:596-613): positive
// regrets normalised by their sum (multiplied by the float reciprocal), uniform
// when no regret is positive; an A3-frozen node plays its frozen action for
// every hand (street_solve.cu:641-643).  The reference's pruning branch only
// maps regrets below -1e4 to 0, which the positive part already does.
// r receives the raw regrets.
__device__ __forceinline__ void regret_match4(const float *__restrict__ R, size_t HS, int fe,
                                              int na, int frozen, int h0,
                                              float r[SS_MAX_ACTIONS][4],
                                              float sig[SS_MAX_ACTIONS][4]) {
    float sum[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < na) {
            const float4 v = ld4(R + static_cast<size_t>(fe + a) * HS + h0);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                r[a][i] = get(v, i);
                sum[i] += r[a][i] > 0.f ? r[a][i] : 0.f;
            }
        }
    }
    const float uni = 1.0f / static_cast<float>(na);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const bool pos = sum[i] > 0.f;
        const float inv = pos ? 1.0f / sum[i] : 0.f;
#pragma unroll
        for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
            if (a < na) {
                float s = pos ? (r[a][i] > 0.f ? r[a][i] : 0.f) * inv : uni;
                if (frozen >= 0) s = (a == frozen) ? 1.0f : 0.0f;
                sig[a][i] = s;
            }
        }
    }
}

// --------------------------------------------------------------------------
// reach: reach[first_edge + a] = reach[parent_row] * sigma_a
// (street_solve.cu:650-683, stored per sequence instead of per node)
// --------------------------------------------------------------------------
// Batched form: a subgame that has left the batch keeps its items in the
// captured launches; their blocks return at once.  Every block serves one
// subgame, so the test is block-uniform (ahead of any barrier).
__device__ __forceinline__ bool retired(const DevCtx *ctxs, int sg) { return ctxs && !ctxs[sg].live; }

__global__ void __launch_bounds__(kHandThreads) k_reach(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                        const ReachItem *__restrict__ items, int nchunk, int H,
                                                        int p) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kHandThreads + threadIdx.x) * 4;
    const ReachItem I = items[it];
    if (retired(ctxs, I.sg)) return;
    // context fields in registers (a reference to either the parameter or a
    // batch entry would send every field read through local memory)
    float *R, *reach;
    int HSi, Hp;
    if (ctxs) {
        const DevCtx &c = ctxs[I.sg];
        R = c.R, reach = c.reach, HSi = c.HS, Hp = c.H[p];
    } else {
        R = c0.R, reach = c0.reach, HSi = c0.HS, Hp = H;
    }
    if (h0 >= Hp) return;
    const size_t HS = static_cast<size_t>(HSi);
    float r[SS_MAX_ACTIONS][4], sig[SS_MAX_ACTIONS][4];
    regret_match4(R, HS, I.first_edge, I.na, I.frozen, h0, r, sig);
    const float4 pr = ld4(reach + static_cast<size_t>(I.parent_row) * HS + h0);
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            float4 o;
            o.x = pr.x * sig[a][0];
            o.y = pr.y * sig[a][1];
            o.z = pr.z * sig[a][2];
            o.w = pr.w * sig[a][3];
            st4(reach + static_cast<size_t>(I.first_edge + a) * HS + h0, o);
        }
    }
}

// --------------------------------------------------------------------------
// cfv: value, regret and strategy-sum update at traverser nodes
// (street_solve.cu:1155-1175): v = sum_a sigma_a ev_a; r_a = (r_a + (ev_a - v))
// * t/(t+1); s_a += t * sigma_a; ev_a = sum of val over frontier(edge a).
// Each lane owns 2 hands, each warp 64 consecutive hands.  S == 1: the four
// warps of a block take four hand chunks and walk whole frontiers, eight row
// loads in flight.  S > 1 (items with long frontiers, which are few): the S
// warps of a block share one hand chunk and each sums every S-th frontier
// row; warp 0 adds the S partial sums in a fixed order and updates.
// --------------------------------------------------------------------------
__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
// a float2 load kept as a separate L1-cached access (not merged with an
// earlier load of the same address, so the value need not stay in registers)
__device__ __forceinline__ float2 ld2_l1(const float *p) {
    float2 v;
    asm volatile("ld.global.ca.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ void add2(float2 &a, float2 b) {
    a.x += b.x;
    a.y += b.y;
}

// context fields of the value/regret kernel, copied into registers (see Cr2View)
struct CfvView {
    float *R, *S, *val;
    const int *fr_off, *fr_items, *iter;
    int HS, H;
};
__device__ __forceinline__ CfvView cfv_view(const DevCtx &c, int H) {
    return CfvView{c.R, c.S, c.val, c.fr_off, c.fr_items, c.iter, c.HS, H};
}


// the first 32 bytes of a CfvItem (the inline frontier rows follow), read
// with two 16-byte loads
struct CfvHead {
    int first_edge, na, frozen, node, sg;
    float scale;
    int nfr, fr_bnd;
};
static_assert(sizeof(CfvItem) == 64 && offsetof(CfvItem, nfr) == 24 && offsetof(CfvItem, fr) == 32,
              "CfvItem layout read by cfv_head");
__device__ __forceinline__ CfvHead cfv_head(const CfvItem *p) {
    const int4 a = __ldg(reinterpret_cast<const int4 *>(p)), b = __ldg(reinterpret_cast<const int4 *>(p) + 1);
    return CfvHead{a.x, a.y, a.z, a.w, b.x, __int_as_float(b.y), b.z, b.w};
}

template <int S>
__global__ void __launch_bounds__(kCfvThreads, 8) k_cfv(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                     const CfvItem *__restrict__ items, int nchunk, int Hl,
                                                     int trav) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const CfvHead I = cfv_head(items + it);
    if (retired(ctxs, I.sg)) return;
    const CfvView V = ctxs ? cfv_view(ctxs[I.sg], ctxs[I.sg].H[trav]) : cfv_view(c0, Hl);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int h0 = (S == 1 ? ch * (kCfvThreads / 32) + warp : ch) * 64 + lane * 2;
    const bool act = h0 < V.H;
    if (S == 1 && !act) return;
    const size_t HS = static_cast<size_t>(V.HS);
    const float *val = V.val + h0;
    const int *__restrict__ fr = V.fr_items;
    // the regret and strategy-sum rows are needed after the frontier sums:
    // start bringing them into L1 now (no registers held)
    if (act && (S == 1 || warp == 0)) {
#pragma unroll
        for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
            if (a < I.na) {
                const size_t off = static_cast<size_t>(I.first_edge + a) * HS + h0;
                asm volatile("prefetch.global.L1 [%0];" ::"l"(V.R + off));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(V.S + off));
            }
        }
    }
    float2 ev[SS_MAX_ACTIONS];
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) ev[a] = make_float2(0.f, 0.f);
    if constexpr (S == 1) {
        if (I.nfr > 0) {
            // a short frontier held in the item: its rows load at once, with
            // no index loads before them; each row adds to its edge in row order
            const unsigned bnd = static_cast<unsigned>(I.fr_bnd);
            static_assert(kCfvInline == 8, "two 16-byte loads of inline rows");
            const int4 *fp = reinterpret_cast<const int4 *>(items + it) + 2;
            const int4 f0 = __ldg(fp), f1 = __ldg(fp + 1);
            const int rows[kCfvInline] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w};
            float2 x[kCfvInline];
#pragma unroll
            for (int i = 0; i < kCfvInline; ++i)
                x[i] = i < I.nfr ? ld2(val + static_cast<size_t>(rows[i]) * HS) : make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < kCfvInline; ++i) {
                if (i < I.nfr) {
                    int e = 0;   // the edge of row i: the edges whose last row (nibble) is before it
#pragma unroll
                    for (int a = 0; a < SS_MAX_ACTIONS - 1; ++a)
                        e += i > static_cast<int>((bnd >> (4 * a)) & 15u) ? 1 : 0;
#pragma unroll
                    for (int a = 0; a < SS_MAX_ACTIONS; ++a)
                        if (e == a) add2(ev[a], x[i]);
                }
            }
        } else {
            // the frontiers of all edges are one contiguous run of rows: walk
            // it eight rows at a time across edge boundaries (short frontiers,
            // one row per edge at the lowest level, would otherwise leave one
            // load in flight); each row adds to its edge in row order
            const int fe = I.first_edge;
            int bnd[SS_MAX_ACTIONS];
#pragma unroll
            for (int a = 0; a < SS_MAX_ACTIONS; ++a) bnd[a] = a < I.na ? V.fr_off[fe + a + 1] : 0x7fffffff;
            const int k0 = V.fr_off[fe], kend = V.fr_off[fe + I.na];
            for (int k = k0; k < kend; k += 8) {
                float2 x[8];
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    x[i] = k + i < kend ? ld2(val + static_cast<size_t>(__ldg(fr + k + i)) * HS)
                                        : make_float2(0.f, 0.f);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    if (k + i < kend) {
                        int e = 0;
#pragma unroll
                        for (int a = 0; a < SS_MAX_ACTIONS - 1; ++a) e += k + i >= bnd[a] ? 1 : 0;
#pragma unroll
                        for (int a = 0; a < SS_MAX_ACTIONS; ++a)
                            if (e == a) add2(ev[a], x[i]);
                    }
                }
            }
        }
    } else {
#pragma unroll
        for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
            if (a < I.na && act) {
                float2 e = make_float2(0.f, 0.f);
                int k = V.fr_off[I.first_edge + a] + warp;
                const int k1 = V.fr_off[I.first_edge + a + 1];
                for (; k + 7 * S < k1; k += 8 * S) {
                    float2 x[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) x[i] = ld2(val + static_cast<size_t>(__ldg(fr + k + i * S)) * HS);
#pragma unroll
                    for (int i = 0; i < 8; ++i) add2(e, x[i]);
                }
                if (k < k1) {
                    // the last (< 8) rows of this warp, loaded together; the
                    // missing ones add +0, so the sum is the row-order sum
                    float2 x[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        x[i] = k + i * S < k1 ? ld2(val + static_cast<size_t>(__ldg(fr + k + i * S)) * HS)
                                              : make_float2(0.f, 0.f);
#pragma unroll
                    for (int i = 0; i < 8; ++i) add2(e, x[i]);
                }
                ev[a] = e;
            }
        }
    }
    if constexpr (S > 1) {
        __shared__ float2 part[S][SS_MAX_ACTIONS][32];
#pragma unroll
        for (int a = 0; a < SS_MAX_ACTIONS; ++a)
            if (a < I.na) part[warp][a][lane] = ev[a];
        __syncthreads();
        if (warp != 0 || !act) return;
#pragma unroll
        for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
            if (a < I.na) {
                float2 e = part[0][a][lane];
#pragma unroll
                for (int w = 1; w < S; ++w) add2(e, part[w][a][lane]);
                ev[a] = e;
            }
        }
    }
    // the regrets are read three times (sum, value, update) instead of being
    // held in registers; the rereads hit L1
    const float *Rh = V.R + static_cast<size_t>(I.first_edge) * HS + h0;
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            const float2 r = ld2_l1(Rh + a * HS);
            s0 += r.x > 0.f ? r.x : 0.f;
            s1 += r.y > 0.f ? r.y : 0.f;
        }
    }
    const float uni = 1.0f / static_cast<float>(I.na);
    const float inv0 = s0 > 0.f ? 1.0f / s0 : 0.f, inv1 = s1 > 0.f ? 1.0f / s1 : 0.f;
    // strategy of action a (regret matching, A3 freeze)
    auto sigma = [&](int a, float ra, float sum, float inv) {
        if (I.frozen >= 0) return a == I.frozen ? 1.0f : 0.0f;
        return sum > 0.f ? (ra > 0.f ? ra : 0.f) * inv : uni;
    };
    float v0 = 0.f, v1 = 0.f;
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            const float2 r = ld2_l1(Rh + a * HS);
            v0 += sigma(a, r.x, s0, inv0) * ev[a].x;
            v1 += sigma(a, r.y, s1, inv1) * ev[a].y;
        }
    }
    const int t = *V.iter;
    const float d = static_cast<float>(t) / (static_cast<float>(t) + 1.0f);
    const float w = static_cast<float>(t);
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            const size_t off = static_cast<size_t>(I.first_edge + a) * HS + h0;
            const float2 r = ld2_l1(Rh + a * HS);
            const float2 sm = ld2(V.S + off);
            float2 nr, ns;
            nr.x = (r.x + (ev[a].x - v0)) * d;
            nr.y = (r.y + (ev[a].y - v1)) * d;
            ns.x = sm.x + w * sigma(a, r.x, s0, inv0);
            ns.y = sm.y + w * sigma(a, r.y, s1, inv1);
            st2(V.R + off, nr);
            st2(V.S + off, ns);
        }
    }
    // scale 1 on a single street (exact: the row equals v); below chance
    // nodes the row carries their 1 / cards weights for the parent's frontier
    st2(V.val + static_cast<size_t>(I.node) * HS + h0, make_float2(v0 * I.scale, v1 * I.scale));
}

// --------------------------------------------------------------------------
// terminals
// --------------------------------------------------------------------------

// per-hand factor: fold payoff, or the leaf value of this traverser hand
__device__ __forceinline__ float term_factor(const DevCtx &c, const TermItem &I, int h) {
    return I.leaf_off >= 0 ? c.leaf_values[I.leaf_off + h] : I.payoff;
}

// The terminal kernels serve the CFR iterations (T = float: reach and values
// in FP32, per-node aggregates in FP64) and the best response (T = double).
template <class T> __device__ __forceinline__ const T *reach_rows(const DevCtx &c);
template <> __device__ __forceinline__ const float *reach_rows<float>(const DevCtx &c) { return c.reach; }
template <> __device__ __forceinline__ const double *reach_rows<double>(const DevCtx &c) { return c.reach_d; }
template <class T> __device__ __forceinline__ T *val_rows(const DevCtx &c);
template <> __device__ __forceinline__ float *val_rows<float>(const DevCtx &c) { return c.val; }
template <> __device__ __forceinline__ double *val_rows<double>(const DevCtx &c) { return c.val_d; }

// value rows of terminals with no opponent coupling: zero, or the factor itself
// (a leaf without a live opponent, street_solve.cu:1062-1065)
template <class T>
__global__ void __launch_bounds__(kHandThreads) k_term_fill(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                            const TermItem *__restrict__ items, int nchunk,
                                                            int trav, int zero) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kHandThreads + threadIdx.x) * 4;
    const TermItem I = items[it];
    if (retired(ctxs, I.sg)) return;
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    if (h0 >= c.HS) return;
    const int Ht = c.H[trav];
    T *out = val_rows<T>(c) + static_cast<size_t>(I.node) * c.HS + h0;
#pragma unroll
    for (int i = 0; i < 4; ++i) out[i] = (zero || h0 + i >= Ht) ? T(0) : static_cast<T>(term_factor(c, I, h0 + i));
}

// Scatter one opponent's reach at a terminal into a 52x52 combo matrix
// (row stride MS): M[a][b] = M[b][a] = reach of the opponent's hand {a, b}.
// Board-blocked hands never count (street_solve.cu:755-757).  A range that
// holds some combo twice accumulates atomically; otherwise each cell has one
// writer and plain stores suffice.
template <class T>
__device__ __forceinline__ void scatter_combo(const DevCtx &c, int opp, int row, T *M) {
    const T *r = reach_rows<T>(c) + static_cast<size_t>(row) * c.HS;
    const int *code = c.hand_code + static_cast<size_t>(opp) * c.HS;
    const int Ho = c.H[opp];
    const bool dup = c.dup[opp] != 0;
    for (int j = threadIdx.x; j < Ho; j += blockDim.x) {
        const int hc = code[j];
        if (hc & 0x10000) continue;
        const int a = hc & 0xff, b = (hc >> 8) & 0xff;
        const T x = r[j];
        if (dup) {
            atomicAdd(&M[a * MS + b], x);
            atomicAdd(&M[b * MS + a], x);
        } else {
            M[a * MS + b] = x;
            M[b * MS + a] = x;
        }
    }
}

__device__ __forceinline__ int bit(unsigned long long m, int b) { return static_cast<int>((m >> b) & 1ull); }

template <class T>
__device__ __forceinline__ void zero_matrix(T *M) {
    float4 *m4 = reinterpret_cast<float4 *>(M);
    const int n = 52 * MS * static_cast<int>(sizeof(T)) / 16;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// four consecutive matrix entries (16-byte aligned)
__device__ __forceinline__ void load4(const double *p, double v[4]) {
    const double2 x = *reinterpret_cast<const double2 *>(p);
    const double2 y = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}
__device__ __forceinline__ void load4(const float *p, float v[4]) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void store4(double *p, const double v[4]) {
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void store4(float *p, const float v[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// Row pass over a combo matrix, one warp per card row r: the row sum u(r) in
// FP64 and the 64-bit mask of the row's positive cells.  The masks give the
// exact number of compatible positive-reach opponent tuples through the same
// inclusion-exclusion as the sums; where that number is 0 the value is
// exactly 0, as in the reference, which only adds positive products
// (street_solve.cu:810-812).  Without it rounding residue of the closed form
// would turn into a pure strategy under regret matching where the reference
// plays uniformly.
template <class T>
__device__ __forceinline__ void row_stats(const T *M, int r, int lane, double *sum_out,
                                          unsigned long long *mask_out, double *x0, double *x1) {
    const T a = M[r * MS + lane];
    const T b = lane + 32 < 52 ? M[r * MS + lane + 32] : T(0);
    const unsigned lo = __ballot_sync(0xffffffffu, a > T(0));
    const unsigned hi = __ballot_sync(0xffffffffu, b > T(0));
    *sum_out = warp_sum(static_cast<double>(a) + static_cast<double>(b));
    *mask_out = static_cast<unsigned long long>(lo) | (static_cast<unsigned long long>(hi) << 32);
    *x0 = a;
    *x1 = b;
}

template <class T>
__device__ __forceinline__ void store_value(T *out, int h, double v) { out[h] = static_cast<T>(v); }

// shared-memory carve-up of the terminal kernels (dynamic, 16-byte aligned)
struct Carve {
    char *p;
    template <class U>
    __device__ __forceinline__ U *take(int n) {
        U *r = reinterpret_cast<U *>(p);
        p += (static_cast<size_t>(n) * sizeof(U) + 15) & ~static_cast<size_t>(15);
        return r;
    }
};

template <class T>
constexpr size_t cr1_smem() {
    return 52 * MS * sizeof(T) + 52 * 8 + 52 * 8 + 64;
}

// One counted opponent: mass(h) = F - u(c1) - u(c2) + f(h), F the opponent's
// total reach, u(c) its reach on hands holding card c, f(h) its reach on the
// traverser's own combo.  Folds: payoff * mass (street_solve.cu:745-761);
// leaves: leaf value * mass (:1047-1066).  This form scatters the opponent's
// reach into a cleared 52x52 matrix (atomically), so it serves ranges that
// hold some combo more than once; k_term_cr1 below covers the others.
template <class T>
__global__ void __launch_bounds__(kTermThreads) k_term_cr1_dup(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                           const TermItem *__restrict__ items, int trav) {
    wait_prior_grid();
    extern __shared__ __align__(16) char smem[];
    Carve cv{smem};
    T *M = cv.take<T>(52 * MS);
    double *u = cv.take<double>(52);
    unsigned long long *B = cv.take<unsigned long long>(52);
    double *F = cv.take<double>(1);
    int *npos = cv.take<int>(1);
    const TermItem I = items[blockIdx.x];
    if (retired(ctxs, I.sg)) return;
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    zero_matrix(M);
    __syncthreads();
    scatter_combo(c, I.opp_player[0], I.opp_row[0], M);
    __syncthreads();
    for (int r = warp; r < 52; r += blockDim.x / 32) {
        double s, x0, x1;
        unsigned long long m;
        row_stats(M, r, lane, &s, &m, &x0, &x1);
        if (lane == 0) {
            u[r] = s;
            B[r] = m;
        }
    }
    __syncthreads();
    if (warp == 0) {
        double s = u[lane] + (lane + 32 < 52 ? u[lane + 32] : 0.0);
        int n = __popcll(B[lane]) + (lane + 32 < 52 ? __popcll(B[lane + 32]) : 0);
        s = warp_sum(s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
        if (lane == 0) {
            *F = 0.5 * s;
            *npos = n / 2;
        }
    }
    __syncthreads();
    const int Ht = c.H[trav];
    const int *tc = c.hand_code + static_cast<size_t>(trav) * c.HS;
    T *out = val_rows<T>(c) + static_cast<size_t>(I.node) * c.HS;
    const double Fv = *F;
    const int np_ = *npos;
    for (int h = tid; h < c.HS; h += blockDim.x) {
        double v = 0.0;
        if (h < Ht) {
            const int hc = tc[h];
            const int a = hc & 0xff, b = (hc >> 8) & 0xff;
            const unsigned long long Ba = B[a], Bb = B[b];
            const int live = np_ - __popcll(Ba) - __popcll(Bb) + bit(Ba, b);
            if (live > 0) {
                const double z = Fv - u[a] - u[b] + static_cast<double>(M[a * MS + b]);
                v = static_cast<double>(term_factor(c, I, h)) * z;
            }
        }
        store_value(out, h, v);
    }
}

// Per-card terms of the two-opponent closed form over the dense deck (the
// non-board cards, renumbered 0 .. deck-1): FP64 sums and integer counts of
// positive-reach cells.  Entry 52 stays zero and stands for a board card of
// the traverser.  The tensor-core form packs the sums per card (Cr2Card);
// k_term_cr2 keeps one array per field.
struct alignas(16) Cr2Card {
    double u1, u2;      // per-card reach sums of opponents 1 and 2
    double g;           // u1 u2 + w - 2 d, w = (M2 u1 + M1 u2)(c), d = sum_b M1[c][b] M2[c][b]
    double d;
};
struct alignas(16) Cr2Cnt {
    int n1, n2;         // positive-reach cells of the card's row in M1, M2
    int pad0, pad1;
};
// block scalars: F_i = sum u_i / 2, QD = D - Q with Q = sum u1 u2, D = sum d / 2,
// and the same on the 0/1 positive-reach matrices
struct Cr2Scalars {
    double F1, F2, QD;
    int IF1, IF2, IQD, pad;
};
constexpr int kCr2Off = 52;   // index of the zero per-card entry
constexpr int kMaxHS = 1344;  // largest row stride: 1326 combos rounded up to 32

// dynamic shared memory of the two-opponent kernel for row stride HS: M1, M2,
// P (whose space first stages the two opponents' reach rows), the first
// terminal's leaf row, per-card terms, staged group items
template <class T>
constexpr size_t cr2_smem(int HS) {
    return 3 * 52 * MS * sizeof(T) + (static_cast<size_t>(HS) + 4) * sizeof(T) + 3 * 56 * sizeof(double) + 53 * sizeof(Cr2Cnt) +
           53 * 16 + 5 * 48 * 4 + sizeof(Cr2Scalars) + 3 * kTermGroupMax * 4 + 8 * 16;
}

// asynchronous global -> shared copies (cp.async): 16-byte chunks and 4-byte words
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// One opponent's staged reach as a symmetric matrix over the dense deck:
// M[a][b] = M[b][a] = reach of the hand {a, b}; board-blocked hands never
// count (street_solve.cu:755-757).  This form serves ranges that hold some
// combo twice (accumulated atomically into a cleared matrix).
template <class T>
__device__ __forceinline__ void scatter_dense(const int *__restrict__ code, int Ho, const T *r, T *M) {
    for (int j = threadIdx.x; j < Ho; j += blockDim.x) {
        const int hc = __ldg(code + j);
        if (hc & 0x10000) continue;
        const int a = (hc >> 20) & 63, b = (hc >> 26) & 63;
        const T x = r[j];
        atomicAdd(&M[a * MS + b], x);
        atomicAdd(&M[b * MS + a], x);
    }
}

// The same matrices gathered instead (ranges without a repeated combo): each
// thread fills 4-column chunks of rows 0 .. Dp-1 through the player's table of
// range indices per dense-card pair (missing pairs index the zero kept after
// the staged row), so every cell is written once, with 16-byte stores and no
// clearing pass.  Cells outside rows and columns 0 .. Dp-1 are left unset;
// nothing reads them.
template <class T>
__device__ __forceinline__ void gather_dense(const int *__restrict__ tab, const T *r, T *M, int Dp) {
    const int chunk = threadIdx.x & 15, c0 = chunk * 4;
    if (c0 >= Dp) return;
    for (int row = threadIdx.x >> 4; row < Dp; row += kTermThreads / 16) {
        const int4 ix = __ldg(reinterpret_cast<const int4 *>(tab + row * 52 + c0));
        const T v[4] = {r[ix.x], r[ix.y], r[ix.z], r[ix.w]};
        store4(M + row * MS + c0, v);
    }
}

// The fields of a subgame context that the two-opponent kernel reads, copied
// into registers.  (A reference bound to either the kernel parameter or a
// batch entry would give the parameter a generic address, and every field
// read would then go through local memory.)
template <class T>
struct Cr2View {
    const T *reach;
    T *val;
    const int *code_t, *code0, *code1;   // hand codes of the traverser and the two opponents
    const int *tab0, *tab1;              // dense-pair tables of the two opponents
    const int *x0, *x1;                  // each traverser hand's index in the two opponents' ranges
    const float *leaf;
    int HS, deck, Ht, H0, H1;
    bool dup;
};
template <class T>
__device__ __forceinline__ Cr2View<T> cr2_view(const DevCtx &c, int trav, int o0, int o1) {
    Cr2View<T> v;
    v.reach = reach_rows<T>(c);
    v.val = val_rows<T>(c);
    v.code_t = c.hand_code + static_cast<size_t>(trav) * c.HS;
    v.code0 = c.hand_code + static_cast<size_t>(o0) * c.HS;
    v.code1 = c.hand_code + static_cast<size_t>(o1) * c.HS;
    v.tab0 = c.pair_idx + static_cast<size_t>(o0) * 52 * 52;
    v.tab1 = c.pair_idx + static_cast<size_t>(o1) * 52 * 52;
    v.x0 = c.cross_idx + (static_cast<size_t>(trav) * c.np + o0) * c.HS;
    v.x1 = c.cross_idx + (static_cast<size_t>(trav) * c.np + o1) * c.HS;
    v.leaf = c.leaf_values;
    v.HS = c.HS;
    v.deck = c.deck;
    v.Ht = c.H[trav];
    v.H0 = c.H[o0];
    v.H1 = c.H[o1];
    v.dup = (c.dup[o0] | c.dup[o1]) != 0;
    return v;
}

// TF32 split of the tensor-core product below: x = hi + lo, hi = x truncated
// to TF32 (10 explicit mantissa bits), lo = the exact FP32 remainder rounded
// to TF32 (half away from zero on the bit pattern).  hi*hi + hi*lo + lo*hi
// then carries about 21 significant bits, close to the FP32 product.
__device__ __forceinline__ void split_tf32(float x, unsigned &hi, unsigned &lo) {
    hi = __float_as_uint(x) & 0xffffe000u;                                        // truncated: x - hi is exact
    lo = (__float_as_uint(x - __uint_as_float(hi)) + 0x1000u) & 0xffffe000u;     // rounded remainder
}
// d += a b, one m16n8k8 TF32 tile (A row-major 16x8, B column-major 8x8)
__device__ __forceinline__ void mma_tf32(float d[4], const unsigned a[4], const unsigned b[2]) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// P = M1 M2 over a dense deck of at most 48 cards on the tensor cores: warp w
// (0..5) owns rows 16 (w / 2) .. +15 and columns 24 (w % 2) .. +23 (three
// 8-column tiles); six k-steps of 8.  Operand fragments are read from the
// FP32 matrices in shared memory (row stride 52 keeps the A-fragment loads
// free of bank conflicts) and split into TF32 pairs in registers.
// Also leaves rsum[h][r] = sum of row r over column half h and csum[s][c] =
// sum of column c over row strip s (FP32, deterministic order).
__device__ __forceinline__ void product_mma48(const float *M1, const float *M2, float *P, float *rsum, float *csum,
                                              int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int m0 = (warp >> 1) * 16, n0 = (warp & 1) * 24;
    float acc[3][4] = {};
#pragma unroll
    for (int k0 = 0; k0 < 48; k0 += 8) {
        unsigned ah[4], al[4];
        split_tf32(M1[(m0 + g) * MS + k0 + t], ah[0], al[0]);
        split_tf32(M1[(m0 + g + 8) * MS + k0 + t], ah[1], al[1]);
        split_tf32(M1[(m0 + g) * MS + k0 + t + 4], ah[2], al[2]);
        split_tf32(M1[(m0 + g + 8) * MS + k0 + t + 4], ah[3], al[3]);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int n = n0 + j * 8 + g;
            unsigned bh[2], bl[2];
            split_tf32(M2[(k0 + t) * MS + n], bh[0], bl[0]);
            split_tf32(M2[(k0 + t + 4) * MS + n], bh[1], bl[1]);
            mma_tf32(acc[j], al, bh);
            mma_tf32(acc[j], ah, bl);
            mma_tf32(acc[j], ah, bh);
        }
    }
    float ra = 0.f, rb = 0.f;   // this lane's share of rows m0 + g and m0 + g + 8
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const int n = n0 + j * 8 + 2 * t;
        *reinterpret_cast<float2 *>(&P[(m0 + g) * MS + n]) = make_float2(acc[j][0], acc[j][1]);
        *reinterpret_cast<float2 *>(&P[(m0 + g + 8) * MS + n]) = make_float2(acc[j][2], acc[j][3]);
        ra += acc[j][0] + acc[j][1];
        rb += acc[j][2] + acc[j][3];
    }
    // row sums over this warp's 24 columns and column sums over its 16 rows
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
        ra += __shfl_xor_sync(0xffffffffu, ra, o);
        rb += __shfl_xor_sync(0xffffffffu, rb, o);
    }
    if (t == 0) {
        rsum[(warp & 1) * 48 + m0 + g] = ra;
        rsum[(warp & 1) * 48 + m0 + g + 8] = rb;
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        float c0 = acc[j][0] + acc[j][2], c1 = acc[j][1] + acc[j][3];
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) {
            c0 += __shfl_xor_sync(0xffffffffu, c0, o);
            c1 += __shfl_xor_sync(0xffffffffu, c1, o);
        }
        if (g == 0) {
            csum[(warp >> 1) * 48 + n0 + j * 8 + 2 * t] = c0;
            csum[(warp >> 1) * 48 + n0 + j * 8 + 2 * t + 1] = c1;
        }
    }
}

// column sums and positive-cell masks of M1 (s < Dp) or M2 (s >= Dp): four
// independent partial sums in T (Dp is a multiple of 4; FP32 keeps the
// relative error near 1e-7), added in FP64 in a fixed order
template <class T>
__device__ __forceinline__ void column_stats(const T *M1, const T *M2, int s, int Dp, double *cu1, double *cu2,
                                             ulonglong2 *Bm) {
    const bool second = s >= Dp;
    const int col = second ? s - Dp : s;
    const T *M = (second ? M2 : M1) + col;
    T u[4] = {T(0), T(0), T(0), T(0)};
    unsigned long long B = 0ull;
    for (int r = 0; r < Dp; r += 4) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const T x = M[(r + i) * MS];
            u[i] += x;
            B |= static_cast<unsigned long long>(x > T(0)) << (r + i);
        }
    }
    const double tot = (static_cast<double>(u[0]) + static_cast<double>(u[1])) +
                       (static_cast<double>(u[2]) + static_cast<double>(u[3]));
    if (second) {
        cu2[col] = tot;
        Bm[col].y = B;
    } else {
        cu1[col] = tot;
        Bm[col].x = B;
    }
}

// 4x4 tile (rows i0.., columns j0..) of P = M1 M2; M1 is symmetric, so row k
// of M1 is its column k.
template <class T>
__device__ __forceinline__ void product_tile(const T *M1, const T *M2, T *P, int i0, int j0, int Dp) {
    T acc[4][4] = {};
#pragma unroll 4
    for (int k = 0; k < Dp; ++k) {
        T xs[4], ys[4];
        load4(&M1[k * MS + i0], xs);
        load4(&M2[k * MS + j0], ys);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] += xs[i] * ys[j];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) P[(i0 + i) * MS + j0 + j] = acc[i][j];
}

// Number of opponent pairs with positive reach that are disjoint from each
// other and from the traverser hand (a, b): the two-opponent formula on the
// 0/1 positive-reach matrices, whose entries are the bits of the card masks
// (row c of M_i = bits of Bm[c]).  The per-card term ng(c) = n1 n2 + nw - 2 nd
// with nw(c) = (I2 n1 + I1 n2)(c) is summed here over the set bits, since the
// count is only needed for the few hands whose mass is near zero.
__device__ __forceinline__ int card_ng(const ulonglong2 *Bm, const Cr2Cnt *cnt, int c) {
    const ulonglong2 Bc = Bm[c];
    int nw = 0;
    for (unsigned long long m = Bc.y; m; m &= m - 1) nw += cnt[__ffsll(static_cast<long long>(m)) - 1].n1;
    for (unsigned long long m = Bc.x; m; m &= m - 1) nw += cnt[__ffsll(static_cast<long long>(m)) - 1].n2;
    return cnt[c].n1 * cnt[c].n2 + nw - 2 * __popcll(Bc.x & Bc.y);
}
__device__ __noinline__ int pair_count(const ulonglong2 *Bm, const Cr2Cnt *cnt, int a, int b, int IF1, int IF2,
                                      int IQD) {
    const ulonglong2 Ba = Bm[a], Bb = Bm[b];
    const int n1a = cnt[a].n1, n1b = cnt[b].n1, n2a = cnt[a].n2, n2b = cnt[b].n2;
    const int j1 = bit(Ba.x, b), j2 = bit(Ba.y, b);
    return (IF1 - n1a - n1b + j1) * (IF2 - n2a - n2b + j2) + IQD + card_ng(Bm, cnt, a) + card_ng(Bm, cnt, b) -
           j2 * (n1a + n1b) - j1 * (n2a + n2b) + 3 * j1 * j2 - (__popcll(Ba.x & Bb.y) + __popcll(Bb.x & Ba.y));
}

// Two counted opponents (1, 2) with combo matrices M1, M2 over the dense
// deck, per-card sums u_i = M_i 1, d(c) = sum_b M1[c][b] M2[c][b],
// w = M2 u1 + M1 u2, P = M1 M2, F_i = sum u_i / 2, Q = sum u1 u2, D = sum d / 2.
// For a traverser hand (a, b), m_i = M_i[a][b], A_i = F_i - u_i(a) - u_i(b) + m_i,
// the mass of opponent pairs disjoint from each other and from (a, b) is
//   A1 A2 - Q + u1(a)u2(a) + u1(b)u2(b) + w(a) + w(b)
//   - m2 (u1(a) + u1(b)) - m1 (u2(a) + u2(b)) - 2 (d(a) + d(b)) + 3 m1 m2
//   - P[a][b] - P[b][a] + D
// (inclusion-exclusion over shared cards), equal to the reference odometer
// sum of street_solve.cu:771-823 / :1079-1127 for two opponents.
//
// Exact zeros: the reference only adds positive reach products, so a hand
// with no compatible positive-reach pair gets exactly 0.  Every term above is
// at most a few F1 F2 in size and the product P carries FP32 accuracy, so a
// computed mass above 1e-4 F1 F2 cannot come from an empty set of pairs; at or
// below it the kernel counts the compatible positive-reach pairs exactly (the
// same formula on the 0/1 positive-reach matrices, via 64-bit card masks) and
// writes 0 when there are none.
//
// One block per group of terminals sharing both opponents' reach rows: the
// masses are computed once and multiplied by each terminal's factor.  A
// chain of groups on the same first-opponent row (TermItem::chain) runs in
// one block, one group after the other: the first opponent's matrix, its
// column sums and masks are built once for the chain.
// Phases per group: cp.async staging of the reach rows (both for the
// chain's first group; the next group's second-opponent row is staged while
// this group's mass is computed); gather (or clear + scatter for ranges that
// repeat a combo); P (tensor cores) alongside per-column sums and masks;
// per-card FP64 terms and block scalars; per-hand mass and one output row
// per terminal (the leaf factors read one hand ahead from global memory).
template <class T>
__global__ void __launch_bounds__(kTermThreads, sizeof(T) == 4 ? 5 : 2) k_term_cr2(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                              const TermItem *__restrict__ items,
                                                              const int *__restrict__ heads, int trav) {
    wait_prior_grid();
    extern __shared__ __align__(16) char smem[];
    const TermItem *I0 = items + (heads ? __ldg(heads + blockIdx.x) : static_cast<int>(blockIdx.x));
    // followers are written by their group's leader, chained groups by the chain's head
    if (I0->follow || I0->chained) return;
    if (retired(ctxs, I0->sg)) return;
    const int o0 = I0->opp_player[0], o1 = I0->opp_player[1];
    const Cr2View<T> V = ctxs ? cr2_view<T>(ctxs[I0->sg], trav, o0, o1) : cr2_view<T>(c0, trav, o0, o1);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int HS = V.HS;
    const int Dp = (V.deck + 3) & ~3;
    const int hc_first = tid < V.Ht ? __ldg(V.code_t + tid) : 0;   // this thread's first hand code
    // shared memory was provisioned for c0's row stride (the largest of a batch)
    if (HS > c0.HS || V.deck > 52) return;
    Carve cv{smem};
    T *M1 = cv.take<T>(52 * MS);
    T *M2 = cv.take<T>(52 * MS);
    T *P = cv.take<T>(52 * MS);
    // per-card terms, one array per field (a hand reads three of them at two
    // cards; separate arrays keep those reads free of bank conflicts)
    double *cu1 = cv.take<double>(56), *cu2 = cv.take<double>(56), *cg = cv.take<double>(56);
    Cr2Cnt *cnt = cv.take<Cr2Cnt>(53);
    ulonglong2 *Bm = cv.take<ulonglong2>(53);   // positive-cell masks of M1 (x) and M2 (y) per card
    float *rsum = cv.take<float>(2 * 48);       // tensor-core path: partial row / column sums of P
    float *csum = cv.take<float>(3 * 48);
    Cr2Scalars *sc = cv.take<Cr2Scalars>(1);
    int *gnode = cv.take<int>(kTermGroupMax);
    int *gleaf = cv.take<int>(kTermGroupMax);
    float *gpay = cv.take<float>(kTermGroupMax);
    // the second opponent's staged reach row, followed by a zero (last: every
    // other offset is a constant); the next group's row lands here while
    // this group's mass is computed.  The first opponent's row is staged in
    // P's space (P is written after the gather).
    T *r2 = cv.take<T>(HS + 16 / sizeof(T));
    T *r1 = P;
    bool mma = false;
    if constexpr (sizeof(T) == 4) mma = Dp <= 48;
    const int Ht = V.Ht;
    const int *__restrict__ tc = V.code_t;

    // staging: a group's second-opponent reach row (16-byte chunks; rows
    // start on 128-byte boundaries), the first opponent's row with with_first
    auto stage_rows = [&](const TermItem *G, bool with_first) {
        constexpr int per = 16 / sizeof(T);
        const T *s1 = V.reach + static_cast<size_t>(G->opp_row[0]) * HS;
        const T *s2 = V.reach + static_cast<size_t>(G->opp_row[1]) * HS;
        for (int i = tid * per; i < HS; i += kTermThreads * per) {
            if (with_first) cp_async16(r1 + i, s1 + i);
            cp_async16(r2 + i, s2 + i);
        }
    };
    // a group's items' fields
    auto stage_items = [&](const TermItem *G) {
        if (tid <= G->gextra) {
            const TermItem &I = G[tid];
            gnode[tid] = I.node;
            gleaf[tid] = I.leaf_off;
            gpay[tid] = I.payoff;
        }
    };
    auto gather_second = [&]() {
        if (V.dup)
            scatter_dense(V.code1, V.H1, r2, M2);
        else
            gather_dense(V.tab1, r2, M2, Dp);
    };

    // the chain's first group: both opponents' matrices
    stage_rows(I0, true);
    stage_items(I0);
    if (tid == 0) {
        r1[HS] = T(0);
        r2[HS] = T(0);
    }
    if (V.dup) {
        zero_matrix(M1);
        zero_matrix(M2);
    }
    cp_async_wait_all();
    __syncthreads();
    if (V.dup)
        scatter_dense(V.code0, V.H0, r1, M1);
    else
        gather_dense(V.tab0, r1, M1, Dp);
    gather_second();
    __syncthreads();

    const TermItem *G = I0;
    const int nchain = I0->chain;
    for (int q = 0;; ++q) {
        const bool first = q == 0;
        const int ng = G->gextra + 1;

        // phase A: P = M1 M2 (tensor cores when the deck fits 48 cards, else
        // 4x4 SIMT tiles); per-column reach sums and positive-cell masks (the
        // first opponent's for the chain's first group only: they stay in
        // cu1 and Bm[].x)
        if (mma) {
            if constexpr (sizeof(T) == 4) {
                if (warp < 6) product_mma48(M1, M2, P, rsum, csum, warp, lane);
            }
            // columns: warps 6-7 take 0..63, warp 0 (after its MMA tiles) 64..95
            const int s = tid >= 6 * 32 ? tid - 6 * 32 : tid < 32 ? 64 + tid : 2 * 52;
            if (s < 2 * Dp && (first || s >= Dp)) column_stats(M1, M2, s, Dp, cu1, cu2, Bm);
        } else {
            const int nt = Dp >> 2;
            if (tid < nt * nt) product_tile(M1, M2, P, (tid / nt) * 4, (tid % nt) * 4, Dp);
            const int s = kTermThreads - 1 - tid;
            if (s < 2 * Dp && (first || s >= Dp)) column_stats(M1, M2, s, Dp, cu1, cu2, Bm);
        }
        __syncthreads();
        // the chain's next group: its second-opponent row is brought in while
        // this group's mass is computed (the gather of this group's is done)
        if (q < nchain) stage_rows(G + ng, false);

        // phase B: per-card terms (w from the row and column sums of P, d from its
        // diagonal: P = M1 M2 with symmetric M1, M2 gives rowsum = M1 u2,
        // colsum = M2 u1, P[c][c] = d(c)); entries beyond the deck are zeroed;
        // the last warp forms the block scalars
        if (tid < Dp) {
            const int col = tid;
            double w;
            if (mma) {
                w = (static_cast<double>(rsum[col]) + static_cast<double>(rsum[48 + col])) +
                    ((static_cast<double>(csum[col]) + static_cast<double>(csum[48 + col])) +
                     static_cast<double>(csum[96 + col]));
            } else {
                w = 0.0;
                for (int b = 0; b < Dp; ++b)
                    w += static_cast<double>(P[col * MS + b]) + static_cast<double>(P[b * MS + col]);
            }
            const double d = P[col * MS + col];
            cg[col] = cu1[col] * cu2[col] + w - 2.0 * d;
            const ulonglong2 Bc = Bm[col];
            cnt[col] = Cr2Cnt{__popcll(Bc.x), __popcll(Bc.y), 0, 0};
        } else if (tid <= kCr2Off) {
            cu1[tid] = 0.0;
            cu2[tid] = 0.0;
            cg[tid] = 0.0;
            cnt[tid] = Cr2Cnt{0, 0, 0, 0};
            Bm[tid] = make_ulonglong2(0ull, 0ull);
        } else if (warp == kTermThreads / 32 - 1) {
            double a1 = 0.0, a2 = 0.0, qq = 0.0, e = 0.0;
            int n1 = 0, n2 = 0, nq = 0, nd = 0;
            for (int k = lane; k < Dp; k += 32) {
                const double u1 = cu1[k], u2 = cu2[k];
                a1 += u1;
                a2 += u2;
                qq += u1 * u2;
                e += static_cast<double>(P[k * MS + k]);
                const ulonglong2 B = Bm[k];
                const int p1 = __popcll(B.x), p2 = __popcll(B.y);
                n1 += p1;
                n2 += p2;
                nq += p1 * p2;
                nd += __popcll(B.x & B.y);
            }
            a1 = warp_sum(a1);
            a2 = warp_sum(a2);
            qq = warp_sum(qq);
            e = warp_sum(e);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                n1 += __shfl_xor_sync(0xffffffffu, n1, o);
                n2 += __shfl_xor_sync(0xffffffffu, n2, o);
                nq += __shfl_xor_sync(0xffffffffu, nq, o);
                nd += __shfl_xor_sync(0xffffffffu, nd, o);
            }
            if (lane == 0) *sc = Cr2Scalars{0.5 * a1, 0.5 * a2, 0.5 * e - qq, n1 / 2, n2 / 2, nd / 2 - nq, 0};
        }
        __syncthreads();

        // phase C: card-removal mass of every traverser hand, written out as
        // factor x mass for every terminal of the group
        const Cr2Scalars S = *sc;
        const double zmin = 1e-4 * S.F1 * S.F2;
        const bool none = !(S.F1 > 0.0 && S.F2 > 0.0);   // an opponent without positive reach: all zero
        const int gl0 = gleaf[0];
        const float gp0 = gpay[0];
        T *out0 = V.val + static_cast<size_t>(gnode[0]) * HS;
        // the next hand's code is loaded one iteration ahead (the first one at
        // the start of the block), so the loop does not wait on it
        int hc_next = hc_first;
        float f_next = tid < Ht ? (gl0 >= 0 ? __ldg(V.leaf + gl0 + tid) : gp0) : 0.f;
        for (int h = tid; h < HS; h += kTermThreads) {
            const int hc = hc_next;
            const float f0 = f_next;
            hc_next = h + kTermThreads < Ht ? __ldg(tc + h + kTermThreads) : 0;
            f_next = h + kTermThreads < Ht ? (gl0 >= 0 ? __ldg(V.leaf + gl0 + h + kTermThreads) : gp0) : 0.f;
            double v = 0.0;
            if (h < Ht && !none) {
                const int a = min((hc >> 20) & 63, kCr2Off), b = min((hc >> 26) & 63, kCr2Off);
                const bool on = (a < kCr2Off) && (b < kCr2Off);
                const double ua1 = cu1[a], ua2 = cu2[a], ub1 = cu1[b], ub2 = cu2[b];
                const double m1 = on ? static_cast<double>(M1[a * MS + b]) : 0.0;
                const double m2 = on ? static_cast<double>(M2[a * MS + b]) : 0.0;
                const double pp = on ? static_cast<double>(P[a * MS + b] + P[b * MS + a]) : 0.0;
                const double A1 = S.F1 - ua1 - ub1 + m1;
                const double A2 = S.F2 - ua2 - ub2 + m2;
                v = A1 * A2 + S.QD + cg[a] + cg[b] - m2 * (ua1 + ub1) - m1 * (ua2 + ub2) + 3.0 * m1 * m2 - pp;
                if (fabs(v) <= zmin && pair_count(Bm, cnt, a, b, S.IF1, S.IF2, S.IQD) <= 0) v = 0.0;
            }
            out0[h] = static_cast<T>(static_cast<double>(f0) * v);
            for (int g = 1; g < ng; ++g) {
                const float f = h >= Ht ? 0.f : gleaf[g] >= 0 ? __ldg(V.leaf + gleaf[g] + h) : gpay[g];
                V.val[static_cast<size_t>(gnode[g]) * HS + h] = static_cast<T>(static_cast<double>(f) * v);
            }
        }
        if (q == nchain) break;
        // the chain's next group: its second-opponent matrix replaces the
        // last one once every thread is done with the shared state
        G += ng;
        __syncthreads();
        stage_items(G);
        if (V.dup) zero_matrix(M2);
        cp_async_wait_all();
        __syncthreads();
        gather_second();
        __syncthreads();
    }
}

#include "ss_cr2_tc.cuh"

template <class T>
constexpr size_t cr1_gather_smem(int HS) {
    return (static_cast<size_t>(HS) + 4) * sizeof(T) + static_cast<size_t>(HS) * 4 + 64 * 8 + 64 * 4 +
           3 * kTermGroupMax * 4 + 2 * 16 + 8 * 16;
}

// One counted opponent over the dense deck, for ranges without a repeated
// combo: u(c) and f(h) are read from the staged reach row through the
// opponent's pair table (row c of the table lists the opponent's hands
// holding card c), so no matrix is built.  Exact zeros: the number of
// compatible positive-reach opponent hands N - n(a) - n(b) + [f(h) > 0]
// decides a value of exactly 0.  One block per group of terminals sharing the
// opponent's reach row (the traverser's own continuation choices).
template <class T>
__global__ void __launch_bounds__(kTermThreads) k_term_cr1(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                           const TermItem *__restrict__ items, int trav) {
    wait_prior_grid();
    extern __shared__ __align__(16) char smem[];
    const TermItem *I0 = items + blockIdx.x;
    if (I0->follow) return;   // written by the block of its group's first item
    if (retired(ctxs, I0->sg)) return;
    const int ng = I0->gextra + 1;
    const int o = I0->opp_player[0];
    const Cr2View<T> V = ctxs ? cr2_view<T>(ctxs[I0->sg], trav, o, o) : cr2_view<T>(c0, trav, o, o);
    const int HS = V.HS;
    if (HS > c0.HS || V.deck > 52) return;   // shared memory was provisioned for c0's row stride
    const int tid = threadIdx.x, lane = tid & 31;
    const int Dp = (V.deck + 3) & ~3;
    Carve cv{smem};
    T *r = cv.take<T>(HS + 4);                 // staged reach row, r[HS] = 0 for missing pairs
    float *leaf0 = cv.take<float>(HS);
    double *u = cv.take<double>(64);
    int *nz = cv.take<int>(64);
    int *gnode = cv.take<int>(kTermGroupMax);
    int *gleaf = cv.take<int>(kTermGroupMax);
    float *gpay = cv.take<float>(kTermGroupMax);
    {
        const T *src = V.reach + static_cast<size_t>(I0->opp_row[0]) * HS;
        constexpr int per = 16 / sizeof(T);
        for (int q = tid * per; q < HS; q += kTermThreads * per) cp_async16(r + q, src + q);
        const int lo = I0->leaf_off;
        if (lo >= 0) {
            const float *ls = V.leaf + lo;
            for (int h = tid; h < V.Ht; h += kTermThreads) cp_async4(leaf0 + h, ls + h);
        }
        if (tid < ng) {
            const TermItem &I = I0[tid];
            gnode[tid] = I.node;
            gleaf[tid] = I.leaf_off;
            gpay[tid] = I.payoff;
        }
        if (tid == 0) r[HS] = T(0);
        if (tid < 64) {
            u[tid] = 0.0;
            nz[tid] = 0;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // per card c: u(c) and the count of positive-reach hands holding c, four
    // lanes per card (a quarter of the table row each, shuffles in a fixed order)
    {
        const int col = tid >> 2, part = tid & 3, q = Dp >> 2;
        double s = 0.0;
        int n = 0;
        if (col < Dp) {
            const int *row = V.tab0 + col * 52 + part * q;
            for (int b = 0; b < q; ++b) {
                const T x = r[__ldg(row + b)];
                s += static_cast<double>(x);
                n += x > T(0) ? 1 : 0;
            }
        }
#pragma unroll
        for (int k = 1; k < 4; k <<= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, k);
            n += __shfl_xor_sync(0xffffffffu, n, k);
        }
        if (part == 0 && col < Dp) {
            u[col] = s;
            nz[col] = n;
        }
    }
    __syncthreads();
    double F;
    int N;
    {
        double s = (lane < Dp ? u[lane] : 0.0) + (lane + 32 < Dp ? u[lane + 32] : 0.0);
        int n = (lane < Dp ? nz[lane] : 0) + (lane + 32 < Dp ? nz[lane + 32] : 0);
        s = warp_sum(s);
#pragma unroll
        for (int k = 16; k > 0; k >>= 1) n += __shfl_xor_sync(0xffffffffu, n, k);
        F = 0.5 * s;
        N = n / 2;
    }
    const int Ht = V.Ht;
    const int *__restrict__ tc = V.code_t;
    const bool leaf_first = gleaf[0] >= 0;
    const float gp0 = gpay[0];
    T *out0 = V.val + static_cast<size_t>(gnode[0]) * HS;
    for (int h = tid; h < HS; h += kTermThreads) {
        double v = 0.0;
        if (h < Ht) {
            const int hc = __ldg(tc + h);
            const int a = min((hc >> 20) & 63, kCr2Off), b = min((hc >> 26) & 63, kCr2Off);
            const T f = r[__ldg(V.x0 + h)];   // 0 for a hand touching the board (index HS)
            const int live = N - nz[a] - nz[b] + (f > T(0) ? 1 : 0);
            if (live > 0) v = F - u[a] - u[b] + static_cast<double>(f);
        }
        const float f0 = h >= Ht ? 0.f : leaf_first ? leaf0[h] : gp0;
        out0[h] = static_cast<T>(static_cast<double>(f0) * v);
        for (int g = 1; g < ng; ++g) {
            const float f = h >= Ht ? 0.f : gleaf[g] >= 0 ? __ldg(V.leaf + gleaf[g] + h) : gpay[g];
            V.val[static_cast<size_t>(gnode[g]) * HS + h] = static_cast<T>(static_cast<double>(f) * v);
        }
    }
}

template <class T>
constexpr size_t sd1_smem() {
    return 1326 * sizeof(T) + 1327 * 8 + 52 * 53 * 8 + 52 * 4 + (kTermThreads / 32) * 8 + 52 * 8 + 64;
}

// Showdown against one live opponent (street_solve.cu:886-903): with W, T, L
// the opponent reach on compatible hands that are weaker, tied and stronger,
// value = (pot - bet) W + (pot/2 - bet) T - bet L.  Combos are ranked once per board; the
// block builds the opponent's reach in rank order, its prefix sums P and
// per-card prefix sums PC[c], and then for a traverser combo (c1, c2) with
// tie group [lo, hi):
//   W = P[lo] - PC[c1][<lo] - PC[c2][<lo]
//   T = P[hi] - P[lo] - (PC[c1][<hi] - PC[c1][<lo]) - (PC[c2][<hi] - PC[c2][<lo]) + f(h)
//   S = P[end] - PC[c1][end] - PC[c2][end] + f(h)
// A traverser hand with no compatible positive-reach opponent hand gets
// exactly 0 (positive-reach masks per card, as in the two-opponent kernels).
template <class T>
__global__ void __launch_bounds__(kTermThreads) k_term_sd1(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                           const TermItem *__restrict__ items, int trav) {
    wait_prior_grid();
    extern __shared__ __align__(16) char smem[];
    Carve cv{smem};
    T *Rr = cv.take<T>(1326);
    double *Pp = cv.take<double>(1327);
    double *PC = cv.take<double>(52 * 53);
    int *clen = cv.take<int>(52);
    double *wsum = cv.take<double>(kTermThreads / 32);
    unsigned long long *B = cv.take<unsigned long long>(52);
    int *npos = cv.take<int>(1);
    const TermItem I = items[blockIdx.x];
    if (retired(ctxs, I.sg)) return;
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nc = c.ncomb;
    for (int i = tid; i < nc; i += blockDim.x) Rr[i] = T(0);
    __syncthreads();
    {
        const int o = I.opp_player[0];
        const T *r = reach_rows<T>(c) + static_cast<size_t>(I.opp_row[0]) * c.HS;
        const int *pos = c.sd_pos + static_cast<size_t>(o) * c.HS;
        const bool dup = c.dup[o] != 0;
        for (int j = tid; j < c.H[o]; j += blockDim.x) {
            const int q = pos[j];
            if (q < 0) continue;
            if (dup)
                atomicAdd(&Rr[q], r[j]);
            else
                Rr[q] = r[j];
        }
    }
    __syncthreads();
    // exclusive prefix over rank positions: each thread scans a contiguous chunk
    {
        const int per = (nc + blockDim.x - 1) / blockDim.x;
        const int b0 = tid * per, b1 = min(nc, b0 + per);
        double local = 0.0;
        for (int i = b0; i < b1; ++i) local += Rr[i];
        double incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        double base = 0.0;
        for (int w = 0; w < warp; ++w) base += wsum[w];
        double run = base + incl - local;
        for (int i = b0; i < b1; ++i) {
            Pp[i] = run;
            run += Rr[i];
        }
        if (tid == blockDim.x - 1) {
            double tot = 0.0;
            for (int w = 0; w < blockDim.x / 32; ++w) tot += wsum[w];
            Pp[nc] = tot;
        }
    }
    // per card: exclusive prefix sums over its combos in rank order, and the
    // mask of partner cards whose combo holds positive reach
    for (int card = warp; card < 52; card += blockDim.x / 32) {
        const short *L = c.sd_card_list + card * 52;
        const short *Pt = c.sd_card_partner + card * 52;
        const int i0 = 2 * lane, i1 = 2 * lane + 1;
        const int q0 = i0 < 52 ? L[i0] : -1, q1 = i1 < 52 ? L[i1] : -1;
        const T f0 = q0 >= 0 ? Rr[q0] : T(0), f1 = q1 >= 0 ? Rr[q1] : T(0);
        const double v0 = f0, v1 = f1;
        const double pair = v0 + v1;
        double incl = pair;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const double ex = incl - pair;
        const int len = __popc(__ballot_sync(0xffffffffu, q0 >= 0)) + __popc(__ballot_sync(0xffffffffu, q1 >= 0));
        if (i0 <= len) PC[card * 53 + i0] = ex;
        if (i1 <= len) PC[card * 53 + i1] = ex + v0;
        unsigned long long m = 0ull;
        if (f0 > T(0)) m |= 1ull << Pt[i0];
        if (f1 > T(0)) m |= 1ull << Pt[i1];
        const unsigned lo = __reduce_or_sync(0xffffffffu, static_cast<unsigned>(m));
        const unsigned hi = __reduce_or_sync(0xffffffffu, static_cast<unsigned>(m >> 32));
        if (lane == 0) {
            clen[card] = len;
            B[card] = static_cast<unsigned long long>(lo) | (static_cast<unsigned long long>(hi) << 32);
        }
    }
    __syncthreads();
    if (warp == 0) {
        int n = __popcll(B[lane]) + (lane + 32 < 52 ? __popcll(B[lane + 32]) : 0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
        if (lane == 0) *npos = n / 2;
    }
    __syncthreads();
    const int Ht = c.H[trav];
    const int *tpos = c.sd_pos + static_cast<size_t>(trav) * c.HS;
    T *out = val_rows<T>(c) + static_cast<size_t>(I.node) * c.HS;
    // payoff per class with the reference's float coefficients (win pot - bet,
    // tie pot * 0.5 - bet, loss -bet): a coefficient that is exactly 0 drops
    // its class exactly, as in the reference's sum
    const double cw = static_cast<double>(I.pot - I.bet), ct = static_cast<double>(I.pot * 0.5f - I.bet);
    const double cl = -static_cast<double>(I.bet);
    const int np_ = *npos;
    for (int h = tid; h < c.HS; h += blockDim.x) {
        double v = 0.0;
        const int q = h < Ht ? tpos[h] : -1;
        if (q >= 0) {
            const SdCombo s = c.sd_combo[q];
            const unsigned long long B1 = B[s.c1], B2 = B[s.c2];
            if (np_ - __popcll(B1) - __popcll(B2) + bit(B1, s.c2) > 0) {
                const double *p1 = PC + s.c1 * 53, *p2 = PC + s.c2 * 53;
                const double self = Rr[q];
                const double W = Pp[s.lo] - p1[s.l1lo] - p2[s.l2lo];
                const double Tt = (Pp[s.hi] - Pp[s.lo]) - (p1[s.l1hi] - p1[s.l1lo]) -
                                  (p2[s.l2hi] - p2[s.l2lo]) + self;
                const double L = (Pp[nc] - Pp[s.hi]) - (p1[clen[s.c1]] - p1[s.l1hi]) - (p2[clen[s.c2]] - p2[s.l2hi]);
                v = cw * W + ct * Tt + cl * L;
            }
        }
        store_value(out, h, v);
    }
}

// ---------------------------------------------------------------------------
// Three-way showdown (two live opponents), street_solve.cu:936-1002: the
// traverser (strength s) against opponents 1, 2 on disjoint hands o1, o2
// wins pot / (1 + number of opponents tying s) - bet if neither opponent is
// stronger, else loses bet.  With D(X, Y) the mass of opponent pairs
// (o1 in X, o2 in Y) disjoint from each other and from the hand, and L / E
// the opponents' hands weaker than / tying s, the classes are W2 = D(L, L)
// (win), T1 = D(E, L) + D(L, E) (two-way tie), T2 = D(E, E) (three-way tie)
// and the rest of Z = D(all, all) (loss).
// D(X, Y) is the two-opponent card-removal closed form on matrices holding
// only X's and Y's hands.  The kernel sweeps the combos in rank order and
// keeps that form's aggregates (P = M1 M2, u_i, w, d, F_i, Q, D; FP64) for
// the opponents' hands added so far; per tie group of the traverser's hands
// it reads A = D(L, L) before the group and C = D(L+E, L+E) after adding
// both opponents' group hands, and sums D(L, E) over opponent 2's group
// hands and D(E, L) over opponent 1's directly (each term an exact four-card
// removal for the other opponent).  With Z read after the sweep:
//   W2 = A, T1 = D(E, L) + D(L, E), T2 = C - A - T1, lose = Z - C,
//   value = (pot - bet) W2 + (pot/2 - bet) T1 + (pot/3 - bet) T2 - bet lose,
// and T2 = 0 exactly when opponent 2 holds nothing in the group (C is then
// B = D(L+E, L), and C - B the empty class).
// Adding a hand changes two rows (or columns) of P, two card sums and every
// w entry, so each phase gives threads fixed ownership (P cells by column
// and row residue, one card's u / d / w, the scalars, matrix cells), each
// accumulating its share of the phase's hands in registers: no atomics, a
// fixed summation order.  The sweep of a terminal is cut into runs of tie
// groups of about equal cost, one block each, starting from a directly
// computed state (the product P as 3x3 FP64 tiles over all 256 threads).
// C of a group and A of the next are read in one phase (the same state); the
// tie sums of a traverser hand are split over eight lanes.
// ---------------------------------------------------------------------------
constexpr int SD2_S = 49;   // row stride of the sweep's card matrices (odd: conflict-free columns)
constexpr int SD2_N = 48;   // cards a matrix covers (dense indices; a river deck has 47)
static_assert(kTermThreads == 256, "the sweep's thread roles assume 256 threads");

// the opponents' reach by rank position; after the sweep the same space holds
// the positive-reach masks, counts and scalars of the exact-zero test
template <class T>
__host__ __device__ constexpr size_t sd2_reach_bytes(int ncomb) {
    return 2 * static_cast<size_t>(ncomb) * sizeof(T) > 53 * sizeof(ulonglong2) + 53 * sizeof(Cr2Cnt) + sizeof(Cr2Scalars)
               ? 2 * static_cast<size_t>(ncomb) * sizeof(T)
               : 53 * sizeof(ulonglong2) + 53 * sizeof(Cr2Cnt) + sizeof(Cr2Scalars);
}

// dynamic shared memory for runs of at most `span` rank positions: P, M1, M2,
// u1, u2, w, d, scalars, per-position classes of the run, reach (masks), the
// cards of each position, the traverser's hand at each position of the run,
// the last positive position; 16 bytes of alignment slack per carve
template <class T>
constexpr size_t sd2_smem(int span, int ncomb) {
    return SD2_S * SD2_S * 8 + 2 * SD2_S * SD2_S * sizeof(T) + 4 * 64 * 8 + 8 * 8 + static_cast<size_t>(span) * 32 +
           sd2_reach_bytes<T>(ncomb) + static_cast<size_t>(ncomb) * 2 + static_cast<size_t>(span) * 2 + 16 +
           13 * 16;
}

struct Sd2State {
    double *P, *u1, *u2, *w, *d, *sc;   // sc: F1, F2, Q, D
};

__device__ __forceinline__ int sd2_c1(unsigned short e) { return e & 255; }
__device__ __forceinline__ int sd2_c2(unsigned short e) { return e >> 8; }

// D(., .) of the hand (a, b) on the current sweep state (the two-opponent
// closed form, see k_term_cr2)
// Written with explicit round-to-nearest operations (no contraction into
// FMAs), so two evaluations on the same state agree bit for bit wherever they
// are inlined: the class masses below are differences of such evaluations and
// must come out exactly 0 when the class is empty and the states coincide.
template <class T>
__device__ __forceinline__ double sd2_mass(Sd2State st, const T *M1, const T *M2, int a, int b) {
    const double u1a = st.u1[a], u1b = st.u1[b], u2a = st.u2[a], u2b = st.u2[b];
    const double m1 = static_cast<double>(M1[a * SD2_S + b]), m2 = static_cast<double>(M2[a * SD2_S + b]);
    const double pp = __dadd_rn(st.P[a * SD2_S + b], st.P[b * SD2_S + a]);
    const double ga = __dsub_rn(__dadd_rn(__dmul_rn(u1a, u2a), st.w[a]), __dmul_rn(2.0, st.d[a]));
    const double gb = __dsub_rn(__dadd_rn(__dmul_rn(u1b, u2b), st.w[b]), __dmul_rn(2.0, st.d[b]));
    const double A1 = __dadd_rn(__dsub_rn(__dsub_rn(st.sc[0], u1a), u1b), m1);
    const double A2 = __dadd_rn(__dsub_rn(__dsub_rn(st.sc[1], u2a), u2b), m2);
    double z = __dmul_rn(A1, A2);
    z = __dadd_rn(z, __dsub_rn(st.sc[3], st.sc[2]));
    z = __dadd_rn(z, __dadd_rn(ga, gb));
    z = __dsub_rn(z, __dmul_rn(m2, __dadd_rn(u1a, u1b)));
    z = __dsub_rn(z, __dmul_rn(m1, __dadd_rn(u2a, u2b)));
    z = __dadd_rn(z, __dmul_rn(3.0, __dmul_rn(m1, m2)));
    return __dsub_rn(z, pp);
}

// Add the hands of opponent `who` (0 or 1) at rank positions [lo, hi) to the
// sweep state.  R: that opponent's reach by rank position; Mo: that
// opponent's matrix, Mx: the other's (symmetric); uo / ux: their card sums.
template <class T>
__device__ __forceinline__ void sd2_add(Sd2State st, const unsigned short *dd, const T *R, T *Mo, const T *Mx,
                                        double *uo, const double *ux, int who, int lo, int hi) {
    const int tid = threadIdx.x;
    if (tid < 4 * SD2_N) {
        // P = M1 M2: opponent 1's hand {x, y} adds r Mx[y][.] to row x and
        // r Mx[x][.] to row y; opponent 2's adds the same to columns x, y.
        // Thread (part, j) owns column (row) j of the rows (columns) x with
        // x % 4 == part: the four suits of a rank fall to different threads.
        const int part = tid / SD2_N, j = tid - part * SD2_N;
        for (int q = lo; q < hi; ++q) {
            const T rt = R[q];
            if (rt == T(0)) continue;
            const double r = static_cast<double>(rt);
            const unsigned short e = dd[q];
            const int x = sd2_c1(e), y = sd2_c2(e);
            if ((x & 3) == part) {
                double *p = who == 0 ? st.P + x * SD2_S + j : st.P + j * SD2_S + x;
                *p += r * static_cast<double>(Mx[y * SD2_S + j]);
            }
            if ((y & 3) == part) {
                double *p = who == 0 ? st.P + y * SD2_S + j : st.P + j * SD2_S + y;
                *p += r * static_cast<double>(Mx[x * SD2_S + j]);
            }
        }
    } else if (tid < 5 * SD2_N) {
        // card c: this opponent's card sum u(c), d(c) = sum_b M1[c][b] M2[c][b]
        // and w(c) = (M2 u1 + M1 u2)(c): the hand changes Mo at (x, y) and uo
        // at x, y
        const int c = tid - 4 * SD2_N;
        double du = 0.0, dd_c = 0.0, dw = 0.0;
        for (int q = lo; q < hi; ++q) {
            const T rt = R[q];
            if (rt == T(0)) continue;
            const double r = static_cast<double>(rt);
            const unsigned short e = dd[q];
            const int x = sd2_c1(e), y = sd2_c2(e);
            const double mx = static_cast<double>(Mx[c * SD2_S + x]), my = static_cast<double>(Mx[c * SD2_S + y]);
            dw += r * (mx + my);
            if (c == x) {
                du += r;
                dd_c += r * my;
                dw += r * ux[y];
            }
            if (c == y) {
                du += r;
                dd_c += r * mx;
                dw += r * ux[x];
            }
        }
        uo[c] += du;
        st.d[c] += dd_c;
        st.w[c] += dw;
    } else if (tid == 5 * SD2_N) {
        // F (this opponent's total), Q = sum u1 u2, D = sum d / 2
        double F = st.sc[who], Q = st.sc[2], D = st.sc[3];
        for (int q = lo; q < hi; ++q) {
            const T rt = R[q];
            if (rt == T(0)) continue;
            const double r = static_cast<double>(rt);
            const unsigned short e = dd[q];
            const int x = sd2_c1(e), y = sd2_c2(e);
            Q += r * (ux[x] + ux[y]);
            D += r * static_cast<double>(Mx[x * SD2_S + y]);
            F += r;
        }
        st.sc[who] = F;
        st.sc[2] = Q;
        st.sc[3] = D;
    } else {
        constexpr int kFirst = 5 * SD2_N + 1, kStep = kTermThreads - kFirst;
        for (int q = lo + tid - kFirst; q < hi; q += kStep) {
            const T r = R[q];
            if (r == T(0)) continue;
            const unsigned short e = dd[q];
            const int x = sd2_c1(e), y = sd2_c2(e);
            Mo[x * SD2_S + y] = r;
            Mo[y * SD2_S + x] = r;
        }
    }
}

// The sweep state for the opponents' hands at rank positions [0, qend),
// computed directly (not by adding them one tie group at a time): the two
// matrices, P = M1 M2 as FP64 3x3 tiles over the 48-card box, the card sums,
// d = diag P, w = column sums + row sums of P, and the scalars, each summed
// in a fixed order.  The caller syncs before; this syncs after.
template <class T>
__device__ __forceinline__ void sd2_direct_state(Sd2State st, T *M1, T *M2, const T *R1, const T *R2,
                                                 const unsigned short *dd, int qend) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (qend == 0) {
        // no hands: every aggregate is zero (the same for every thread of the
        // block, so the early return passes no barrier unevenly)
        for (int i = tid; i < SD2_S * SD2_S; i += kTermThreads) {
            M1[i] = T(0);
            M2[i] = T(0);
            st.P[i] = 0.0;
        }
        if (tid < 64) {
            st.u1[tid] = 0.0;
            st.u2[tid] = 0.0;
            st.w[tid] = 0.0;
            st.d[tid] = 0.0;
        }
        if (tid < 8) st.sc[tid] = 0.0;
        __syncthreads();
        return;
    }
    for (int i = tid; i < SD2_S * SD2_S; i += kTermThreads) {
        M1[i] = T(0);
        M2[i] = T(0);
    }
    __syncthreads();
    for (int q = tid; q < qend; q += kTermThreads) {
        const unsigned short e = dd[q];
        const int x = sd2_c1(e), y = sd2_c2(e);
        const T r1 = R1[q], r2 = R2[q];
        if (r1 != T(0)) {
            M1[x * SD2_S + y] = r1;
            M1[y * SD2_S + x] = r1;
        }
        if (r2 != T(0)) {
            M2[x * SD2_S + y] = r2;
            M2[y * SD2_S + x] = r2;
        }
    }
    __syncthreads();
    {
        const int i0 = (tid >> 4) * 3, j0 = (tid & 15) * 3;
        double acc[3][3] = {};
        for (int k = 0; k < SD2_N; ++k) {
            double xs[3], ys[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                xs[i] = static_cast<double>(M1[(i0 + i) * SD2_S + k]);
                ys[i] = static_cast<double>(M2[k * SD2_S + j0 + i]);
            }
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) acc[i][j] += xs[i] * ys[j];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) st.P[(i0 + i) * SD2_S + j0 + j] = acc[i][j];
    }
    __syncthreads();
    if (tid < SD2_N) {
        const int c = tid;
        double u = 0.0;
        for (int r = 0; r < SD2_N; ++r) u += static_cast<double>(M1[r * SD2_S + c]);
        st.u1[c] = u;
        st.d[c] = st.P[c * SD2_S + c];
    } else if (tid >= 64 && tid < 64 + SD2_N) {
        const int c = tid - 64;
        double u = 0.0;
        for (int r = 0; r < SD2_N; ++r) u += static_cast<double>(M2[r * SD2_S + c]);
        st.u2[c] = u;
    } else if (tid >= 128 && tid < 128 + SD2_N) {
        const int c = tid - 128;
        double w = 0.0;   // (M2 u1)(c) = sum_r P[r][c]
        for (int r = 0; r < SD2_N; ++r) w += st.P[r * SD2_S + c];
        st.w[c] = w;
    }
    __syncthreads();
    if (tid < SD2_N) {
        const int c = tid;
        double w = 0.0;   // (M1 u2)(c) = sum_r P[c][r]
        for (int r = 0; r < SD2_N; ++r) w += st.P[c * SD2_S + r];
        st.w[c] += w;
    } else if (warp == kTermThreads / 32 - 1) {
        double f1 = 0.0, f2 = 0.0, q = 0.0, e = 0.0;
        for (int c = lane; c < SD2_N; c += 32) {
            f1 += st.u1[c];
            f2 += st.u2[c];
            q += st.u1[c] * st.u2[c];
            e += st.d[c];
        }
        f1 = warp_sum(f1);
        f2 = warp_sum(f2);
        q = warp_sum(q);
        e = warp_sum(e);
        if (lane == 0) {
            st.sc[0] = 0.5 * f1;
            st.sc[1] = 0.5 * f2;
            st.sc[2] = q;
            st.sc[3] = 0.5 * e;
        }
    }
    __syncthreads();
}

// For the traverser's hands at positions [lo, hi) (a tie group), on the state
// before the group: A = D(L, L); T1 = D(L, E) + D(E, L), summing over
// opponent 2's group hands (opponent 1's weaker hands avoiding four cards)
// and over opponent 1's (opponent 2's avoiding four cards); whether opponent 2
// holds any group hand.  Eight lanes per hand, each taking every eighth group
// position, combined in a fixed order.  Classes of position q at
// cls[4 (q - base)]: A, T1, opponent 2 present, (C).
template <class T>
__device__ __forceinline__ void sd2_phase_a(Sd2State st, const T *M1, const T *M2, const T *R1, const T *R2,
                                            const unsigned short *dd, const short *pt, double *cls, int base,
                                            int lo, int hi) {
    const int l8 = threadIdx.x & 7, team = threadIdx.x >> 3;
    const int tbit = threadIdx.x & 24;   // the team's first lane in its warp
    for (int q0 = lo; q0 < hi; q0 += kTermThreads / 8) {
        const int q = q0 + team;
        const bool mine = q < hi && pt[q - base] >= 0;   // the same for all lanes of a team
        double t1 = 0.0;
        bool any2 = false;
        int a = 0, b = 0;
        if (mine) {
            const unsigned short e = dd[q];
            a = sd2_c1(e);
            b = sd2_c2(e);
            const double F1 = st.sc[0], F2 = st.sc[1];
            const double u1a = st.u1[a], u1b = st.u1[b], u2a = st.u2[a], u2b = st.u2[b];
            const double m1ab = static_cast<double>(M1[a * SD2_S + b]), m2ab = static_cast<double>(M2[a * SD2_S + b]);
            double dle = 0.0, del = 0.0;
            for (int q2 = lo + l8; q2 < hi; q2 += 8) {
                const T r1 = R1[q2], r2 = R2[q2];
                any2 = any2 || r2 != T(0);
                if (r1 == T(0) && r2 == T(0)) continue;
                const unsigned short e2 = dd[q2];
                const int x = sd2_c1(e2), y = sd2_c2(e2);
                if (x == a || x == b || y == a || y == b) continue;
                if (r2 != T(0))
                    dle += static_cast<double>(r2) *
                           (F1 - u1a - u1b - st.u1[x] - st.u1[y] + m1ab + static_cast<double>(M1[a * SD2_S + x]) +
                            static_cast<double>(M1[a * SD2_S + y]) + static_cast<double>(M1[b * SD2_S + x]) +
                            static_cast<double>(M1[b * SD2_S + y]) + static_cast<double>(M1[x * SD2_S + y]));
                if (r1 != T(0))
                    del += static_cast<double>(r1) *
                           (F2 - u2a - u2b - st.u2[x] - st.u2[y] + m2ab + static_cast<double>(M2[a * SD2_S + x]) +
                            static_cast<double>(M2[a * SD2_S + y]) + static_cast<double>(M2[b * SD2_S + x]) +
                            static_cast<double>(M2[b * SD2_S + y]) + static_cast<double>(M2[x * SD2_S + y]));
            }
            t1 = dle + del;
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) t1 += __shfl_xor_sync(0xffffffffu, t1, o);
        const unsigned bal = __ballot_sync(0xffffffffu, any2);
        if (mine && l8 == 0) {
            double *k4 = cls + 4 * (q - base);
            k4[0] = sd2_mass(st, M1, M2, a, b);
            k4[1] = t1;
            k4[2] = ((bal >> tbit) & 0xffu) ? 1.0 : 0.0;
        }
    }
}

// mass on the current state for the traverser's hands at [lo, hi), into
// class slot k
template <class T>
__device__ __forceinline__ void sd2_phase_mass(Sd2State st, const T *M1, const T *M2, const unsigned short *dd,
                                               const short *pt, double *cls, int base, int lo, int hi, int k) {
    for (int q = lo + threadIdx.x; q < hi; q += kTermThreads)
        if (pt[q - base] >= 0) cls[4 * (q - base) + k] = sd2_mass(st, M1, M2, sd2_c1(dd[q]), sd2_c2(dd[q]));
}

// One block per 2^lgm consecutive runs of a terminal's sweep (grid: items x
// kSd2Chunks / 2^lgm).  With bmap (batches), block b serves item bmap[b].x,
// run group bmap[b].y, with that item's own lgm (its subgame's solo choice).
template <class T>
__global__ void __launch_bounds__(kTermThreads, 4) k_term_sd2(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                              const TermItem *__restrict__ items, int trav, int lgm,
                                                              const int2 *__restrict__ bmap) {
    wait_prior_grid();
    extern __shared__ __align__(16) char smem[];
    int it_idx, grp;
    if (bmap) {
        const int2 m = bmap[blockIdx.x];
        it_idx = m.x;
        grp = m.y;
        lgm = items[it_idx].kind_detail;
    } else {
        const int per = kSd2Chunks >> lgm;
        it_idx = blockIdx.x / per;
        grp = blockIdx.x % per;
    }
    const TermItem I = items[it_idx];
    if (retired(ctxs, I.sg)) return;
    const int o1 = I.opp_player[0], o2 = I.opp_player[1];
    const T *reach;
    T *val;
    const int *pos_hand, *seg, *sd_pos;
    const SdCombo *cb;
    int HS, nc, Ht, s0, s1, span;
    {
        const DevCtx &c = ctxs ? ctxs[I.sg] : c0;   // read once into registers below
        reach = reach_rows<T>(c);
        val = val_rows<T>(c);
        pos_hand = c.pos_hand;
        seg = c.sd_seg;
        sd_pos = c.sd_pos;
        cb = c.sd_combo;
        HS = c.HS;
        nc = c.ncomb;
        span = c.sd_span[lgm];
        Ht = c.H[trav];
        const int *ch = c.sd_chunk + static_cast<size_t>(trav) * (kSd2Chunks + 1);
        s0 = ch[grp << lgm];
        s1 = ch[(grp + 1) << lgm];
    }
    // the launch provisioned shared memory for c0's rank table and run span
    // (the largest of a batch); a block needing more must not run
    if (HS > c0.HS || nc > c0.ncomb || span > c0.sd_span[lgm]) return;
    if (s0 >= s1) return;   // an unused run (the player has few tie groups)
    const int4 *seg4 = reinterpret_cast<const int4 *>(seg);   // {lo, hi, holds a traverser hand, 0}
    int4 sg = __ldg(seg4 + s0);
    const int run_lo = sg.x, run_hi = __ldg(seg + 4 * (s1 - 1) + 1);
    const int tid = threadIdx.x, lane = tid & 31;
    Carve cv{smem};
    Sd2State st;
    st.P = cv.take<double>(SD2_S * SD2_S);
    T *M1 = cv.take<T>(SD2_S * SD2_S);
    T *M2 = cv.take<T>(SD2_S * SD2_S);
    st.u1 = cv.take<double>(64);
    st.u2 = cv.take<double>(64);
    st.w = cv.take<double>(64);
    st.d = cv.take<double>(64);
    st.sc = cv.take<double>(8);
    double *cls = cv.take<double>(4 * span);   // per position of the run: A, T1, opponent 2 present, C
    char *rbuf = cv.take<char>(static_cast<int>(sd2_reach_bytes<T>(nc)));
    T *R1 = reinterpret_cast<T *>(rbuf);
    T *R2 = R1 + nc;
    unsigned short *dd = cv.take<unsigned short>(nc);
    short *pt = cv.take<short>(span);   // the traverser's hand at each position of the run, -1 if none
    int *last_pos = cv.take<int>(4);

    // opponents' reach and the cards by rank position, and the last position
    // holding positive reach of either opponent
    if (tid == 0) *last_pos = -1;
    if (tid < 64) {
        st.u1[tid] = 0.0;
        st.u2[tid] = 0.0;
        st.w[tid] = 0.0;
        st.d[tid] = 0.0;
    }
    __syncthreads();
    {
        const T *ra = reach + static_cast<size_t>(I.opp_row[0]) * HS;
        const T *rb = reach + static_cast<size_t>(I.opp_row[1]) * HS;
        const int *pa = pos_hand + static_cast<size_t>(o1) * nc, *pb = pos_hand + static_cast<size_t>(o2) * nc;
        int lp = -1;
#pragma unroll 4
        for (int q = tid; q < nc; q += kTermThreads) {
            const int ha = __ldg(pa + q), hb = __ldg(pb + q);
            const T x = ha >= 0 ? ra[ha] : T(0), y = hb >= 0 ? rb[hb] : T(0);
            R1[q] = x;
            R2[q] = y;
            dd[q] = static_cast<unsigned short>(cb[q].d1 | (cb[q].d2 << 8));
            if (x > T(0) || y > T(0)) lp = q;
        }
        atomicMax(last_pos, lp);
        const int *ph_t = pos_hand + static_cast<size_t>(trav) * nc + run_lo;
        for (int k = tid; k < run_hi - run_lo; k += kTermThreads) pt[k] = static_cast<short>(__ldg(ph_t + k));
    }
    __syncthreads();
    // this run starts from the state of every hand ranked below it
    sd2_direct_state(st, M1, M2, R1, R2, dd, run_lo);

    // segment entries come from global memory a step ahead of their use
    int4 nsg = s0 + 1 < s1 ? __ldg(seg4 + s0 + 1) : make_int4(0, 0, 0, 0);
    if (sg.z) {
        sd2_phase_a(st, M1, M2, R1, R2, dd, pt, cls, run_lo, sg.x, sg.y);
        __syncthreads();
    }
    for (int si = s0; si < s1; ++si) {
        const int lo = sg.x, hi = sg.y;
        const bool has = sg.z != 0, nhas = si + 1 < s1 && nsg.z != 0;
        sd2_add(st, dd, R1, M1, M2, st.u1, st.u2, 0, lo, hi);
        __syncthreads();
        sd2_add(st, dd, R2, M2, M1, st.u2, st.u1, 1, lo, hi);
        __syncthreads();
        // C of this group and A of the next group: the same state
        if (has) sd2_phase_mass(st, M1, M2, dd, pt, cls, run_lo, lo, hi, 3);
        if (nhas) sd2_phase_a(st, M1, M2, R1, R2, dd, pt, cls, run_lo, nsg.x, nsg.y);
        if (has || nhas) __syncthreads();
        sg = nsg;   // the next segment's entry is loaded a full step before its use
        if (si + 2 < s1) nsg = __ldg(seg4 + si + 2);
    }

    // all hands added (directly, unless this run ends the rank order): Z, and
    // the exact positive-pair count for hands whose mass is within the error
    // bound of zero (masks over the 47-card matrices, in the reach space)
    if (run_hi < nc) sd2_direct_state(st, M1, M2, R1, R2, dd, nc);
    ulonglong2 *Bm = reinterpret_cast<ulonglong2 *>(rbuf);
    Cr2Cnt *cnt = reinterpret_cast<Cr2Cnt *>(rbuf + 53 * sizeof(ulonglong2));
    Cr2Scalars *sc2 = reinterpret_cast<Cr2Scalars *>(rbuf + 53 * sizeof(ulonglong2) + 53 * sizeof(Cr2Cnt));
    if (tid < 2 * 64) {
        const int col = tid & 63;
        const T *M = tid < 64 ? M1 : M2;
        unsigned long long B = 0ull;
        if (col < SD2_S - 2)
            for (int r = 0; r < SD2_S - 2; ++r) B |= static_cast<unsigned long long>(M[r * SD2_S + col] > T(0)) << r;
        if (col <= kCr2Off) {
            if (tid < 64)
                Bm[col].x = B;
            else
                Bm[col].y = B;
        }
    }
    __syncthreads();
    if (tid <= kCr2Off) cnt[tid] = Cr2Cnt{__popcll(Bm[tid].x), __popcll(Bm[tid].y), 0, 0};
    __syncthreads();
    if (tid < 32) {
        int n1 = 0, n2 = 0, nq = 0, nd = 0;
        for (int k = lane; k <= kCr2Off; k += 32) {
            n1 += cnt[k].n1;
            n2 += cnt[k].n2;
            nq += cnt[k].n1 * cnt[k].n2;
            nd += __popcll(Bm[k].x & Bm[k].y);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n1 += __shfl_xor_sync(0xffffffffu, n1, o);
            n2 += __shfl_xor_sync(0xffffffffu, n2, o);
            nq += __shfl_xor_sync(0xffffffffu, nq, o);
            nd += __shfl_xor_sync(0xffffffffu, nd, o);
        }
        if (lane == 0) *sc2 = Cr2Scalars{0.0, 0.0, 0.0, n1 / 2, n2 / 2, nd / 2 - nq, 0};
    }
    __syncthreads();
    const Cr2Scalars S2 = *sc2;
    const double zmin = 1e-4 * st.sc[0] * st.sc[1];
    // payoff per class with the reference's float coefficients (pot / winners
    // - bet, or -bet): a coefficient that is exactly 0 drops its class exactly
    const double cw = static_cast<double>(I.pot - I.bet), c1 = static_cast<double>(I.pot / 2.0f - I.bet);
    const double c2 = static_cast<double>(I.pot / 3.0f - I.bet), cl = -static_cast<double>(I.bet);
    T *out = val + static_cast<size_t>(I.node) * HS;
    const int lastp = *last_pos;
    // the traverser's hands at this run's positions
    for (int q = run_lo + tid; q < run_hi; q += kTermThreads) {
        const int h = pt[q - run_lo];
        if (h < 0) continue;
        const unsigned short e = dd[q];
        const int a = sd2_c1(e), b = sd2_c2(e);
        const double Z = sd2_mass(st, M1, M2, a, b);
        const double *k4 = cls + 4 * (q - run_lo);
        const double A = k4[0], T1 = k4[1], C = k4[3];
        // no positive-reach opponent hand ranked above the group: the loss
        // class is empty, exactly (Z and C may come from different runs)
        const double L = __ldg(&cb[q].hi) > lastp ? 0.0 : Z - C;
        const double T2 = k4[2] != 0.0 ? (C - A) - T1 : 0.0;
        double v = cw * A + c1 * T1 + c2 * T2 + cl * L;
        if (fabs(Z) <= zmin && pair_count(Bm, cnt, a, b, S2.IF1, S2.IF2, S2.IQD) <= 0) v = 0.0;
        out[h] = static_cast<T>(v);
    }
    // the first block of the terminal also writes the hands without a rank
    // position (board-blocked) and the padding
    if (grp == 0) {
        const int *tp = sd_pos + static_cast<size_t>(trav) * HS;
        for (int h = tid; h < HS; h += kTermThreads)
            if (h >= Ht || __ldg(tp + h) < 0) out[h] = T(0);
    }
}

// Exact enumeration of opponent hand tuples, with the reference validity
// rules and payoffs (street_solve.cu:771-823 fold, :936-1002 showdown,
// :1079-1127 leaf).  One warp per (terminal, traverser hand): the tuple space
// (the opponents' hands in odometer order, the last opponent fastest) is cut
// into 32 contiguous runs, one per lane; each lane walks its run with an
// odometer and adds the positive products in FP64, and the lanes' sums are
// combined in a fixed order.  A block of 4 warps serves 4 hands; the blocks
// of a terminal stride over the subgame's hands.  Cost is the product of the
// opponents' range sizes; the planner only routes small cases here.
constexpr int kEnumWarps = 4;
template <class T>
__global__ void __launch_bounds__(32 * kEnumWarps) k_term_enum(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                               const TermItem *__restrict__ items, int nchunk,
                                                               int trav) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const TermItem I = items[it];
    if (retired(ctxs, I.sg)) return;
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    T *out = val_rows<T>(c) + static_cast<size_t>(I.node) * c.HS;
    const T *reach = reach_rows<T>(c);
    const int Ht = c.H[trav], HSs = c.HS;
    const size_t HS = static_cast<size_t>(HSs);
    const int k = I.k;
    const bool sd = I.kind_detail == 2;
    int radix[SS_MAX_PLAYERS - 1] = {1, 1, 1, 1, 1};
    long long ntup = 1;
    for (int i = 0; i < k; ++i) {
        radix[i] = c.H[I.opp_player[i]];
        ntup *= radix[i];
    }
    const long long per = (ntup + 31) / 32;
    const double tb = static_cast<double>(static_cast<T>(I.bet));
    for (int hb = ch; hb * kEnumWarps < HSs; hb += nchunk) {
        const int h = hb * kEnumWarps + warp;
        if (h >= HSs) break;
        if (h >= Ht) {
            if (lane == 0) out[h] = T(0);
            continue;
        }
        const int hc = c.hand_code[trav * HS + h];
        const int t0 = hc & 0xff, t1 = (hc >> 8) & 0xff;
        unsigned hs = 0;
        if (sd) {
            hs = c.strength[trav * HS + h];
            if (hs == 0) {
                if (lane == 0) out[h] = T(0);
                continue;
            }
        }
        // this lane's run of tuples [q0, q1), its first tuple's digits (an
        // opponent without hands leaves no tuple at all)
        const long long q0 = lane * per, q1 = q0 + per < ntup ? q0 + per : ntup;
        int idx[SS_MAX_PLAYERS - 1] = {0, 0, 0, 0, 0};
        if (q0 < q1) {
            long long q = q0;
            for (int i = k - 1; i >= 0; --i) {
                idx[i] = static_cast<int>(q % radix[i]);
                q /= radix[i];
            }
        }
        double total = 0.0;
        for (long long q = q0; q < q1; ++q) {
            int cards[SS_MAX_PLAYERS - 1][2];
            unsigned os[SS_MAX_PLAYERS - 1];
            T prod = T(1);
            bool ok = true;
            for (int i = 0; i < k && ok; ++i) {
                const int p = I.opp_player[i], o = idx[i];
                const int code = c.hand_code[p * HS + o];
                const int a0 = code & 0xff, a1 = (code >> 8) & 0xff;
                cards[i][0] = a0;
                cards[i][1] = a1;
                if (t0 == a0 || t0 == a1 || t1 == a0 || t1 == a1) { ok = false; break; }
                if (sd) {
                    os[i] = c.strength[p * HS + o];
                    if (os[i] == 0) { ok = false; break; }
                } else if (code & 0x10000) {
                    ok = false;
                    break;
                }
                prod *= reach[static_cast<size_t>(I.opp_row[i]) * HS + o];
                for (int j = 0; j < i; ++j)
                    if (a0 == cards[j][0] || a0 == cards[j][1] || a1 == cards[j][0] || a1 == cards[j][1]) {
                        ok = false;
                        break;
                    }
            }
            if (ok && prod > T(0)) {
                if (!sd) {
                    total += static_cast<double>(prod);
                } else {
                    unsigned best = hs;
                    for (int i = 0; i < k; ++i) best = os[i] > best ? os[i] : best;
                    if (hs < best) {
                        total += static_cast<double>(prod) * (-tb);
                    } else {
                        int wins = 1;
                        for (int i = 0; i < k; ++i) wins += os[i] == best ? 1 : 0;
                        // the reference's float payoff pot / winners - bet
                        const double pay = static_cast<double>(static_cast<T>(I.pot) / static_cast<T>(wins) -
                                                               static_cast<T>(I.bet));
                        total += static_cast<double>(prod) * pay;
                    }
                }
            }
            for (int j = k - 1; j >= 0; --j) {
                if (++idx[j] < radix[j]) break;
                idx[j] = 0;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
        if (lane == 0)
            out[h] = sd ? static_cast<T>(total) : static_cast<T>(static_cast<double>(term_factor(c, I, h)) * total);
    }
}

// Folds and leaves with three counted opponents (4+ player subgames): the
// card-removal mass by conditioning on the third opponent (ss_cr3.cuh), in
// FP64, one block per (group of terminals, chunk of kTermThreads traverser
// hands), one thread per hand; the first two opponents' aggregates are
// rebuilt by every chunk's block (O(deck^3), small beside the O(H3) walk of
// each hand).  A hand whose mass is within rounding of 0 takes the exact
// tuple count, and 0 when there is none (the reference adds only positive
// products).  Terminals on the same opponent reach rows (the traverser's own
// continuation choices) form a group: its first item's blocks write every
// member's row, each with its own factor.
constexpr size_t cr3_smem(int HS) {
    return (4 * cr3::kS * cr3::kS + 4 * cr3::kS + 8) * sizeof(double) + 4 * cr3::kS * sizeof(int) +
           2 * cr3::kS * sizeof(unsigned long long) + 8 * sizeof(long long) +
           static_cast<size_t>(HS) * (sizeof(double) + sizeof(unsigned short)) + 16 * 16;
}

template <class T>
__global__ void __launch_bounds__(kTermThreads, 2) k_term_cr3(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                             const TermItem *__restrict__ items, int nchunk,
                                                             int trav) {
    wait_prior_grid();
    extern __shared__ __align__(16) char smem[];
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const TermItem *I0 = items + it;
    if (I0->follow) return;   // written by the blocks of its group's first item
    if (retired(ctxs, I0->sg)) return;
    const int ng = I0->gextra + 1;
    const TermItem I = *I0;
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    const int HS = c.HS;
    // shared memory was provisioned for c0's row stride (the largest of a batch)
    if (HS > c0.HS || c.deck > cr3::kS - 1) return;
    const int h0 = ch * kTermThreads;
    if (h0 >= HS) return;
    Carve cv{smem};
    cr3::Tables t;
    t.A = cv.take<double>(cr3::kS * cr3::kS);
    t.B = cv.take<double>(cr3::kS * cr3::kS);
    t.P = cv.take<double>(cr3::kS * cr3::kS);
    t.PT = cv.take<double>(cr3::kS * cr3::kS);
    t.uA = cv.take<double>(cr3::kS);
    t.uB = cv.take<double>(cr3::kS);
    t.w = cv.take<double>(cr3::kS);
    t.d = cv.take<double>(cr3::kS);
    t.sc = cv.take<double>(8);
    t.iuA = cv.take<int>(cr3::kS);
    t.iuB = cv.take<int>(cr3::kS);
    t.iw = cv.take<int>(cr3::kS);
    t.id = cv.take<int>(cr3::kS);
    t.mA = cv.take<unsigned long long>(cr3::kS);
    t.mB = cv.take<unsigned long long>(cr3::kS);
    t.isc = cv.take<long long>(8);
    t.r3 = cv.take<double>(HS);
    t.xy = cv.take<unsigned short>(HS);
    const T *reach = reach_rows<T>(c);
    const size_t hs = static_cast<size_t>(HS);
    cr3::Opp3<T> in;
    in.r1 = reach + static_cast<size_t>(I.opp_row[0]) * hs;
    in.r2 = reach + static_cast<size_t>(I.opp_row[1]) * hs;
    in.r3 = reach + static_cast<size_t>(I.opp_row[2]) * hs;
    in.pair1 = c.pair_idx + static_cast<size_t>(I.opp_player[0]) * 52 * 52;
    in.pair2 = c.pair_idx + static_cast<size_t>(I.opp_player[1]) * 52 * 52;
    in.code3 = c.hand_code + static_cast<size_t>(I.opp_player[2]) * hs;
    in.H3 = c.H[I.opp_player[2]];
    in.HS = HS;
    in.deck = c.deck;
    const int tid = threadIdx.x;
    static_assert(kTermThreads == 256, "the device build steps assume 256 threads");
    cr3::gather_dev(tid, in, t, nullptr, 0, 0, nullptr, 0, 0);
    __syncthreads();
    cr3::build_step1(tid, t);
    if (tid == kTermThreads - 1) cr3::compact_third_list(in, t);
    __syncthreads();
    cr3::build_step2(tid, t);
    __syncthreads();
    const int h = h0 + tid;
    if (h >= HS) return;
    T *val = val_rows<T>(c);
    if (h >= c.H[trav]) {
        for (int g = 0; g < ng; ++g) val[static_cast<size_t>(I0[g].node) * hs + h] = T(0);
        return;
    }
    const double m = cr3::cr3_hand_value_mass(c.hand_code[static_cast<size_t>(trav) * hs + h], c.deck, t);
    for (int g = 0; g < ng; ++g) {
        const TermItem &Ig = I0[g];
        val[static_cast<size_t>(Ig.node) * hs + h] = static_cast<T>(static_cast<double>(term_factor(c, Ig, h)) * m);
    }
}

// Four-way showdowns (three live opponents): the traverser's class masses
// (ss_cr3.cuh) in FP64.  One block per (terminal, 256 rank positions), one
// thread per position (the traverser's hand there, if any).  The block
// builds the tables of the first two opponents' full matrices once (every
// tuple's mass, for the loss class and the exact zero), then walks the tie
// groups that meet its positions and, for a group holding a traverser hand,
// rebuilds them for the four pairs of the opponents' weaker / tying parts;
// the group's threads add the third opponent's hands by class.  A class
// mass within rounding of 0 takes its exact tuple count (0: exactly 0).
constexpr int kSd3Positions = 1081;   // C(47, 2): rank positions on every river board
constexpr int kSd3Warps = kTermThreads / 32;
// a tie group whose tying parts hold at most this many positive-reach hands
// of each of the first two opponents takes the sparse steps (grown weaker
// parts, tying pairs evaluated directly); a longer one rebuilds tables
constexpr int kSd3MaxE = 64;
// a table build in units of one D2 evaluation (the sparse steps' cost model)
constexpr double kSd3BuildCost = 3000.0;
constexpr size_t sd3_smem(int HS) {
    return cr3_smem(HS) + static_cast<size_t>(HS) * sizeof(int) + 16 + 3 * kTermThreads +
           2 * kSd3Warps * (sizeof(double) + sizeof(long long)) + 64 + 2 * kSd3MaxE * sizeof(cr3::EHand) + 16 + 64;
}

template <class T>
__global__ void __launch_bounds__(kTermThreads, 2) k_term_sd3(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                             const TermItem *__restrict__ items, int nchunk,
                                                             int trav) {
    wait_prior_grid();
    extern __shared__ __align__(16) char smem[];
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const TermItem I = items[it];
    if (retired(ctxs, I.sg)) return;
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    const int HS = c.HS;
    if (HS > c0.HS || c.deck > cr3::kS - 1) return;
    const size_t hs = static_cast<size_t>(HS);
    const int tid = threadIdx.x;
    T *out = val_rows<T>(c) + static_cast<size_t>(I.node) * hs;
    const int *tpos = c.sd_pos + static_cast<size_t>(trav) * hs;
    // the first chunk writes the hands without a rank position and the padding
    if (ch == 0)
        for (int h = tid; h < HS; h += kTermThreads)
            if (h >= c.H[trav] || tpos[h] < 0) out[h] = T(0);
    const int nc = c.ncomb;
    const int q0 = ch * kTermThreads;
    if (q0 >= nc) return;
    const int qend = min(q0 + kTermThreads, nc);
    Carve cv{smem};
    cr3::Tables t;
    t.A = cv.take<double>(cr3::kS * cr3::kS);
    t.B = cv.take<double>(cr3::kS * cr3::kS);
    t.P = cv.take<double>(cr3::kS * cr3::kS);
    t.PT = cv.take<double>(cr3::kS * cr3::kS);
    t.uA = cv.take<double>(cr3::kS);
    t.uB = cv.take<double>(cr3::kS);
    t.w = cv.take<double>(cr3::kS);
    t.d = cv.take<double>(cr3::kS);
    t.sc = cv.take<double>(8);
    t.iuA = cv.take<int>(cr3::kS);
    t.iuB = cv.take<int>(cr3::kS);
    t.iw = cv.take<int>(cr3::kS);
    t.id = cv.take<int>(cr3::kS);
    t.mA = cv.take<unsigned long long>(cr3::kS);
    t.mB = cv.take<unsigned long long>(cr3::kS);
    t.isc = cv.take<long long>(8);
    t.r3 = cv.take<double>(HS);
    t.xy = cv.take<unsigned short>(HS);
    int *p3 = cv.take<int>(HS);
    // per warp: the two class partials of one (hand, slice) of a tie group
    double *part = cv.take<double>(2 * kSd3Warps);
    long long *partc = cv.take<long long>(2 * kSd3Warps);
    // the traverser hand at each of the block's rank positions
    unsigned char *ga = cv.take<unsigned char>(kTermThreads);
    unsigned char *gb = cv.take<unsigned char>(kTermThreads);
    unsigned char *ghas = cv.take<unsigned char>(kTermThreads);
    // the current tie group's tying hands of the first two opponents, and their numbers
    cr3::EHand *elist1 = cv.take<cr3::EHand>(kSd3MaxE);
    cr3::EHand *elist2 = cv.take<cr3::EHand>(kSd3MaxE);
    int *en = cv.take<int>(2);
    const int lane = tid & 31, warp = tid >> 5;
    const T *reach = reach_rows<T>(c);
    const int o1 = I.opp_player[0], o2 = I.opp_player[1], o3 = I.opp_player[2];
    cr3::Opp3<T> in;
    in.r1 = reach + static_cast<size_t>(I.opp_row[0]) * hs;
    in.r2 = reach + static_cast<size_t>(I.opp_row[1]) * hs;
    in.r3 = reach + static_cast<size_t>(I.opp_row[2]) * hs;
    in.pair1 = c.pair_idx + static_cast<size_t>(o1) * 52 * 52;
    in.pair2 = c.pair_idx + static_cast<size_t>(o2) * 52 * 52;
    in.code3 = c.hand_code + static_cast<size_t>(o3) * hs;
    in.H3 = c.H[o3];
    in.HS = HS;
    in.deck = c.deck;
    const int *posA = c.sd_pos + static_cast<size_t>(o1) * hs;
    const int *posB = c.sd_pos + static_cast<size_t>(o2) * hs;
    const int *pre1 = c.pos_prefix + static_cast<size_t>(o1) * (nc + 1);
    const int *pre2 = c.pos_prefix + static_cast<size_t>(o2) * (nc + 1);
    // this thread's rank position and the traverser's hand there
    cr3::Sd3Thread st;
    cr3::sd3_thread_init(q0 + tid, qend, c.pos_hand + static_cast<size_t>(trav) * nc,
                         c.hand_code + static_cast<size_t>(trav) * hs, c.sd_combo, st);
    ga[tid] = static_cast<unsigned char>(st.a);
    gb[tid] = static_cast<unsigned char>(st.b);
    ghas[tid] = st.h >= 0;
    constexpr int kAll = 1 << 30;
    auto build = [&](int lo1, int hi1, int lo2, int hi2) {
        cr3::gather_dev(tid, in, t, posA, lo1, hi1, posB, lo2, hi2);
        __syncthreads();
        cr3::build_step1(tid, t);
        __syncthreads();
        cr3::build_step2(tid, t);
        __syncthreads();
    };
    cr3::compact_third(tid, in, t, c.sd_pos + static_cast<size_t>(o3) * hs, p3);
    build(0, kAll, 0, kAll);
    cr3::sd3_thread_total(st, t, p3);
    __syncthreads();
    // The tie groups meeting [q0, qend), the same walk in every thread.  For
    // each of a group's four pairs, its hands' class masses are sums over the
    // third opponent's list: the group's hands and slices of that list are
    // spread over the block's warps (per warps per hand, lanes splitting a
    // slice), and each hand's owner thread combines its warps' partials in
    // warp order.  A mass within rounding of 0 takes the exact tuple count
    // (a second pass of the same shape over the 0/1 tables).
    // the weaker parts' tables (positions [0, t_hi) of the first two
    // opponents), grown group by group while the groups' tying parts are short
    bool t_valid = false;
    int t_hi = 0;
    for (int g = q0; g < qend;) {
        const int lo = c.sd_combo[g].lo, hi = c.sd_combo[g].hi;
        const bool mine = st.h >= 0 && st.glo == lo;
        const int nmine = __syncthreads_count(mine);   // the traverser's hands of this group in the block
        const bool any = nmine > 0;
        // the group's tying hands of the first two opponents with positive
        // reach, in rank order (warp 0: first opponent, warp 1: second)
        if (warp < 2) {
            const int *ph = c.pos_hand + static_cast<size_t>(warp == 0 ? o1 : o2) * nc;
            const T *rr = warp == 0 ? in.r1 : in.r2;
            const int *code = c.hand_code + static_cast<size_t>(warp == 0 ? o1 : o2) * hs;
            cr3::EHand *E = warp == 0 ? elist1 : elist2;
            int n = 0;
            for (int base = lo; base < hi; base += 32) {
                const int q = base + lane;
                const int hh = q < hi ? ph[q] : -1;
                const T rv = hh >= 0 ? rr[hh] : T(0);
                const bool ok = hh >= 0 && rv > T(0);
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                const int at = n + __popc(bal & ((1u << lane) - 1u));
                if (ok && at < kSd3MaxE) {
                    const int hc = code[hh];
                    E[at] = cr3::EHand{static_cast<double>(rv), (hc >> 20) & 63, (hc >> 26) & 63};
                }
                n += __popc(bal);
            }
            if (lane == 0) en[warp] = n;
        }
        __syncthreads();
        const int n1 = en[0], n2 = en[1];
        const bool small = n1 <= kSd3MaxE && n2 <= kSd3MaxE;
        if (any) {
            // LL from the weaker parts' tables (grown along the walk, or built
            // here); a pair with a tying part is evaluated directly from them
            // when that costs less than building its own tables (direct: a
            // six-card one-opponent mass per tying hand and third-opponent
            // hand; built: a table build shared by the group's hands, then one
            // D2 per third-opponent hand) -- sparse ranges go direct, full
            // ranges build; the direct pairs run first, while the tables
            // still hold the weaker parts
            if (!(t_valid && t_hi == lo)) {
                build(0, lo, 0, lo);
                t_valid = true;
                t_hi = lo;
            }
            const double work = static_cast<double>(nmine) * static_cast<double>(t.isc[4]);
            auto go_direct = [&](int pr) {
                if (!small) return false;
                const double terms = pr == 1 ? n1 : pr == 2 ? n2 : 0.125 * n1 * n2;
                return work * (0.8 * terms) <= kSd3BuildCost + work;
            };
            int order[4] = {0, 0, 0, 0}, no = 1;
            for (int pr = 1; pr < 4; ++pr)
                if (go_direct(pr)) order[no++] = pr;
            for (int pr = 1; pr < 4; ++pr)
                if (!go_direct(pr)) order[no++] = pr;
            const int j0 = max(lo, q0) - q0, ng = min(hi, qend) - q0 - j0;
            const int per = ng >= kSd3Warps ? 1 : kSd3Warps / ng;   // warps per hand
            const int hpr = kSd3Warps / per;                          // hands per round
            const int r = warp / per, sl = warp - r * per;
            const int jl = tid - j0;                                  // this thread's index in the group
            auto walk = [&](int pr, bool direct, int base, bool want_count) {
                const int j = j0 + base + r;
                double o[2] = {0.0, 0.0};
                long long n[2] = {0, 0};
                if (r < hpr && base + r < ng && ghas[j]) {
                    if (direct)
                        cr3::e_pair_slice(pr, ga[j], gb[j], t, elist1, n1, elist2, n2, p3, lo, hi, sl * 32 + lane,
                                          per * 32, o, n);
                    else
                        cr3::hand_mass_cls_slice(ga[j], gb[j], t, p3, lo, hi, sl * 32 + lane, per * 32, o, n,
                                                 want_count);
                }
                for (int off = 16; off > 0; off >>= 1) {
                    o[0] += __shfl_xor_sync(0xffffffffu, o[0], off);
                    o[1] += __shfl_xor_sync(0xffffffffu, o[1], off);
                    n[0] += __shfl_xor_sync(0xffffffffu, n[0], off);
                    n[1] += __shfl_xor_sync(0xffffffffu, n[1], off);
                }
                if (lane == 0) {
                    part[2 * warp] = o[0];
                    part[2 * warp + 1] = o[1];
                    partc[2 * warp] = n[0];
                    partc[2 * warp + 1] = n[1];
                }
                __syncthreads();
            };
            for (int step = 0; step < 4; ++step) {
                const int pr = order[step];
                int lo1, hi1, lo2, hi2;
                cr3::sd3_pair_bounds(pr, lo, hi, &lo1, &hi1, &lo2, &hi2);
                // an opponent without a hand in its part of the pair: no
                // tuple, both class masses exactly 0 (what the tables and the
                // exact count would give), no tables to build
                if (pre1[hi1] == pre1[lo1] || pre2[hi2] == pre2[lo2]) {
                    if (mine) st.m[pr][0] = st.m[pr][1] = 0.0;
                    continue;
                }
                // direct: a pair with a short tying part, from the weaker
                // parts' tables and the lists (masses and exact counts in one
                // walk); otherwise the pair's own tables
                const bool direct = pr > 0 && go_direct(pr);
                if (pr > 0 && !direct) {
                    build(lo1, hi1, lo2, hi2);
                    t_valid = false;   // the pair's tables replace the weaker parts'
                }
                const double zb = cr3::zero_bound(t);
                bool near_zero = false;
                for (int base = 0; base < ng; base += hpr) {
                    walk(pr, direct, base, false);
                    if (mine && jl >= base && jl < base + hpr) {
                        double m0 = 0.0, m1 = 0.0;
                        long long c0 = 0, c1 = 0;
                        for (int k = 0; k < per; ++k) {
                            m0 += part[2 * ((jl - base) * per + k)];
                            m1 += part[2 * ((jl - base) * per + k) + 1];
                            c0 += partc[2 * ((jl - base) * per + k)];
                            c1 += partc[2 * ((jl - base) * per + k) + 1];
                        }
                        if (direct) {
                            st.m[pr][0] = c0 == 0 ? 0.0 : m0;
                            st.m[pr][1] = c1 == 0 ? 0.0 : m1;
                        } else {
                            st.m[pr][0] = m0;
                            st.m[pr][1] = m1;
                            near_zero = fabs(m0) <= zb || fabs(m1) <= zb;
                        }
                    }
                    __syncthreads();
                }
                if (__syncthreads_or(near_zero)) {
                    for (int base = 0; base < ng; base += hpr) {
                        walk(pr, false, base, true);
                        if (mine && jl >= base && jl < base + hpr)
                            for (int cls = 0; cls < 2; ++cls) {
                                long long n = 0;
                                for (int k = 0; k < per; ++k) n += partc[2 * ((jl - base) * per + k) + cls];
                                if (fabs(st.m[pr][cls]) <= zb && n == 0) st.m[pr][cls] = 0.0;
                            }
                        __syncthreads();
                    }
                }
            }
        }
        // advance the weaker parts' tables past this group: its tying hands
        // join the first opponent's side, then the second's
        if (t_valid && t_hi == lo) {
            if (!small) {
                t_valid = false;
            } else {
                if (n1 > 0) {
                    cr3::add_hands(tid, kTermThreads, t, 0, elist1, n1);
                    __syncthreads();
                }
                if (n2 > 0) {
                    cr3::add_hands(tid, kTermThreads, t, 1, elist2, n2);
                    __syncthreads();
                }
                t_hi = hi;
            }
        }
        g = hi;
    }
    if (st.h >= 0) out[st.h] = static_cast<T>(cr3::sd3_thread_value(st, I.pot, I.bet));
}

// --------------------------------------------------------------------------
// best response (FP64): exploitability of an average-strategy profile
// avg[(di * 8 + a) * max_h + h] (the SSOutput layout)
// --------------------------------------------------------------------------

__device__ __forceinline__ double avg_sigma(const float *avg, int di, int a, int h, int max_h, int frozen) {
    if (frozen >= 0) return a == frozen ? 1.0 : 0.0;
    return static_cast<double>(avg[(static_cast<size_t>(di) * SS_MAX_ACTIONS + a) * max_h + h]);
}

// reach of one player under the average strategy
__global__ void __launch_bounds__(128) k_br_reach(DevCtx c, const ReachItem *__restrict__ items, int nchunk,
                                                  int H, const float *__restrict__ avg,
                                                  const int *__restrict__ edge_di, int max_h) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const int h = (blockIdx.x - it * nchunk) * blockDim.x + threadIdx.x;
    if (h >= H) return;
    const ReachItem I = items[it];
    const size_t HS = static_cast<size_t>(c.HS);
    const int di = edge_di[I.first_edge];
    const double pr = c.reach_d[static_cast<size_t>(I.parent_row) * HS + h];
    for (int a = 0; a < I.na; ++a)
        c.reach_d[static_cast<size_t>(I.first_edge + a) * HS + h] = pr * avg_sigma(avg, di, a, h, max_h, I.frozen);
}

// value of the traverser's nodes: mode 0 follows the profile, mode 1 takes
// the best action (a pure best response per information set; a frozen node
// keeps its frozen action)
__global__ void __launch_bounds__(128) k_br_value(DevCtx c, const CfvItem *__restrict__ items, int nchunk,
                                                  int H, const float *__restrict__ avg,
                                                  const int *__restrict__ edge_di, int max_h, int mode) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const int h = (blockIdx.x - it * nchunk) * blockDim.x + threadIdx.x;
    if (h >= H) return;
    const CfvItem I = items[it];
    const size_t HS = static_cast<size_t>(c.HS);
    const int di = edge_di[I.first_edge];
    double v = mode == 1 ? -1e300 : 0.0;
    double vf = 0.0;
    for (int a = 0; a < I.na; ++a) {
        double e = 0.0;
        for (int k = c.fr_off[I.first_edge + a]; k < c.fr_off[I.first_edge + a + 1]; ++k)
            e += c.val_d[static_cast<size_t>(c.fr_items[k]) * HS + h];
        if (mode == 1) {
            v = e > v ? e : v;
            if (a == I.frozen) vf = e;
        } else {
            v += avg_sigma(avg, di, a, h, max_h, I.frozen) * e;
        }
    }
    if (mode == 1 && I.frozen >= 0 && I.frozen < I.na) v = vf;
    c.val_d[static_cast<size_t>(I.node) * HS + h] = v;
}

// out = sum over hands h < H of weight(h) * (sum over rows of val_d[row][h]);
// the weights are the traverser's range (reach_d row weight_row); with
// skip_blocked, hands touching the board do not count.  One block, fixed
// reduction order.
__global__ void __launch_bounds__(1024) k_br_root(DevCtx c, const int *__restrict__ rows, int n, int H,
                                                  int weight_row, int trav, int skip_blocked, double *out) {
    wait_prior_grid();
    __shared__ double part[32];
    const size_t HS = static_cast<size_t>(c.HS);
    double acc = 0.0;
    for (int h = threadIdx.x; h < H; h += blockDim.x) {
        if (skip_blocked && (c.hand_code[trav * HS + h] & 0x10000)) continue;
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += c.val_d[static_cast<size_t>(rows[k]) * HS + h];
        acc += c.reach_d[static_cast<size_t>(weight_row) * HS + h] * s;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < blockDim.x / 32 ? part[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) *out = v;
    }
}

// Batched best response: the kernels above with every item reading its own
// subgame's context (its FP64 rows, profile and tables); blocks of subgames
// that have left the batch return at once.
__global__ void __launch_bounds__(128) k_avg_many(const DevCtx *__restrict__ ctxs,
                                                  const AvgItem *__restrict__ items, int nchunk) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const AvgItem I = items[it];
    if (!ctxs[I.sg].live) return;
    const DevCtx &c = ctxs[I.sg];
    const int h = (blockIdx.x - it * nchunk) * blockDim.x + threadIdx.x;
    const int max_h = c.max_h;
    if (h >= max_h) return;
    const int fe = c.dec_fe[I.di], na = c.dec_na[I.di], p = c.dec_pl[I.di];
    float *o = c.avg_br + static_cast<size_t>(I.di) * SS_MAX_ACTIONS * max_h;
    if (h >= c.H[p]) {
        for (int a = 0; a < SS_MAX_ACTIONS; ++a) o[static_cast<size_t>(a) * max_h + h] = 0.f;
        return;
    }
    float v[SS_MAX_ACTIONS];
    float sum = 0.f;
    for (int a = 0; a < na; ++a) {
        float x = c.S[static_cast<size_t>(fe + a) * c.HS + h];
        x = x < 0.f ? 0.f : x;
        v[a] = x;
        sum += x;
    }
    const float inv = sum > 0.f ? 1.0f / sum : 1.0f / static_cast<float>(na);
    for (int a = 0; a < SS_MAX_ACTIONS; ++a)
        o[static_cast<size_t>(a) * max_h + h] = a < na ? (sum > 0.f ? v[a] * inv : inv) : 0.f;
}

__global__ void __launch_bounds__(128) k_br_reach_many(const DevCtx *__restrict__ ctxs,
                                                       const ReachItem *__restrict__ items, int nchunk, int p) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const ReachItem I = items[it];
    if (!ctxs[I.sg].live) return;
    const DevCtx &c = ctxs[I.sg];
    const int h = (blockIdx.x - it * nchunk) * blockDim.x + threadIdx.x;
    if (h >= c.H[p]) return;
    const size_t HS = static_cast<size_t>(c.HS);
    const int di = c.edge_di[I.first_edge];
    const double pr = c.reach_d[static_cast<size_t>(I.parent_row) * HS + h];
    for (int a = 0; a < I.na; ++a)
        c.reach_d[static_cast<size_t>(I.first_edge + a) * HS + h] = pr * avg_sigma(c.avg_br, di, a, h, c.max_h, I.frozen);
}

__global__ void __launch_bounds__(128) k_br_value_many(const DevCtx *__restrict__ ctxs,
                                                       const CfvItem *__restrict__ items, int nchunk, int trav,
                                                       int mode) {
    wait_prior_grid();
    const int it = blockIdx.x / nchunk;
    const CfvItem I = items[it];
    if (!ctxs[I.sg].live) return;
    const DevCtx &c = ctxs[I.sg];
    const int h = (blockIdx.x - it * nchunk) * blockDim.x + threadIdx.x;
    if (h >= c.H[trav]) return;
    const size_t HS = static_cast<size_t>(c.HS);
    const int di = c.edge_di[I.first_edge];
    double v = mode == 1 ? -1e300 : 0.0;
    double vf = 0.0;
    for (int a = 0; a < I.na; ++a) {
        double e = 0.0;
        for (int k = c.fr_off[I.first_edge + a]; k < c.fr_off[I.first_edge + a + 1]; ++k)
            e += c.val_d[static_cast<size_t>(c.fr_items[k]) * HS + h];
        if (mode == 1) {
            v = e > v ? e : v;
            if (a == I.frozen) vf = e;
        } else {
            v += avg_sigma(c.avg_br, di, a, h, c.max_h, I.frozen) * e;
        }
    }
    if (mode == 1 && I.frozen >= 0 && I.frozen < I.na) v = vf;
    c.val_d[static_cast<size_t>(I.node) * HS + h] = v;
}

// one block per item, same fixed reduction order as k_br_root
__global__ void __launch_bounds__(1024) k_br_root_many(const DevCtx *__restrict__ ctxs,
                                                       const RootItem *__restrict__ items, double *out) {
    wait_prior_grid();
    __shared__ double part[32];
    const RootItem I = items[blockIdx.x];
    if (!ctxs[I.sg].live) return;
    const DevCtx &c = ctxs[I.sg];
    const size_t HS = static_cast<size_t>(c.HS);
    const int H = c.H[I.trav];
    double acc = 0.0;
    for (int h = threadIdx.x; h < H; h += blockDim.x) {
        if (I.skip_blocked && (c.hand_code[I.trav * HS + h] & 0x10000)) continue;
        double s = 0.0;
        for (int k = 0; k < I.n; ++k) s += c.val_d[static_cast<size_t>(I.rows[k]) * HS + h];
        acc += c.reach_d[static_cast<size_t>(I.weight_row) * HS + h] * s;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < blockDim.x / 32 ? part[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) out[I.slot] = v;
    }
}

// batched form: advance the iteration counter of every listed subgame
__global__ void k_bump_many(const DevCtx *__restrict__ ctxs, const int *__restrict__ sgs, int n) {
    wait_prior_grid();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && ctxs[sgs[i]].live) *const_cast<int *>(ctxs[sgs[i]].iter) += 1;
}

// batched form: root strategy snapshot (regret matching of the root node)
// of every listed subgame, one block per subgame, into its ctx.snap
__global__ void __launch_bounds__(128) k_snapshot_many(const DevCtx *__restrict__ ctxs,
                                                       const int *__restrict__ sgs) {
    wait_prior_grid();
    const DevCtx &c = ctxs[sgs[blockIdx.x]];
    if (!c.live) return;
    const int H = c.H[c.root_player];
    for (int h0 = threadIdx.x * 4; h0 < H; h0 += blockDim.x * 4) {
        float r[SS_MAX_ACTIONS][4], sig[SS_MAX_ACTIONS][4];
        regret_match4(c.R, static_cast<size_t>(c.HS), c.root_fe, c.root_na, c.root_frozen, h0, r, sig);
        for (int a = 0; a < c.root_na; ++a)
            for (int i = 0; i < 4; ++i)
                if (h0 + i < H) c.snap[static_cast<size_t>(a) * H + h0 + i] = sig[a][i];
    }
}

__global__ void k_bump(int *iter) {
    wait_prior_grid(); *iter += 1; }

// out[h] = sum over rows of val[row][h]
__global__ void __launch_bounds__(kHandThreads) k_sum_rows(DevCtx c, const int *__restrict__ rows, int n,
                                                           float *out, int H) {
    wait_prior_grid();
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= H) return;
    float s = 0.f;
    for (int k = 0; k < n; ++k) s += c.val[static_cast<size_t>(rows[k]) * c.HS + h];
    out[h] = s;
}

// regret-matched (and frozen) strategy of one node, [na][H] (street_solve.cu:1564-1573)
__global__ void __launch_bounds__(kHandThreads) k_root_strategy(DevCtx c, int fe, int na, int frozen,
                                                                int H, float *out) {
    wait_prior_grid();
    const int h0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (h0 >= H) return;
    float r[SS_MAX_ACTIONS][4], sig[SS_MAX_ACTIONS][4];
    regret_match4(c.R, static_cast<size_t>(c.HS), fe, na, frozen, h0, r, sig);
    for (int a = 0; a < na; ++a)
        for (int i = 0; i < 4; ++i)
            if (h0 + i < H) out[static_cast<size_t>(a) * H + h0 + i] = sig[a][i];
}

// normalised strategy sums of every decision node in the output layout
// [num_dec][8][max_h] (street_solve.cu:1589-1612)
__global__ void __launch_bounds__(128) k_avg_strategy(DevCtx c, const int *__restrict__ dec_fe,
                                                      const int *__restrict__ dec_na,
                                                      const int *__restrict__ dec_player, int nchunk,
                                                      int max_h, float *out) {
    wait_prior_grid();
    const int di = blockIdx.x / nchunk;
    const int h = (blockIdx.x - di * nchunk) * blockDim.x + threadIdx.x;
    if (h >= max_h) return;
    const int fe = dec_fe[di], na = dec_na[di], p = dec_player[di];
    float *o = out + static_cast<size_t>(di) * SS_MAX_ACTIONS * max_h;
    if (h >= c.H[p]) {
        for (int a = 0; a < SS_MAX_ACTIONS; ++a) o[static_cast<size_t>(a) * max_h + h] = 0.f;
        return;
    }
    float v[SS_MAX_ACTIONS];
    float sum = 0.f;
    for (int a = 0; a < na; ++a) {
        float x = c.S[static_cast<size_t>(fe + a) * c.HS + h];
        x = x < 0.f ? 0.f : x;
        v[a] = x;
        sum += x;
    }
    const float inv = sum > 0.f ? 1.0f / sum : 1.0f / static_cast<float>(na);
    for (int a = 0; a < SS_MAX_ACTIONS; ++a)
        o[static_cast<size_t>(a) * max_h + h] = a < na ? (sum > 0.f ? v[a] * inv : inv) : 0.f;
}

inline int chunks(int H) { return (H + kHandsPerBlock - 1) / kHandsPerBlock; }

// The tensor-core form of the two-opponent terminals serves dense decks of
// at most 48 cards (turn and river boards) without repeated combos; c is the
// launch's context (for a batch: the largest deck and the OR of every
// member's repeated-combo flags).  It is taken only with SSB_CR2_TENSOR=1 in
// the environment: measured on the 3-player turn it is slower than the
// mma.sync form (0.70 vs 0.55 ms of two-opponent terminals per iteration) --
// its operand space (55 KB per block) leaves four blocks per SM instead of
// five, and a block's time is set by its serial phases, not the product.
bool tensor_product_serves(const DevCtx &c) {
    static const bool on = [] {
        const char *v = std::getenv("SSB_CR2_TENSOR");
        return v && v[0] == '1';
    }();
    if (!on || c.deck <= 0 || c.deck > kTcRows) return false;
    for (int p = 0; p < SS_MAX_PLAYERS; ++p)
        if (c.dup[p]) return false;
    return true;
}

}  // namespace

bool cr2_tensor_form(const DevCtx &c) { return tensor_product_serves(c); }

cudaError_t read_device_fault(unsigned *code, cudaStream_t s) {
    *code = 0;
    cudaError_t e = cudaMemcpyFromSymbolAsync(code, g_ss_fault, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && *code) {
        static const unsigned zero = 0;
        e = cudaMemcpyToSymbolAsync(g_ss_fault, &zero, sizeof(unsigned), 0, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    return e;
}

cudaError_t launch_reach(const DevCtx &c, const ReachItem *items, int n, int H, cudaStream_t s,
                         const DevCtx *ctxs, int player) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = chunks(H);
    SSB_LAUNCH(k_reach, n * nc, kHandThreads, 0, s, c, ctxs, items, nc, H, player);
    return cudaGetLastError();
}

cudaError_t launch_cfv(const DevCtx &c, const CfvItem *items, int n, int n_long, int H, cudaStream_t s,
                       const DevCtx *ctxs, int trav) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    n_long = n_long < 0 ? 0 : n_long > n ? n : n_long;
    const int n_short = n - n_long;
    if (n_short > 0) {
        const int nc = (H + 2 * kCfvThreads - 1) / (2 * kCfvThreads);
        SSB_LAUNCH(k_cfv<1>, n_short * nc, kCfvThreads, 0, s, c, ctxs, items, nc, H, trav);
    }
    if (n_long > 0) {
        const int nc = (H + 63) / 64;
        static_assert(32 * kCfvSplit == kCfvThreads, "the split form fills one block of kCfvThreads");
        SSB_LAUNCH(k_cfv<kCfvSplit>, n_long * nc, kCfvThreads, 0, s, c, ctxs, items + n_short, nc, H, trav);
    }
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_terms_t(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                           cudaStream_t s, const DevCtx *ctxs, const int *heads = nullptr, int n_heads = 0) {
    if (n <= 0 || (heads && n_heads <= 0)) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    switch (kind) {
        case TK_ZERO:
        case TK_LEAF0: {
            const int nc = chunks(c.HS);
            SSB_LAUNCH(k_term_fill<T>, n * nc, kHandThreads, 0, s, c, ctxs, items, nc, trav, kind == TK_ZERO);
            break;
        }
        case TK_CR1: {
            const size_t sm = cr1_gather_smem<T>(c.HS);
            if (sm > 48 * 1024)
                e = cudaFuncSetAttribute(k_term_cr1<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(cr1_gather_smem<T>(kMaxHS)));
            if (e != cudaSuccess) return e;
            SSB_LAUNCH(k_term_cr1<T>, n, kTermThreads, sm, s, c, ctxs, items, trav);
            break;
        }
        case TK_CR1D:
            SSB_LAUNCH(k_term_cr1_dup<T>, n, kTermThreads, cr1_smem<T>(), s, c, ctxs, items, trav);
            break;
        case TK_CR2: {
            // c.HS: the row stride (the largest of a batch); the staging of two
            // reach rows in the product's space needs HS <= kMaxHS
            if (c.HS > kMaxHS) return cudaErrorInvalidValue;
            if constexpr (sizeof(T) == 4) {
                if (tensor_product_serves(c)) {
                    e = cudaFuncSetAttribute(k_term_cr2_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(cr2_tc_smem(kMaxHS)));
                    if (e != cudaSuccess) return e;
                    SSB_LAUNCH(k_term_cr2_tc, n, kTermThreads, cr2_tc_smem(c.HS), s, c, ctxs, items, trav);
                    break;
                }
            }
            const size_t sm = cr2_smem<T>(c.HS);
            if (sm > 48 * 1024)
                e = cudaFuncSetAttribute(k_term_cr2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(cr2_smem<T>(kMaxHS)));
            if (e != cudaSuccess) return e;
            SSB_LAUNCH(k_term_cr2<T>, heads ? n_heads : n, kTermThreads, sm, s, c, ctxs, items, heads, trav);
            break;
        }
        case TK_SD1:
            if (sd1_smem<T>() > 48 * 1024)
                e = cudaFuncSetAttribute(k_term_sd1<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(sd1_smem<T>()));
            if (e != cudaSuccess) return e;
            SSB_LAUNCH(k_term_sd1<T>, n, kTermThreads, sd1_smem<T>(), s, c, ctxs, items, trav);
            break;
        case TK_SD2: {
            // runs per block: about two waves of four blocks per SM at most
            const int lgm = sd2_merge_of(n);
            const size_t sm = sd2_smem<T>(c.sd_span[lgm], c.ncomb);
            e = cudaFuncSetAttribute(k_term_sd2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
            if (e != cudaSuccess) return e;
            SSB_LAUNCH(k_term_sd2<T>, n * (kSd2Chunks >> lgm), kTermThreads, sm, s, c, ctxs, items, trav, lgm, nullptr);
            break;
        }
        case TK_ENUM: {
            // blocks per terminal: one per 4 hands, at most 16 (they stride
            // over a larger range; a batch's c.HS is its largest row stride)
            const int nc = std::min((c.HS + kEnumWarps - 1) / kEnumWarps, 16);
            SSB_LAUNCH(k_term_enum<T>, n * nc, 32 * kEnumWarps, 0, s, c, ctxs, items, nc, trav);
            break;
        }
        case TK_SD3: {
            // the grid covers the 1081 rank positions of a river board
            if (c.HS > kMaxHS || c.ncomb > kSd3Positions) return cudaErrorInvalidValue;
            const int nc = (kSd3Positions + kTermThreads - 1) / kTermThreads;
            e = cudaFuncSetAttribute(k_term_sd3<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(sd3_smem(kMaxHS)));
            if (e != cudaSuccess) return e;
            SSB_LAUNCH(k_term_sd3<T>, n * nc, kTermThreads, sd3_smem(c.HS), s, c, ctxs, items, nc, trav);
            break;
        }
        case TK_CR3: {
            if (c.HS > kMaxHS) return cudaErrorInvalidValue;
            const int nc = (c.HS + kTermThreads - 1) / kTermThreads;
            e = cudaFuncSetAttribute(k_term_cr3<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(cr3_smem(kMaxHS)));
            if (e != cudaSuccess) return e;
            SSB_LAUNCH(k_term_cr3<T>, n * nc, kTermThreads, cr3_smem(c.HS), s, c, ctxs, items, nc, trav);
            break;
        }
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_terms(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                         cudaStream_t s, const DevCtx *ctxs, const int *heads, int n_heads) {
    return launch_terms_t<float>(c, kind, items, n, trav, s, ctxs, heads, n_heads);
}

template <class T>
cudaError_t launch_sd2_mapped_t(const DevCtx &c, const TermItem *items, const int2 *bmap, int nblocks, int lg_max,
                                int trav, cudaStream_t s, const DevCtx *ctxs) {
    if (nblocks <= 0) return cudaSuccess;
    const size_t sm = sd2_smem<T>(c.sd_span[lg_max], c.ncomb);
    cudaError_t e =
        cudaFuncSetAttribute(k_term_sd2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
    if (e != cudaSuccess) return e;
    SSB_LAUNCH(k_term_sd2<T>, nblocks, kTermThreads, sm, s, c, ctxs, items, trav, 0, bmap);
    return cudaGetLastError();
}

cudaError_t launch_sd2_mapped(const DevCtx &c, const TermItem *items, const int2 *bmap, int nblocks, int lg_max,
                              int trav, cudaStream_t s, const DevCtx *ctxs, bool fp64) {
    return fp64 ? launch_sd2_mapped_t<double>(c, items, bmap, nblocks, lg_max, trav, s, ctxs)
                : launch_sd2_mapped_t<float>(c, items, bmap, nblocks, lg_max, trav, s, ctxs);
}

cudaError_t launch_terms_fp64(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                              cudaStream_t s, const DevCtx *ctxs) {
    return launch_terms_t<double>(c, kind, items, n, trav, s, ctxs);
}

cudaError_t launch_avg_many(const DevCtx *ctxs, const AvgItem *items, int n, int max_h, cudaStream_t s) {
    if (n <= 0 || max_h <= 0) return cudaSuccess;
    const int nc = (max_h + 127) / 128;
    SSB_LAUNCH(k_avg_many, n * nc, 128, 0, s, ctxs, items, nc);
    return cudaGetLastError();
}

cudaError_t launch_br_reach_many(const DevCtx *ctxs, const ReachItem *items, int n, int H, int player,
                                 cudaStream_t s) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = (H + 127) / 128;
    SSB_LAUNCH(k_br_reach_many, n * nc, 128, 0, s, ctxs, items, nc, player);
    return cudaGetLastError();
}

cudaError_t launch_br_value_many(const DevCtx *ctxs, const CfvItem *items, int n, int H, int trav, int mode,
                                 cudaStream_t s) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = (H + 127) / 128;
    SSB_LAUNCH(k_br_value_many, n * nc, 128, 0, s, ctxs, items, nc, trav, mode);
    return cudaGetLastError();
}

cudaError_t launch_br_root_many(const DevCtx *ctxs, const RootItem *items, int n, double *out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    SSB_LAUNCH(k_br_root_many, n, 1024, 0, s, ctxs, items, out);
    return cudaGetLastError();
}

cudaError_t launch_bump(int *iter, cudaStream_t s) {
    SSB_LAUNCH(k_bump, 1, 1, 0, s, iter);
    return cudaGetLastError();
}

cudaError_t launch_sum_rows(const DevCtx &c, const int *rows, int n, float *out, int H,
                            cudaStream_t s) {
    if (H <= 0) return cudaSuccess;
    SSB_LAUNCH(k_sum_rows, (H + kHandThreads - 1) / kHandThreads, kHandThreads, 0, s, c, rows, n, out, H);
    return cudaGetLastError();
}

cudaError_t launch_root_strategy(const DevCtx &c, int first_edge, int na, int frozen, int H,
                                 float *out, cudaStream_t s) {
    if (H <= 0) return cudaSuccess;
    SSB_LAUNCH(k_root_strategy, (H + kHandsPerBlock - 1) / kHandsPerBlock, kHandThreads, 0, s,
               c, first_edge, na, frozen, H, out);
    return cudaGetLastError();
}

cudaError_t launch_avg_strategy(const DevCtx &c, const int *dec_fe, const int *dec_na,
                                const int *dec_player, int num_dec, int max_h, float *out,
                                cudaStream_t s) {
    if (num_dec <= 0) return cudaSuccess;
    const int nc = (max_h + 127) / 128;
    SSB_LAUNCH(k_avg_strategy, num_dec * nc, 128, 0, s, c, dec_fe, dec_na, dec_player, nc, max_h, out);
    return cudaGetLastError();
}

cudaError_t launch_br_reach(const DevCtx &c, const ReachItem *items, int n, int H, const float *avg,
                            const int *edge_di, int max_h, cudaStream_t s) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = (H + 127) / 128;
    SSB_LAUNCH(k_br_reach, n * nc, 128, 0, s, c, items, nc, H, avg, edge_di, max_h);
    return cudaGetLastError();
}

cudaError_t launch_br_value(const DevCtx &c, const CfvItem *items, int n, int H, const float *avg,
                            const int *edge_di, int max_h, int mode, cudaStream_t s) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = (H + 127) / 128;
    SSB_LAUNCH(k_br_value, n * nc, 128, 0, s, c, items, nc, H, avg, edge_di, max_h, mode);
    return cudaGetLastError();
}

cudaError_t launch_br_root(const DevCtx &c, const int *rows, int n, int H, int weight_row, int trav,
                           int skip_blocked, double *out, cudaStream_t s) {
    SSB_LAUNCH(k_br_root, 1, 1024, 0, s, c, rows, n, H, weight_row, trav, skip_blocked, out);
    return cudaGetLastError();
}

cudaError_t launch_bump_many(const DevCtx *ctxs, const int *sgs, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    SSB_LAUNCH(k_bump_many, (n + 127) / 128, 128, 0, s, ctxs, sgs, n);
    return cudaGetLastError();
}

cudaError_t launch_snapshot_many(const DevCtx *ctxs, const int *sgs, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    SSB_LAUNCH(k_snapshot_many, n, 128, 0, s, ctxs, sgs);
    return cudaGetLastError();
}

}  // namespace ssb
