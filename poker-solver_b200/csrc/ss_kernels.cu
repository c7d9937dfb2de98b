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

namespace ssb {

namespace {

constexpr int MS = 52;  // shared-memory row stride of a 52x52 combo matrix (16-byte rows)

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
__global__ void __launch_bounds__(kHandThreads) k_reach(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                        const ReachItem *__restrict__ items, int nchunk, int H,
                                                        int p) {
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kHandThreads + threadIdx.x) * 4;
    const ReachItem I = items[it];
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    if (h0 >= (ctxs ? c.H[p] : H)) return;
    const size_t HS = static_cast<size_t>(c.HS);
    float r[SS_MAX_ACTIONS][4], sig[SS_MAX_ACTIONS][4];
    regret_match4(c.R, HS, I.first_edge, I.na, I.frozen, h0, r, sig);
    const float4 pr = ld4(c.reach + static_cast<size_t>(I.parent_row) * HS + h0);
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            float4 o;
            o.x = pr.x * sig[a][0];
            o.y = pr.y * sig[a][1];
            o.z = pr.z * sig[a][2];
            o.w = pr.w * sig[a][3];
            st4(c.reach + static_cast<size_t>(I.first_edge + a) * HS + h0, o);
        }
    }
}

// --------------------------------------------------------------------------
// cfv: value, regret and strategy-sum update at traverser nodes
// (street_solve.cu:1155-1175): v = sum_a sigma_a ev_a; r_a = (r_a + (ev_a - v))
// * t/(t+1); s_a += t * sigma_a; ev_a = sum of val over frontier(edge a).
// Each thread owns 2 hands.  Edge values are gathered first (four frontier
// rows in flight at a time), then the regrets are loaded and matched, which
// keeps the live state to the edge values and regrets.
// --------------------------------------------------------------------------
__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }

__global__ void __launch_bounds__(kCfvThreads) k_cfv(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                     const CfvItem *__restrict__ items, int nchunk, int Hl,
                                                     int trav) {
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kCfvThreads + threadIdx.x) * 2;
    const CfvItem I = items[it];
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    const int H = ctxs ? c.H[trav] : Hl;
    if (h0 >= H) return;
    const size_t HS = static_cast<size_t>(c.HS);
    const float *val = c.val + h0;
    float2 ev[SS_MAX_ACTIONS];
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            float2 e = make_float2(0.f, 0.f);
            int k = c.fr_off[I.first_edge + a];
            const int k1 = c.fr_off[I.first_edge + a + 1];
            for (; k + 4 <= k1; k += 4) {
                const int n0 = c.fr_items[k], n1 = c.fr_items[k + 1];
                const int n2 = c.fr_items[k + 2], n3 = c.fr_items[k + 3];
                const float2 x0 = ld2(val + static_cast<size_t>(n0) * HS);
                const float2 x1 = ld2(val + static_cast<size_t>(n1) * HS);
                const float2 x2 = ld2(val + static_cast<size_t>(n2) * HS);
                const float2 x3 = ld2(val + static_cast<size_t>(n3) * HS);
                e.x += x0.x; e.y += x0.y;
                e.x += x1.x; e.y += x1.y;
                e.x += x2.x; e.y += x2.y;
                e.x += x3.x; e.y += x3.y;
            }
            for (; k < k1; ++k) {
                const float2 x = ld2(val + static_cast<size_t>(c.fr_items[k]) * HS);
                e.x += x.x; e.y += x.y;
            }
            ev[a] = e;
        }
    }
    float2 r[SS_MAX_ACTIONS];
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            r[a] = ld2(c.R + static_cast<size_t>(I.first_edge + a) * HS + h0);
            s0 += r[a].x > 0.f ? r[a].x : 0.f;
            s1 += r[a].y > 0.f ? r[a].y : 0.f;
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
            v0 += sigma(a, r[a].x, s0, inv0) * ev[a].x;
            v1 += sigma(a, r[a].y, s1, inv1) * ev[a].y;
        }
    }
    const int t = *c.iter;
    const float d = static_cast<float>(t) / (static_cast<float>(t) + 1.0f);
    const float w = static_cast<float>(t);
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            const size_t off = static_cast<size_t>(I.first_edge + a) * HS + h0;
            const float2 sm = ld2(c.S + off);
            float2 nr, ns;
            nr.x = (r[a].x + (ev[a].x - v0)) * d;
            nr.y = (r[a].y + (ev[a].y - v1)) * d;
            ns.x = sm.x + w * sigma(a, r[a].x, s0, inv0);
            ns.y = sm.y + w * sigma(a, r[a].y, s1, inv1);
            st2(c.R + off, nr);
            st2(c.S + off, ns);
        }
    }
    st2(c.val + static_cast<size_t>(I.node) * HS + h0, make_float2(v0, v1));
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
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kHandThreads + threadIdx.x) * 4;
    const TermItem I = items[it];
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
// leaves: leaf value * mass (:1047-1066).
template <class T>
__global__ void __launch_bounds__(kTermThreads) k_term_cr1(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                           const TermItem *__restrict__ items, int trav) {
    extern __shared__ __align__(16) char smem[];
    Carve cv{smem};
    T *M = cv.take<T>(52 * MS);
    double *u = cv.take<double>(52);
    unsigned long long *B = cv.take<unsigned long long>(52);
    double *F = cv.take<double>(1);
    int *npos = cv.take<int>(1);
    const TermItem I = items[blockIdx.x];
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

// Per-card aggregates of the two-opponent closed form, packed so a hand
// needs two 16-byte shared loads per card.
struct alignas(16) CardAgg {
    double u1, u2;      // per-card reach sums of opponents 1 and 2
    double w, d;        // (M2 u1 + M1 u2)(c), sum_b M1[c][b] M2[c][b]
};
struct alignas(16) CardCnt {
    int u1, u2, w, d;   // the same on the 0/1 positive-reach matrices
};
struct Cr2Scalars {
    double F1, F2, Q, D;
    long long IF1, IF2, IQ, ID;
};

template <class T>
constexpr size_t cr2_smem() {
    return 3 * 52 * MS * sizeof(T) + 52 * sizeof(CardAgg) + 52 * sizeof(CardCnt) + 52 * 16 +
           sizeof(Cr2Scalars) + 64;
}

// Two counted opponents (1, 2) with combo matrices M1, M2, per-card sums
// u_i = M_i 1, d(c) = sum_b M1[c][b] M2[c][b], w = M2 u1 + M1 u2,
// P = M1 M2, F_i = sum u_i / 2, Q = sum u1 u2, D = sum d / 2.  For a traverser
// hand (a, b), m_i = M_i[a][b], A_i = F_i - u_i(a) - u_i(b) + m_i, the mass of
// opponent pairs disjoint from each other and from (a, b) is
//   A1 A2 - Q + u1(a)u2(a) + u1(b)u2(b) + w(a) + w(b)
//   - m2 (u1(a) + u1(b)) - m1 (u2(a) + u2(b)) - 2 (d(a) + d(b)) + 3 m1 m2
//   - P[a][b] - P[b][a] + D
// (inclusion-exclusion over shared cards), equal to the reference odometer
// sum of street_solve.cu:771-823 / :1079-1127 for two opponents.
template <class T>
__global__ void __launch_bounds__(kTermThreads, sizeof(T) == 4 ? 6 : 2) k_term_cr2(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                              const TermItem *__restrict__ items, int trav) {
    extern __shared__ __align__(16) char smem[];
    Carve cv{smem};
    T *M1 = cv.take<T>(52 * MS);
    T *M2 = cv.take<T>(52 * MS);
    T *P = cv.take<T>(52 * MS);
    CardAgg *agg = cv.take<CardAgg>(52);
    CardCnt *cnt = cv.take<CardCnt>(52);
    ulonglong2 *Bm = cv.take<ulonglong2>(52);   // positive-reach masks of M1 (x) and M2 (y)
    Cr2Scalars *sc = cv.take<Cr2Scalars>(1);
    const TermItem I = items[blockIdx.x];
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarp = blockDim.x / 32;
    zero_matrix(M1);
    zero_matrix(M2);
    __syncthreads();
    scatter_combo(c, I.opp_player[0], I.opp_row[0], M1);
    scatter_combo(c, I.opp_player[1], I.opp_row[1], M2);
    __syncthreads();
    for (int r = warp; r < 52; r += nwarp) {
        double s1, s2, a0, a1, e0, e1;
        unsigned long long b1, b2;
        row_stats(M1, r, lane, &s1, &b1, &a0, &a1);
        row_stats(M2, r, lane, &s2, &b2, &e0, &e1);
        const double sd = warp_sum(a0 * e0 + a1 * e1);
        if (lane == 0) {
            agg[r].u1 = s1;
            agg[r].u2 = s2;
            agg[r].d = sd;
            Bm[r] = make_ulonglong2(b1, b2);
            cnt[r].u1 = __popcll(b1);
            cnt[r].u2 = __popcll(b2);
            cnt[r].d = __popcll(b1 & b2);
        }
    }
    __syncthreads();
    if (tid < 169) {
        // P = M1 M2 in 4x4 tiles; M1 is symmetric, so row b of M1 is column b
        const int i0 = (tid / 13) * 4, j0 = (tid % 13) * 4;
        T acc[4][4] = {};
        for (int b = 0; b < 52; ++b) {
            T xs[4], ys[4];
            load4(&M1[b * MS + i0], xs);
            load4(&M2[b * MS + j0], ys);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += xs[i] * ys[j];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) P[(i0 + i) * MS + j0 + j] = acc[i][j];
    } else if (tid < 169 + 52) {
        const int col = tid - 169;
        double s = 0.0;
        int n = 0;
        for (int b = 0; b < 52; ++b) {
            const CardAgg g = agg[b];
            s += g.u1 * static_cast<double>(M2[b * MS + col]) + g.u2 * static_cast<double>(M1[b * MS + col]);
            const ulonglong2 m = Bm[b];
            n += bit(m.y, col) * cnt[b].u1 + bit(m.x, col) * cnt[b].u2;
        }
        agg[col].w = s;
        cnt[col].w = n;
    } else if (warp == nwarp - 1) {
        double a1 = 0, a2 = 0, q = 0, e = 0;
        long long n1 = 0, n2 = 0, nq = 0, nd = 0;
        for (int k = lane; k < 52; k += 32) {
            const CardAgg g = agg[k];
            a1 += g.u1;
            a2 += g.u2;
            q += g.u1 * g.u2;
            e += g.d;
            const CardCnt m = cnt[k];
            n1 += m.u1;
            n2 += m.u2;
            nq += static_cast<long long>(m.u1) * m.u2;
            nd += m.d;
        }
        a1 = warp_sum(a1);
        a2 = warp_sum(a2);
        q = warp_sum(q);
        e = warp_sum(e);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n1 += __shfl_xor_sync(0xffffffffu, n1, o);
            n2 += __shfl_xor_sync(0xffffffffu, n2, o);
            nq += __shfl_xor_sync(0xffffffffu, nq, o);
            nd += __shfl_xor_sync(0xffffffffu, nd, o);
        }
        if (lane == 0) {
            sc->F1 = 0.5 * a1;
            sc->F2 = 0.5 * a2;
            sc->Q = q;
            sc->D = 0.5 * e;
            sc->IF1 = n1 / 2;
            sc->IF2 = n2 / 2;
            sc->IQ = nq;
            sc->ID = nd / 2;
        }
    }
    __syncthreads();
    const Cr2Scalars S = *sc;
    const int Ht = c.H[trav];
    const int *tc = c.hand_code + static_cast<size_t>(trav) * c.HS;
    T *out = val_rows<T>(c) + static_cast<size_t>(I.node) * c.HS;
    for (int h = tid; h < c.HS; h += blockDim.x) {
        double v = 0.0;
        if (h < Ht) {
            const int hc = tc[h];
            const int a = hc & 0xff, b = (hc >> 8) & 0xff;
            const ulonglong2 Ba = Bm[a], Bb = Bm[b];
            const CardCnt na = cnt[a], nb = cnt[b];
            const long long j1 = bit(Ba.x, b), j2 = bit(Ba.y, b);
            const long long JA1 = S.IF1 - na.u1 - nb.u1 + j1, JA2 = S.IF2 - na.u2 - nb.u2 + j2;
            const long long live = JA1 * JA2 - S.IQ + static_cast<long long>(na.u1) * na.u2 +
                                   static_cast<long long>(nb.u1) * nb.u2 + na.w + nb.w -
                                   j2 * (na.u1 + nb.u1) - j1 * (na.u2 + nb.u2) - 2 * (na.d + nb.d) +
                                   3 * j1 * j2 - (__popcll(Ba.x & Bb.y) + __popcll(Bb.x & Ba.y)) + S.ID;
            if (live > 0) {
                const CardAgg ga = agg[a], gb = agg[b];
                const double m1 = M1[a * MS + b], m2 = M2[a * MS + b];
                const double A1 = S.F1 - ga.u1 - gb.u1 + m1;
                const double A2 = S.F2 - ga.u2 - gb.u2 + m2;
                const double z = A1 * A2 - S.Q + ga.u1 * ga.u2 + gb.u1 * gb.u2 + ga.w + gb.w -
                                 m2 * (ga.u1 + gb.u1) - m1 * (ga.u2 + gb.u2) - 2.0 * (ga.d + gb.d) +
                                 3.0 * m1 * m2 -
                                 (static_cast<double>(P[a * MS + b]) + static_cast<double>(P[b * MS + a])) +
                                 S.D;
                v = static_cast<double>(term_factor(c, I, h)) * z;
            }
        }
        store_value(out, h, v);
    }
}

template <class T>
constexpr size_t sd1_smem() {
    return 1326 * sizeof(T) + 1327 * 8 + 52 * 53 * 8 + 52 * 4 + (kTermThreads / 32) * 8 + 52 * 8 + 64;
}

// Showdown against one live opponent (street_solve.cu:886-903): with W, T, S
// the opponent reach on compatible hands that are weaker, tied and in total,
// value = pot W + pot/2 T - bet S.  Combos are ranked once per board; the
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
    const double pot = I.pot, bet = I.bet;
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
                const double S = Pp[nc] - p1[clen[s.c1]] - p2[clen[s.c2]] + self;
                v = pot * W + 0.5 * pot * Tt - bet * S;
            }
        }
        store_value(out, h, v);
    }
}

// Exact enumeration of opponent hand tuples for one (terminal, traverser hand)
// per thread, with the reference validity rules and payoffs
// (street_solve.cu:771-823 fold, :936-1002 showdown, :1079-1127 leaf).  Cost
// is the product of the opponents' range sizes; the planner only routes small
// cases here.
template <class T>
__global__ void __launch_bounds__(128) k_term_enum(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                   const TermItem *__restrict__ items, int nchunk, int trav) {
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h = ch * blockDim.x + threadIdx.x;
    const TermItem I = items[it];
    const DevCtx &c = ctxs ? ctxs[I.sg] : c0;
    if (h >= c.HS) return;
    T *out = val_rows<T>(c) + static_cast<size_t>(I.node) * c.HS;
    const T *reach = reach_rows<T>(c);
    const int Ht = c.H[trav];
    if (h >= Ht) {
        out[h] = T(0);
        return;
    }
    const size_t HS = static_cast<size_t>(c.HS);
    const int hc = c.hand_code[trav * HS + h];
    const int t0 = hc & 0xff, t1 = (hc >> 8) & 0xff;
    const int k = I.k;
    const bool sd = I.kind_detail == 2;
    unsigned hs = 0;
    if (sd) {
        hs = c.strength[trav * HS + h];
        if (hs == 0) {
            out[h] = T(0);
            return;
        }
    }
    int idx[SS_MAX_PLAYERS - 1] = {0, 0, 0, 0, 0};
    T total = T(0);
    const T pot = I.pot, tb = I.bet;
    for (;;) {
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
                total += prod;
            } else {
                unsigned best = hs;
                for (int i = 0; i < k; ++i) best = os[i] > best ? os[i] : best;
                if (hs < best) {
                    total += prod * (-tb);
                } else {
                    int wins = 1;
                    for (int i = 0; i < k; ++i) wins += os[i] == best ? 1 : 0;
                    total += prod * (pot / static_cast<T>(wins) - tb);
                }
            }
        }
        int j = k - 1;
        while (j >= 0) {
            if (++idx[j] < c.H[I.opp_player[j]]) break;
            idx[j] = 0;
            --j;
        }
        if (j < 0) break;
    }
    out[h] = sd ? total : static_cast<T>(term_factor(c, I, h)) * total;
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

// batched form: advance the iteration counter of every listed subgame
__global__ void k_bump_many(const DevCtx *__restrict__ ctxs, const int *__restrict__ sgs, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) *const_cast<int *>(ctxs[sgs[i]].iter) += 1;
}

// batched form: root strategy snapshot (regret matching of the root node)
// of every listed subgame, one block per subgame, into its ctx.snap
__global__ void __launch_bounds__(128) k_snapshot_many(const DevCtx *__restrict__ ctxs,
                                                       const int *__restrict__ sgs) {
    const DevCtx &c = ctxs[sgs[blockIdx.x]];
    const int H = c.H[c.root_player];
    for (int h0 = threadIdx.x * 4; h0 < H; h0 += blockDim.x * 4) {
        float r[SS_MAX_ACTIONS][4], sig[SS_MAX_ACTIONS][4];
        regret_match4(c.R, static_cast<size_t>(c.HS), c.root_fe, c.root_na, c.root_frozen, h0, r, sig);
        for (int a = 0; a < c.root_na; ++a)
            for (int i = 0; i < 4; ++i)
                if (h0 + i < H) c.snap[static_cast<size_t>(a) * H + h0 + i] = sig[a][i];
    }
}

__global__ void k_bump(int *iter) { *iter += 1; }

// out[h] = sum over rows of val[row][h]
__global__ void __launch_bounds__(kHandThreads) k_sum_rows(DevCtx c, const int *__restrict__ rows, int n,
                                                           float *out, int H) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= H) return;
    float s = 0.f;
    for (int k = 0; k < n; ++k) s += c.val[static_cast<size_t>(rows[k]) * c.HS + h];
    out[h] = s;
}

// regret-matched (and frozen) strategy of one node, [na][H] (street_solve.cu:1564-1573)
__global__ void __launch_bounds__(kHandThreads) k_root_strategy(DevCtx c, int fe, int na, int frozen,
                                                                int H, float *out) {
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

}  // namespace

cudaError_t launch_reach(const DevCtx &c, const ReachItem *items, int n, int H, cudaStream_t s,
                         const DevCtx *ctxs, int player) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = chunks(H);
    k_reach<<<n * nc, kHandThreads, 0, s>>>(c, ctxs, items, nc, H, player);
    return cudaGetLastError();
}

cudaError_t launch_cfv(const DevCtx &c, const CfvItem *items, int n, int H, cudaStream_t s,
                       const DevCtx *ctxs, int trav) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = (H + 2 * kCfvThreads - 1) / (2 * kCfvThreads);
    k_cfv<<<n * nc, kCfvThreads, 0, s>>>(c, ctxs, items, nc, H, trav);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_terms_t(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                           cudaStream_t s, const DevCtx *ctxs) {
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    switch (kind) {
        case TK_ZERO:
        case TK_LEAF0: {
            const int nc = chunks(c.HS);
            k_term_fill<T><<<n * nc, kHandThreads, 0, s>>>(c, ctxs, items, nc, trav, kind == TK_ZERO);
            break;
        }
        case TK_CR1:
            k_term_cr1<T><<<n, kTermThreads, cr1_smem<T>(), s>>>(c, ctxs, items, trav);
            break;
        case TK_CR2:
            if (cr2_smem<T>() > 48 * 1024)
                e = cudaFuncSetAttribute(k_term_cr2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(cr2_smem<T>()));
            if (e != cudaSuccess) return e;
            k_term_cr2<T><<<n, kTermThreads, cr2_smem<T>(), s>>>(c, ctxs, items, trav);
            break;
        case TK_SD1:
            if (sd1_smem<T>() > 48 * 1024)
                e = cudaFuncSetAttribute(k_term_sd1<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(sd1_smem<T>()));
            if (e != cudaSuccess) return e;
            k_term_sd1<T><<<n, kTermThreads, sd1_smem<T>(), s>>>(c, ctxs, items, trav);
            break;
        case TK_ENUM: {
            const int nc = (c.HS + 127) / 128;
            k_term_enum<T><<<n * nc, 128, 0, s>>>(c, ctxs, items, nc, trav);
            break;
        }
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_terms(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                         cudaStream_t s, const DevCtx *ctxs) {
    return launch_terms_t<float>(c, kind, items, n, trav, s, ctxs);
}

cudaError_t launch_terms_fp64(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                              cudaStream_t s) {
    return launch_terms_t<double>(c, kind, items, n, trav, s, nullptr);
}

cudaError_t launch_bump(int *iter, cudaStream_t s) {
    k_bump<<<1, 1, 0, s>>>(iter);
    return cudaGetLastError();
}

cudaError_t launch_sum_rows(const DevCtx &c, const int *rows, int n, float *out, int H,
                            cudaStream_t s) {
    if (H <= 0) return cudaSuccess;
    k_sum_rows<<<(H + kHandThreads - 1) / kHandThreads, kHandThreads, 0, s>>>(c, rows, n, out, H);
    return cudaGetLastError();
}

cudaError_t launch_root_strategy(const DevCtx &c, int first_edge, int na, int frozen, int H,
                                 float *out, cudaStream_t s) {
    if (H <= 0) return cudaSuccess;
    k_root_strategy<<<(H + kHandsPerBlock - 1) / kHandsPerBlock, kHandThreads, 0, s>>>(
        c, first_edge, na, frozen, H, out);
    return cudaGetLastError();
}

cudaError_t launch_avg_strategy(const DevCtx &c, const int *dec_fe, const int *dec_na,
                                const int *dec_player, int num_dec, int max_h, float *out,
                                cudaStream_t s) {
    if (num_dec <= 0) return cudaSuccess;
    const int nc = (max_h + 127) / 128;
    k_avg_strategy<<<num_dec * nc, 128, 0, s>>>(c, dec_fe, dec_na, dec_player, nc, max_h, out);
    return cudaGetLastError();
}

cudaError_t launch_br_reach(const DevCtx &c, const ReachItem *items, int n, int H, const float *avg,
                            const int *edge_di, int max_h, cudaStream_t s) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = (H + 127) / 128;
    k_br_reach<<<n * nc, 128, 0, s>>>(c, items, nc, H, avg, edge_di, max_h);
    return cudaGetLastError();
}

cudaError_t launch_br_value(const DevCtx &c, const CfvItem *items, int n, int H, const float *avg,
                            const int *edge_di, int max_h, int mode, cudaStream_t s) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = (H + 127) / 128;
    k_br_value<<<n * nc, 128, 0, s>>>(c, items, nc, H, avg, edge_di, max_h, mode);
    return cudaGetLastError();
}

cudaError_t launch_br_root(const DevCtx &c, const int *rows, int n, int H, int weight_row, int trav,
                           int skip_blocked, double *out, cudaStream_t s) {
    k_br_root<<<1, 1024, 0, s>>>(c, rows, n, H, weight_row, trav, skip_blocked, out);
    return cudaGetLastError();
}

cudaError_t launch_bump_many(const DevCtx *ctxs, const int *sgs, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_bump_many<<<(n + 127) / 128, 128, 0, s>>>(ctxs, sgs, n);
    return cudaGetLastError();
}

cudaError_t launch_snapshot_many(const DevCtx *ctxs, const int *sgs, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_snapshot_many<<<n, 128, 0, s>>>(ctxs, sgs);
    return cudaGetLastError();
}

}  // namespace ssb
