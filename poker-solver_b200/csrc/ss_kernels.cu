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
__global__ void __launch_bounds__(kHandThreads) k_reach(DevCtx c, const ReachItem *__restrict__ items,
                                                        int nchunk, int H) {
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kHandThreads + threadIdx.x) * 4;
    if (h0 >= H) return;
    const ReachItem I = items[it];
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

__global__ void __launch_bounds__(kCfvThreads) k_cfv(DevCtx c, const CfvItem *__restrict__ items,
                                                     int nchunk, int H) {
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kCfvThreads + threadIdx.x) * 2;
    if (h0 >= H) return;
    const CfvItem I = items[it];
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

// value rows of terminals with no opponent coupling: zero, or the factor itself
// (a leaf without a live opponent, street_solve.cu:1062-1065)
__global__ void __launch_bounds__(kHandThreads) k_term_fill(DevCtx c, const TermItem *__restrict__ items,
                                                            int nchunk, int trav, int zero) {
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kHandThreads + threadIdx.x) * 4;
    if (h0 >= c.HS) return;
    const TermItem I = items[it];
    const int Ht = c.H[trav];
    float o[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = (zero || h0 + i >= Ht) ? 0.f : term_factor(c, I, h0 + i);
    st4(c.val + static_cast<size_t>(I.node) * c.HS + h0, make_float4(o[0], o[1], o[2], o[3]));
}

// Scatter one opponent's reach at a terminal into a 52x52 combo matrix
// (row stride MS): M[a][b] = M[b][a] = reach of the opponent's hand {a, b}.
// Board-blocked hands never count (street_solve.cu:755-757).  A range that
// holds some combo twice accumulates atomically; otherwise each cell has one
// writer and plain stores suffice.
__device__ __forceinline__ void scatter_combo(const DevCtx &c, int opp, int row, float *M) {
    const float *r = c.reach + static_cast<size_t>(row) * c.HS;
    const int *code = c.hand_code + static_cast<size_t>(opp) * c.HS;
    const int Ho = c.H[opp];
    const bool dup = c.dup[opp] != 0;
    for (int j = threadIdx.x; j < Ho; j += blockDim.x) {
        const int hc = code[j];
        if (hc & 0x10000) continue;
        const int a = hc & 0xff, b = (hc >> 8) & 0xff;
        const float x = r[j];
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

__device__ __forceinline__ void zero_matrix(float *M) {
    float4 *m4 = reinterpret_cast<float4 *>(M);
    for (int i = threadIdx.x; i < 52 * MS / 4; i += blockDim.x) m4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Row pass over a combo matrix, one warp per card row r: the row sum u(r) in
// FP64 and the 64-bit mask of the row's positive cells.  The masks give the
// exact number of compatible positive-reach opponent tuples through the same
// inclusion-exclusion as the float sums; where that number is 0 the value is
// exactly 0, as in the reference, which only adds positive products
// (street_solve.cu:810-812).  Without it rounding residue of the closed form
// would turn into a pure strategy under regret matching where the reference
// plays uniformly.
__device__ __forceinline__ void row_stats(const float *M, int r, int lane, double *sum_out,
                                          unsigned long long *mask_out, float *x0, float *x1) {
    const float a = M[r * MS + lane];
    const float b = lane + 32 < 52 ? M[r * MS + lane + 32] : 0.f;
    const unsigned lo = __ballot_sync(0xffffffffu, a > 0.f);
    const unsigned hi = __ballot_sync(0xffffffffu, b > 0.f);
    *sum_out = warp_sum(static_cast<double>(a) + static_cast<double>(b));
    *mask_out = static_cast<unsigned long long>(lo) | (static_cast<unsigned long long>(hi) << 32);
    *x0 = a;
    *x1 = b;
}

// One counted opponent: mass(h) = F - u(c1) - u(c2) + f(h), F the opponent's
// total reach, u(c) its reach on hands holding card c, f(h) its reach on the
// traverser's own combo.  Folds: payoff * mass (street_solve.cu:745-761);
// leaves: leaf value * mass (:1047-1066).
__global__ void __launch_bounds__(kTermThreads) k_term_cr1(DevCtx c, const TermItem *__restrict__ items,
                                                           int trav) {
    __shared__ __align__(16) float M[52 * MS];
    __shared__ double u[52];
    __shared__ unsigned long long B[52];
    __shared__ double F;
    __shared__ int npos;
    const TermItem I = items[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    zero_matrix(M);
    __syncthreads();
    scatter_combo(c, I.opp_player[0], I.opp_row[0], M);
    __syncthreads();
    for (int r = warp; r < 52; r += blockDim.x / 32) {
        double s;
        unsigned long long m;
        float x0, x1;
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
            F = 0.5 * s;
            npos = n / 2;
        }
    }
    __syncthreads();
    const int Ht = c.H[trav];
    const int *tc = c.hand_code + static_cast<size_t>(trav) * c.HS;
    float *out = c.val + static_cast<size_t>(I.node) * c.HS;
    for (int h = tid; h < c.HS; h += blockDim.x) {
        float v = 0.f;
        if (h < Ht) {
            const int hc = tc[h];
            const int a = hc & 0xff, b = (hc >> 8) & 0xff;
            const unsigned long long Ba = B[a], Bb = B[b];
            const int live = npos - __popcll(Ba) - __popcll(Bb) + bit(Ba, b);
            if (live > 0) {
                const double z = F - u[a] - u[b] + static_cast<double>(M[a * MS + b]);
                v = static_cast<float>(static_cast<double>(term_factor(c, I, h)) * z);
            }
        }
        out[h] = v;
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
__global__ void __launch_bounds__(kTermThreads, 6) k_term_cr2(DevCtx c, const TermItem *__restrict__ items,
                                                           int trav) {
    __shared__ __align__(16) float M1[52 * MS];
    __shared__ __align__(16) float M2[52 * MS];
    __shared__ __align__(16) float P[52 * MS];
    __shared__ CardAgg agg[52];
    __shared__ CardCnt cnt[52];
    __shared__ ulonglong2 Bm[52];   // positive-reach masks of M1 (x) and M2 (y)
    __shared__ double F1, F2, Q, D;
    __shared__ long long IF1, IF2, IQ, ID;
    const TermItem I = items[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarp = blockDim.x / 32;
    zero_matrix(M1);
    zero_matrix(M2);
    __syncthreads();
    scatter_combo(c, I.opp_player[0], I.opp_row[0], M1);
    scatter_combo(c, I.opp_player[1], I.opp_row[1], M2);
    __syncthreads();
    for (int r = warp; r < 52; r += nwarp) {
        double s1, s2;
        unsigned long long b1, b2;
        float a0, a1, e0, e1;
        row_stats(M1, r, lane, &s1, &b1, &a0, &a1);
        row_stats(M2, r, lane, &s2, &b2, &e0, &e1);
        const double sd = warp_sum(static_cast<double>(a0) * e0 + static_cast<double>(a1) * e1);
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
        float acc[4][4] = {};
        for (int b = 0; b < 52; ++b) {
            const float4 x = *reinterpret_cast<const float4 *>(&M1[b * MS + i0]);
            const float4 y = *reinterpret_cast<const float4 *>(&M2[b * MS + j0]);
            const float xs[4] = {x.x, x.y, x.z, x.w}, ys[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += xs[i] * ys[j];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            *reinterpret_cast<float4 *>(&P[(i0 + i) * MS + j0]) =
                make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
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
            F1 = 0.5 * a1;
            F2 = 0.5 * a2;
            Q = q;
            D = 0.5 * e;
            IF1 = n1 / 2;
            IF2 = n2 / 2;
            IQ = nq;
            ID = nd / 2;
        }
    }
    __syncthreads();
    const int Ht = c.H[trav];
    const int *tc = c.hand_code + static_cast<size_t>(trav) * c.HS;
    float *out = c.val + static_cast<size_t>(I.node) * c.HS;
    for (int h = tid; h < c.HS; h += blockDim.x) {
        float v = 0.f;
        if (h < Ht) {
            const int hc = tc[h];
            const int a = hc & 0xff, b = (hc >> 8) & 0xff;
            const ulonglong2 Ba = Bm[a], Bb = Bm[b];
            const CardCnt na = cnt[a], nb = cnt[b];
            const long long j1 = bit(Ba.x, b), j2 = bit(Ba.y, b);
            const long long JA1 = IF1 - na.u1 - nb.u1 + j1, JA2 = IF2 - na.u2 - nb.u2 + j2;
            const long long live = JA1 * JA2 - IQ + static_cast<long long>(na.u1) * na.u2 +
                                   static_cast<long long>(nb.u1) * nb.u2 + na.w + nb.w -
                                   j2 * (na.u1 + nb.u1) - j1 * (na.u2 + nb.u2) - 2 * (na.d + nb.d) +
                                   3 * j1 * j2 - (__popcll(Ba.x & Bb.y) + __popcll(Bb.x & Ba.y)) + ID;
            if (live > 0) {
                const CardAgg ga = agg[a], gb = agg[b];
                const double m1 = M1[a * MS + b], m2 = M2[a * MS + b];
                const double A1 = F1 - ga.u1 - gb.u1 + m1;
                const double A2 = F2 - ga.u2 - gb.u2 + m2;
                const double z = A1 * A2 - Q + ga.u1 * ga.u2 + gb.u1 * gb.u2 + ga.w + gb.w -
                                 m2 * (ga.u1 + gb.u1) - m1 * (ga.u2 + gb.u2) - 2.0 * (ga.d + gb.d) +
                                 3.0 * m1 * m2 -
                                 (static_cast<double>(P[a * MS + b]) + static_cast<double>(P[b * MS + a])) + D;
                v = static_cast<float>(static_cast<double>(term_factor(c, I, h)) * z);
            }
        }
        out[h] = v;
    }
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
__global__ void __launch_bounds__(kTermThreads) k_term_sd1(DevCtx c, const TermItem *__restrict__ items,
                                                           int trav) {
    __shared__ float Rr[1326];
    __shared__ double Pp[1327];
    __shared__ double PC[52 * 53];
    __shared__ int clen[52];
    __shared__ double wsum[kTermThreads / 32];
    __shared__ unsigned long long B[52];
    __shared__ int npos;
    const TermItem I = items[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nc = c.ncomb;
    for (int i = tid; i < nc; i += blockDim.x) Rr[i] = 0.f;
    __syncthreads();
    {
        const int o = I.opp_player[0];
        const float *r = c.reach + static_cast<size_t>(I.opp_row[0]) * c.HS;
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
        const float f0 = q0 >= 0 ? Rr[q0] : 0.f, f1 = q1 >= 0 ? Rr[q1] : 0.f;
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
        if (f0 > 0.f) m |= 1ull << Pt[i0];
        if (f1 > 0.f) m |= 1ull << Pt[i1];
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
        if (lane == 0) npos = n / 2;
    }
    __syncthreads();
    const int Ht = c.H[trav];
    const int *tpos = c.sd_pos + static_cast<size_t>(trav) * c.HS;
    float *out = c.val + static_cast<size_t>(I.node) * c.HS;
    const double pot = I.pot, bet = I.bet;
    for (int h = tid; h < c.HS; h += blockDim.x) {
        float v = 0.f;
        const int q = h < Ht ? tpos[h] : -1;
        if (q >= 0) {
            const SdCombo s = c.sd_combo[q];
            const unsigned long long B1 = B[s.c1], B2 = B[s.c2];
            if (npos - __popcll(B1) - __popcll(B2) + bit(B1, s.c2) > 0) {
                const double *p1 = PC + s.c1 * 53, *p2 = PC + s.c2 * 53;
                const double self = Rr[q];
                const double W = Pp[s.lo] - p1[s.l1lo] - p2[s.l2lo];
                const double T = (Pp[s.hi] - Pp[s.lo]) - (p1[s.l1hi] - p1[s.l1lo]) -
                                 (p2[s.l2hi] - p2[s.l2lo]) + self;
                const double S = Pp[nc] - p1[clen[s.c1]] - p2[clen[s.c2]] + self;
                v = static_cast<float>(pot * W + 0.5 * pot * T - bet * S);
            }
        }
        out[h] = v;
    }
}

// Exact enumeration of opponent hand tuples for one (terminal, traverser hand)
// per thread, with the reference validity rules and payoffs
// (street_solve.cu:771-823 fold, :936-1002 showdown, :1079-1127 leaf).  Cost
// is the product of the opponents' range sizes; the planner only routes small
// cases here.
__global__ void __launch_bounds__(128) k_term_enum(DevCtx c, const TermItem *__restrict__ items,
                                                   int nchunk, int trav) {
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h = ch * blockDim.x + threadIdx.x;
    if (h >= c.HS) return;
    const TermItem I = items[it];
    float *out = c.val + static_cast<size_t>(I.node) * c.HS;
    const int Ht = c.H[trav];
    if (h >= Ht) {
        out[h] = 0.f;
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
            out[h] = 0.f;
            return;
        }
    }
    int idx[SS_MAX_PLAYERS - 1] = {0, 0, 0, 0, 0};
    float total = 0.f;
    const float pot = I.pot, tb = I.bet;
    for (;;) {
        int cards[SS_MAX_PLAYERS - 1][2];
        unsigned os[SS_MAX_PLAYERS - 1];
        float prod = 1.0f;
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
            prod *= c.reach[static_cast<size_t>(I.opp_row[i]) * HS + o];
            for (int j = 0; j < i; ++j)
                if (a0 == cards[j][0] || a0 == cards[j][1] || a1 == cards[j][0] || a1 == cards[j][1]) {
                    ok = false;
                    break;
                }
        }
        if (ok && prod > 0.f) {
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
                    total += prod * (pot / static_cast<float>(wins) - tb);
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
    out[h] = sd ? total : term_factor(c, I, h) * total;
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

cudaError_t launch_reach(const DevCtx &c, const ReachItem *items, int n, int H, cudaStream_t s) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = chunks(H);
    k_reach<<<n * nc, kHandThreads, 0, s>>>(c, items, nc, H);
    return cudaGetLastError();
}

cudaError_t launch_cfv(const DevCtx &c, const CfvItem *items, int n, int H, cudaStream_t s) {
    if (n <= 0 || H <= 0) return cudaSuccess;
    const int nc = (H + 2 * kCfvThreads - 1) / (2 * kCfvThreads);
    k_cfv<<<n * nc, kCfvThreads, 0, s>>>(c, items, nc, H);
    return cudaGetLastError();
}

cudaError_t launch_terms(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                         cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    switch (kind) {
        case TK_ZERO:
        case TK_LEAF0: {
            const int nc = chunks(c.HS);
            k_term_fill<<<n * nc, kHandThreads, 0, s>>>(c, items, nc, trav, kind == TK_ZERO);
            break;
        }
        case TK_CR1:
            k_term_cr1<<<n, kTermThreads, 0, s>>>(c, items, trav);
            break;
        case TK_CR2:
            k_term_cr2<<<n, kTermThreads, 0, s>>>(c, items, trav);
            break;
        case TK_SD1:
            k_term_sd1<<<n, kTermThreads, 0, s>>>(c, items, trav);
            break;
        case TK_ENUM: {
            const int nc = (c.HS + 127) / 128;
            k_term_enum<<<n * nc, 128, 0, s>>>(c, items, nc, trav);
            break;
        }
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
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

}  // namespace ssb
