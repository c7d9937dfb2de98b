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

constexpr int MS = 56;  // shared-memory row stride of a 52x52 combo matrix

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
// * t/(t+1); s_a += t * sigma_a; ev_a = sum of val over frontier(edge a)
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(kHandThreads) k_cfv(DevCtx c, const CfvItem *__restrict__ items,
                                                      int nchunk, int H) {
    const int it = blockIdx.x / nchunk;
    const int ch = blockIdx.x - it * nchunk;
    const int h0 = (ch * kHandThreads + threadIdx.x) * 4;
    if (h0 >= H) return;
    const CfvItem I = items[it];
    const size_t HS = static_cast<size_t>(c.HS);
    float r[SS_MAX_ACTIONS][4], sig[SS_MAX_ACTIONS][4], ev[SS_MAX_ACTIONS][4];
    regret_match4(c.R, HS, I.first_edge, I.na, I.frozen, h0, r, sig);
    float v[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            float e[4] = {0.f, 0.f, 0.f, 0.f};
            const int k0 = c.fr_off[I.first_edge + a], k1 = c.fr_off[I.first_edge + a + 1];
            for (int k = k0; k < k1; ++k) {
                const float4 x = ld4(c.val + static_cast<size_t>(c.fr_items[k]) * HS + h0);
                e[0] += x.x;
                e[1] += x.y;
                e[2] += x.z;
                e[3] += x.w;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ev[a][i] = e[i];
                v[i] += sig[a][i] * e[i];
            }
        }
    }
    const int t = *c.iter;
    const float d = static_cast<float>(t) / (static_cast<float>(t) + 1.0f);
    const float w = static_cast<float>(t);
#pragma unroll
    for (int a = 0; a < SS_MAX_ACTIONS; ++a) {
        if (a < I.na) {
            const size_t off = static_cast<size_t>(I.first_edge + a) * HS + h0;
            float4 nr, ns;
            const float4 s = ld4(c.S + off);
            nr.x = (r[a][0] + (ev[a][0] - v[0])) * d;
            nr.y = (r[a][1] + (ev[a][1] - v[1])) * d;
            nr.z = (r[a][2] + (ev[a][2] - v[2])) * d;
            nr.w = (r[a][3] + (ev[a][3] - v[3])) * d;
            ns.x = s.x + w * sig[a][0];
            ns.y = s.y + w * sig[a][1];
            ns.z = s.z + w * sig[a][2];
            ns.w = s.w + w * sig[a][3];
            st4(c.R + off, nr);
            st4(c.S + off, ns);
        }
    }
    st4(c.val + static_cast<size_t>(I.node) * HS + h0, make_float4(v[0], v[1], v[2], v[3]));
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

// Scatter one opponent's reach at a terminal into a 52x52 combo matrix, and
// mark the combos holding positive reach in per-card 64-bit masks (bit b of
// B[a] = combo {a, b}).  The masks give the exact number of compatible
// positive-reach opponent tuples through the same inclusion-exclusion as the
// float sums, with popcounts; where that number is 0 the value is exactly 0,
// as the reference's enumeration returns (it only adds positive products,
// street_solve.cu:810-812).  Without it the float formula would leave rounding
// residue there, and regret matching turns a residue into a pure strategy
// where the reference plays uniformly.
__device__ __forceinline__ void scatter_combo(const DevCtx &c, int opp, int row, float *M,
                                              unsigned long long *B) {
    const float *r = c.reach + static_cast<size_t>(row) * c.HS;
    const int *code = c.hand_code + static_cast<size_t>(opp) * c.HS;
    const int Ho = c.H[opp];
    for (int j = threadIdx.x; j < Ho; j += blockDim.x) {
        const int hc = code[j];
        if (hc & 0x10000) continue;  // board-blocked hands never count (street_solve.cu:755-757)
        const int a = hc & 0xff, b = (hc >> 8) & 0xff;
        const float x = r[j];
        atomicAdd(&M[a * MS + b], x);
        atomicAdd(&M[b * MS + a], x);
        if (x > 0.f) {
            atomicOr(&B[a], 1ull << b);
            atomicOr(&B[b], 1ull << a);
        }
    }
}

__device__ __forceinline__ int bit(unsigned long long m, int b) { return static_cast<int>((m >> b) & 1ull); }

// One counted opponent: mass(h) = F - u(c1) - u(c2) + f(h), F the opponent's
// total reach, u(c) its reach on hands holding card c, f(h) its reach on the
// traverser's own combo.  Folds: payoff * mass (street_solve.cu:745-761);
// leaves: leaf value * mass (:1047-1066).
__global__ void __launch_bounds__(kTermThreads) k_term_cr1(DevCtx c, const TermItem *__restrict__ items,
                                                           int trav) {
    __shared__ float M[52 * MS];
    __shared__ unsigned long long B[52];
    __shared__ double u[52];
    __shared__ double F;
    __shared__ int npos;
    const TermItem I = items[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < 52 * MS; i += blockDim.x) M[i] = 0.f;
    if (tid < 52) B[tid] = 0ull;
    __syncthreads();
    scatter_combo(c, I.opp_player[0], I.opp_row[0], M, B);
    __syncthreads();
    for (int r = warp; r < 52; r += blockDim.x / 32) {
        double s = static_cast<double>(M[r * MS + lane]) +
                   (lane + 32 < 52 ? static_cast<double>(M[r * MS + lane + 32]) : 0.0);
        s = warp_sum(s);
        if (lane == 0) u[r] = s;
    }
    __syncthreads();
    if (warp == 0) {
        double s = u[lane] + (lane + 32 < 52 ? u[lane + 32] : 0.0);
        s = warp_sum(s);
        int n = __popcll(B[lane]) + (lane + 32 < 52 ? __popcll(B[lane + 32]) : 0);
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
            const int live = npos - __popcll(B[a]) - __popcll(B[b]) + bit(B[a], b);
            if (live > 0) {
                const double z = F - u[a] - u[b] + static_cast<double>(M[a * MS + b]);
                v = static_cast<float>(static_cast<double>(term_factor(c, I, h)) * z);
            }
        }
        out[h] = v;
    }
}

// Two counted opponents (1, 2) with combo matrices M1, M2, per-card sums
// u_i = M_i 1, d(c) = sum_b M1[c][b] M2[c][b], w12 = M2 u1, w21 = M1 u2,
// P = M1 M2, F_i = sum u_i / 2, Q = sum u1 u2, D = sum d / 2.  For a traverser
// hand (a, b), m_i = M_i[a][b], A_i = F_i - u_i(a) - u_i(b) + m_i, the mass of
// opponent pairs disjoint from each other and from (a, b) is
//   A1 A2 - Q + u1(a)u2(a) + u1(b)u2(b) + w12(a) + w12(b) + w21(a) + w21(b)
//   - m2 (u1(a) + u1(b)) - m1 (u2(a) + u2(b)) - 2 (d(a) + d(b)) + 3 m1 m2
//   - P[a][b] - P[b][a] + D
// (inclusion-exclusion over shared cards), equal to the reference odometer
// sum of street_solve.cu:771-823 / :1079-1127 for two opponents.
__global__ void __launch_bounds__(kTermThreads) k_term_cr2(DevCtx c, const TermItem *__restrict__ items,
                                                           int trav) {
    __shared__ __align__(16) float M1[52 * MS];
    __shared__ __align__(16) float M2[52 * MS];
    __shared__ __align__(16) float P[52 * MS];
    __shared__ double u1[52], u2[52], dd[52], w12[52], w21[52];
    __shared__ double F1, F2, Q, D;
    // exact counts of positive-reach combos, same formula on 0/1 matrices
    __shared__ unsigned long long B1[52], B2[52];
    __shared__ int iu1[52], iu2[52], idd[52], iw12[52], iw21[52];
    __shared__ long long IF1, IF2, IQ, ID;
    const TermItem I = items[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarp = blockDim.x / 32;
    for (int i = tid; i < 52 * MS; i += blockDim.x) {
        M1[i] = 0.f;
        M2[i] = 0.f;
    }
    if (tid < 52) {
        B1[tid] = 0ull;
        B2[tid] = 0ull;
    }
    __syncthreads();
    scatter_combo(c, I.opp_player[0], I.opp_row[0], M1, B1);
    scatter_combo(c, I.opp_player[1], I.opp_row[1], M2, B2);
    __syncthreads();
    if (tid < 52) {
        iu1[tid] = __popcll(B1[tid]);
        iu2[tid] = __popcll(B2[tid]);
        idd[tid] = __popcll(B1[tid] & B2[tid]);
    }
    for (int r = warp; r < 52; r += nwarp) {
        const double x1 = M1[r * MS + lane], x2 = M2[r * MS + lane];
        const double y1 = lane + 32 < 52 ? M1[r * MS + lane + 32] : 0.0;
        const double y2 = lane + 32 < 52 ? M2[r * MS + lane + 32] : 0.0;
        const double s1 = warp_sum(x1 + y1);
        const double s2 = warp_sum(x2 + y2);
        const double sd = warp_sum(x1 * x2 + y1 * y2);
        if (lane == 0) {
            u1[r] = s1;
            u2[r] = s2;
            dd[r] = sd;
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
    } else {
        for (int q = tid - 169; q < 104; q += blockDim.x - 169) {
            const int col = q % 52;
            double s = 0.0;
            int n = 0;
            if (q < 52) {
                for (int b = 0; b < 52; ++b) {
                    s += u1[b] * static_cast<double>(M2[b * MS + col]);
                    n += bit(B2[b], col) * __popcll(B1[b]);
                }
                w12[col] = s;
                iw12[col] = n;
            } else {
                for (int b = 0; b < 52; ++b) {
                    s += u2[b] * static_cast<double>(M1[b * MS + col]);
                    n += bit(B1[b], col) * __popcll(B2[b]);
                }
                w21[col] = s;
                iw21[col] = n;
            }
        }
    }
    if (warp == 0) {
        const double a1 = u1[lane] + (lane + 32 < 52 ? u1[lane + 32] : 0.0);
        const double a2 = u2[lane] + (lane + 32 < 52 ? u2[lane + 32] : 0.0);
        const double q = u1[lane] * u2[lane] + (lane + 32 < 52 ? u1[lane + 32] * u2[lane + 32] : 0.0);
        const double e = dd[lane] + (lane + 32 < 52 ? dd[lane + 32] : 0.0);
        const double s1 = warp_sum(a1), s2 = warp_sum(a2), sq = warp_sum(q), se = warp_sum(e);
        long long n1 = 0, n2 = 0, nq = 0, nd = 0;
        for (int k = lane; k < 52; k += 32) {
            const int x1 = __popcll(B1[k]), x2 = __popcll(B2[k]);
            n1 += x1;
            n2 += x2;
            nq += static_cast<long long>(x1) * x2;
            nd += __popcll(B1[k] & B2[k]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n1 += __shfl_xor_sync(0xffffffffu, n1, o);
            n2 += __shfl_xor_sync(0xffffffffu, n2, o);
            nq += __shfl_xor_sync(0xffffffffu, nq, o);
            nd += __shfl_xor_sync(0xffffffffu, nd, o);
        }
        if (lane == 0) {
            F1 = 0.5 * s1;
            F2 = 0.5 * s2;
            Q = sq;
            D = 0.5 * se;
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
            const long long j1 = bit(B1[a], b), j2 = bit(B2[a], b);
            const long long ja1 = iu1[a], jb1 = iu1[b], ja2 = iu2[a], jb2 = iu2[b];
            const long long JA1 = IF1 - ja1 - jb1 + j1, JA2 = IF2 - ja2 - jb2 + j2;
            const long long live = JA1 * JA2 - IQ + ja1 * ja2 + jb1 * jb2 +
                                   (iw12[a] + iw12[b] + iw21[a] + iw21[b]) - j2 * (ja1 + jb1) -
                                   j1 * (ja2 + jb2) - 2 * (idd[a] + idd[b]) + 3 * j1 * j2 -
                                   (__popcll(B1[a] & B2[b]) + __popcll(B1[b] & B2[a])) + ID;
            if (live <= 0) {
                out[h] = 0.f;
                continue;
            }
            const double m1 = M1[a * MS + b], m2 = M2[a * MS + b];
            const double ua1 = u1[a], ub1 = u1[b], ua2 = u2[a], ub2 = u2[b];
            const double A1 = F1 - ua1 - ub1 + m1;
            const double A2 = F2 - ua2 - ub2 + m2;
            const double z = A1 * A2 - Q + ua1 * ua2 + ub1 * ub2 + (w12[a] + w12[b] + w21[a] + w21[b]) -
                             m2 * (ua1 + ub1) - m1 * (ua2 + ub2) - 2.0 * (dd[a] + dd[b]) +
                             3.0 * m1 * m2 -
                             (static_cast<double>(P[a * MS + b]) + static_cast<double>(P[b * MS + a])) + D;
            v = static_cast<float>(static_cast<double>(term_factor(c, I, h)) * z);
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
    if (tid < 52) B[tid] = 0ull;
    __syncthreads();
    {
        const int o = I.opp_player[0];
        const float *r = c.reach + static_cast<size_t>(I.opp_row[0]) * c.HS;
        const int *pos = c.sd_pos + static_cast<size_t>(o) * c.HS;
        const int *code = c.hand_code + static_cast<size_t>(o) * c.HS;
        for (int j = tid; j < c.H[o]; j += blockDim.x) {
            const int q = pos[j];
            if (q < 0) continue;
            const float x = r[j];
            atomicAdd(&Rr[q], x);
            if (x > 0.f) {
                const int a = code[j] & 0xff, b = (code[j] >> 8) & 0xff;
                atomicOr(&B[a], 1ull << b);
                atomicOr(&B[b], 1ull << a);
            }
        }
    }
    __syncthreads();
    if (warp == 0) {
        int n = __popcll(B[lane]) + (lane + 32 < 52 ? __popcll(B[lane + 32]) : 0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
        if (lane == 0) npos = n / 2;
    }
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
    // per-card exclusive prefix sums over each card's combos in rank order
    for (int card = warp; card < 52; card += blockDim.x / 32) {
        const short *L = c.sd_card_list + card * 52;
        const int i0 = 2 * lane, i1 = 2 * lane + 1;
        const int q0 = i0 < 52 ? L[i0] : -1, q1 = i1 < 52 ? L[i1] : -1;
        const double v0 = q0 >= 0 ? static_cast<double>(Rr[q0]) : 0.0;
        const double v1 = q1 >= 0 ? static_cast<double>(Rr[q1]) : 0.0;
        const double pair = v0 + v1;
        double incl = pair;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const double ex = incl - pair;
        const unsigned have = __ballot_sync(0xffffffffu, q0 >= 0);
        const unsigned have1 = __ballot_sync(0xffffffffu, q1 >= 0);
        const int len = __popc(have) + __popc(have1);
        if (i0 <= len) PC[card * 53 + i0] = ex;
        if (i1 <= len) PC[card * 53 + i1] = ex + v0;
        if (lane == 0) clen[card] = len;
    }
    __syncthreads();
    const int Ht = c.H[trav];
    const int *tpos = c.sd_pos + static_cast<size_t>(trav) * c.HS;
    float *out = c.val + static_cast<size_t>(I.node) * c.HS;
    const double pot = I.pot, bet = I.bet;
    for (int h = tid; h < c.HS; h += blockDim.x) {
        float v = 0.f;
        const int q = h < Ht ? tpos[h] : -1;
        if (q >= 0 &&
            npos - __popcll(B[c.sd_combo[q].c1]) - __popcll(B[c.sd_combo[q].c2]) +
                    bit(B[c.sd_combo[q].c1], c.sd_combo[q].c2) > 0) {
            const SdCombo s = c.sd_combo[q];
            const double *p1 = PC + s.c1 * 53, *p2 = PC + s.c2 * 53;
            const double self = Rr[q];
            const double W = Pp[s.lo] - p1[s.l1lo] - p2[s.l2lo];
            const double T = (Pp[s.hi] - Pp[s.lo]) - (p1[s.l1hi] - p1[s.l1lo]) -
                             (p2[s.l2hi] - p2[s.l2lo]) + self;
            const double S = Pp[nc] - p1[clen[s.c1]] - p2[clen[s.c2]] + self;
            v = static_cast<float>(pot * W + 0.5 * pot * T - bet * S);
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
    const int nc = chunks(H);
    k_cfv<<<n * nc, kHandThreads, 0, s>>>(c, items, nc, H);
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
