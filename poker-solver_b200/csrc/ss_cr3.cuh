// ss_cr3.cuh -- card-removal mass of three counted opponents (folds and
// leaves of 4+ player subgames), the block phases of k_term_cr3.
//
// The reference sums, per traverser hand h, the reach products of every
// tuple of opponent hands (o1, o2, o3) that are pairwise disjoint and
// disjoint from h (street_solve.cu:771-823 folds, :1079-1127 leaves): O(H^3)
// per hand.  Conditioning on the third opponent's hand gives it in O(H):
//   M3(h) = sum_{o3 disjoint from h} r3(o3) * D2(h + o3),
// where D2(S), the two-opponent mass avoiding a card set S, takes O(|S|^2)
// lookups of aggregates of the first two opponents' combo matrices A, B
// (symmetric, zero diagonal, over the dense deck):
//   D2(S) = F_A(S) F_B(S) - Q(S) + E(S)
//   F_A(S) = F_A - sum_{c in S} u_A(c) + sum_{pairs in S} A
//   Q(S)   = Q - sum_{e in S} w(e) + sum_{e, f in S} P[e][f] - sum_{c in S} u~_A(c) u~_B(c),
//            u~_A(c) = u_A(c) - sum_{e in S} A[c][e]
//   E(S)   = E - sum_{c in S} d(c) + sum_{pairs in S} A B
// with u = A 1, F = sum u / 2, P = A B, w = A u_B + B u_A, Q = u_A . u_B,
// d = diag P, E = sum d / 2.  The same formula on the 0/1 matrices of
// positive reach counts the tuples exactly (integers), which gives the
// reference's exact zero: a hand with no tuple of positive products gets 0.
//
// A board card of the traverser's hand maps to the dummy index `deck`,
// whose rows, columns and vectors are zero, so it drops out of every sum
// (opponent hands never hold board cards).
//
// Each phase is a function of (thread index, thread count) whose work items
// are independent within the phase; the kernel separates phases with block
// barriers, and a host build runs them one after another (the check in
// tests/native/cr3_emul.cpp).
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define SSB_CR3_HD __host__ __device__ __forceinline__
#else
#define SSB_CR3_HD inline
#endif

namespace ssb {
namespace cr3 {

constexpr int kS = 52;   // table stride (cards 0 .. deck, deck <= 49 plus the dummy)

SSB_CR3_HD int popc64(unsigned long long x) {
#if defined(__CUDA_ARCH__)
    return __popcll(x);
#else
    return __builtin_popcountll(x);
#endif
}

// the block's shared tables
struct Tables {
    double *A, *B, *P, *PT;           // [kS][kS]; PT[x][a] = P[a][x]
    double *uA, *uB, *w, *d;          // [kS]
    int *iuA, *iuB, *iw, *id;         // [kS]: the same on the 0/1 matrices
    unsigned long long *mA, *mB;      // [kS]: positive cells of each row
    double *r3;                       // [HS]: the third opponent's positive reach, compacted
    unsigned short *xy;               // [HS]: its dense cards x | y << 8
    double *sc;                       // [5]: F_A, F_B, Q, E, F3 (sum of the compacted r3)
    long long *isc;                   // [5]: the same on the 0/1 matrices, then the number of o3 entries
};

// the inputs of one terminal: reach rows of the three counted opponents and
// their pair tables ([52][52] dense-card pair -> range index, HS if none)
template <class T>
struct Opp3 {
    const T *r1, *r2, *r3;
    const int *pair1, *pair2;
    const int *code3;                 // hand codes of the third opponent ([HS])
    int H3, HS, deck;
};

// phase 1: the combo matrices A, B (zero outside 0..deck-1) and PT cleared
template <class T>
SSB_CR3_HD void phase_gather(int tid, int nt, const Opp3<T> &in, const Tables &t) {
    for (int i = tid; i < kS * kS; i += nt) {
        const int c = i / kS, e = i - c * kS;
        double a = 0.0, b = 0.0;
        if (c < in.deck && e < in.deck) {
            const int j1 = in.pair1[c * 52 + e], j2 = in.pair2[c * 52 + e];
            if (j1 < in.HS) a = static_cast<double>(in.r1[j1]);
            if (j2 < in.HS) b = static_cast<double>(in.r2[j2]);
        }
        t.A[i] = a;
        t.B[i] = b;
    }
}

// phase 2: per card c (one item each): u, the positive-cell masks and counts
SSB_CR3_HD void phase_rows(int tid, int nt, const Tables &t) {
    for (int c = tid; c < kS; c += nt) {
        double sa = 0.0, sb = 0.0;
        unsigned long long ma = 0ull, mb = 0ull;
        for (int e = 0; e < kS; ++e) {
            const double a = t.A[c * kS + e], b = t.B[c * kS + e];
            sa += a;
            sb += b;
            if (a > 0.0) ma |= 1ull << e;
            if (b > 0.0) mb |= 1ull << e;
        }
        t.uA[c] = sa;
        t.uB[c] = sb;
        t.mA[c] = ma;
        t.mB[c] = mb;
        t.iuA[c] = popc64(ma);
        t.iuB[c] = popc64(mb);
    }
}

// phase 3: P = A B and its transpose, one cell per item (fixed order over c)
SSB_CR3_HD void phase_product(int tid, int nt, const Tables &t) {
    for (int i = tid; i < kS * kS; i += nt) {
        const int e = i / kS, f = i - e * kS;
        double s = 0.0;
        for (int c = 0; c < kS; ++c) s += t.A[e * kS + c] * t.B[c * kS + f];
        t.P[i] = s;
        t.PT[f * kS + e] = s;
    }
}

// phase 3, tiled: the same P and PT, 4 x 4 cells per item (13 x 13 items):
// A is symmetric, so row c of A is its column c, and each cell still sums
// over c = 0 .. kS-1 in order (the same value as phase_product), with a
// quarter of the table reads
SSB_CR3_HD void phase_product_tiled(int tid, int nt, const Tables &t) {
    constexpr int kT = kS / 4;
    for (int q = tid; q < kT * kT; q += nt) {
        const int e0 = (q / kT) * 4, f0 = (q % kT) * 4;
        double acc[4][4] = {};
        for (int c = 0; c < kS; ++c) {
            double xs[4], ys[4];
            for (int i = 0; i < 4; ++i) {
                xs[i] = t.A[c * kS + e0 + i];
                ys[i] = t.B[c * kS + f0 + i];
            }
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j) acc[i][j] += xs[i] * ys[j];
        }
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                t.P[(e0 + i) * kS + f0 + j] = acc[i][j];
                t.PT[(f0 + j) * kS + e0 + i] = acc[i][j];
            }
    }
}

// phase 4: per card w and d, and on item kS the third opponent's compacted
// list (in hand order) -- done by one item, so its order is fixed
template <class T>
SSB_CR3_HD void phase_vectors(int tid, int nt, const Opp3<T> &in, const Tables &t, bool compact = true) {
    for (int c = tid; c <= kS; c += nt) {
        if (c == kS) {
            if (!compact) continue;
            long long n = 0;
            double f3 = 0.0;
            for (int h = 0; h < in.H3; ++h) {
                const int code = in.code3[h];
                if (code & 0x10000) continue;   // touches the board
                const T r = in.r3[h];
                if (!(r > T(0))) continue;
                t.r3[n] = static_cast<double>(r);
                f3 += t.r3[n];
                t.xy[n] = static_cast<unsigned short>(((code >> 20) & 63) | (((code >> 26) & 63) << 8));
                ++n;
            }
            t.isc[4] = n;
            t.sc[4] = f3;
            continue;
        }
        double w = 0.0;
        int iw = 0;
        for (int f = 0; f < kS; ++f) {
            w += t.A[c * kS + f] * t.uB[f] + t.B[c * kS + f] * t.uA[f];
            iw += ((t.mA[c] >> f) & 1ull ? t.iuB[f] : 0) + ((t.mB[c] >> f) & 1ull ? t.iuA[f] : 0);
        }
        t.w[c] = w;
        t.iw[c] = iw;
        t.d[c] = t.P[c * kS + c];
        t.id[c] = popc64(t.mA[c] & t.mB[c]);
    }
}

// the third opponent's compacted positive-reach list in hand order (the
// kS item of phase_vectors, on its own)
template <class T>
SSB_CR3_HD void compact_third_list(const Opp3<T> &in, const Tables &t) {
    long long n = 0;
    double f3 = 0.0;
    for (int h = 0; h < in.H3; ++h) {
        const int code = in.code3[h];
        if (code & 0x10000) continue;   // touches the board
        const T r = in.r3[h];
        if (!(r > T(0))) continue;
        t.r3[n] = static_cast<double>(r);
        f3 += t.r3[n];
        t.xy[n] = static_cast<unsigned short>(((code >> 20) & 63) | (((code >> 26) & 63) << 8));
        ++n;
    }
    t.isc[4] = n;
    t.sc[4] = f3;
}

// phase 5 (one item): the scalars
SSB_CR3_HD void phase_scalars(int tid, const Tables &t) {
    if (tid != 0) return;
    double fa = 0.0, fb = 0.0, q = 0.0, e = 0.0;
    long long ifa = 0, ifb = 0, iq = 0, ie = 0;
    for (int c = 0; c < kS; ++c) {
        fa += t.uA[c];
        fb += t.uB[c];
        q += t.uA[c] * t.uB[c];
        e += t.d[c];
        ifa += t.iuA[c];
        ifb += t.iuB[c];
        iq += static_cast<long long>(t.iuA[c]) * t.iuB[c];
        ie += t.id[c];
    }
    t.sc[0] = 0.5 * fa;
    t.sc[1] = 0.5 * fb;
    t.sc[2] = q;
    t.sc[3] = 0.5 * e;
    t.isc[0] = ifa / 2;
    t.isc[1] = ifb / 2;
    t.isc[2] = iq;
    t.isc[3] = ie / 2;
}

#if defined(__CUDACC__)
// Device form of phases 2-5 for a block of 256 threads, in two barrier-
// separated steps after the gather (3 barriers per table build instead of 5):
//   step 1: per card u and counts, four lanes per card (13 cells each,
//           partial sums combined by shuffles in a fixed order), beside the
//           tiled product, which skips the card indices whose cells of the
//           tile are zero (sparse ranges; the masks come from the gather);
//   step 2: per card w, d and their counts, four lanes per card, and the
//           block scalars by the last warp (one lane per card pair of slots,
//           shuffle sums in a fixed order).
// The integer parts are exact; the FP64 sums differ from the one-item phases
// only in summation order.
__device__ __forceinline__ double quad_sum(double v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v + __shfl_xor_sync(0xffffffffu, v, 2);
}
// Device gather (phase 1 with or without rank-position bounds): each warp
// fills whole rows c of A and B (columns 0-31, then 32-51) and takes each
// row's positive-cell masks from two ballots, so the masks exist before the
// product.  Cells outside rows / columns 0 .. deck-1 are 0.
template <class T>
__device__ __forceinline__ void gather_dev(int tid, const Opp3<T> &in, const Tables &t, const int *pos1, int lo1,
                                           int hi1, const int *pos2, int lo2, int hi2) {
    const int warp = tid >> 5, lane = tid & 31;
    for (int c = warp; c < kS; c += 8) {
        unsigned long long ma = 0ull, mb = 0ull;
        for (int half = 0; half < 2; ++half) {
            const int e = half * 32 + lane;
            double a = 0.0, b = 0.0;
            if (e < kS && c < in.deck && e < in.deck) {
                const int j1 = in.pair1[c * 52 + e], j2 = in.pair2[c * 52 + e];
                if (j1 < in.HS && (!pos1 || (pos1[j1] >= lo1 && pos1[j1] < hi1))) a = static_cast<double>(in.r1[j1]);
                if (j2 < in.HS && (!pos2 || (pos2[j2] >= lo2 && pos2[j2] < hi2))) b = static_cast<double>(in.r2[j2]);
            }
            if (e < kS) {
                t.A[c * kS + e] = a;
                t.B[c * kS + e] = b;
            }
            ma |= static_cast<unsigned long long>(__ballot_sync(0xffffffffu, a > 0.0)) << (32 * half);
            mb |= static_cast<unsigned long long>(__ballot_sync(0xffffffffu, b > 0.0)) << (32 * half);
        }
        if (lane == 0) {
            t.mA[c] = ma;
            t.mB[c] = mb;
        }
    }
}

// the tiled product skipping card indices c whose four A cells (rows e0..,
// column c: A is symmetric) or four B cells are all zero: their terms are
// exact +0, so every cell keeps phase_product's value
__device__ __forceinline__ void product_masked(int tid, const Tables &t) {
    constexpr int kT = kS / 4;
    if (tid >= kT * kT) return;
    const int e0 = (tid / kT) * 4, f0 = (tid % kT) * 4;
    double acc[4][4] = {};
    for (int c = 0; c < kS; ++c) {
        if (!((t.mA[c] >> e0) & 0xfull) || !((t.mB[c] >> f0) & 0xfull)) continue;
        double xs[4], ys[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            xs[i] = t.A[c * kS + e0 + i];
            ys[i] = t.B[c * kS + f0 + i];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] += xs[i] * ys[j];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            t.P[(e0 + i) * kS + f0 + j] = acc[i][j];
            t.PT[(f0 + j) * kS + e0 + i] = acc[i][j];
        }
}

// step 1 after gather_dev: per card u and counts (masks from the gather)
// beside the masked product
__device__ __forceinline__ void build_step1(int tid, const Tables &t) {
    if (tid < 224) {   // warps 0-6: cards tid / 4 < kS (lanes of cards 52-55 add zeros)
        const int c = tid >> 2, part = tid & 3;
        double sa = 0.0, sb = 0.0;
        if (c < kS)
            for (int e = part * 13; e < part * 13 + 13; ++e) {
                sa += t.A[c * kS + e];
                sb += t.B[c * kS + e];
            }
        sa = quad_sum(sa);
        sb = quad_sum(sb);
        if (part == 0 && c < kS) {
            t.uA[c] = sa;
            t.uB[c] = sb;
            t.iuA[c] = __popcll(t.mA[c]);
            t.iuB[c] = __popcll(t.mB[c]);
        }
    }
    product_masked(tid, t);
}
__device__ __forceinline__ void build_step2(int tid, const Tables &t) {
    if (tid < 224) {
        const int c = tid >> 2, part = tid & 3;
        double w = 0.0;
        int iw = 0;
        if (c < kS) {
            const unsigned long long mAc = t.mA[c], mBc = t.mB[c];
            for (int f = part * 13; f < part * 13 + 13; ++f) {
                w += t.A[c * kS + f] * t.uB[f] + t.B[c * kS + f] * t.uA[f];
                iw += ((mAc >> f) & 1ull ? t.iuB[f] : 0) + ((mBc >> f) & 1ull ? t.iuA[f] : 0);
            }
        }
        w = quad_sum(w);
        iw += __shfl_xor_sync(0xffffffffu, iw, 1);
        iw += __shfl_xor_sync(0xffffffffu, iw, 2);
        if (part == 0 && c < kS) {
            t.w[c] = w;
            t.iw[c] = iw;
            t.d[c] = t.P[c * kS + c];
            t.id[c] = __popcll(t.mA[c] & t.mB[c]);
        }
    } else {
        // the scalars from step 1's vectors and P's diagonal
        const int lane = tid & 31;
        double fa = 0.0, fb = 0.0, q = 0.0, e = 0.0;
        long long ifa = 0, ifb = 0, iq = 0, ie = 0;
        for (int c = lane; c < kS; c += 32) {
            fa += t.uA[c];
            fb += t.uB[c];
            q += t.uA[c] * t.uB[c];
            e += t.P[c * kS + c];
            ifa += t.iuA[c];
            ifb += t.iuB[c];
            iq += static_cast<long long>(t.iuA[c]) * t.iuB[c];
            ie += __popcll(t.mA[c] & t.mB[c]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            fa += __shfl_xor_sync(0xffffffffu, fa, o);
            fb += __shfl_xor_sync(0xffffffffu, fb, o);
            q += __shfl_xor_sync(0xffffffffu, q, o);
            e += __shfl_xor_sync(0xffffffffu, e, o);
            ifa += __shfl_xor_sync(0xffffffffu, ifa, o);
            ifb += __shfl_xor_sync(0xffffffffu, ifb, o);
            iq += __shfl_xor_sync(0xffffffffu, iq, o);
            ie += __shfl_xor_sync(0xffffffffu, ie, o);
        }
        if (lane == 0) {
            t.sc[0] = 0.5 * fa;
            t.sc[1] = 0.5 * fb;
            t.sc[2] = q;
            t.sc[3] = 0.5 * e;
            t.isc[0] = ifa / 2;
            t.isc[1] = ifb / 2;
            t.isc[2] = iq;
            t.isc[3] = ie / 2;
        }
    }
}
#endif

// The traverser's part of every sum in D2(S), S = {a, b} + {x, y}: computed
// once per hand, reused for every third-opponent hand (x, y).
struct HandPart {
    double Aab, Bab, fa, fb, Phh, wd, dd;
};

SSB_CR3_HD HandPart hand_part(int a, int b, const Tables &t) {
    const double *A = t.A, *B = t.B, *P = t.P;
    HandPart hp;
    hp.Aab = A[a * kS + b];
    hp.Bab = B[a * kS + b];
    hp.fa = t.sc[0] - t.uA[a] - t.uA[b] + hp.Aab;
    hp.fb = t.sc[1] - t.uB[a] - t.uB[b] + hp.Bab;
    hp.Phh = P[a * kS + a] + P[a * kS + b] + P[b * kS + a] + P[b * kS + b];
    hp.wd = t.w[a] + t.w[b];
    hp.dd = t.d[a] + t.d[b];
    return hp;
}

// D2({a, b, x, y}) of the tables' two matrices; (x, y) disjoint from (a, b).
// The cross terms between {a, b} and {x, y} read rows x and y of the
// symmetric A, B and of P and P^T.
SSB_CR3_HD double d2_at(const HandPart &hp, int a, int b, int x, int y, const Tables &t) {
    const double *A = t.A, *B = t.B, *P = t.P, *PT = t.PT;
    const double Aax = A[x * kS + a], Aay = A[y * kS + a], Abx = A[x * kS + b], Aby = A[y * kS + b];
    const double Bax = B[x * kS + a], Bay = B[y * kS + a], Bbx = B[x * kS + b], Bby = B[y * kS + b];
    const double Axy = A[x * kS + y], Bxy = B[x * kS + y];
    const double Px = P[x * kS + a] + P[x * kS + b] + PT[x * kS + a] + PT[x * kS + b];
    const double Py = P[y * kS + a] + P[y * kS + b] + PT[y * kS + a] + PT[y * kS + b];
    const double Poo = P[x * kS + x] + P[x * kS + y] + P[y * kS + x] + P[y * kS + y];
    const double FAS = hp.fa - t.uA[x] - t.uA[y] + Axy + (Aax + Aay + Abx + Aby);
    const double FBS = hp.fb - t.uB[x] - t.uB[y] + Bxy + (Bax + Bay + Bbx + Bby);
    const double ua = t.uA[a] - hp.Aab - Aax - Aay, ub = t.uA[b] - hp.Aab - Abx - Aby;
    const double ux = t.uA[x] - Axy - Aax - Abx, uy = t.uA[y] - Axy - Aay - Aby;
    const double va = t.uB[a] - hp.Bab - Bax - Bay, vb = t.uB[b] - hp.Bab - Bbx - Bby;
    const double vx = t.uB[x] - Bxy - Bax - Bbx, vy = t.uB[y] - Bxy - Bay - Bby;
    const double QS = t.sc[2] - (hp.wd + t.w[x] + t.w[y]) + (hp.Phh + Poo + Px + Py) -
                      (ua * va + ub * vb + ux * vx + uy * vy);
    const double ES = t.sc[3] - (hp.dd + t.d[x] + t.d[y]) + hp.Aab * hp.Bab + Axy * Bxy + Aax * Bax + Aay * Bay +
                      Abx * Bbx + Aby * Bby;
    return FAS * FBS - QS + ES;
}

// the same on the 0/1 matrices: the number of disjoint (o1, o2) pairs of
// positive reach avoiding {a, b, x, y}
struct HandCount {
    long long fa, fb;
    int iAab, iBab, Phh, wd, dd;
};

SSB_CR3_HD HandCount hand_count_part(int a, int b, const Tables &t) {
    const unsigned long long mAa = t.mA[a], mAb = t.mA[b], mBa = t.mB[a], mBb = t.mB[b];
    HandCount hc;
    hc.iAab = static_cast<int>((mAa >> b) & 1ull);
    hc.iBab = static_cast<int>((mBa >> b) & 1ull);
    hc.fa = t.isc[0] - t.iuA[a] - t.iuA[b] + hc.iAab;
    hc.fb = t.isc[1] - t.iuB[a] - t.iuB[b] + hc.iBab;
    hc.Phh = popc64(mAa & mBa) + popc64(mAa & mBb) + popc64(mAb & mBa) + popc64(mAb & mBb);
    hc.wd = t.iw[a] + t.iw[b];
    hc.dd = t.id[a] + t.id[b];
    return hc;
}

SSB_CR3_HD long long c2_at(const HandCount &hc, int a, int b, int x, int y, const Tables &t) {
    const unsigned long long mAa = t.mA[a], mAb = t.mA[b], mBa = t.mB[a], mBb = t.mB[b];
    const unsigned long long mAx = t.mA[x], mAy = t.mA[y], mBx = t.mB[x], mBy = t.mB[y];
    const int Aax = static_cast<int>((mAx >> a) & 1ull), Aay = static_cast<int>((mAy >> a) & 1ull);
    const int Abx = static_cast<int>((mAx >> b) & 1ull), Aby = static_cast<int>((mAy >> b) & 1ull);
    const int Bax = static_cast<int>((mBx >> a) & 1ull), Bay = static_cast<int>((mBy >> a) & 1ull);
    const int Bbx = static_cast<int>((mBx >> b) & 1ull), Bby = static_cast<int>((mBy >> b) & 1ull);
    const int Axy = static_cast<int>((mAx >> y) & 1ull), Bxy = static_cast<int>((mBx >> y) & 1ull);
    const int Px = popc64(mAx & mBa) + popc64(mAx & mBb) + popc64(mAa & mBx) + popc64(mAb & mBx);
    const int Py = popc64(mAy & mBa) + popc64(mAy & mBb) + popc64(mAa & mBy) + popc64(mAb & mBy);
    const int Poo = popc64(mAx & mBx) + popc64(mAx & mBy) + popc64(mAy & mBx) + popc64(mAy & mBy);
    const long long FAS = hc.fa - t.iuA[x] - t.iuA[y] + Axy + (Aax + Aay + Abx + Aby);
    const long long FBS = hc.fb - t.iuB[x] - t.iuB[y] + Bxy + (Bax + Bay + Bbx + Bby);
    const long long ua = t.iuA[a] - hc.iAab - Aax - Aay, ub = t.iuA[b] - hc.iAab - Abx - Aby;
    const long long ux = t.iuA[x] - Axy - Aax - Abx, uy = t.iuA[y] - Axy - Aay - Aby;
    const long long va = t.iuB[a] - hc.iBab - Bax - Bay, vb = t.iuB[b] - hc.iBab - Bbx - Bby;
    const long long vx = t.iuB[x] - Bxy - Bax - Bbx, vy = t.iuB[y] - Bxy - Bay - Bby;
    const long long QS = t.isc[2] - (hc.wd + t.iw[x] + t.iw[y]) + (hc.Phh + Poo + Px + Py) -
                         (ua * va + ub * vb + ux * vx + uy * vy);
    const long long ES = t.isc[3] - (hc.dd + t.id[x] + t.id[y]) + hc.iAab * hc.iBab + Axy * Bxy + Aax * Bax +
                         Aay * Bay + Abx * Bbx + Aby * Bby;
    return FAS * FBS - QS + ES;
}

// the mass of one traverser hand with dense cards (a, b), a board card
// given as the dummy index (the deck size)
SSB_CR3_HD double hand_mass(int a, int b, const Tables &t) {
    const HandPart hp = hand_part(a, b, t);
    double mass = 0.0;
    const long long n3 = t.isc[4];
    for (long long k = 0; k < n3; ++k) {
        const int x = t.xy[k] & 0xff, y = t.xy[k] >> 8;
        if (x == a || x == b || y == a || y == b) continue;   // shares a card with the traverser
        mass += t.r3[k] * d2_at(hp, a, b, x, y, t);
    }
    return mass;
}

// the number of disjoint tuples with positive reach products: the same
// formula on the 0/1 matrices, exact in integers
SSB_CR3_HD long long hand_count(int a, int b, const Tables &t) {
    const HandCount hc = hand_count_part(a, b, t);
    long long count = 0;
    const long long n3 = t.isc[4];
    for (long long k = 0; k < n3; ++k) {
        const int x = t.xy[k] & 0xff, y = t.xy[k] >> 8;
        if (x == a || x == b || y == a || y == b) continue;
        count += c2_at(hc, a, b, x, y, t);
    }
    return count;
}

// ---------------------------------------------------------------------------
// four-way showdowns (three live opponents): class masses by rank position
// ---------------------------------------------------------------------------
// With the traverser's tie group at rank positions [lo, hi), an opponent
// hand is weaker (L) below lo and ties (E) inside.  The traverser wins when
// all three opponents are weaker and splits with the tying ones when none is
// stronger, so its value is a sum over classes of the reference's
// coefficient times the mass of the tuples in the class.  Conditioning on
// the third opponent's class (L or E) and splitting the first two
// opponents' matrices into their L and E parts gives every class mass as a
// sum of D2 masses of matrix pairs (X, Y), X, Y in {L, E}; each pair's mass
// is exact-zeroed by its own count.

// phase 1 for a class pair: A restricted to the first opponent's hands at
// positions [lo1, hi1), B to the second's at [lo2, hi2) (pos1 / pos2: the
// opponents' rank positions per hand, -1 for a hand the board blocks)
template <class T>
SSB_CR3_HD void phase_gather_cls(int tid, int nt, const Opp3<T> &in, const Tables &t, const int *pos1, int lo1,
                                 int hi1, const int *pos2, int lo2, int hi2) {
    for (int i = tid; i < kS * kS; i += nt) {
        const int c = i / kS, e = i - c * kS;
        double a = 0.0, b = 0.0;
        if (c < in.deck && e < in.deck) {
            const int j1 = in.pair1[c * 52 + e], j2 = in.pair2[c * 52 + e];
            if (j1 < in.HS && pos1[j1] >= lo1 && pos1[j1] < hi1) a = static_cast<double>(in.r1[j1]);
            if (j2 < in.HS && pos2[j2] >= lo2 && pos2[j2] < hi2) b = static_cast<double>(in.r2[j2]);
        }
        t.A[i] = a;
        t.B[i] = b;
    }
}

// the third opponent's positive-reach live hands in hand order with their
// rank positions (one item; run once per block)
template <class T>
SSB_CR3_HD void compact_third(int tid, const Opp3<T> &in, const Tables &t, const int *pos3, int *p3) {
    if (tid != 0) return;
    long long n = 0;
    double f3 = 0.0;
    for (int h = 0; h < in.H3; ++h) {
        const int code = in.code3[h];
        if ((code & 0x10000) || pos3[h] < 0) continue;
        const T r = in.r3[h];
        if (!(r > T(0))) continue;
        t.r3[n] = static_cast<double>(r);
        t.xy[n] = static_cast<unsigned short>(((code >> 20) & 63) | (((code >> 26) & 63) << 8));
        p3[n] = pos3[h];
        f3 += t.r3[n];
        ++n;
    }
    t.isc[4] = n;
    t.sc[4] = f3;
}

// r3 * D2 of the current pair summed over the third opponent's hands:
// out[0] over positions below lo, out[1] over [lo, hi), out[2] over all;
// cnt[] the same tuple counts on the 0/1 matrices (only when want_count)
SSB_CR3_HD void hand_mass_cls(int a, int b, const Tables &t, const int *p3, int lo, int hi, double out[3],
                              long long cnt[3], bool want_count) {
    const HandPart hp = hand_part(a, b, t);
    const HandCount hc = hand_count_part(a, b, t);
    out[0] = out[1] = out[2] = 0.0;
    cnt[0] = cnt[1] = cnt[2] = 0;
    const long long n3 = t.isc[4];
    for (long long k = 0; k < n3; ++k) {
        const int x = t.xy[k] & 0xff, y = t.xy[k] >> 8;
        if (x == a || x == b || y == a || y == b) continue;
        const double v = t.r3[k] * d2_at(hp, a, b, x, y, t);
        const int cls = p3[k] < lo ? 0 : (p3[k] < hi ? 1 : 2);
        if (cls < 2) out[cls] += v;
        out[2] += v;
        if (want_count) {
            const long long n = c2_at(hc, a, b, x, y, t);
            if (cls < 2) cnt[cls] += n;
            cnt[2] += n;
        }
    }
}

// The class masses of hand_mass_cls below a tie group (out[0]: third
// opponent weaker, out[1]: tying), summed over the third opponent's entries
// k = k0, k0 + kstep, ... only; entries stronger than the group are skipped
// (no class of a pair uses them).  k_term_sd3 spreads a tie group's hands
// and these slices over its warps; slices combined in a fixed order give the
// same sums up to the order of the additions.
SSB_CR3_HD void hand_mass_cls_slice(int a, int b, const Tables &t, const int *p3, int lo, int hi, long long k0,
                                    long long kstep, double out[2], long long cnt[2], bool want_count) {
    const HandPart hp = hand_part(a, b, t);
    HandCount hc{};
    if (want_count) hc = hand_count_part(a, b, t);
    out[0] = out[1] = 0.0;
    cnt[0] = cnt[1] = 0;
    const long long n3 = t.isc[4];
    for (long long k = k0; k < n3; k += kstep) {
        if (p3[k] >= hi) continue;
        const int x = t.xy[k] & 0xff, y = t.xy[k] >> 8;
        if (x == a || x == b || y == a || y == b) continue;
        const int cls = p3[k] < lo ? 0 : 1;
        if (want_count)
            cnt[cls] += c2_at(hc, a, b, x, y, t);
        else
            out[cls] += t.r3[k] * d2_at(hp, a, b, x, y, t);
    }
}

// ---------------------------------------------------------------------------
// four-way showdowns on sparse ranges: the weaker parts' tables grown along
// the walk, and the tying parts' pairs evaluated from them directly
// ---------------------------------------------------------------------------
// An opponent hand added to one side of the tables: dense cards x, y and a
// positive reach r.
struct EHand {
    double r;
    int x, y;
};

// Adds hands to the first opponent's matrix A (side 0) or the second's B
// (side 1), keeping every table equal to a direct build of the larger
// sets (up to the order of the FP64 additions; the counts exactly).  Work
// items f = 0 .. kS-1 own card f -- for side 0 column f of P (rows x, y),
// row f of A and PT, for side 1 row f of P and column f of PT, row f of B --
// plus w[f], iw[f], d[f], id[f]; item kS adds to the scalars.  Within a call
// only the other side's tables are read, so the items are independent:
// side 0, then (after a block barrier) side 1 adds the product's cross
// terms through the updated A.
SSB_CR3_HD void add_hands(int tid, int nt, const Tables &t, int side, const EHand *L, int n) {
    double *X = side == 0 ? t.A : t.B;            // the matrix that grows
    const double *Y = side == 0 ? t.B : t.A;      // the other one
    double *uX = side == 0 ? t.uA : t.uB;
    const double *uY = side == 0 ? t.uB : t.uA;
    int *iuX = side == 0 ? t.iuA : t.iuB;
    const int *iuY = side == 0 ? t.iuB : t.iuA;
    unsigned long long *mX = side == 0 ? t.mA : t.mB;
    const unsigned long long *mY = side == 0 ? t.mB : t.mA;
    for (int f = tid; f <= kS; f += nt) {
        if (f == kS) {
            double s0 = 0.0, s2 = 0.0, s3 = 0.0;
            long long i2 = 0, i3 = 0;
            for (int k = 0; k < n; ++k) {
                const int x = L[k].x, y = L[k].y;
                const double r = L[k].r;
                s0 += r;
                s2 += r * (uY[x] + uY[y]);
                s3 += r * Y[x * kS + y];
                i2 += iuY[x] + iuY[y];
                i3 += static_cast<long long>((mY[x] >> y) & 1ull);
            }
            t.sc[side] += s0;
            t.sc[2] += s2;
            t.sc[3] += s3;
            t.isc[side] += n;
            t.isc[2] += i2;
            t.isc[3] += i3;
            continue;
        }
        double wf = 0.0;
        int iwf = 0;
        for (int k = 0; k < n; ++k) {
            const int x = L[k].x, y = L[k].y;
            const double r = L[k].r;
            if (side == 0) {
                // P = A B: rows x and y gain r * rows y and x of B
                t.P[x * kS + f] += r * Y[y * kS + f];
                t.P[y * kS + f] += r * Y[x * kS + f];
                t.PT[f * kS + x] = t.P[x * kS + f];
                t.PT[f * kS + y] = t.P[y * kS + f];
            } else {
                // columns x and y gain r * columns y and x of A
                t.P[f * kS + x] += t.A[f * kS + y] * r;
                t.P[f * kS + y] += t.A[f * kS + x] * r;
                t.PT[x * kS + f] = t.P[f * kS + x];
                t.PT[y * kS + f] = t.P[f * kS + y];
            }
            // w = A uB + B uA: the grown u at x, y times the other matrix's column
            wf += r * (Y[f * kS + x] + Y[f * kS + y]);
            iwf += static_cast<int>((mY[f] >> x) & 1ull) + static_cast<int>((mY[f] >> y) & 1ull);
            if (f == x || f == y) {
                const int o = f == x ? y : x;
                X[f * kS + o] = r;
                mX[f] |= 1ull << o;
                uX[f] += r;
                iuX[f] += 1;
                wf += r * uY[o];
                iwf += iuY[o];
            }
        }
        t.w[f] += wf;
        t.iw[f] += iwf;
        t.d[f] = t.P[f * kS + f];
        t.id[f] = popc64(t.mA[f] & t.mB[f]);
    }
}

// One opponent's mass (and count of positive-reach hands) avoiding the six
// cards c[0..5], from its side of the tables: F - sum u + sum of the matrix
// over the pairs of the six (a hand touches at most two of them).
SSB_CR3_HD void one_opp_avoid6(const double *M, const double *u, const unsigned long long *m, const int *iu, double F,
                               long long iF, const int c[6], double *mass, long long *count) {
    double s = F;
    long long n = iF;
    for (int i = 0; i < 6; ++i) {
        s -= u[c[i]];
        n -= iu[c[i]];
    }
    for (int i = 0; i < 6; ++i)
        for (int j = i + 1; j < 6; ++j) {
            s += M[c[i] * kS + c[j]];
            n += static_cast<long long>((m[c[i]] >> c[j]) & 1ull);
        }
    *mass = s;
    *count = n;
}

// Class masses and exact tuple counts of pair pr (EL 1, LE 2, EE 3) for the
// traverser hand (a, b) when the tables hold the weaker parts L1 (A) and L2
// (B) and the tying parts are the short lists E1, E2: EL sums over E1 the
// second opponent's L2 mass avoiding the six cards, LE over E2 the first's
// L1 mass, EE enumerates E1 x E2.  Third-opponent entries k0, k0 + kstep, ...
// below hi, split by class as in hand_mass_cls_slice; a term without a tuple
// adds nothing, so a class whose count is 0 has mass exactly 0.
SSB_CR3_HD void e_pair_slice(int pr, int a, int b, const Tables &t, const EHand *E1, int n1, const EHand *E2, int n2,
                             const int *p3, int lo, int hi, long long k0, long long kstep, double out[2],
                             long long cnt[2]) {
    out[0] = out[1] = 0.0;
    cnt[0] = cnt[1] = 0;
    const long long n3 = t.isc[4];
    const EHand *E = pr == 1 ? E1 : E2;
    const int nE = pr == 1 ? n1 : n2;
    for (long long k = k0; k < n3; k += kstep) {
        if (p3[k] >= hi) continue;
        const int x = t.xy[k] & 0xff, y = t.xy[k] >> 8;
        if (x == a || x == b || y == a || y == b) continue;
        const int cls = p3[k] < lo ? 0 : 1;
        const double r3 = t.r3[k];
        if (pr == 3) {
            for (int i = 0; i < n1; ++i) {
                const int e = E1[i].x, f = E1[i].y;
                if (e == a || e == b || e == x || e == y || f == a || f == b || f == x || f == y) continue;
                for (int j = 0; j < n2; ++j) {
                    const int g = E2[j].x, h = E2[j].y;
                    if (g == a || g == b || g == x || g == y || g == e || g == f || h == a || h == b || h == x ||
                        h == y || h == e || h == f)
                        continue;
                    out[cls] += r3 * (E1[i].r * E2[j].r);
                    cnt[cls] += 1;
                }
            }
            continue;
        }
        for (int i = 0; i < nE; ++i) {
            const int e = E[i].x, f = E[i].y;
            if (e == a || e == b || e == x || e == y || f == a || f == b || f == x || f == y) continue;
            const int c6[6] = {a, b, x, y, e, f};
            double m;
            long long n;
            if (pr == 1)
                one_opp_avoid6(t.B, t.uB, t.mB, t.iuB, t.sc[1], t.isc[1], c6, &m, &n);
            else
                one_opp_avoid6(t.A, t.uA, t.mA, t.iuA, t.sc[0], t.isc[0], c6, &m, &n);
            if (n > 0) {
                out[cls] += r3 * (E[i].r * m);
                cnt[cls] += n;
            }
        }
    }
}

// The largest FP64 rounding of hand_mass on a tuple set that is empty: each
// of its ~H3 terms is a few F_A F_B in size times r3 <= F3, so 1e-9 of
// F_A F_B F3 bounds it with a wide margin; a hand whose mass is at or below
// this bound takes the exact count to decide whether it is 0.
SSB_CR3_HD double zero_bound(const Tables &t) {
    return 1e-9 * (t.sc[0] + 1.0) * (t.sc[1] + 1.0) * (t.sc[4] + 1.0);
}

}  // namespace cr3
}  // namespace ssb

namespace ssb {
namespace cr3 {

// The traverser's value at a four-way showdown from its class masses:
// m[pair][cls] with pairs LL, EL, LE, EE (first opponent's class, second's)
// and cls 0 = third opponent weaker, 1 = tying; total = every tuple's mass.
// Coefficients as the reference computes them (pot / winners - bet in
// float, -bet for a loss); a class whose coefficient is 0 adds exactly 0.
struct Sd3Coef {
    double win, two, three, four, loss;
};

SSB_CR3_HD double sd3_value(const double m[4][2], double total, const Sd3Coef &k) {
    const double win = m[0][0];
    const double two = (m[1][0] + m[2][0]) + m[0][1];
    const double three = m[3][0] + (m[1][1] + m[2][1]);
    const double four = m[3][1];
    const double loss = total - ((m[0][0] + m[1][0] + m[2][0] + m[3][0]) + (m[0][1] + m[1][1] + m[2][1] + m[3][1]));
    return k.win * win + k.two * two + k.three * three + k.four * four + k.loss * loss;
}

}  // namespace cr3
}  // namespace ssb

namespace ssb {
namespace cr3 {

// ---------------------------------------------------------------------------
// per-thread steps of the four-way showdown block (k_term_sd3), shared with
// the host check: the kernel runs them between its barriers
// ---------------------------------------------------------------------------

struct Sd3Thread {
    int h;               // the traverser's hand at this thread's rank position, -1 if none
    int a, b;            // its dense cards
    int glo, ghi;        // its tie group [glo, ghi)
    double total;        // every tuple's mass (third opponent of any class)
    double m[4][2];      // class masses: pairs LL, EL, LE, EE x third opponent weaker / tying
};

// the thread at rank position q (q < qend): hand, cards and tie group from
// the showdown tables (pos_hand [np][ncomb], hand codes, SdCombo groups)
template <class Combo>
SSB_CR3_HD void sd3_thread_init(int q, int qend, const int *pos_hand_t, const int *hand_code_t,
                                const Combo *sd_combo, Sd3Thread &s) {
    s.h = q < qend ? pos_hand_t[q] : -1;
    s.a = s.b = s.glo = s.ghi = 0;
    s.total = 0.0;
    for (int p = 0; p < 4; ++p) s.m[p][0] = s.m[p][1] = 0.0;
    if (s.h >= 0) {
        const int hc = hand_code_t[s.h];
        s.a = (hc >> 20) & 63;
        s.b = (hc >> 26) & 63;
        s.glo = sd_combo[q].lo;
        s.ghi = sd_combo[q].hi;
    }
}

// after the full pair's tables: the total, exact 0 when no tuple exists
SSB_CR3_HD void sd3_thread_total(Sd3Thread &s, const Tables &t, const int *p3) {
    if (s.h < 0) return;
    double o[3];
    long long cnt[3];
    hand_mass_cls(s.a, s.b, t, p3, s.glo, s.ghi, o, cnt, false);
    s.total = o[2];
    if (fabs(s.total) <= zero_bound(t)) {
        hand_mass_cls(s.a, s.b, t, p3, s.glo, s.ghi, o, cnt, true);
        if (cnt[2] == 0) s.total = 0.0;
    }
}

// the first / second opponent's position ranges of pair pr (LL, EL, LE, EE)
// for the tie group [lo, hi): weaker [0, lo), tying [lo, hi)
SSB_CR3_HD void sd3_pair_bounds(int pr, int lo, int hi, int *lo1, int *hi1, int *lo2, int *hi2) {
    *lo1 = (pr & 1) ? lo : 0;
    *hi1 = (pr & 1) ? hi : lo;
    *lo2 = (pr & 2) ? lo : 0;
    *hi2 = (pr & 2) ? hi : lo;
}

// after pair pr's tables, for a thread of the group [lo, hi): its two class
// masses, each exact 0 when its count is 0
SSB_CR3_HD void sd3_thread_pair(Sd3Thread &s, const Tables &t, const int *p3, int pr, int lo, int hi) {
    double o[3];
    long long cnt[3];
    hand_mass_cls(s.a, s.b, t, p3, lo, hi, o, cnt, false);
    const double zb = zero_bound(t);
    if (fabs(o[0]) <= zb || fabs(o[1]) <= zb) {
        double oc[3];
        hand_mass_cls(s.a, s.b, t, p3, lo, hi, oc, cnt, true);
        for (int k = 0; k < 2; ++k)
            if (fabs(o[k]) <= zb && cnt[k] == 0) o[k] = 0.0;
    }
    s.m[pr][0] = o[0];
    s.m[pr][1] = o[1];
}

// the value from the class masses, with the reference's float coefficients
SSB_CR3_HD double sd3_thread_value(const Sd3Thread &s, float pot, float bet) {
    const Sd3Coef k{static_cast<double>(pot - bet), static_cast<double>(pot / 2.0f - bet),
                    static_cast<double>(pot / 3.0f - bet), static_cast<double>(pot / 4.0f - bet),
                    -static_cast<double>(bet)};
    return sd3_value(s.m, s.total, k);
}

// the three-opponent fold / leaf mass of a traverser hand from its hand code
// (a board card maps to the zero dummy row `deck`), exact 0 without a tuple
SSB_CR3_HD double cr3_hand_value_mass(int hand_code, int deck, const Tables &t) {
    int a = (hand_code >> 20) & 63, b = (hand_code >> 26) & 63;
    if (a >= deck) a = deck;
    if (b >= deck) b = deck;
    double m = hand_mass(a, b, t);
    if (fabs(m) <= zero_bound(t) && hand_count(a, b, t) == 0) m = 0.0;
    return m;
}

}  // namespace cr3
}  // namespace ssb
