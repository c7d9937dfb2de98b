// ss_cr2_tc.cuh -- two counted opponents with the card-pair product
// P = M1 M2 on the 5th-generation tensor cores (tcgen05.mma, kind::tf32,
// accumulator in tensor memory).  Included by ss_kernels.cu inside its
// anonymous namespace, after k_term_cr2, whose closed form, per-card structs
// and exact-zero count this kernel shares; only the way the block builds its
// matrices and P differs:
//
//  * no FP32 combo matrices: the gather writes M1 and M2 straight into the
//    tensor-core operand layout as TF32 pairs (x = hi + lo), two threads per
//    row, and reduces each row to its reach sum and positive-cell mask on the
//    way (the matrices are symmetric, so row sums are the per-card sums u_i);
//  * one thread issues 18 MMAs (three split-TF32 passes x six K steps of 8)
//    into a 128 x 48 FP32 accumulator in tensor memory and commits them to an
//    mbarrier; warps 0-1 read the 48 valid accumulator rows back (one row per
//    thread) into shared memory, with the row sums of P;
//  * the hand phase reads m_i = M_i[a][b] from the staged reach rows at the
//    traverser hand's index in each opponent's range (one coalesced load).
//
// Shared memory stays near 55 KB for a 1152-hand row stride (four blocks per
// SM, 64 tensor-memory columns each: at most 8 x 64 = 512 columns for the 8
// blocks of 256 threads an SM can hold, so an allocation never waits).

constexpr int kTcRows = 48;                   // dense deck bound of this path (turn and river boards)
constexpr int kTcLbo = 6 * 128 + 16;          // K-direction core-matrix stride (bytes), see below
constexpr int kTcSbo = 128;                   // row-group stride (bytes)
constexpr int kTcMat = 12 * kTcLbo;           // one 48 x 48 TF32 operand (bytes)
constexpr int kTcCols = 64;                   // tensor-memory columns (a power of two >= 48)
constexpr int kTcPS = 52;                     // row stride of P in shared memory (floats)
// instruction descriptor of kind::tf32: FP32 accumulator (bits 4-5 = 1), A
// and B TF32 (bits 7-9, 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at
// bit 17, M >> 4 at bit 24; M = 128, N = 48
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((48u >> 3) << 17) | ((128u >> 4) << 24);

// Operand layout (K-major, no swizzle, the canonical form of the shared-memory
// matrix descriptor): core matrices of 8 rows x 16 bytes (4 TF32 along K),
// rows 16 bytes apart inside; row group g = row / 8 and K chunk q = col / 4 at
// byte offset q * kTcLbo + g * kTcSbo.  The 16 bytes of padding in kTcLbo put
// the chunks of one row in different shared-memory bank groups.  With M = 128
// the MMA reads 128 rows of A: rows 48..127 lie in the bytes after the A
// operand (the next operand) and only feed accumulator rows that are never
// read.
__device__ __forceinline__ int tc_offset(int row, int kc) { return kc * kTcLbo + (row >> 3) * kTcSbo + (row & 7) * 16; }

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// shared-memory matrix descriptor: start address, leading (K) and stride
// (row-group) byte offsets, all >> 4; version 1 (bits 46-47); no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr) {
    return static_cast<uint64_t>((addr & 0x3ffffu) >> 4) | (static_cast<uint64_t>(kTcLbo >> 4) << 16) |
           (static_cast<uint64_t>(kTcSbo >> 4) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate));
}
__device__ __forceinline__ void tc_commit(void *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(void *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(void *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// 16 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

constexpr size_t rup16(size_t b) { return (b + 15) & ~static_cast<size_t>(15); }
// dynamic shared memory for row stride HS (the Carve order of the kernel)
constexpr size_t cr2_tc_smem(int HS) {
    return rup16(4 * kTcMat) + 2 * rup16((static_cast<size_t>(HS) + 4) * 4) + rup16(static_cast<size_t>(HS) * 4) +
           rup16(53 * sizeof(Cr2Card)) + rup16(53 * sizeof(Cr2Cnt)) + rup16(53 * 16) + rup16(kTcRows * 4) +
           rup16(sizeof(Cr2Scalars)) + 3 * rup16(kTermGroupMax * 4) + rup16(8) + rup16(4);
}
static_assert(kTcRows * kTcPS * 4 <= 4 * kTcMat, "P fits in the operand space");

// spin limit of the wait for the MMAs (each try_wait may also suspend a while)
constexpr int kTcWaitLimit = 1 << 22;

__global__ void __launch_bounds__(kTermThreads, 4) k_term_cr2_tc(DevCtx c0, const DevCtx *__restrict__ ctxs,
                                                                  const TermItem *__restrict__ items, int trav) {
    wait_prior_grid();
    extern __shared__ __align__(16) char smem[];
    const TermItem *I0 = items + blockIdx.x;
    if (I0->follow) return;   // written by the block of its group's first item
    if (retired(ctxs, I0->sg)) return;
    const int ng = I0->gextra + 1;
    const int o0 = I0->opp_player[0], o1 = I0->opp_player[1];
    const Cr2View<float> V = ctxs ? cr2_view<float>(ctxs[I0->sg], trav, o0, o1) : cr2_view<float>(c0, trav, o0, o1);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int HS = V.HS;
    // the launcher sends only subgames this path serves (shared memory sized
    // for c0's row stride, dense deck of at most 48 cards, no repeated combo)
    if (HS > c0.HS || V.deck > kTcRows || V.dup) {
        if (tid == 0) atomicOr(&g_ss_fault, kFaultTcInput);
        return;
    }
    Carve cv{smem};
    char *ops = cv.take<char>(4 * kTcMat);       // A hi, A lo (M1), B hi, B lo (M2)
    float *P = reinterpret_cast<float *>(ops);   // the product, once the MMAs are done
    float *r1 = cv.take<float>(HS + 4);
    float *r2 = cv.take<float>(HS + 4);
    float *leaf0 = cv.take<float>(HS);
    Cr2Card *card = cv.take<Cr2Card>(53);
    Cr2Cnt *cnt = cv.take<Cr2Cnt>(53);
    ulonglong2 *Bm = cv.take<ulonglong2>(53);   // positive-cell masks of M1 (x) and M2 (y) per card
    float *rsum = cv.take<float>(kTcRows);      // row sums of P
    Cr2Scalars *sc = cv.take<Cr2Scalars>(1);
    int *gnode = cv.take<int>(kTermGroupMax);
    int *gleaf = cv.take<int>(kTermGroupMax);
    float *gpay = cv.take<float>(kTermGroupMax);
    unsigned long long *bar = cv.take<unsigned long long>(1);
    uint32_t *tslot = cv.take<uint32_t>(1);

    // accumulator columns (warp 0) and the MMA completion barrier
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) mbar_init(bar, 1);
    // staging: both opponents' reach rows, each followed by a zero (the pair
    // tables index it for missing pairs), and the first terminal's leaf row
    {
        const float *s1 = V.reach + static_cast<size_t>(I0->opp_row[0]) * HS;
        const float *s2 = V.reach + static_cast<size_t>(I0->opp_row[1]) * HS;
        for (int q = tid * 4; q < HS; q += kTermThreads * 4) {
            cp_async16(r1 + q, s1 + q);
            cp_async16(r2 + q, s2 + q);
        }
        const int lo = I0->leaf_off;
        if (lo >= 0) {
            const float *src = V.leaf + lo;
            for (int h = tid; h < V.Ht; h += kTermThreads) cp_async4(leaf0 + h, src + h);
        }
        if (tid < ng) {
            const TermItem &I = I0[tid];
            gnode[tid] = I.node;
            gleaf[tid] = I.leaf_off;
            gpay[tid] = I.payoff;
        }
        if (tid == 0) {
            r1[HS] = 0.f;
            r2[HS] = 0.f;
        }
    }
    cp_async_wait_all();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    // gather: two threads per matrix row (six 4-column chunks each) write it
    // as TF32 pairs into the operand layout (eight consecutive rows fill one
    // 128-byte core-matrix column, so a warp's stores spread over the banks)
    // and reduce it to its sum (FP32 chunk sums, FP64 across them, fixed
    // order) and its positive-cell mask
    if (tid < 4 * kTcRows) {
        const int m = tid >= 2 * kTcRows ? 1 : 0;
        const int row = (tid >> 1) - m * kTcRows, half = tid & 1;
        const float *r = m ? r2 : r1;
        const int *tab = (m ? V.tab1 : V.tab0) + row * 52;
        char *hb = ops + (2 * m) * kTcMat, *lb = ops + (2 * m + 1) * kTcMat;
        double s = 0.0;
        unsigned long long mask = 0ull;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const int kc = half * 6 + j;
            const int4 ix = __ldg(reinterpret_cast<const int4 *>(tab + kc * 4));
            const float x0 = r[ix.x], x1 = r[ix.y], x2 = r[ix.z], x3 = r[ix.w];
            uint4 hi, lo;
            split_tf32(x0, hi.x, lo.x);
            split_tf32(x1, hi.y, lo.y);
            split_tf32(x2, hi.z, lo.z);
            split_tf32(x3, hi.w, lo.w);
            const int off = tc_offset(row, kc);
            *reinterpret_cast<uint4 *>(hb + off) = hi;
            *reinterpret_cast<uint4 *>(lb + off) = lo;
            s += static_cast<double>((x0 + x1) + (x2 + x3));
            const unsigned bits = (x0 > 0.f ? 1u : 0u) | (x1 > 0.f ? 2u : 0u) | (x2 > 0.f ? 4u : 0u) |
                                  (x3 > 0.f ? 8u : 0u);
            mask |= static_cast<unsigned long long>(bits) << (4 * kc);
        }
        const double so = __shfl_xor_sync(0xffffffffu, s, 1);
        mask |= __shfl_xor_sync(0xffffffffu, mask, 1);
        if (half == 0) {
            const double u = s + so;   // the first half's sum first
            if (m == 0) {
                card[row].u1 = u;
                Bm[row].x = mask;
            } else {
                card[row].u2 = u;
                Bm[row].y = mask;
            }
        }
    }
    fence_async_smem();   // the operands, written by ordinary stores, are read by the tensor core
    __syncthreads();

    // P = A_lo B_hi + A_hi B_lo + A_hi B_hi (the split product, small terms
    // first), six K steps of 8 each; one thread issues, the barrier tracks
    if (tid == 0) {
        tc_fence_after();
        const uint32_t base = smem_u32(ops);
#pragma unroll
        for (int pass = 0; pass < 3; ++pass) {
            const uint32_t a = base + (pass == 0 ? kTcMat : 0);
            const uint32_t b = base + 2 * kTcMat + (pass == 1 ? kTcMat : 0);
#pragma unroll
            for (int s = 0; s < 6; ++s)
                tc_mma(tmem, tc_desc(a + 2 * s * kTcLbo), tc_desc(b + 2 * s * kTcLbo), (pass | s) != 0 ? 1u : 0u);
        }
        tc_commit(bar);
    }
    // meanwhile: per-card counts, entries beyond the deck zeroed
    const int Dp = (V.deck + 3) & ~3;
    if (tid >= 64 && tid < 64 + kTcRows) {
        const int col = tid - 64;
        const ulonglong2 Bc = Bm[col];
        cnt[col] = Cr2Cnt{__popcll(Bc.x), __popcll(Bc.y), 0, 0};
    } else if (tid >= 128 && tid < 128 + kCr2Off + 1 - kTcRows) {
        const int col = kTcRows + tid - 128;
        card[col] = Cr2Card{0.0, 0.0, 0.0, 0.0};
        cnt[col] = Cr2Cnt{0, 0, 0, 0};
        Bm[col] = make_ulonglong2(0ull, 0ull);
    }
    // read-back: warps 0-1 own accumulator lanes 0-63 (row = lane); rows
    // 0..47 are P's
    if (warp < 2) {
        bool done = false;
        for (int i = 0; i < kTcWaitLimit && !done; ++i) done = mbar_try_wait(bar, 0);
        if (!done) atomicOr(&g_ss_fault, kFaultTcWait);
        __syncwarp();   // the tensor-memory loads below are warp-collective
        tc_fence_after();
        const int row = 32 * warp + lane;
        float s = 0.f;
#pragma unroll
        for (int c = 0; c < 48; c += 16) {
            float v[16];
            tmem_ld16(tmem + (static_cast<uint32_t>(32 * warp) << 16) + c, v);
            if (!done) {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.f;
            }
            if (row < kTcRows) {
#pragma unroll
                for (int i = 0; i < 16; ++i) s += v[i];
#pragma unroll
                for (int i = 0; i < 16; i += 4)
                    *reinterpret_cast<float4 *>(P + row * kTcPS + c + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            }
        }
        if (row < kTcRows) rsum[row] = s;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
    }

    // per-card terms: w = row sum + column sum of P (P = M1 M2 with symmetric
    // M1, M2: rowsum = M1 u2, colsum = M2 u1), d = P[c][c]; the last warp
    // forms the block scalars
    if (tid < Dp) {
        const int col = tid;
        float cs = 0.f;
        for (int r = 0; r < Dp; ++r) cs += P[r * kTcPS + col];
        const double w = static_cast<double>(rsum[col]) + static_cast<double>(cs);
        const double d = P[col * kTcPS + col];
        const double u1 = card[col].u1, u2 = card[col].u2;
        card[col].g = u1 * u2 + w - 2.0 * d;
        card[col].d = d;
    } else if (warp == kTermThreads / 32 - 1) {
        double a1 = 0.0, a2 = 0.0, qq = 0.0, e = 0.0;
        int n1 = 0, n2 = 0, nq = 0, nd = 0;
        for (int k = lane; k < Dp; k += 32) {
            const double u1 = card[k].u1, u2 = card[k].u2;
            a1 += u1;
            a2 += u2;
            qq += u1 * u2;
            e += static_cast<double>(P[k * kTcPS + k]);
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

    // card-removal mass of every traverser hand (the closed form of
    // k_term_cr2), written out as factor x mass for every terminal of the group
    const Cr2Scalars S = *sc;
    const double zmin = 1e-4 * S.F1 * S.F2;
    const bool none = !(S.F1 > 0.0 && S.F2 > 0.0);
    const int Ht = V.Ht;
    const int *__restrict__ tc = V.code_t;
    const bool leaf_first = gleaf[0] >= 0;
    const float gp0 = gpay[0];
    float *out0 = V.val + static_cast<size_t>(gnode[0]) * HS;
    for (int h = tid; h < HS; h += kTermThreads) {
        double v = 0.0;
        if (h < Ht && !none) {
            const int hc = __ldg(tc + h);
            const int a = min((hc >> 20) & 63, kCr2Off), b = min((hc >> 26) & 63, kCr2Off);
            const bool on = (a < kCr2Off) && (b < kCr2Off);
            const Cr2Card ga = card[a], gb = card[b];
            // the opponents' reach at this combo (index HS, a zero, when the
            // hand touches the board or an opponent lacks it)
            const double m1 = static_cast<double>(r1[__ldg(V.x0 + h)]);
            const double m2 = static_cast<double>(r2[__ldg(V.x1 + h)]);
            const double pp = on ? static_cast<double>(P[a * kTcPS + b] + P[b * kTcPS + a]) : 0.0;
            const double A1 = S.F1 - ga.u1 - gb.u1 + m1;
            const double A2 = S.F2 - ga.u2 - gb.u2 + m2;
            v = A1 * A2 + S.QD + ga.g + gb.g - m2 * (ga.u1 + gb.u1) - m1 * (ga.u2 + gb.u2) + 3.0 * m1 * m2 - pp;
            if (fabs(v) <= zmin && pair_count(Bm, cnt, a, b, S.IF1, S.IF2, S.IQD) <= 0) v = 0.0;
        }
        const float f0 = h >= Ht ? 0.f : leaf_first ? leaf0[h] : gp0;
        out0[h] = static_cast<float>(static_cast<double>(f0) * v);
        for (int g = 1; g < ng; ++g) {
            const float f = h >= Ht ? 0.f : gleaf[g] >= 0 ? __ldg(V.leaf + gleaf[g] + h) : gpay[g];
            V.val[static_cast<size_t>(gnode[g]) * HS + h] = static_cast<float>(static_cast<double>(f) * v);
        }
    }
}
