// ss_noalloc.cu -- ss_solve_gpu_noalloc: a solve that allocates no GPU memory.
//
// Who needs it: callers that cannot call cudaMalloc at solve time -- a
// process whose device memory is owned by another allocator (a framework's
// caching pool that must not be bypassed), code running under a strict
// no-allocation policy on a serving path, or a host that must not grow its
// CUDA footprint after start-up.  ss_solve_gpu allocates its device state per
// call (stream-ordered pool), creates a stream and instantiates CUDA graphs;
// this entry point does none of that.
//
// How: every byte of device state -- tables, ranges, leaf values, regrets,
// strategy sums, reach, values and output staging -- lives in one file-scope
// `static __device__` array of kArenaBytes (64 MiB).  Every GPU that loads the
// library reserves that array until the process exits.  Host code cannot use
// the array's name as a device address, so the first call on each device
// (with that device current) resolves it once with cudaGetSymbolAddress and
// caches the pointer; make that first call before any stream capture.  The
// kernels are the same as ss_solve_gpu's, launched one by one on the legacy
// default stream; copies are synchronous cudaMemcpy.  Subgames whose state
// does not fit in the arena are rejected with SS_ERR_NOMEM and a message
// giving the size they need.
//
// All calls on a device share the arena and it keeps the last call's data:
// each call re-initialises everything it reads, and two calls that overlap
// on the same GPU (from different host threads) race on the arena.  Host
// memory is used for planning (ordinary heap); nothing is allocated on the
// device, pinned or managed.
#include "ss_kernels.h"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace ssb {

namespace {

constexpr size_t kArenaBytes = 64ull << 20;

static __device__ __align__(256) unsigned char g_arena[kArenaBytes];

std::mutex g_arena_mu;
unsigned char *g_arena_ptr[64] = {};

#define NA_CK(call)                                                                   \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            set_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #call); \
            return SS_ERR_CUDA;                                                       \
        }                                                                             \
    } while (0)

// device address of the arena on the current device (resolved once per device)
int arena_base(int device, unsigned char **out) {
    if (device < 0 || device >= 64) {
        set_error("device ordinal out of range");
        return SS_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(g_arena_mu);
    if (!g_arena_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_arena);
        if (e != cudaSuccess) {
            set_error(std::string("cudaGetSymbolAddress of the static arena failed: ") +
                      cudaGetErrorString(e));
            return SS_ERR_CUDA;
        }
        g_arena_ptr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_arena_ptr[device];
    return SS_OK;
}

// bump layout of the arena: offsets only, checked against kArenaBytes
struct Layout {
    size_t used = 0;
    size_t take(size_t bytes) {
        size_t off = (used + 255) & ~static_cast<size_t>(255);
        used = off + bytes;
        return off;
    }
};

}  // namespace

int solve_noalloc(const Problem &pb, int iterations, SSOutput *out) {
    if (iterations < 0) {
        set_error("max_iterations must be >= 0");
        return SS_ERR_INVALID;
    }
    if (!out || !out->root_strategy || !out->root_ev || !out->avg_strategies ||
        !out->avg_strategy_node_ids) {
        set_error("ss_solve_gpu_noalloc: the caller provides every output array (see street_solve.h)");
        return SS_ERR_INVALID;
    }
    Plan P;
    int rc = build_plan(pb, &P);
    if (rc != SS_OK) return rc;
    if (P.enum_work > 4e9 || P.enum_work * iterations > 2e11) {
        set_error("terminals with three or more counted opponents need too many tuple visits");
        return SS_ERR_UNSUPPORTED;
    }
    int device = 0, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device");
        return SS_ERR_NO_DEVICE;
    }
    NA_CK(cudaGetDevice(&device));
    unsigned char *base = nullptr;
    rc = arena_base(device, &base);
    if (rc != SS_OK) return rc;

    const int np = P.np;
    const size_t HS = static_cast<size_t>(P.HS), E = static_cast<size_t>(P.E), N = static_cast<size_t>(P.N);

    // ---- host images of the tables (same content as a session's) --------
    std::vector<ReachItem> reach_all[SS_MAX_PLAYERS];
    std::vector<std::pair<int, int>> reach_lv[SS_MAX_PLAYERS];
    std::vector<CfvItem> cfv_all[SS_MAX_PLAYERS];
    std::vector<std::pair<int, int>> cfv_lv[SS_MAX_PLAYERS];
    for (int p = 0; p < np; ++p) {
        for (auto &lv : P.reach_levels[p]) {
            reach_lv[p].push_back({static_cast<int>(reach_all[p].size()), static_cast<int>(lv.size())});
            reach_all[p].insert(reach_all[p].end(), lv.begin(), lv.end());
        }
        for (auto &lv : P.cfv_levels[p]) {
            cfv_lv[p].push_back({static_cast<int>(cfv_all[p].size()), static_cast<int>(lv.size())});
            cfv_all[p].insert(cfv_all[p].end(), lv.begin(), lv.end());
        }
    }
    std::vector<int> dfe, dna, dpl;
    for (int x : P.dec_nodes) {
        dfe.push_back(P.first_edge[x]);
        dna.push_back(pb.nodes[x].num_children);
        dpl.push_back(pb.nodes[x].player);
    }
    std::vector<float> w(static_cast<size_t>(np) * HS, 0.f);
    for (int p = 0; p < np; ++p)
        for (int h = 0; h < P.H[p]; ++h) w[p * HS + h] = pb.weights[p][h];
    const size_t n_leaf = (pb.leaf_values && pb.num_leaves > 0)
                              ? static_cast<size_t>(pb.num_leaves) * np * P.max_h : 0;
    const size_t n_avg = static_cast<size_t>(P.num_dec) * SS_MAX_ACTIONS * P.max_h;
    const size_t n_rs = static_cast<size_t>(P.root_na) * P.H[P.root_player];

    // ---- arena layout ----------------------------------------------------
    struct Piece {
        size_t off;
        const void *src;
        size_t bytes;
    };
    std::vector<Piece> uploads;
    Layout L;
    auto up = [&](const void *src, size_t bytes) {
        size_t off = L.take(bytes);
        uploads.push_back({off, src, bytes});
        return off;
    };
    size_t o_reach[SS_MAX_PLAYERS], o_cfv[SS_MAX_PLAYERS], o_term[SS_MAX_PLAYERS][TK_COUNT],
        o_rootfr[SS_MAX_PLAYERS];
    for (int p = 0; p < np; ++p) {
        o_reach[p] = up(reach_all[p].data(), reach_all[p].size() * sizeof(ReachItem));
        o_cfv[p] = up(cfv_all[p].data(), cfv_all[p].size() * sizeof(CfvItem));
        for (int k = 0; k < TK_COUNT; ++k)
            o_term[p][k] = up(P.term[p][k].data(), P.term[p][k].size() * sizeof(TermItem));
        o_rootfr[p] = up(P.root_fr[p].data(), P.root_fr[p].size() * sizeof(int));
    }
    const size_t o_fr_off = up(P.fr_off.data(), P.fr_off.size() * sizeof(int));
    const size_t o_fr_items = up(P.fr_items.data(), P.fr_items.size() * sizeof(int));
    const size_t o_code = up(P.hand_code.data(), P.hand_code.size() * sizeof(int));
    const size_t o_pair = up(P.pair_idx.data(), P.pair_idx.size() * sizeof(int));
    const size_t o_cross = up(P.cross_idx.data(), P.cross_idx.size() * sizeof(int));
    const size_t o_sdpos = up(P.sd_pos.data(), P.sd_pos.size() * sizeof(int));
    const size_t o_str = up(P.strength.data(), P.strength.size() * sizeof(uint32_t));
    const size_t o_sdc = up(P.sd_combo.data(), P.sd_combo.size() * sizeof(SdCombo));
    const size_t o_sdl = up(P.sd_card_list.data(), P.sd_card_list.size() * sizeof(short));
    const size_t o_sdp = up(P.sd_card_partner.data(), P.sd_card_partner.size() * sizeof(short));
    const size_t o_ph = up(P.pos_hand.data(), P.pos_hand.size() * sizeof(int));
    const size_t o_pp = up(P.pos_prefix.data(), P.pos_prefix.size() * sizeof(int));
    const size_t o_seg = up(P.sd_seg.data(), P.sd_seg.size() * sizeof(int));
    const size_t o_chunk = up(P.sd_chunk.data(), P.sd_chunk.size() * sizeof(int));
    const size_t o_dfe = up(dfe.data(), dfe.size() * sizeof(int));
    const size_t o_dna = up(dna.data(), dna.size() * sizeof(int));
    const size_t o_dpl = up(dpl.data(), dpl.size() * sizeof(int));
    const size_t o_leaf = up(pb.leaf_values, n_leaf * sizeof(float));
    const size_t nR = E * HS, nReach = (E + np) * HS, nVal = N * HS;
    const size_t o_state = L.take((2 * nR + nReach + nVal) * sizeof(float));
    const size_t o_weights = o_state + (2 * nR + E * HS) * sizeof(float);  // last np reach rows
    const size_t o_iter = L.take(sizeof(int));
    const size_t o_rs = L.take((n_rs + HS) * sizeof(float));
    const size_t o_avg = L.take(n_avg * sizeof(float));
    if (L.used > kArenaBytes) {
        set_error("ss_solve_gpu_noalloc: this subgame needs " + std::to_string(L.used) +
                  " bytes of device state, the static arena holds " + std::to_string(kArenaBytes));
        return SS_ERR_NOMEM;
    }

    // ---- upload and clear (everything the solve reads is rewritten) -----
    for (const Piece &pc : uploads)
        if (pc.bytes) NA_CK(cudaMemcpy(base + pc.off, pc.src, pc.bytes, cudaMemcpyHostToDevice));
    NA_CK(cudaMemset(base + o_state, 0, (2 * nR + E * HS) * sizeof(float)));
    NA_CK(cudaMemcpy(base + o_weights, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
    NA_CK(cudaMemset(base + o_weights + np * HS * sizeof(float), 0, nVal * sizeof(float)));
    NA_CK(cudaMemset(base + o_iter, 0, sizeof(int)));
    NA_CK(cudaMemset(base + o_rs, 0, (n_rs + HS) * sizeof(float)));

    DevCtx c{};
    float *state = reinterpret_cast<float *>(base + o_state);
    c.R = state;
    c.S = state + nR;
    c.reach = state + 2 * nR;
    c.val = state + 2 * nR + nReach;
    c.fr_off = reinterpret_cast<const int *>(base + o_fr_off);
    c.fr_items = reinterpret_cast<const int *>(base + o_fr_items);
    c.hand_code = reinterpret_cast<const int *>(base + o_code);
    c.pair_idx = reinterpret_cast<const int *>(base + o_pair);
    c.cross_idx = reinterpret_cast<const int *>(base + o_cross);
    c.sd_pos = reinterpret_cast<const int *>(base + o_sdpos);
    c.strength = reinterpret_cast<const unsigned *>(base + o_str);
    c.sd_combo = reinterpret_cast<const SdCombo *>(base + o_sdc);
    c.sd_card_list = reinterpret_cast<const short *>(base + o_sdl);
    c.sd_card_partner = reinterpret_cast<const short *>(base + o_sdp);
    c.pos_hand = reinterpret_cast<const int *>(base + o_ph);
    c.pos_prefix = reinterpret_cast<const int *>(base + o_pp);
    c.sd_seg = reinterpret_cast<const int *>(base + o_seg);
    c.sd_chunk = reinterpret_cast<const int *>(base + o_chunk);
    for (int p = 0; p <= SS_MAX_PLAYERS; ++p) c.sd_seg_off[p] = P.sd_seg_off[p];
    c.leaf_values = n_leaf ? reinterpret_cast<const float *>(base + o_leaf) : nullptr;
    c.iter = reinterpret_cast<int *>(base + o_iter);
    c.HS = P.HS;
    c.np = np;
    c.ncomb = P.ncomb;
    for (int lg = 0; lg < kSd2Merge; ++lg) c.sd_span[lg] = P.sd_span[lg];
    c.deck = P.deck;
    for (int p = 0; p < SS_MAX_PLAYERS; ++p) {
        c.H[p] = p < np ? P.H[p] : 0;
        c.dup[p] = p < np ? P.dup[p] : 0;
    }
    int *iter_ptr = reinterpret_cast<int *>(base + o_iter);
    float *d_rs = reinterpret_cast<float *>(base + o_rs), *d_rev = d_rs + n_rs;
    float *d_avg = reinterpret_cast<float *>(base + o_avg);
    const int frozen_root = pb.frozen ? pb.frozen[0] : -1;
    cudaStream_t s0 = 0;  // legacy default stream

    auto reach = [&](int p) {
        for (auto &lv : reach_lv[p]) {
            cudaError_t e = launch_reach(c, reinterpret_cast<const ReachItem *>(base + o_reach[p]) + lv.first,
                                         lv.second, P.H[p], s0);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    for (int p = 0; p < np; ++p) NA_CK(reach(p));
    for (int it = 1; it <= iterations; ++it) {
        NA_CK(launch_bump(iter_ptr, s0));
        for (int t = 0; t < np; ++t) {
            if (it == iterations && t == np - 1)
                NA_CK(launch_root_strategy(c, P.first_edge[0], P.root_na, frozen_root,
                                           P.H[P.root_player], d_rs, s0));
            for (int k = 0; k < TK_COUNT; ++k)
                NA_CK(launch_terms(c, k, reinterpret_cast<const TermItem *>(base + o_term[t][k]),
                                   static_cast<int>(P.term[t][k].size()), t, s0));
            for (size_t l = 0; l < cfv_lv[t].size(); ++l)
                NA_CK(launch_cfv(c, reinterpret_cast<const CfvItem *>(base + o_cfv[t]) + cfv_lv[t][l].first,
                                 cfv_lv[t][l].second, P.cfv_nlong[t][l], P.H[t], s0));
            NA_CK(reach(t));
        }
    }
    const int tl = np - 1;
    if (iterations >= 1)
        NA_CK(launch_sum_rows(c, reinterpret_cast<const int *>(base + o_rootfr[tl]),
                              static_cast<int>(P.root_fr[tl].size()), d_rev, P.H[tl], s0));
    NA_CK(launch_avg_strategy(c, reinterpret_cast<const int *>(base + o_dfe),
                              reinterpret_cast<const int *>(base + o_dna),
                              reinterpret_cast<const int *>(base + o_dpl), P.num_dec, P.max_h, d_avg, s0));

    // ---- outputs into the caller's arrays --------------------------------
    NA_CK(cudaMemcpy(out->avg_strategies, d_avg, n_avg * sizeof(float), cudaMemcpyDeviceToHost));
    std::memset(out->root_ev, 0, static_cast<size_t>(np) * P.max_h * sizeof(float));
    if (iterations >= 1) {
        NA_CK(cudaMemcpy(out->root_strategy, d_rs, n_rs * sizeof(float), cudaMemcpyDeviceToHost));
        NA_CK(cudaMemcpy(out->root_ev, d_rev, static_cast<size_t>(P.H[tl]) * sizeof(float),
                         cudaMemcpyDeviceToHost));
    } else {
        std::memset(out->root_strategy, 0, n_rs * sizeof(float));
    }
    for (int i = 0; i < P.num_dec; ++i) out->avg_strategy_node_ids[i] = P.dec_nodes[i];
    out->root_num_actions = P.root_na;
    out->root_player = P.root_player;
    out->num_avg_nodes = P.num_dec;
    out->num_players = np;
    out->max_hands = P.max_h;
    return SS_OK;
}

}  // namespace ssb
