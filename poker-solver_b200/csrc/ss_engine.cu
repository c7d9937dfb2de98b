// ss_engine.cu -- host orchestration: one resident subgame per Session.
//
// Replaces the per-iteration launch loop of the reference (street_solve.cu:
// 1471-1550), which re-runs regret matching for every node and re-propagates
// every opponent's reach for every traverser, with blocking copies in between.
// Here:
//   * regret matching is fused into the kernels that consume the strategy
//     (reach propagation and the traverser's value/regret update), so no
//     strategy array exists;
//   * a player's strategy only changes when that player traverses (the
//     reference's regret pruning never changes a strategy), so each player's
//     reach is re-propagated once per iteration, right after its own regret
//     update, instead of once per other traverser;
//   * an iteration (terminals, bottom-up updates, reach) is captured once as
//     a CUDA graph and replayed; the iteration number lives on the device;
//   * plan, tables and state stay resident in a Session, so a solve can be
//     extended, reset or read without re-uploading.
#include "ss_session.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace ssb {

namespace {

thread_local std::string g_err;

struct Blob {
    std::vector<char> host;
    // append bytes at the next 256-byte boundary; a null source reserves zeros
    size_t add(const void *src, size_t bytes) {
        size_t off = (host.size() + 255) & ~static_cast<size_t>(255);
        host.resize(off + bytes);
        if (bytes && src) std::memcpy(host.data() + off, src, bytes);
        return off;
    }
    template <class T>
    size_t add(const std::vector<T> &v) {
        return add(v.data(), v.size() * sizeof(T));
    }
};

void keep_pool_warm(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = 8ull << 30;  // keep up to 8 GiB cached between solves
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done[device] = true;
}

const char *kClassName[SS_PROFILE_CLASSES] = {"reach", "cfv", "term_fill", "term_cr1",
                                             "term_cr2", "term_sd", "term_enum", "other"};

}  // namespace

void set_error(const std::string &msg) { g_err = msg; }
const char *last_error() { return g_err.c_str(); }

// Average strategies are the one large output (200 MB for a full-range
// 3-player turn).  Written into a freshly allocated buffer, the copy first
// faults in every page and stages through pageable memory; instead the
// buffer comes from a pool of page-locked blocks that ss_free_output hands
// back, so a later solve of similar size copies straight into mapped,
// locked pages.  The pool is never destroyed (it would outlive the CUDA
// runtime at exit); at most kPoolIdleBytes wait idle.
namespace {
constexpr size_t kPoolIdleBytes = size_t(2) << 30;
constexpr size_t kPoolGrain = size_t(2) << 20;

struct HostPool {
    struct Block {
        size_t bytes;
        bool locked;
    };
    std::mutex mu;
    std::vector<std::pair<void *, Block>> out, idle;
    size_t idle_bytes = 0;

    static void release(void *p, const Block &b) {
        if (b.locked) cudaHostUnregister(p);
        std::free(p);
    }
};
HostPool &host_pool() {
    static HostPool *pool = new HostPool;
    return *pool;
}
}  // namespace

void *host_block_take(size_t bytes) {
    HostPool &hp = host_pool();
    const size_t cap = (std::max<size_t>(bytes, 1) + kPoolGrain - 1) / kPoolGrain * kPoolGrain;
    {
        std::lock_guard<std::mutex> lk(hp.mu);
        // the smallest idle block that fits and wastes at most half of itself
        size_t best = hp.idle.size();
        for (size_t i = 0; i < hp.idle.size(); ++i) {
            const size_t b = hp.idle[i].second.bytes;
            if (b >= cap && b <= 2 * cap && (best == hp.idle.size() || b < hp.idle[best].second.bytes)) best = i;
        }
        if (best < hp.idle.size()) {
            auto blk = hp.idle[best];
            hp.idle.erase(hp.idle.begin() + static_cast<std::ptrdiff_t>(best));
            hp.idle_bytes -= blk.second.bytes;
            hp.out.push_back(blk);
            return blk.first;
        }
    }
    void *p = std::aligned_alloc(4096, cap);
    if (!p) return nullptr;
    const bool locked = cudaHostRegister(p, cap, cudaHostRegisterPortable) == cudaSuccess;
    if (!locked) cudaGetLastError();   // stays pageable; clear the error
    std::lock_guard<std::mutex> lk(hp.mu);
    hp.out.push_back({p, HostPool::Block{cap, locked}});
    return p;
}

bool host_block_give(void *p) {
    if (!p) return false;
    HostPool &hp = host_pool();
    std::pair<void *, HostPool::Block> blk{nullptr, {0, false}};
    {
        std::lock_guard<std::mutex> lk(hp.mu);
        auto it = std::find_if(hp.out.begin(), hp.out.end(), [p](const auto &e) { return e.first == p; });
        if (it == hp.out.end()) return false;
        blk = *it;
        hp.out.erase(it);
        if (hp.idle_bytes + blk.second.bytes <= kPoolIdleBytes) {
            hp.idle.push_back(blk);
            hp.idle_bytes += blk.second.bytes;
            return true;
        }
    }
    HostPool::release(blk.first, blk.second);
    return true;
}

#define CK(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            set_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #call); \
            return e_ == cudaErrorMemoryAllocation ? SS_ERR_NOMEM : SS_ERR_CUDA;      \
        }                                                                             \
    } while (0)


int Session::init(const Problem &pb, const SolveConfig &cfg) {
    int rc = build_plan(pb, &P);
    if (rc != SS_OK) return rc;
    if (P.enum_work > kEnumLimitPerIter) {
        set_error("terminals with three or more counted opponents (or multiway showdowns) need " +
                  std::to_string(P.enum_work) +
                  " tuple visits per iteration; only small ranges are supported for them");
        return SS_ERR_UNSUPPORTED;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device");
        return SS_ERR_NO_DEVICE;
    }
    if (cfg.device < 0 || cfg.device >= ndev) {
        set_error("device ordinal out of range");
        return SS_ERR_INVALID;
    }
    device = cfg.device;
    graph_iters = std::max(1, cfg.graph_iterations);
    CK(cudaSetDevice(device));
    keep_pool_warm(device);
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    if (!cfg.batch_member) {
        // side streams of the session's own captured iterations (a batch
        // member's launches are the batch's)
        CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        for (int k = 0; k < TK_COUNT; ++k) {
            CK(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
        }
    }
    const int np = P.np;
    const size_t HS = static_cast<size_t>(P.HS);
    const size_t E = static_cast<size_t>(P.E), N = static_cast<size_t>(P.N);

    // ---- static tables and the minimum bytes of every launch ------------
    Blob b;
    size_t o_heads[SS_MAX_PLAYERS][TK_COUNT] = {};
    size_t o_reach[SS_MAX_PLAYERS], o_cfv[SS_MAX_PLAYERS], o_term[SS_MAX_PLAYERS][TK_COUNT],
        o_rootfr[SS_MAX_PLAYERS];
    for (int p = 0; p < np; ++p) {
        std::vector<ReachItem> all;
        for (auto &lv : P.reach_levels[p]) {
            reach_lv[p].push_back({static_cast<int>(all.size()), static_cast<int>(lv.size())});
            double by = 0;
            for (auto &it : lv) by += (2.0 * it.na + 1.0) * 4.0 * P.H[p];
            reach_bytes[p].push_back(by);
            all.insert(all.end(), lv.begin(), lv.end());
        }
        o_reach[p] = b.add(all);
        std::vector<CfvItem> call;
        for (auto &lv : P.cfv_levels[p]) {
            cfv_lv[p].push_back({static_cast<int>(call.size()), static_cast<int>(lv.size())});
            double by = 0;
            for (auto &it : lv) {
                const int nfr = P.fr_off[it.first_edge + it.na] - P.fr_off[it.first_edge];
                by += (4.0 * it.na + nfr + 1.0) * 4.0 * P.H[p];
            }
            cfv_bytes[p].push_back(by);
            call.insert(call.end(), lv.begin(), lv.end());
        }
        o_cfv[p] = b.add(call);
        for (int k = 0; k < TK_COUNT; ++k) {
            double by = 0;
            for (auto &it : P.term[p][k]) {
                by += 4.0 * HS;  // value row
                if (it.leaf_off >= 0 && k != TK_ZERO) by += 4.0 * P.H[p];
                if (k != TK_ZERO && k != TK_LEAF0)
                    for (int i = 0; i < it.k; ++i) by += 4.0 * P.H[it.opp_player[i]];
            }
            term_bytes[p][k] = by;
            o_term[p][k] = b.add(P.term[p][k]);
            if (!P.term_heads[p][k].empty()) o_heads[p][k] = b.add(P.term_heads[p][k]);
        }
        o_rootfr[p] = b.add(P.root_fr[p]);
    }
    const size_t o_fr_off = b.add(P.fr_off);
    const size_t o_fr_items = b.add(P.fr_items);
    const size_t o_code = b.add(P.hand_code);
    const size_t o_pair = b.add(P.pair_idx);
    const size_t o_cross = b.add(P.cross_idx);
    const size_t o_sdpos = b.add(P.sd_pos);
    const size_t o_str = b.add(P.strength);
    const size_t o_sdc = b.add(P.sd_combo);
    const size_t o_sdl = b.add(P.sd_card_list);
    const size_t o_sdp = b.add(P.sd_card_partner);
    const size_t o_ph = b.add(P.pos_hand);
    const size_t o_pp = b.add(P.pos_prefix);
    const size_t o_seg = b.add(P.sd_seg);
    const size_t o_chunk = b.add(P.sd_chunk);
    std::vector<int> dfe, dna, dpl;
    for (int x : P.dec_nodes) {
        dfe.push_back(P.first_edge[x]);
        dna.push_back(pb.nodes[x].num_children);
        dpl.push_back(pb.nodes[x].player);
    }
    const size_t o_dfe = b.add(dfe), o_dna = b.add(dna), o_dpl = b.add(dpl);
    dec_na_host = dna;
    dec_player_host = dpl;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&dbase), std::max<size_t>(b.host.size(), 256), stream));
    CK(cudaMemcpyAsync(dbase, b.host.data(), b.host.size(), cudaMemcpyHostToDevice, stream));
    for (int p = 0; p < np; ++p) {
        reach_items[p] = reinterpret_cast<const ReachItem *>(dbase + o_reach[p]);
        cfv_items[p] = reinterpret_cast<const CfvItem *>(dbase + o_cfv[p]);
        for (int k = 0; k < TK_COUNT; ++k) {
            term_items[p][k] = reinterpret_cast<const TermItem *>(dbase + o_term[p][k]);
            term_heads[p][k] = P.term_heads[p][k].empty() ? nullptr
                                                          : reinterpret_cast<const int *>(dbase + o_heads[p][k]);
        }
        root_fr[p] = reinterpret_cast<const int *>(dbase + o_rootfr[p]);
    }
    dec_fe = reinterpret_cast<const int *>(dbase + o_dfe);
    dec_na = reinterpret_cast<const int *>(dbase + o_dna);
    dec_pl = reinterpret_cast<const int *>(dbase + o_dpl);
    c.dec_fe = dec_fe;
    c.dec_na = dec_na;
    c.dec_pl = dec_pl;
    c.live = 1;

    // ---- state: regrets, strategy sums, reach (weights in the last np rows), values
    nR = E * HS;
    nReach = (E + np) * HS;
    nVal = N * HS;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&dstate), (2 * nR + nReach + nVal) * sizeof(float), stream));
    CK(cudaMemsetAsync(dstate, 0, (2 * nR + nReach + nVal) * sizeof(float), stream));
    CK(cudaMallocAsync(reinterpret_cast<void **>(&diter), sizeof(int), stream));
    float *R = dstate, *S = R + nR, *reach = S + nR, *val = reach + nReach;
    {
        std::vector<float> w(static_cast<size_t>(np) * HS, 0.f);
        for (int p = 0; p < np; ++p)
            for (int h = 0; h < P.H[p]; ++h) w[p * HS + h] = pb.weights[p][h];
        CK(cudaMemcpyAsync(reach + E * HS, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice,
                           stream));
        CK(cudaStreamSynchronize(stream));  // the staging vector must outlive the copy
        host_w = w;
    }
    if (pb.leaf_values && pb.num_leaves > 0) {
        const size_t n = static_cast<size_t>(pb.num_leaves) * np * P.max_h;
        CK(cudaMallocAsync(reinterpret_cast<void **>(&dleaf), n * sizeof(float), stream));
        CK(cudaMemcpyAsync(dleaf, pb.leaf_values, n * sizeof(float), cudaMemcpyHostToDevice, stream));
    }
    n_rs = static_cast<size_t>(P.root_na) * P.H[P.root_player];
    CK(cudaMallocAsync(reinterpret_cast<void **>(&dsmall), (n_rs + HS) * sizeof(float), stream));

    c.R = R;
    c.S = S;
    c.reach = reach;
    c.val = val;
    c.fr_off = reinterpret_cast<const int *>(dbase + o_fr_off);
    c.fr_items = reinterpret_cast<const int *>(dbase + o_fr_items);
    c.hand_code = reinterpret_cast<const int *>(dbase + o_code);
    c.pair_idx = reinterpret_cast<const int *>(dbase + o_pair);
    c.cross_idx = reinterpret_cast<const int *>(dbase + o_cross);
    c.sd_pos = reinterpret_cast<const int *>(dbase + o_sdpos);
    c.strength = reinterpret_cast<const unsigned *>(dbase + o_str);
    c.sd_combo = reinterpret_cast<const SdCombo *>(dbase + o_sdc);
    c.sd_card_list = reinterpret_cast<const short *>(dbase + o_sdl);
    c.sd_card_partner = reinterpret_cast<const short *>(dbase + o_sdp);
    c.pos_hand = reinterpret_cast<const int *>(dbase + o_ph);
    c.pos_prefix = reinterpret_cast<const int *>(dbase + o_pp);
    c.sd_seg = reinterpret_cast<const int *>(dbase + o_seg);
    c.sd_chunk = reinterpret_cast<const int *>(dbase + o_chunk);
    for (int p = 0; p <= SS_MAX_PLAYERS; ++p) c.sd_seg_off[p] = P.sd_seg_off[p];
    c.leaf_values = dleaf;
    c.iter = diter;
    c.HS = P.HS;
    c.np = np;
    c.ncomb = P.ncomb;
    for (int lg = 0; lg < kSd2Merge; ++lg) c.sd_span[lg] = P.sd_span[lg];
    c.deck = P.deck;
    for (int p = 0; p < SS_MAX_PLAYERS; ++p) {
        c.H[p] = p < np ? P.H[p] : 0;
        c.dup[p] = p < np ? P.dup[p] : 0;
    }
    frozen_root = pb.frozen ? pb.frozen[0] : -1;
    c.snap = dsmall;
    c.root_fe = P.first_edge[0];
    c.root_na = P.root_na;
    c.root_frozen = frozen_root;
    c.root_player = P.root_player;
    return reset();
}

int Session::reset() {
    CK(cudaSetDevice(device));
    CK(cudaMemsetAsync(dstate, 0, 2 * nR * sizeof(float), stream));
    CK(cudaMemsetAsync(c.val, 0, nVal * sizeof(float), stream));
    CK(cudaMemsetAsync(diter, 0, sizeof(int), stream));
    CK(cudaMemsetAsync(dsmall, 0, (n_rs + P.HS) * sizeof(float), stream));
    for (int p = 0; p < P.np; ++p) CK(reach(p));  // all regrets zero: uniform (or frozen) play
    iterations = 0;
    return SS_OK;
}

int Session::run(int iters) {
    if (iters < 0) {
        set_error("iterations must be >= 0");
        return SS_ERR_INVALID;
    }
    if (iters == 0) return SS_OK;
    if (P.enum_work * (iterations + iters) > kEnumLimitTotal) {
        set_error("enumerated terminals would need more than " + std::to_string(kEnumLimitTotal) +
                  " tuple visits; only small ranges are supported for them");
        return SS_ERR_UNSUPPORTED;
    }
    CK(cudaSetDevice(device));
    const int rest = iters - 1;
    const int qA = rest / graph_iters, rC = rest % graph_iters;
    if (qA > 0 && !gA) CK(capture(graph_iters, false, &gA));
    if (rC > 0 && !gC) CK(capture(1, false, &gC));
    if (!gB) CK(capture(1, true, &gB));
    for (int i = 0; i < qA; ++i) CK(cudaGraphLaunch(gA, stream));
    for (int i = 0; i < rC; ++i) CK(cudaGraphLaunch(gC, stream));
    CK(cudaGraphLaunch(gB, stream));
    iterations += iters;
    return SS_OK;
}

int Session::output(SSOutput *out) {
    std::memset(out, 0, sizeof(*out));
    CK(cudaSetDevice(device));
    const int np = P.np, tl = np - 1;
    const size_t n_avg = static_cast<size_t>(P.num_dec) * SS_MAX_ACTIONS * P.max_h;
    float *davg = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&davg), std::max<size_t>(n_avg, 1) * sizeof(float), stream));
    float *d_rev = dsmall + n_rs;
    cudaError_t e = cudaSuccess;
    if (iterations >= 1)
        e = launch_sum_rows(c, root_fr[tl], static_cast<int>(P.root_fr[tl].size()), d_rev, P.H[tl], stream);
    if (e == cudaSuccess)
        e = launch_avg_strategy(c, dec_fe, dec_na, dec_pl, P.num_dec, P.max_h, davg, stream);
    float *h_rs = static_cast<float *>(std::calloc(std::max<size_t>(n_rs, 1), sizeof(float)));
    float *h_rev = static_cast<float *>(std::calloc(static_cast<size_t>(np) * P.max_h, sizeof(float)));
    float *h_avg = static_cast<float *>(host_block_take(std::max<size_t>(n_avg, 1) * sizeof(float)));
    int *h_ids = static_cast<int *>(std::malloc(std::max<size_t>(P.num_dec, 1) * sizeof(int)));
    if (!h_rs || !h_rev || !h_avg || !h_ids) {
        std::free(h_rs);
        std::free(h_rev);
        host_block_give(h_avg);
        std::free(h_ids);
        cudaFreeAsync(davg, stream);
        set_error("host allocation of the outputs failed");
        return SS_ERR_NOMEM;
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_avg, davg, n_avg * sizeof(float), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && iterations >= 1)
        e = cudaMemcpyAsync(h_rs, dsmall, n_rs * sizeof(float), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && iterations >= 1)
        e = cudaMemcpyAsync(h_rev, d_rev, static_cast<size_t>(P.H[tl]) * sizeof(float),
                            cudaMemcpyDeviceToHost, stream);
    cudaFreeAsync(davg, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    unsigned fault = 0;
    if (e == cudaSuccess) e = read_device_fault(&fault, stream);
    if (e != cudaSuccess || fault) {
        std::free(h_rs);
        std::free(h_rev);
        host_block_give(h_avg);
        std::free(h_ids);
        if (e != cudaSuccess)
            set_error(std::string("CUDA: ") + cudaGetErrorString(e));
        else
            set_error("a kernel recorded a device fault (code " + std::to_string(fault) +
                      "): the tensor-core product's completion wait ran out or it got a subgame it does not serve");
        return SS_ERR_CUDA;
    }
    for (int i = 0; i < P.num_dec; ++i) h_ids[i] = P.dec_nodes[i];
    out->root_strategy = h_rs;
    out->root_num_actions = P.root_na;
    out->root_player = P.root_player;
    out->root_ev = h_rev;
    out->avg_strategies = h_avg;
    out->avg_strategy_node_ids = h_ids;
    out->num_avg_nodes = P.num_dec;
    out->num_players = np;
    out->max_hands = P.max_h;
    return SS_OK;
}

int Session::profile(SSKernelProfile *prof) {
    std::memset(prof, 0, sizeof(*prof));
    CK(cudaSetDevice(device));
    std::vector<Mark> ms;
    marks = &ms;
    cudaGraphExec_t g = nullptr;
    cudaError_t e = capture(1, true, &g);
    marks = nullptr;
    cudaEvent_t end = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&end);
    if (e == cudaSuccess) e = cudaGraphLaunch(g, stream);
    if (e == cudaSuccess) e = cudaEventRecord(end, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) {
        iterations += 1;
        prof->num_classes = SS_PROFILE_CLASSES;
        for (int k = 0; k < SS_PROFILE_CLASSES; ++k)
            std::strncpy(prof->name[k], kClassName[k], sizeof(prof->name[k]) - 1);
        last_launches.clear();
        for (size_t i = 0; i < ms.size() && e == cudaSuccess; ++i) {
            float t = 0.f;
            e = cudaEventElapsedTime(&t, ms[i].ev, i + 1 < ms.size() ? ms[i + 1].ev : end);
            prof->ms[ms[i].cls] += t;
            prof->bytes[ms[i].cls] += ms[i].bytes;
            prof->launches[ms[i].cls] += 1;
            last_launches.push_back(SSLaunchRecord{ms[i].cls, ms[i].items, static_cast<double>(t), ms[i].bytes});
        }
        float tot = 0.f;
        if (e == cudaSuccess && !ms.empty()) e = cudaEventElapsedTime(&tot, ms.front().ev, end);
        prof->iteration_ms = tot;
    }
    for (auto &m : ms) cudaEventDestroy(m.ev);
    if (end) cudaEventDestroy(end);
    if (g) cudaGraphExecDestroy(g);
    CK(e);
    return SS_OK;
}

int Session::profile_launches(SSLaunchRecord *rec, int max_records, int *num_records) const {
    const int n = static_cast<int>(last_launches.size());
    if (num_records) *num_records = n;
    if (rec)
        for (int i = 0; i < n && i < max_records; ++i) rec[i] = last_launches[i];
    return SS_OK;
}

// Best-response buffers (FP64 reach and values, the profile, the edge ->
// decision table, the deal-mass item and the root sums), allocated on first
// use and kept; also points the context at them, so that the batched checks
// can run this session's best response from the batch's context array.
int Session::ensure_br() {
    if (dbr) return SS_OK;
    const int np = P.np;
    const size_t HS = static_cast<size_t>(P.HS), E = static_cast<size_t>(P.E), N = static_cast<size_t>(P.N);
    const size_t n_avg = static_cast<size_t>(P.num_dec) * SS_MAX_ACTIONS * P.max_h;
    // deal mass term: the players' ranges against each other (valid deals)
    std::memset(&deal, 0, sizeof(deal));
    deal.node = P.N;
    deal.leaf_off = -1;
    deal.payoff = 1.f;
    deal.k = np - 1;
    for (int o = 1; o < np; ++o) {
        deal.opp_row[o - 1] = P.E + o;
        deal.opp_player[o - 1] = o;
    }
    const bool deal_cr3 = np == 4 && !P.dup[1] && !P.dup[2] && P.H[1] >= kCr3MinHands &&
                          P.H[2] >= kCr3MinHands && P.H[3] >= kCr3MinHands;
    deal_kind = np == 1   ? TK_LEAF0
                : np == 2 ? (P.dup[1] ? TK_CR1D : TK_CR1)
                : np == 3 ? TK_CR2
                : deal_cr3 ? TK_CR3
                           : TK_ENUM;
    if (deal_kind == TK_ENUM) {
        double w = P.H[0];
        for (int o = 1; o < np; ++o) w *= std::max(1, P.H[o]);
        if (w > kEnumLimitPerIter) {
            set_error("exploitability: the deal mass of " + std::to_string(np) +
                      " players needs the multiway closed form; only small ranges are supported");
            return SS_ERR_UNSUPPORTED;
        }
    }
    CK(cudaSetDevice(device));
    CK(cudaMallocAsync(reinterpret_cast<void **>(&dbr), ((E + np) + (N + 1)) * HS * sizeof(double), stream));
    CK(cudaMemsetAsync(dbr, 0, ((E + np) + (N + 1)) * HS * sizeof(double), stream));
    std::vector<double> w(host_w.begin(), host_w.end());
    CK(cudaMemcpyAsync(dbr + E * HS, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    Blob t;
    std::vector<int> node_di(P.N, -1), edge_di(P.E);
    for (int i = 0; i < P.num_dec; ++i) node_di[P.dec_nodes[i]] = i;
    for (int e = 0; e < P.E; ++e) edge_di[e] = node_di[P.edge_node[e]];
    const size_t o_edge = t.add(edge_di);
    const size_t o_deal = t.add(&deal, sizeof(deal));
    const int nrow = P.N;
    const size_t o_row = t.add(&nrow, sizeof(int));
    const size_t o_sc = t.add(nullptr, (2 * SS_MAX_PLAYERS + 2) * sizeof(double));
    CK(cudaMallocAsync(reinterpret_cast<void **>(&dbr_tab), t.host.size(), stream));
    CK(cudaMemcpyAsync(dbr_tab, t.host.data(), t.host.size(), cudaMemcpyHostToDevice, stream));
    CK(cudaMallocAsync(reinterpret_cast<void **>(&davg_br), std::max<size_t>(n_avg, 1) * sizeof(float), stream));
    CK(cudaStreamSynchronize(stream));  // host staging must outlive the copies
    br_edge_di = reinterpret_cast<const int *>(dbr_tab + o_edge);
    br_deal = reinterpret_cast<const TermItem *>(dbr_tab + o_deal);
    br_row = reinterpret_cast<const int *>(dbr_tab + o_row);
    br_sc = reinterpret_cast<double *>(dbr_tab + o_sc);
    c.reach_d = dbr;
    c.val_d = dbr + (E + np) * HS;
    c.avg_br = davg_br;
    c.edge_di = br_edge_di;
    c.max_h = P.max_h;
    return SS_OK;
}

// NashConv of an average-strategy profile (the session's own when host_avg is
// null, else avg given in the SSOutput layout), FP64 throughout: every
// player's reach under the profile, then per player the terminal values
// (same closed forms as the CFR path, in double), the profile value and the
// best-response value at its own nodes, and the root sums weighted by the
// player's range.  Exploitability = NashConv / np / starting pot * 100.
int Session::exploitability(const float *host_avg, double *pct, double *nash, double *br, double *cur,
                            double *deal_mass) {
    int rc = ensure_br();
    if (rc != SS_OK) return rc;
    CK(cudaSetDevice(device));
    const int np = P.np;
    const size_t n_avg = static_cast<size_t>(P.num_dec) * SS_MAX_ACTIONS * P.max_h;
    if (host_avg)
        CK(cudaMemcpyAsync(davg_br, host_avg, n_avg * sizeof(float), cudaMemcpyHostToDevice, stream));
    else
        CK(launch_avg_strategy(c, dec_fe, dec_na, dec_pl, P.num_dec, P.max_h, davg_br, stream));
    for (int p = 0; p < np; ++p)
        for (size_t l = 0; l < reach_lv[p].size(); ++l)
            CK(launch_br_reach(c, reach_items[p] + reach_lv[p][l].first, reach_lv[p][l].second, P.H[p],
                               davg_br, br_edge_di, P.max_h, stream));
    for (int t = 0; t < np; ++t) {
        for (int k = 0; k < TK_COUNT; ++k)
            CK(launch_terms_fp64(c, k, term_items[t][k], static_cast<int>(P.term[t][k].size()), t, stream));
        for (int mode = 0; mode < 2; ++mode) {
            for (size_t l = 0; l < cfv_lv[t].size(); ++l)
                CK(launch_br_value(c, cfv_items[t] + cfv_lv[t][l].first, cfv_lv[t][l].second, P.H[t],
                                   davg_br, br_edge_di, P.max_h, mode, stream));
            CK(launch_br_root(c, root_fr[t], static_cast<int>(P.root_fr[t].size()), P.H[t], P.E + t, t, 0,
                              br_sc + 2 * t + mode, stream));
        }
    }
    CK(launch_terms_fp64(c, deal_kind, br_deal, 1, 0, stream));
    CK(launch_br_root(c, br_row, 1, P.H[0], P.E, 0, 1, br_sc + 2 * SS_MAX_PLAYERS, stream));
    double sc[2 * SS_MAX_PLAYERS + 2] = {};
    CK(cudaMemcpyAsync(sc, br_sc, sizeof(sc), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    nashconv_from_sums(sc, pct, nash, br, cur, deal_mass);
    return SS_OK;
}

// sc: per traverser t, [2t] profile value and [2t + 1] best-response value;
// [2 * SS_MAX_PLAYERS] the deal mass
void Session::nashconv_from_sums(const double *sc, double *pct, double *nash, double *br, double *cur,
                                 double *deal_mass) const {
    const int np = P.np;
    double nc = 0.0;
    for (int t = 0; t < np; ++t) {
        if (cur) cur[t] = sc[2 * t];
        if (br) br[t] = sc[2 * t + 1];
        nc += sc[2 * t + 1] - sc[2 * t];
    }
    const double z = sc[2 * SS_MAX_PLAYERS];
    if (deal_mass) *deal_mass = z;
    const double nash_v = z > 0 ? nc / z : 0.0;
    if (nash) *nash = nash_v;
    if (pct) *pct = P.starting_pot > 0 ? nash_v / np / P.starting_pot * 100.0 : 0.0;
}

// ---------------------------------------------------------------------------
// entry points used by the ABI layer
// ---------------------------------------------------------------------------

int session_create(const Problem &pb, const SolveConfig &cfg, Session **out) {
    *out = nullptr;
    Session *s = new Session();
    int rc = s->init(pb, cfg);
    if (rc != SS_OK) {
        delete s;
        return rc;
    }
    *out = s;
    return SS_OK;
}

int session_run(Session *s, int iters) { return s->run(iters); }

int session_sync(Session *s) {
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    return SS_OK;
}

int session_reset(Session *s) { return s->reset(); }
int session_iterations(const Session *s) { return s->iterations; }
int session_output(Session *s, SSOutput *out) { return s->output(out); }
int session_profile(Session *s, SSKernelProfile *p) { return s->profile(p); }
int session_profile_launches(const Session *s, SSLaunchRecord *rec, int max_records, int *num_records) {
    return s->profile_launches(rec, max_records, num_records);
}
int session_exploitability(Session *s, const float *host_avg, double *pct, double *nash, double *br,
                           double *cur, double *z) {
    return s->exploitability(host_avg, pct, nash, br, cur, z);
}
void session_destroy(Session *s) { delete s; }
void *session_stream(Session *s) { return static_cast<void *>(s->stream); }

int solve(const Problem &pb, int iterations, const SolveConfig &cfg, SSOutput *out,
          SSSolveStats *stats) {
    std::memset(out, 0, sizeof(*out));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->exploitability_pct = -1.0;
        stats->nashconv = -1.0;
    }
    if (iterations < 0) {
        set_error("max_iterations must be >= 0");
        return SS_ERR_INVALID;
    }
    Session *s = nullptr;
    int rc = session_create(pb, cfg, &s);
    if (rc != SS_OK) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float ms = 0.f;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        set_error("cudaEventCreate failed");
        rc = SS_ERR_CUDA;
    }
    double pct = -1.0, nash = -1.0;
    int done = 0;
    if (cfg.target_exploitability > 0.f) {
        // run in blocks of check_every iterations until the profile is within
        // the target (or max_iterations); solve time covers the CFR blocks only
        const int step = std::max(1, cfg.check_every);
        float acc = 0.f;
        while (rc == SS_OK && done < iterations) {
            const int n = std::min(step, iterations - done);
            if (cudaEventRecord(e0, s->stream) != cudaSuccess) rc = SS_ERR_CUDA;
            if (rc == SS_OK) rc = s->run(n);
            if (rc == SS_OK && cudaEventRecord(e1, s->stream) != cudaSuccess) rc = SS_ERR_CUDA;
            if (rc == SS_OK) rc = s->exploitability(nullptr, &pct, &nash, nullptr, nullptr, nullptr);
            if (rc == SS_OK && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) acc += ms;
            done += n;
            if (rc == SS_OK && pct <= cfg.target_exploitability) break;
        }
        ms = acc;
    } else {
        if (rc == SS_OK && cudaEventRecord(e0, s->stream) != cudaSuccess) rc = SS_ERR_CUDA;
        if (rc == SS_OK) rc = s->run(iterations);
        if (rc == SS_OK && cudaEventRecord(e1, s->stream) != cudaSuccess) rc = SS_ERR_CUDA;
        if (rc == SS_OK && cudaEventSynchronize(e1) == cudaSuccess &&
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            ms = -1.f;
        done = iterations;
        if (rc == SS_OK && cfg.compute_exploitability)
            rc = s->exploitability(nullptr, &pct, &nash, nullptr, nullptr, nullptr);
    }
    if (rc == SS_OK) rc = s->output(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc == SS_OK && stats) {
        stats->iterations_run = done;
        stats->solve_ms = ms;
        stats->node_hand_updates = s->P.node_hands * done;
        stats->exploitability_pct = pct;
        stats->nashconv = nash;
    }
    session_destroy(s);
    return rc;
}

int exploitability(const Problem &pb, const float *avg, double *pct, double *nash, double *br,
                   double *cur, double *z) {
    SolveConfig cfg;
    Session *s = nullptr;
    int rc = session_create(pb, cfg, &s);
    if (rc != SS_OK) return rc;
    rc = s->exploitability(avg, pct, nash, br, cur, z);
    session_destroy(s);
    return rc;
}

}  // namespace ssb
