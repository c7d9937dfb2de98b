// ss_batch.cu -- batched and served forms.
//
// Batch: many resident subgames (Sessions) of different size, street and
// player count advance together.  Their per-level work lists are merged, so
// one launch covers level l of traverser t for every member (each item reads
// its subgame's context, item.sg); one launch advances every member's
// iteration counter and one per pass snapshots the root strategies.  A block
// of iterations is captured as one CUDA graph; members can be added or
// retired between blocks, each keeps its own iteration count, and arithmetic
// per subgame is identical to a solve alone (three-way showdown sweeps keep
// each subgame's own run merge through a block map).
//
// Server: continuous batching on one GPU.  Requests are copied at submission
// and admitted into the running batch while their estimated device footprint
// fits the memory budget; the worker runs iteration blocks, checks each
// member's FP64 exploitability at block ends, and retires a member when it
// reaches the target (or the iteration cap), freeing its memory for the next
// requests.  Latency = submission to retirement.
#include "ss_session.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

namespace ssb {

#define BCK(call)                                                                     \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            set_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #call); \
            return e_ == cudaErrorMemoryAllocation ? SS_ERR_NOMEM : SS_ERR_CUDA;      \
        }                                                                             \
    } while (0)

class Batch {
  public:
    int device = 0;
    int graph_iters = 10;
    cudaStream_t stream = nullptr;
    std::vector<Session *> subs;   // members (owned); nullptr once released
    std::vector<char> active;
    std::vector<int> iters_run;

    ~Batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (br_graph) cudaGraphExecDestroy(br_graph);
        if (stream) {
            if (dctx) cudaFreeAsync(dctx, stream);
            if (dlists) cudaFreeAsync(dlists, stream);
            if (dsc) cudaFreeAsync(dsc, stream);
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        if (hsc) cudaFreeHost(hsc);
        for (Session *s : subs) delete s;
    }

    int init(int dev, int g) {
        device = dev;
        graph_iters = std::max(1, g);
        BCK(cudaSetDevice(device));
        BCK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        return SS_OK;
    }

    // a member gets its best-response buffers here, so that every check of
    // the batch is one merged launch sequence
    int add(Session *s, int *slot) {
        int rc = s->ensure_br();
        if (rc != SS_OK) return rc;
        subs.push_back(s);
        active.push_back(1);
        iters_run.push_back(0);
        work.push_back(0.0);
        dirty = true;
        *slot = static_cast<int>(subs.size()) - 1;
        return SS_OK;
    }

    // stop iterating member i (its state stays readable until released): its
    // live flag in the device context array turns 0, so its items in the
    // captured graphs return at once; the graphs are rebuilt without the
    // retired members only once they hold most of the captured work
    int retire(int i) {
        active[i] = 0;
        if (dctx && i < built_members) {
            static const int zero = 0;
            BCK(cudaMemcpyAsync(reinterpret_cast<char *>(dctx + i) + offsetof(DevCtx, live), &zero, sizeof(int),
                                cudaMemcpyHostToDevice, stream));
        }
        live_work -= work[i];
        if (live_work < 0.5 * built_work) dirty = true;
        return SS_OK;
    }

    void release(int i) {
        delete subs[i];
        subs[i] = nullptr;
    }

    int num_active() const {
        int n = 0;
        for (char a : active) n += a;
        return n;
    }

    // wait for queued blocks (before reading members on their own streams)
    int sync() {
        BCK(cudaSetDevice(device));
        BCK(cudaStreamSynchronize(stream));
        return SS_OK;
    }

    int run(int iters) {
        if (iters <= 0 || num_active() == 0) return SS_OK;
        BCK(cudaSetDevice(device));
        if (dirty) {
            int rc = rebuild();
            if (rc != SS_OK) return rc;
        }
        int done = 0;
        while (iters - done >= graph_iters) {
            BCK(cudaGraphLaunch(graph, stream));
            done += graph_iters;
        }
        for (; done < iters; ++done) BCK(iteration());
        for (size_t i = 0; i < subs.size(); ++i)
            if (active[i]) {
                iters_run[i] += iters;
                subs[i]->iterations = iters_run[i];
            }
        return SS_OK;
    }

    // FP64 exploitability of every active member's average strategy: one
    // replay of the merged best-response graph, one copy of the root sums,
    // one synchronisation.  pct / nash are indexed by member.
    int check(std::vector<double> &pct, std::vector<double> &nash) {
        if (num_active() == 0) return SS_OK;
        BCK(cudaSetDevice(device));
        if (dirty) {
            int rc = rebuild();
            if (rc != SS_OK) return rc;
        }
        BCK(cudaGraphLaunch(br_graph, stream));
        BCK(cudaMemcpyAsync(hsc, dsc, static_cast<size_t>(built_members) * kSlots * sizeof(double),
                            cudaMemcpyDeviceToHost, stream));
        BCK(cudaStreamSynchronize(stream));
        pct.resize(subs.size(), -1.0);
        nash.resize(subs.size(), -1.0);
        for (size_t i = 0; i < subs.size(); ++i)
            if (active[i])
                subs[i]->nashconv_from_sums(hsc + i * kSlots, &pct[i], &nash[i], nullptr, nullptr, nullptr);
        return SS_OK;
    }

  private:
    static constexpr int kSlots = 2 * SS_MAX_PLAYERS + 2;   // root sums per member (nashconv_from_sums)
    enum LaunchType { L_BUMP, L_SNAP, L_TERM, L_CFV, L_REACH, L_AVG, L_BR_REACH, L_BR_TERM, L_BR_VALUE, L_BR_ROOT };
    struct Launch {
        int type;
        int kind;   // terminal kind; value/regret launches: long items at the end; best-response values: mode
        int t;      // traverser / player
        size_t off; // item offset in dlists
        int n;
        int H;      // largest hand count of the launch
        // three-way showdowns: block -> (item, run group) map, blocks, largest merge
        size_t map_off = 0;
        int map_blocks = 0;
        int map_lg = 0;
        int cr2_form = -1;  // two-opponent terminals: 1 tensor-core form, 0 mma.sync form
        // grouped terminal kinds: the items that start work, one block each
        size_t heads_off = 0;
        int n_heads = 0;
    };
    DevCtx *dctx = nullptr;
    char *dlists = nullptr;
    double *dsc = nullptr, *hsc = nullptr;
    DevCtx cmax{};
    std::vector<Launch> seq, br_seq;
    cudaGraphExec_t graph = nullptr, br_graph = nullptr;
    bool dirty = true;
    int built_members = 0;
    std::vector<double> work;      // per member: work items in the captured launches
    double built_work = 0, live_work = 0;

    cudaError_t launch(const Launch &L) {
        switch (L.type) {
            case L_BUMP: return launch_bump_many(dctx, reinterpret_cast<const int *>(dlists + L.off), L.n, stream);
            case L_SNAP: return launch_snapshot_many(dctx, reinterpret_cast<const int *>(dlists + L.off), L.n, stream);
            case L_TERM:
                if (L.kind == TK_SD2)
                    return launch_sd2_mapped(cmax, reinterpret_cast<const TermItem *>(dlists + L.off),
                                             reinterpret_cast<const int2 *>(dlists + L.map_off), L.map_blocks,
                                             L.map_lg, L.t, stream, dctx, false);
                {
                    const int *heads = L.n_heads > 0 ? reinterpret_cast<const int *>(dlists + L.heads_off) : nullptr;
                    if (L.cr2_form >= 0) {
                        // the launch context picks the form: a dense deck of 48 and no
                        // repeated combo for the tensor-core one, no deck for the other
                        DevCtx cl = cmax;
                        cl.deck = L.cr2_form == 1 ? 48 : 0;
                        for (int p = 0; p < SS_MAX_PLAYERS; ++p) cl.dup[p] = 0;
                        return launch_terms(cl, L.kind, reinterpret_cast<const TermItem *>(dlists + L.off), L.n,
                                            L.t, stream, dctx, heads, L.n_heads);
                    }
                    return launch_terms(cmax, L.kind, reinterpret_cast<const TermItem *>(dlists + L.off), L.n, L.t,
                                        stream, dctx, heads, L.n_heads);
                }
            case L_CFV:
                return launch_cfv(cmax, reinterpret_cast<const CfvItem *>(dlists + L.off), L.n, L.kind, L.H, stream,
                                  dctx, L.t);
            case L_REACH:
                return launch_reach(cmax, reinterpret_cast<const ReachItem *>(dlists + L.off), L.n, L.H, stream,
                                    dctx, L.t);
            case L_AVG:
                return launch_avg_many(dctx, reinterpret_cast<const AvgItem *>(dlists + L.off), L.n, L.H, stream);
            case L_BR_REACH:
                return launch_br_reach_many(dctx, reinterpret_cast<const ReachItem *>(dlists + L.off), L.n, L.H,
                                            L.t, stream);
            case L_BR_TERM:
                if (L.kind == TK_SD2)
                    return launch_sd2_mapped(cmax, reinterpret_cast<const TermItem *>(dlists + L.off),
                                             reinterpret_cast<const int2 *>(dlists + L.map_off), L.map_blocks,
                                             L.map_lg, L.t, stream, dctx, true);
                return launch_terms_fp64(cmax, L.kind, reinterpret_cast<const TermItem *>(dlists + L.off), L.n, L.t,
                                         stream, dctx);
            case L_BR_VALUE:
                return launch_br_value_many(dctx, reinterpret_cast<const CfvItem *>(dlists + L.off), L.n, L.H, L.t,
                                            L.kind, stream);
            default:
                return launch_br_root_many(dctx, reinterpret_cast<const RootItem *>(dlists + L.off), L.n, dsc,
                                           stream);
        }
    }

    cudaError_t iteration() {
        for (const Launch &L : seq) {
            cudaError_t e = launch(L);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    cudaError_t br_pass() {
        for (const Launch &L : br_seq) {
            cudaError_t e = launch(L);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    int capture(cudaError_t (Batch::*body_fn)(), int reps, cudaGraphExec_t *exec) {
        cudaGraph_t g = nullptr;
        BCK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t body = cudaSuccess;
        for (int r = 0; r < reps && body == cudaSuccess; ++r) body = (this->*body_fn)();
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (body != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            BCK(body);
        }
        BCK(e);
        e = cudaGraphInstantiate(exec, g, 0);
        cudaGraphDestroy(g);
        BCK(e);
        return SS_OK;
    }

    int rebuild() {
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        if (br_graph) {
            cudaGraphExecDestroy(br_graph);
            br_graph = nullptr;
        }
        const int K = static_cast<int>(subs.size());
        std::vector<DevCtx> ctx(K);
        cmax = DevCtx{};
        for (int i = 0; i < K; ++i)
            if (subs[i]) {
                ctx[i] = subs[i]->c;
                ctx[i].live = active[i];
                // launch-time sizes (grids, dynamic shared memory) come from
                // cmax: the largest row stride, rank table and sweep run of the batch
                cmax.HS = std::max(cmax.HS, subs[i]->c.HS);
                cmax.ncomb = std::max(cmax.ncomb, subs[i]->c.ncomb);
                for (int lg = 0; lg < kSd2Merge; ++lg)
                    cmax.sd_span[lg] = std::max(cmax.sd_span[lg], subs[i]->c.sd_span[lg]);
            }
        // merged lists, in launch order
        std::vector<char> blob;
        seq.clear();
        br_seq.clear();
        auto put = [&](const void *src, size_t bytes) {
            size_t off = (blob.size() + 255) & ~static_cast<size_t>(255);
            blob.resize(off + bytes);
            if (bytes) std::memcpy(blob.data() + off, src, bytes);
            return off;
        };
        // a terminal launch over merged items; three-way showdowns also get the
        // block map that sweeps each subgame with its own run merge
        auto term_launch = [&](int type, int k, int t, const std::vector<TermItem> &items) {
            Launch L{type, k, t, put(items.data(), items.size() * sizeof(TermItem)), static_cast<int>(items.size()),
                     0};
            if (type == L_TERM && k == TK_CR2) {
                std::vector<int> heads;
                for (size_t i = 0; i < items.size(); ++i)
                    if (!items[i].follow && !items[i].chained) heads.push_back(static_cast<int>(i));
                L.heads_off = put(heads.data(), heads.size() * sizeof(int));
                L.n_heads = static_cast<int>(heads.size());
            }
            if (k == TK_SD2) {
                std::vector<int2> bmap;
                for (size_t i = 0; i < items.size(); ++i) {
                    const int lg = items[i].kind_detail;
                    L.map_lg = std::max(L.map_lg, lg);
                    for (int g = 0; g < (kSd2Chunks >> lg); ++g) bmap.push_back(make_int2(static_cast<int>(i), g));
                }
                L.map_off = put(bmap.data(), bmap.size() * sizeof(int2));
                L.map_blocks = static_cast<int>(bmap.size());
            }
            return L;
        };
        std::vector<int> act;
        int maxnp = 0, maxh = 0;
        for (int i = 0; i < K; ++i) {
            work[i] = 0.0;
            if (active[i]) {
                act.push_back(i);
                maxnp = std::max(maxnp, subs[i]->P.np);
                maxh = std::max(maxh, subs[i]->P.max_h);
            }
        }
        auto add_work = [&](int i, size_t n) { work[i] += static_cast<double>(n); };
        seq.push_back({L_BUMP, 0, 0, put(act.data(), act.size() * sizeof(int)), static_cast<int>(act.size()), 0});
        for (int t = 0; t < maxnp; ++t) {
            std::vector<int> snap;
            for (int i : act)
                if (subs[i]->P.np - 1 == t) snap.push_back(i);
            if (!snap.empty())
                seq.push_back({L_SNAP, 0, t, put(snap.data(), snap.size() * sizeof(int)), static_cast<int>(snap.size()),
                               0});
            for (int k = 0; k < TK_COUNT; ++k) {
                // two-opponent terminals: one launch per product form, so each
                // subgame's terminals take the form they take in a solo solve
                for (int form = (k == TK_CR2 ? 1 : -1); form >= (k == TK_CR2 ? 0 : -1); --form) {
                    std::vector<TermItem> items;
                    for (int i : act) {
                        if (subs[i]->P.np <= t) continue;
                        if (form >= 0 && cr2_tensor_form(subs[i]->c) != (form == 1)) continue;
                        for (TermItem it : subs[i]->P.term[t][k]) {
                            it.sg = i;
                            items.push_back(it);
                        }
                        add_work(i, subs[i]->P.term[t][k].size());
                    }
                    if (items.empty()) continue;
                    Launch L = term_launch(L_TERM, k, t, items);
                    L.cr2_form = form;
                    seq.push_back(L);
                }
            }
            size_t lv = 0;
            for (int i : act)
                if (subs[i]->P.np > t) lv = std::max(lv, subs[i]->P.cfv_levels[t].size());
            for (size_t l = 0; l < lv; ++l) {
                // every subgame's short items, then every subgame's long ones
                // (each item keeps its own subgame's class, so it is summed as
                // in a solo solve)
                std::vector<CfvItem> items, longs;
                int H = 0;
                for (int i : act) {
                    const Plan &P = subs[i]->P;
                    if (P.np <= t || l >= P.cfv_levels[t].size()) continue;
                    const auto &v = P.cfv_levels[t][l];
                    const size_t n_short = v.size() - static_cast<size_t>(P.cfv_nlong[t][l]);
                    for (size_t j = 0; j < v.size(); ++j) {
                        CfvItem it = v[j];
                        it.sg = i;
                        (j < n_short ? items : longs).push_back(it);
                    }
                    add_work(i, v.size());
                    H = std::max(H, P.H[t]);
                }
                const int n_long = static_cast<int>(longs.size());
                items.insert(items.end(), longs.begin(), longs.end());
                if (!items.empty())
                    seq.push_back({L_CFV, n_long, t, put(items.data(), items.size() * sizeof(CfvItem)),
                                   static_cast<int>(items.size()), H});
            }
            lv = 0;
            for (int i : act)
                if (subs[i]->P.np > t) lv = std::max(lv, subs[i]->P.reach_levels[t].size());
            for (size_t l = 0; l < lv; ++l) {
                std::vector<ReachItem> items;
                int H = 0;
                for (int i : act) {
                    const Plan &P = subs[i]->P;
                    if (P.np <= t || l >= P.reach_levels[t].size()) continue;
                    for (ReachItem it : P.reach_levels[t][l]) {
                        it.sg = i;
                        items.push_back(it);
                    }
                    add_work(i, P.reach_levels[t][l].size());
                    H = std::max(H, P.H[t]);
                }
                if (!items.empty())
                    seq.push_back({L_REACH, 0, t, put(items.data(), items.size() * sizeof(ReachItem)),
                                   static_cast<int>(items.size()), H});
            }
        }
        // the merged best response (Session::exploitability for every member)
        {
            std::vector<AvgItem> avg;
            for (int i : act)
                for (int di = 0; di < subs[i]->P.num_dec; ++di) avg.push_back({i, di});
            if (!avg.empty())
                br_seq.push_back({L_AVG, 0, 0, put(avg.data(), avg.size() * sizeof(AvgItem)),
                                  static_cast<int>(avg.size()), maxh});
        }
        for (int p = 0; p < maxnp; ++p) {
            size_t lv = 0;
            for (int i : act)
                if (subs[i]->P.np > p) lv = std::max(lv, subs[i]->P.reach_levels[p].size());
            for (size_t l = 0; l < lv; ++l) {
                std::vector<ReachItem> items;
                int H = 0;
                for (int i : act) {
                    const Plan &P = subs[i]->P;
                    if (P.np <= p || l >= P.reach_levels[p].size()) continue;
                    for (ReachItem it : P.reach_levels[p][l]) {
                        it.sg = i;
                        items.push_back(it);
                    }
                    H = std::max(H, P.H[p]);
                }
                if (!items.empty())
                    br_seq.push_back({L_BR_REACH, 0, p, put(items.data(), items.size() * sizeof(ReachItem)),
                                      static_cast<int>(items.size()), H});
            }
        }
        for (int t = 0; t < maxnp; ++t) {
            for (int k = 0; k < TK_COUNT; ++k) {
                std::vector<TermItem> items;
                for (int i : act) {
                    if (subs[i]->P.np <= t) continue;
                    for (TermItem it : subs[i]->P.term[t][k]) {
                        it.sg = i;
                        items.push_back(it);
                    }
                }
                if (!items.empty()) br_seq.push_back(term_launch(L_BR_TERM, k, t, items));
            }
            size_t lv = 0;
            for (int i : act)
                if (subs[i]->P.np > t) lv = std::max(lv, subs[i]->P.cfv_levels[t].size());
            for (int mode = 0; mode < 2; ++mode) {
                for (size_t l = 0; l < lv; ++l) {
                    std::vector<CfvItem> items;
                    int H = 0;
                    for (int i : act) {
                        const Plan &P = subs[i]->P;
                        if (P.np <= t || l >= P.cfv_levels[t].size()) continue;
                        for (CfvItem it : P.cfv_levels[t][l]) {
                            it.sg = i;
                            items.push_back(it);
                        }
                        H = std::max(H, P.H[t]);
                    }
                    if (!items.empty())
                        br_seq.push_back({L_BR_VALUE, mode, t, put(items.data(), items.size() * sizeof(CfvItem)),
                                          static_cast<int>(items.size()), H});
                }
                std::vector<RootItem> roots;
                for (int i : act) {
                    const Plan &P = subs[i]->P;
                    if (P.np <= t) continue;
                    roots.push_back({subs[i]->root_fr[t], static_cast<int>(P.root_fr[t].size()), i, t, P.E + t, 0,
                                     i * kSlots + 2 * t + mode});
                }
                if (!roots.empty())
                    br_seq.push_back({L_BR_ROOT, 0, t, put(roots.data(), roots.size() * sizeof(RootItem)),
                                      static_cast<int>(roots.size()), 0});
            }
        }
        {
            // deal mass: each member's own item, merged by kind
            std::vector<RootItem> roots;
            for (int k = 0; k < TK_COUNT; ++k) {
                std::vector<TermItem> items;
                for (int i : act)
                    if (subs[i]->deal_kind == k) {
                        TermItem it = subs[i]->deal;
                        it.sg = i;
                        items.push_back(it);
                    }
                if (!items.empty()) br_seq.push_back(term_launch(L_BR_TERM, k, 0, items));
            }
            for (int i : act)
                roots.push_back({subs[i]->br_row, 1, i, 0, subs[i]->P.E, 1, i * kSlots + 2 * SS_MAX_PLAYERS});
            if (!roots.empty())
                br_seq.push_back({L_BR_ROOT, 0, 0, put(roots.data(), roots.size() * sizeof(RootItem)),
                                  static_cast<int>(roots.size()), 0});
        }
        built_work = live_work = 0;
        for (int i : act) built_work += work[i];
        live_work = built_work;
        if (dctx) cudaFreeAsync(dctx, stream);
        if (dlists) cudaFreeAsync(dlists, stream);
        if (dsc) cudaFreeAsync(dsc, stream);
        dctx = nullptr;
        dlists = nullptr;
        dsc = nullptr;
        if (hsc && built_members < K) {
            cudaFreeHost(hsc);
            hsc = nullptr;
        }
        built_members = K;
        BCK(cudaMallocAsync(reinterpret_cast<void **>(&dctx), std::max(1, K) * sizeof(DevCtx), stream));
        BCK(cudaMallocAsync(reinterpret_cast<void **>(&dlists), std::max<size_t>(blob.size(), 256), stream));
        BCK(cudaMallocAsync(reinterpret_cast<void **>(&dsc), std::max(1, K) * kSlots * sizeof(double), stream));
        BCK(cudaMemsetAsync(dsc, 0, std::max(1, K) * kSlots * sizeof(double), stream));
        if (!hsc) BCK(cudaMallocHost(reinterpret_cast<void **>(&hsc), std::max(1, K) * kSlots * sizeof(double)));
        BCK(cudaMemcpyAsync(dctx, ctx.data(), K * sizeof(DevCtx), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(dlists, blob.data(), blob.size(), cudaMemcpyHostToDevice, stream));
        // members were initialised on their own streams
        for (int i : act) BCK(cudaStreamSynchronize(subs[i]->stream));
        BCK(cudaStreamSynchronize(stream));  // host staging must outlive the copies
        int rc = capture(&Batch::iteration, graph_iters, &graph);
        if (rc == SS_OK) rc = capture(&Batch::br_pass, 1, &br_graph);
        if (rc != SS_OK) return rc;
        dirty = false;
        return SS_OK;
    }
};

// ---------------------------------------------------------------------------
// batched form: solve n subgames together
// ---------------------------------------------------------------------------

// Sessions of many subgames, created on several host threads (the host plan
// dominates their creation); the first failure is returned.
int create_sessions(const std::vector<const Problem *> &pbs, const SolveConfig &cfg, std::vector<Session *> *out) {
    const size_t n = pbs.size();
    out->assign(n, nullptr);
    std::vector<int> rcs(n, SS_OK);
    std::vector<std::string> errs(n);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>(n, std::min(16u, hw));
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (;;) {
            const size_t i = next++;
            if (i >= n) return;
            rcs[i] = session_create(*pbs[i], cfg, &(*out)[i]);
            if (rcs[i] != SS_OK) errs[i] = last_error();
        }
    };
    std::vector<std::thread> th;
    for (size_t k = 1; k < nt; ++k) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
    for (size_t i = 0; i < n; ++i)
        if (rcs[i] != SS_OK) {
            for (Session *s : *out) delete s;
            out->assign(n, nullptr);
            set_error(errs[i]);
            return rcs[i];
        }
    return SS_OK;
}

int batch_solve(const std::vector<Problem> &pbs, int max_iterations, const SolveConfig &cfg, SSOutput *outs,
                SSSolveStats *stats) {
    for (size_t i = 0; i < pbs.size(); ++i) {
        std::memset(&outs[i], 0, sizeof(SSOutput));
        if (stats) {
            std::memset(&stats[i], 0, sizeof(SSSolveStats));
            stats[i].exploitability_pct = -1.0;
            stats[i].nashconv = -1.0;
        }
    }
    if (max_iterations < 0) {
        set_error("max_iterations must be >= 0");
        return SS_ERR_INVALID;
    }
    Batch b;
    int rc = b.init(cfg.device, cfg.graph_iterations);
    if (rc != SS_OK) return rc;
    {
        std::vector<const Problem *> ptrs;
        for (const Problem &pb : pbs) ptrs.push_back(&pb);
        SolveConfig mcfg = cfg;
        mcfg.batch_member = 1;
        std::vector<Session *> made;
        rc = create_sessions(ptrs, mcfg, &made);
        if (rc != SS_OK) return rc;
        for (size_t i = 0; i < made.size(); ++i) {
            int slot = -1;
            rc = b.add(made[i], &slot);
            if (rc != SS_OK) {
                for (size_t j = i; j < made.size(); ++j) delete made[j];
                return rc;
            }
        }
    }
    const bool target = cfg.target_exploitability > 0.f;
    const int step = target ? std::max(1, cfg.check_every) : std::max(1, max_iterations);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    float total_ms = 0.f;
    std::vector<double> pct(pbs.size(), -1.0), nash(pbs.size(), -1.0);
    while (b.num_active() > 0) {
        int n = step;
        for (size_t i = 0; i < pbs.size(); ++i)
            if (b.active[i]) n = std::min(n, max_iterations - b.iters_run[i]);
        if (n <= 0) break;
        BCK(cudaEventRecord(e0, b.stream));
        rc = b.run(n);
        if (rc != SS_OK) break;
        BCK(cudaEventRecord(e1, b.stream));
        bool any_last = false;
        for (size_t i = 0; i < pbs.size(); ++i)
            if (b.active[i] && b.iters_run[i] >= max_iterations) any_last = true;
        if (target || (any_last && cfg.compute_exploitability))
            rc = b.check(pct, nash);
        else
            rc = b.sync();
        if (rc != SS_OK) break;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) total_ms += ms;
        for (size_t i = 0; i < pbs.size() && rc == SS_OK; ++i) {
            if (!b.active[i]) continue;
            const bool last = b.iters_run[i] >= max_iterations;
            if (last || (target && pct[i] <= cfg.target_exploitability)) rc = b.retire(static_cast<int>(i));
        }
        if (rc != SS_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != SS_OK) return rc;
    rc = b.sync();
    if (rc != SS_OK) return rc;
    for (size_t i = 0; i < pbs.size(); ++i) {
        rc = b.subs[i]->output(&outs[i]);
        if (rc != SS_OK) {
            for (size_t j = 0; j < i; ++j) {
                std::free(outs[j].root_strategy);
                std::free(outs[j].root_ev);
                if (!host_block_give(outs[j].avg_strategies)) std::free(outs[j].avg_strategies);
                std::free(outs[j].avg_strategy_node_ids);
                std::memset(&outs[j], 0, sizeof(SSOutput));
            }
            return rc;
        }
        if (stats) {
            stats[i].iterations_run = b.iters_run[i];
            stats[i].exploitability_pct = pct[i];
            stats[i].nashconv = nash[i];
            stats[i].solve_ms = total_ms;  // device time of the whole batch
            stats[i].node_hand_updates = b.subs[i]->P.node_hands * b.iters_run[i];
        }
    }
    return SS_OK;
}

// ---------------------------------------------------------------------------
// served form
// ---------------------------------------------------------------------------

namespace {

// owned copy of one request (the caller's buffers may go away after submit)
struct Request {
    long long id = 0;
    std::vector<SSNode> nodes;
    std::vector<int> children;
    std::vector<int> hands[SS_MAX_PLAYERS];
    std::vector<float> weights[SS_MAX_PLAYERS];
    std::vector<float> leaf;
    std::vector<int> frozen;
    Problem pb;
    size_t bytes = 0;
    std::chrono::steady_clock::time_point t_submit, t_admit, t_done;
    int slot = -1;
    int iters_done = 0;  // iterations run so far (updated after each block)
    int state = 0;  // 0 pending, 1 running, 2 done, <0 failed with that code
    std::string error;
    SSOutput out{};
    SSSolveStats stats{};
};

size_t footprint(const Problem &pb) {
    size_t E = 0, mh = 0;
    for (int i = 0; i < pb.num_nodes; ++i)
        if (pb.nodes[i].type == SS_NODE_DECISION) E += static_cast<size_t>(pb.nodes[i].num_children);
    for (int p = 0; p < pb.num_players; ++p) mh = std::max(mh, static_cast<size_t>(pb.num_hands[p]));
    const size_t HS = (mh + 31) / 32 * 32, N = static_cast<size_t>(pb.num_nodes), np = pb.num_players;
    size_t b = (3 * E + np + N) * HS * 4;           // regrets, sums, reach, values
    b += (E + np + N + 1) * HS * 8;                 // best-response reach and values
    b += static_cast<size_t>(pb.num_leaves) * np * mh * 4 * (pb.leaf_values ? 1 : 0);
    b += E * 200 + N * 64 + (8u << 20);             // tables and slack
    return b;
}

}  // namespace

class Server {
  public:
    SSServerOptions opt{};
    Batch batch;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_admit;
    std::deque<Request *> pending;                     // submitted, not yet admitted
    std::deque<std::pair<Request *, Session *>> ready;  // admitted, session built, not yet in the batch
    std::map<long long, std::unique_ptr<Request>> reqs;
    std::vector<Request *> slot_req;
    size_t used = 0;
    int building = 0;                                  // requests whose session is being built
    long long next_id = 1;
    bool stop = false;
    std::thread worker, admitter;
    int fatal = SS_OK;
    std::string fatal_msg;

    int start(const SSServerOptions &o) {
        opt = o;
        int rc = batch.init(o.device, o.graph_iterations);
        if (rc != SS_OK) return rc;
        worker = std::thread([this] { loop(); });
        admitter = std::thread([this] { admit_loop(); });
        return SS_OK;
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_work.notify_all();
        cv_admit.notify_all();
        if (admitter.joinable()) admitter.join();
        if (worker.joinable()) worker.join();
        for (auto &rs : ready) delete rs.second;
        for (auto &kv : reqs) {
            SSOutput &o = kv.second->out;
            std::free(o.root_strategy);
            std::free(o.root_ev);
            if (!host_block_give(o.avg_strategies)) std::free(o.avg_strategies);
            std::free(o.avg_strategy_node_ids);
        }
    }

    int submit(const Problem &src, long long *id) {
        auto r = std::make_unique<Request>();
        r->nodes.assign(src.nodes, src.nodes + src.num_nodes);
        r->children.assign(src.children, src.children + src.num_children_total);
        r->pb = src;
        r->pb.nodes = r->nodes.data();
        r->pb.children = r->children.data();
        for (int p = 0; p < src.num_players; ++p) {
            r->hands[p].assign(src.hands[p], src.hands[p] + 2 * src.num_hands[p]);
            r->weights[p].assign(src.weights[p], src.weights[p] + src.num_hands[p]);
            r->pb.hands[p] = r->hands[p].data();
            r->pb.weights[p] = r->weights[p].data();
        }
        if (src.leaf_values && src.num_leaves > 0) {
            int mh = 0;
            for (int p = 0; p < src.num_players; ++p) mh = std::max(mh, src.num_hands[p]);
            r->leaf.assign(src.leaf_values, src.leaf_values + static_cast<size_t>(src.num_leaves) * src.num_players * mh);
            r->pb.leaf_values = r->leaf.data();
        }
        if (src.frozen) {
            r->frozen.assign(src.frozen, src.frozen + src.num_nodes);
            r->pb.frozen = r->frozen.data();
        }
        r->bytes = footprint(r->pb);
        r->t_submit = std::chrono::steady_clock::now();
        std::lock_guard<std::mutex> lk(mu);
        if (fatal != SS_OK) {
            set_error(fatal_msg);
            return fatal;
        }
        r->id = next_id++;
        *id = r->id;
        pending.push_back(r.get());
        reqs[r->id] = std::move(r);
        cv_admit.notify_one();
        return SS_OK;
    }

    // 0 done (outputs handed over), 1 pending or running, < 0 failed
    int poll(long long id, SSOutput *out, SSSolveStats *stats, double *latency_ms, bool wait) {
        std::unique_lock<std::mutex> lk(mu);
        auto it = reqs.find(id);
        if (it == reqs.end()) {
            set_error("unknown request id");
            return SS_ERR_INVALID;
        }
        Request *r = it->second.get();
        if (wait) cv_done.wait(lk, [&] { return r->state == 2 || r->state < 0 || fatal != SS_OK; });
        if (r->state < 0) {
            set_error(r->error);
            int rc = r->state;
            reqs.erase(it);
            return rc;
        }
        if (r->state != 2) {
            if (fatal != SS_OK) {
                set_error(fatal_msg);
                return fatal;
            }
            return 1;
        }
        if (out) {
            *out = r->out;
        } else {
            std::free(r->out.root_strategy);
            std::free(r->out.root_ev);
            if (!host_block_give(r->out.avg_strategies)) std::free(r->out.avg_strategies);
            std::free(r->out.avg_strategy_node_ids);
        }
        std::memset(&r->out, 0, sizeof(SSOutput));
        if (stats) *stats = r->stats;
        if (latency_ms)
            *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
        reqs.erase(it);
        return 0;
    }

    int progress(long long id, int *state, int *iters) {
        std::lock_guard<std::mutex> lk(mu);
        auto it = reqs.find(id);
        if (it == reqs.end()) {
            set_error("unknown request id");
            return SS_ERR_INVALID;
        }
        const Request *r = it->second.get();
        if (r->state < 0) {
            set_error(r->error);
            return r->state;
        }
        if (state) *state = r->state;
        if (iters) *iters = r->iters_done;
        return SS_OK;
    }

  private:
    // whether the device context still works after a failed call (a sticky
    // error, such as an illegal address, ends every request)
    static bool context_usable() {
        cudaGetLastError();   // clears a non-sticky error of the last call
        return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess;
    }

    void fail(Request *r, int rc, const std::string &msg) {
        r->state = rc;
        r->error = msg;
        r->t_done = std::chrono::steady_clock::now();
    }

    // Admission: takes pending requests in order while their estimated
    // footprint fits the memory budget (or nothing else is resident) and
    // builds their sessions -- host plan, allocation, upload on the session's
    // own stream -- off the worker thread, so the batch keeps running
    // meanwhile; the worker adds them between iteration blocks.
    void admit_loop() {
        cudaSetDevice(opt.device);
        const size_t budget = static_cast<size_t>(opt.memory_budget_gb * 1e9);
        SolveConfig cfg;
        cfg.device = opt.device;
        cfg.graph_iterations = opt.graph_iterations;
        cfg.batch_member = 1;
        for (;;) {
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_admit.wait(lk, [&] {
                    if (stop || fatal != SS_OK) return true;
                    if (pending.empty()) return false;
                    const bool alone = used == 0;
                    return alone || used + pending.front()->bytes <= budget;
                });
                if (stop || fatal != SS_OK) return;
                r = pending.front();
                pending.pop_front();
                used += r->bytes;
                ++building;
            }
            Session *s = nullptr;
            int rc = session_create(r->pb, cfg, &s);
            if (rc == SS_OK) rc = s->ensure_br();
            std::string msg = rc == SS_OK ? std::string() : std::string(last_error());
            std::lock_guard<std::mutex> lk(mu);
            --building;
            if (rc != SS_OK) {
                delete s;
                used -= r->bytes;
                fail(r, rc, msg);
                cv_done.notify_all();
                cv_admit.notify_all();
                continue;
            }
            ready.emplace_back(r, s);
            cv_work.notify_one();
        }
    }

    void loop() {
        cudaSetDevice(opt.device);
        const int block = std::max(1, opt.block_iterations);
        std::vector<double> pct, nash;
        for (;;) {
            std::vector<std::pair<Request *, Session *>> add;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || !ready.empty() || batch.num_active() > 0; });
                if (stop) return;
                while (!ready.empty()) {
                    add.push_back(ready.front());
                    ready.pop_front();
                }
            }
            for (auto &rs : add) {
                Request *r = rs.first;
                int slot = -1;
                int rc = batch.add(rs.second, &slot);
                std::lock_guard<std::mutex> lk(mu);
                if (rc != SS_OK) {
                    delete rs.second;
                    used -= r->bytes;
                    fail(r, rc, last_error());
                    cv_done.notify_all();
                    cv_admit.notify_all();
                    continue;
                }
                r->slot = slot;
                r->state = 1;
                r->t_admit = std::chrono::steady_clock::now();
                if (static_cast<int>(slot_req.size()) <= slot) slot_req.resize(slot + 1, nullptr);
                slot_req[slot] = r;
            }
            if (batch.num_active() == 0) continue;
            int rc = batch.run(block);
            if (rc == SS_OK) rc = batch.check(pct, nash);
            if (rc != SS_OK && !add.empty() && context_usable()) {
                // a failure that left the context usable (an allocation or a
                // graph build for the members admitted before this block):
                // those members leave with the error, the rest carries on
                const std::string msg = last_error();
                for (auto &rs : add) {
                    Request *r = rs.first;
                    if (r->slot < 0 || r->state != 1) continue;
                    batch.retire(r->slot);
                    batch.release(r->slot);
                    std::lock_guard<std::mutex> lk(mu);
                    used -= r->bytes;
                    slot_req[r->slot] = nullptr;
                    fail(r, rc, msg);
                }
                std::lock_guard<std::mutex> lk(mu);
                cv_done.notify_all();
                cv_admit.notify_all();
                continue;
            }
            if (rc != SS_OK) {
                std::lock_guard<std::mutex> lk(mu);
                fatal = rc;
                fatal_msg = last_error();
                for (Request *r : slot_req)
                    if (r && r->state == 1) fail(r, rc, fatal_msg);
                cv_done.notify_all();
                cv_admit.notify_all();
                return;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                for (size_t i = 0; i < batch.subs.size(); ++i)
                    if (batch.active[i]) slot_req[i]->iters_done = batch.iters_run[i];
            }
            for (size_t i = 0; i < batch.subs.size(); ++i) {
                if (!batch.active[i]) continue;
                Request *r = slot_req[i];
                const bool cap = batch.iters_run[i] >= opt.max_iterations;
                if (!std::isfinite(pct[i])) {
                    // non-finite values (a caller's NaN or infinite leaf value
                    // spreads through the regrets): this request fails, the
                    // others never read its rows
                    batch.retire(static_cast<int>(i));
                    batch.release(static_cast<int>(i));
                    std::lock_guard<std::mutex> lk(mu);
                    used -= r->bytes;
                    fail(r, SS_ERR_INVALID,
                         "non-finite exploitability after " + std::to_string(batch.iters_run[i]) +
                             " iterations: the subgame's inputs (leaf values, weights) hold NaN or infinity");
                    slot_req[i] = nullptr;
                    cv_done.notify_all();
                    cv_admit.notify_all();
                    continue;
                }
                if (!(cap || pct[i] <= opt.target_exploitability)) continue;
                rc = batch.retire(static_cast<int>(i));
                SSOutput o{};
                if (rc == SS_OK) rc = batch.subs[i]->output(&o);
                const std::string msg = rc == SS_OK ? std::string() : std::string(last_error());
                const double nhu = batch.subs[i]->P.node_hands * batch.iters_run[i];
                batch.release(static_cast<int>(i));
                std::lock_guard<std::mutex> lk(mu);
                used -= r->bytes;
                if (rc != SS_OK) {
                    fail(r, rc, msg);
                } else {
                    r->out = o;
                    r->stats.iterations_run = batch.iters_run[i];
                    r->stats.exploitability_pct = pct[i];
                    r->stats.nashconv = nash[i];
                    r->stats.node_hand_updates = nhu;
                    r->stats.queue_ms = std::chrono::duration<double, std::milli>(r->t_admit - r->t_submit).count();
                    r->t_done = std::chrono::steady_clock::now();
                    r->state = 2;
                }
                slot_req[i] = nullptr;
                cv_done.notify_all();
                cv_admit.notify_all();
            }
        }
    }
};

int server_create(const SSServerOptions &o, Server **out) {
    *out = nullptr;
    auto s = std::make_unique<Server>();
    int rc = s->start(o);
    if (rc != SS_OK) return rc;
    *out = s.release();
    return SS_OK;
}

int server_submit(Server *s, const Problem &pb, long long *id) { return s->submit(pb, id); }

int server_poll(Server *s, long long id, SSOutput *out, SSSolveStats *stats, double *lat, int wait) {
    return s->poll(id, out, stats, lat, wait != 0);
}

int server_progress(Server *s, long long id, int *state, int *iters) { return s->progress(id, state, iters); }

void server_destroy(Server *s) { delete s; }

}  // namespace ssb
