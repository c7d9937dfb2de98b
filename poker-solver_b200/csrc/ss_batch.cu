// ss_batch.cu -- batched and served forms.
//
// Batch: many resident subgames (Sessions) of different size, street and
// player count advance together.  Their per-level work lists are merged, so
// one launch covers level l of traverser t for every member (each item reads
// its subgame's context, item.sg); one launch advances every member's
// iteration counter and one per pass snapshots the root strategies.  A block
// of iterations is captured as one CUDA graph; members can be added or
// retired between blocks (the graph is rebuilt), each keeps its own iteration
// count, and arithmetic per subgame is identical to a solve alone.
//
// Server: continuous batching on one GPU.  Requests are copied at submission
// and admitted into the running batch while their estimated device footprint
// fits the memory budget; the worker runs iteration blocks, checks each
// member's FP64 exploitability at block ends, and retires a member when it
// reaches the target (or the iteration cap), freeing its memory for the next
// requests.  Latency = submission to retirement.
#include "ss_session.h"

#include <algorithm>
#include <chrono>
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
        if (stream) {
            if (dctx) cudaFreeAsync(dctx, stream);
            if (dlists) cudaFreeAsync(dlists, stream);
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        for (Session *s : subs) delete s;
    }

    int init(int dev, int g) {
        device = dev;
        graph_iters = std::max(1, g);
        BCK(cudaSetDevice(device));
        BCK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        return SS_OK;
    }

    int add(Session *s) {
        subs.push_back(s);
        active.push_back(1);
        iters_run.push_back(0);
        dirty = true;
        return static_cast<int>(subs.size()) - 1;
    }

    // stop iterating member i (its state stays readable until released)
    void retire(int i) {
        active[i] = 0;
        dirty = true;
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

  private:
    struct Launch {
        int type;   // 0 bump, 1 snapshot, 2 terminals, 3 cfv, 4 reach
        int kind;   // terminal kind; value/regret launches: number of long items (at the end)
        int t;      // traverser / player
        size_t off; // item offset in dlists
        int n;
        int H;      // largest hand count of the launch
    };
    DevCtx *dctx = nullptr;
    char *dlists = nullptr;
    DevCtx cmax{};
    std::vector<Launch> seq;
    cudaGraphExec_t graph = nullptr;
    bool dirty = true;

    cudaError_t launch(const Launch &L) {
        switch (L.type) {
            case 0: return launch_bump_many(dctx, reinterpret_cast<const int *>(dlists + L.off), L.n, stream);
            case 1: return launch_snapshot_many(dctx, reinterpret_cast<const int *>(dlists + L.off), L.n, stream);
            case 2:
                return launch_terms(cmax, L.kind, reinterpret_cast<const TermItem *>(dlists + L.off), L.n, L.t,
                                    stream, dctx);
            case 3:
                return launch_cfv(cmax, reinterpret_cast<const CfvItem *>(dlists + L.off), L.n, L.kind, L.H, stream,
                                  dctx, L.t);
            default:
                return launch_reach(cmax, reinterpret_cast<const ReachItem *>(dlists + L.off), L.n, L.H, stream,
                                    dctx, L.t);
        }
    }

    cudaError_t iteration() {
        for (const Launch &L : seq) {
            cudaError_t e = launch(L);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    int rebuild() {
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        const int K = static_cast<int>(subs.size());
        std::vector<DevCtx> ctx(K);
        cmax = DevCtx{};
        for (int i = 0; i < K; ++i)
            if (subs[i]) {
                ctx[i] = subs[i]->c;
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
        auto put = [&](const void *src, size_t bytes) {
            size_t off = (blob.size() + 255) & ~static_cast<size_t>(255);
            blob.resize(off + bytes);
            if (bytes) std::memcpy(blob.data() + off, src, bytes);
            return off;
        };
        std::vector<int> act;
        int maxnp = 0;
        for (int i = 0; i < K; ++i)
            if (active[i]) {
                act.push_back(i);
                maxnp = std::max(maxnp, subs[i]->P.np);
            }
        seq.push_back({0, 0, 0, put(act.data(), act.size() * sizeof(int)), static_cast<int>(act.size()), 0});
        for (int t = 0; t < maxnp; ++t) {
            std::vector<int> snap;
            for (int i : act)
                if (subs[i]->P.np - 1 == t) snap.push_back(i);
            if (!snap.empty())
                seq.push_back({1, 0, t, put(snap.data(), snap.size() * sizeof(int)), static_cast<int>(snap.size()), 0});
            for (int k = 0; k < TK_COUNT; ++k) {
                std::vector<TermItem> items;
                for (int i : act) {
                    if (subs[i]->P.np <= t) continue;
                    for (TermItem it : subs[i]->P.term[t][k]) {
                        it.sg = i;
                        items.push_back(it);
                    }
                }
                if (!items.empty())
                    seq.push_back({2, k, t, put(items.data(), items.size() * sizeof(TermItem)),
                                   static_cast<int>(items.size()), 0});
            }
            size_t lv = 0;
            for (int i : act)
                if (subs[i]->P.np > t) lv = std::max(lv, subs[i]->P.cfv_levels[t].size());
            for (size_t l = 0; l < lv; ++l) {
                // every subgame's short items, then every subgame's long ones
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
                    H = std::max(H, P.H[t]);
                }
                const int n_long = static_cast<int>(longs.size());
                items.insert(items.end(), longs.begin(), longs.end());
                if (!items.empty())
                    seq.push_back({3, n_long, t, put(items.data(), items.size() * sizeof(CfvItem)),
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
                    H = std::max(H, P.H[t]);
                }
                if (!items.empty())
                    seq.push_back({4, 0, t, put(items.data(), items.size() * sizeof(ReachItem)),
                                   static_cast<int>(items.size()), H});
            }
        }
        if (dctx) cudaFreeAsync(dctx, stream);
        if (dlists) cudaFreeAsync(dlists, stream);
        dctx = nullptr;
        dlists = nullptr;
        BCK(cudaMallocAsync(reinterpret_cast<void **>(&dctx), std::max(1, K) * sizeof(DevCtx), stream));
        BCK(cudaMallocAsync(reinterpret_cast<void **>(&dlists), std::max<size_t>(blob.size(), 256), stream));
        BCK(cudaMemcpyAsync(dctx, ctx.data(), K * sizeof(DevCtx), cudaMemcpyHostToDevice, stream));
        BCK(cudaMemcpyAsync(dlists, blob.data(), blob.size(), cudaMemcpyHostToDevice, stream));
        // members were initialised on their own streams
        for (int i : act) BCK(cudaStreamSynchronize(subs[i]->stream));
        BCK(cudaStreamSynchronize(stream));  // host staging must outlive the copies
        cudaGraph_t g = nullptr;
        BCK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t body = cudaSuccess;
        for (int r = 0; r < graph_iters && body == cudaSuccess; ++r) body = iteration();
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (body != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            BCK(body);
        }
        BCK(e);
        e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        BCK(e);
        dirty = false;
        return SS_OK;
    }
};

// ---------------------------------------------------------------------------
// batched form: solve n subgames together
// ---------------------------------------------------------------------------

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
    for (const Problem &pb : pbs) {
        Session *s = nullptr;
        rc = session_create(pb, cfg, &s);
        if (rc != SS_OK) return rc;
        b.add(s);
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
        rc = b.sync();
        if (rc != SS_OK) break;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) total_ms += ms;
        for (size_t i = 0; i < pbs.size() && rc == SS_OK; ++i) {
            if (!b.active[i]) continue;
            const bool last = b.iters_run[i] >= max_iterations;
            if (target || (last && cfg.compute_exploitability))
                rc = b.subs[i]->exploitability(nullptr, &pct[i], &nash[i], nullptr, nullptr, nullptr);
            if (last || (target && pct[i] <= cfg.target_exploitability)) b.retire(static_cast<int>(i));
        }
        if (rc != SS_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
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
    std::chrono::steady_clock::time_point t_submit, t_done;
    int slot = -1;
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
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;
    std::map<long long, std::unique_ptr<Request>> reqs;
    std::vector<Request *> slot_req;
    size_t used = 0;
    long long next_id = 1;
    bool stop = false;
    std::thread worker;
    int fatal = SS_OK;
    std::string fatal_msg;

    int start(const SSServerOptions &o) {
        opt = o;
        int rc = batch.init(o.device, o.graph_iterations);
        if (rc != SS_OK) return rc;
        worker = std::thread([this] { loop(); });
        return SS_OK;
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_work.notify_all();
        if (worker.joinable()) worker.join();
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
        cv_work.notify_one();
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

  private:
    void fail(Request *r, int rc) {
        r->state = rc;
        r->error = last_error();
        r->t_done = std::chrono::steady_clock::now();
    }

    void loop() {
        cudaSetDevice(opt.device);
        const size_t budget = static_cast<size_t>(opt.memory_budget_gb * 1e9);
        const int block = std::max(1, opt.block_iterations);
        for (;;) {
            std::vector<Request *> admit;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || !pending.empty() || batch.num_active() > 0; });
                if (stop) return;
                while (!pending.empty()) {
                    Request *r = pending.front();
                    if (batch.num_active() + static_cast<int>(admit.size()) > 0 && used + r->bytes > budget) break;
                    pending.pop_front();
                    used += r->bytes;
                    admit.push_back(r);
                }
            }
            for (Request *r : admit) {
                SolveConfig cfg;
                cfg.device = opt.device;
                cfg.graph_iterations = opt.graph_iterations;
                Session *s = nullptr;
                int rc = session_create(r->pb, cfg, &s);
                std::lock_guard<std::mutex> lk(mu);
                if (rc != SS_OK) {
                    used -= r->bytes;
                    fail(r, rc);
                    cv_done.notify_all();
                    continue;
                }
                r->slot = batch.add(s);
                r->state = 1;
                if (static_cast<int>(slot_req.size()) <= r->slot) slot_req.resize(r->slot + 1, nullptr);
                slot_req[r->slot] = r;
            }
            if (batch.num_active() == 0) continue;
            int rc = batch.run(block);
            if (rc == SS_OK) rc = batch.sync();
            if (rc != SS_OK) {
                std::lock_guard<std::mutex> lk(mu);
                fatal = rc;
                fatal_msg = last_error();
                cv_done.notify_all();
                return;
            }
            for (size_t i = 0; i < batch.subs.size(); ++i) {
                if (!batch.active[i]) continue;
                Request *r = slot_req[i];
                double pct = -1, nash = -1;
                rc = batch.subs[i]->exploitability(nullptr, &pct, &nash, nullptr, nullptr, nullptr);
                const bool cap = batch.iters_run[i] >= opt.max_iterations;
                if (rc == SS_OK && !(cap || pct <= opt.target_exploitability)) continue;
                batch.retire(static_cast<int>(i));
                SSOutput o{};
                if (rc == SS_OK) rc = batch.subs[i]->output(&o);
                const double nhu = batch.subs[i]->P.node_hands * batch.iters_run[i];
                batch.release(static_cast<int>(i));
                std::lock_guard<std::mutex> lk(mu);
                used -= r->bytes;
                if (rc != SS_OK) {
                    fail(r, rc);
                } else {
                    r->out = o;
                    r->stats.iterations_run = batch.iters_run[i];
                    r->stats.exploitability_pct = pct;
                    r->stats.nashconv = nash;
                    r->stats.node_hand_updates = nhu;
                    r->t_done = std::chrono::steady_clock::now();
                    r->state = 2;
                }
                slot_req[i] = nullptr;
                cv_done.notify_all();
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

void server_destroy(Server *s) { delete s; }

}  // namespace ssb
