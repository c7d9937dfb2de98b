// ss_session.h -- a resident subgame on one GPU (internal).
//
// The Session owns the plan, the device tables and state, and the CUDA graphs
// of one subgame; the batched and served forms (ss_batch.cu) drive many
// sessions with merged launches.
#pragma once

#include "ss_kernels.h"

#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <utility>
#include <vector>

namespace ssb {

// tuple visits of the enumeration kernel that one solve may spend
constexpr double kEnumLimitPerIter = 4e9;
constexpr double kEnumLimitTotal = 2e11;

enum ProfClass { PC_REACH = 0, PC_CFV, PC_FILL, PC_CR1, PC_CR2, PC_SD1, PC_ENUM, PC_OTHER };
inline int term_class(int kind) {
    switch (kind) {
        case TK_ZERO:
        case TK_LEAF0: return PC_FILL;
        case TK_CR1:
        case TK_CR1D: return PC_CR1;
        case TK_CR2: return PC_CR2;
        case TK_SD1:
        case TK_SD2:
        case TK_SD3: return PC_SD1;
        case TK_CR3:   // the class of terminals with three or more counted opponents
        default: return PC_ENUM;
    }
}

class Session {
  public:
    Plan P;
    int device = 0;
    int graph_iters = 10;
    int iterations = 0;
    cudaStream_t stream = nullptr;
    char *dbase = nullptr;    // static tables
    float *dstate = nullptr;  // R, S, reach, val
    float *dleaf = nullptr;
    float *dsmall = nullptr;  // root strategy snapshot + root values
    int *diter = nullptr;
    size_t nR = 0, nReach = 0, nVal = 0, n_rs = 0;
    int frozen_root = -1;
    DevCtx c{};
    const ReachItem *reach_items[SS_MAX_PLAYERS] = {};
    std::vector<std::pair<int, int>> reach_lv[SS_MAX_PLAYERS];
    const CfvItem *cfv_items[SS_MAX_PLAYERS] = {};
    std::vector<std::pair<int, int>> cfv_lv[SS_MAX_PLAYERS];
    const TermItem *term_items[SS_MAX_PLAYERS][TK_COUNT] = {};
    const int *term_heads[SS_MAX_PLAYERS][TK_COUNT] = {};   // null for kinds without P.term_heads
    const int *root_fr[SS_MAX_PLAYERS] = {};
    const int *dec_fe = nullptr, *dec_na = nullptr, *dec_pl = nullptr;
    std::vector<int> dec_na_host, dec_player_host;   // per decision node (index order): actions, acting player
    // per (player, level) / (traverser, kind) minimum bytes, for the profile
    std::vector<double> reach_bytes[SS_MAX_PLAYERS], cfv_bytes[SS_MAX_PLAYERS];
    double term_bytes[SS_MAX_PLAYERS][TK_COUNT] = {};
    cudaGraphExec_t gA = nullptr, gC = nullptr, gB = nullptr;  // G iters, 1 iter, 1 iter + snapshot
    // best response state (allocated on first use, ensure_br)
    std::vector<float> host_w;          // range weights [np][HS]
    double *dbr = nullptr;              // reach_d [E + np][HS], val_d [N + 1][HS]
    char *dbr_tab = nullptr;            // edge -> decision index, deal item, row list, scalars
    float *davg_br = nullptr;           // profile in the output layout
    const int *br_edge_di = nullptr;    // in dbr_tab: [E] decision index of each edge's node
    const TermItem *br_deal = nullptr;  // in dbr_tab: the deal-mass item (val_d row N)
    const int *br_row = nullptr;        // in dbr_tab: {N}
    double *br_sc = nullptr;            // in dbr_tab: root sums (nashconv_from_sums layout)
    TermItem deal{};
    int deal_kind = TK_ENUM;

    // profiling hook: when set, every launch is preceded by an event record
    struct Mark {
        int cls;
        double bytes;
        int items;
        cudaEvent_t ev;
    };
    std::vector<Mark> *marks = nullptr;
    std::vector<SSLaunchRecord> last_launches;   // per launch of the last profiled iteration

    // terminal kinds of one pass write disjoint value rows and only read
    // reach: in the captured iteration all but one run on side streams
    // (fork / join through events), so short kinds overlap the long one
    cudaStream_t side[TK_COUNT] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[TK_COUNT] = {};

    ~Session() {
        if (gA) cudaGraphExecDestroy(gA);
        if (gB) cudaGraphExecDestroy(gB);
        if (gC) cudaGraphExecDestroy(gC);
        for (int k = 0; k < TK_COUNT; ++k) {
            if (side[k]) cudaStreamDestroy(side[k]);
            if (ev_join[k]) cudaEventDestroy(ev_join[k]);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (stream) {
            if (dbase) cudaFreeAsync(dbase, stream);
            if (dstate) cudaFreeAsync(dstate, stream);
            if (dleaf) cudaFreeAsync(dleaf, stream);
            if (dsmall) cudaFreeAsync(dsmall, stream);
            if (diter) cudaFreeAsync(diter, stream);
            if (dbr) cudaFreeAsync(dbr, stream);
            if (dbr_tab) cudaFreeAsync(dbr_tab, stream);
            if (davg_br) cudaFreeAsync(davg_br, stream);
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }

    cudaError_t mark(int cls, double bytes, int items = 0) {
        if (!marks) return cudaSuccess;
        Mark m{cls, bytes, items, nullptr};
        cudaError_t e = cudaEventCreate(&m.ev);
        if (e != cudaSuccess) return e;
        marks->push_back(m);
        // an external record becomes an event-record node of the captured graph
        return cudaEventRecordWithFlags(m.ev, stream, cudaEventRecordExternal);
    }

    cudaError_t reach(int p) {
        for (size_t l = 0; l < reach_lv[p].size(); ++l) {
            cudaError_t e = mark(PC_REACH, reach_bytes[p][l], reach_lv[p][l].second);
            if (e == cudaSuccess)
                e = launch_reach(c, reach_items[p] + reach_lv[p][l].first, reach_lv[p][l].second,
                                 P.H[p], stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    // traverser t's terminals of kind k (grouped kinds: one block per head)
    cudaError_t terms(int t, int k, cudaStream_t s) {
        return launch_terms(c, k, term_items[t][k], static_cast<int>(P.term[t][k].size()), t, s, nullptr,
                            term_heads[t][k], static_cast<int>(P.term_heads[t][k].size()));
    }

    cudaError_t pass(int t, bool snapshot_root) {
        cudaError_t e = cudaSuccess;
        if (snapshot_root) {
            e = mark(PC_OTHER, 0);
            if (e == cudaSuccess)
                e = launch_root_strategy(c, P.first_edge[0], P.root_na, frozen_root,
                                         P.H[P.root_player], dsmall, stream);
            if (e != cudaSuccess) return e;
        }
        int kinds[TK_COUNT], nk = 0, main_k = -1;
        for (int k = 0; k < TK_COUNT; ++k) {
            const int n = static_cast<int>(P.term[t][k].size());
            if (n == 0) continue;
            kinds[nk++] = k;
            if (main_k < 0 || n > static_cast<int>(P.term[t][main_k].size())) main_k = k;
        }
        if (marks || nk <= 1 || !ev_fork) {
            // one kind after the other (the profile times each class)
            for (int i = 0; i < nk; ++i) {
                const int k = kinds[i];
                e = mark(term_class(k), term_bytes[t][k], static_cast<int>(P.term[t][k].size()));
                if (e == cudaSuccess) e = terms(t, k, stream);
                if (e != cudaSuccess) return e;
            }
        } else {
            e = cudaEventRecord(ev_fork, stream);
            for (int i = 0; i < nk && e == cudaSuccess; ++i) {
                const int k = kinds[i];
                if (k == main_k) continue;
                e = cudaStreamWaitEvent(side[k], ev_fork, 0);
                if (e == cudaSuccess) e = terms(t, k, side[k]);
                if (e == cudaSuccess) e = cudaEventRecord(ev_join[k], side[k]);
            }
            if (e == cudaSuccess) e = terms(t, main_k, stream);
            for (int i = 0; i < nk && e == cudaSuccess; ++i)
                if (kinds[i] != main_k) e = cudaStreamWaitEvent(stream, ev_join[kinds[i]], 0);
            if (e != cudaSuccess) return e;
        }
        for (size_t l = 0; l < cfv_lv[t].size(); ++l) {
            e = mark(PC_CFV, cfv_bytes[t][l], cfv_lv[t][l].second);
            if (e == cudaSuccess)
                e = launch_cfv(c, cfv_items[t] + cfv_lv[t][l].first, cfv_lv[t][l].second, P.cfv_nlong[t][l],
                               P.H[t], stream);
            if (e != cudaSuccess) return e;
        }
        return reach(t);
    }

    cudaError_t iteration(bool last) {
        cudaError_t e = mark(PC_OTHER, 0);
        if (e == cudaSuccess) e = launch_bump(diter, stream);
        for (int t = 0; t < P.np && e == cudaSuccess; ++t) e = pass(t, last && t == P.np - 1);
        return e;
    }

    cudaError_t capture(int iters, bool last, cudaGraphExec_t *exec) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        cudaError_t body = cudaSuccess;
        for (int i = 0; i < iters && body == cudaSuccess; ++i) body = iteration(last && i == iters - 1);
        e = cudaStreamEndCapture(stream, &g);
        if (body != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return body;
        }
        if (e != cudaSuccess) return e;
        e = cudaGraphInstantiate(exec, g, 0);
        cudaGraphDestroy(g);
        return e;
    }

    int init(const Problem &pb, const SolveConfig &cfg);
    int ensure_br();
    int exploitability(const float *host_avg, double *pct, double *nash, double *br, double *cur,
                       double *deal_mass);
    void nashconv_from_sums(const double *sc, double *pct, double *nash, double *br, double *cur,
                            double *deal_mass) const;
    int reset();
    int run(int iters);
    int output(SSOutput *out);
    int profile(SSKernelProfile *prof);
    int profile_launches(SSLaunchRecord *rec, int max_records, int *num_records) const;
};

}  // namespace ssb
