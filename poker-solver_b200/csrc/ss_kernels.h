// ss_kernels.h -- device context and kernel launchers of the street solver.
#pragma once

#include "ss_engine.h"

#include <cuda_runtime.h>

namespace ssb {

// Everything a kernel needs about one solve, passed by value.
struct DevCtx {
    float *R;              // regrets            [E][HS]
    float *S;              // strategy sums      [E][HS]
    float *reach;          // reach per sequence [E + np][HS]
    float *val;            // node values        [N][HS]
    double *reach_d;       // best response: reach under the average strategy [E + np][HS]
    double *val_d;         // best response: node values [N + 1][HS]
    const int *fr_off;     // [E + 1]
    const int *fr_items;
    const int *hand_code;  // [np][HS]
    const int *pair_idx;   // [np][52][52] range index of each dense-card pair, HS if none
    const int *cross_idx;  // [np][np][HS] index in opponent o's range of traverser t's hand h, HS if none
    const int *sd_pos;     // [np][HS]
    const unsigned *strength;    // [np][HS]
    const SdCombo *sd_combo;     // [ncomb]
    const short *sd_card_list;   // [52][52]
    const short *sd_card_partner;// [52][52]
    const int *pos_hand;         // [np][ncomb] hand index at each rank position, -1 if none
    const int *pos_prefix;       // [np][ncomb + 1] hands of the player below each rank position
    const int *sd_seg;           // three-way showdown sweep segments, 4 ints each
    const int *sd_chunk;         // [np][kSd2Chunks + 1] runs of segments
    int sd_seg_off[SS_MAX_PLAYERS + 1];
    const float *leaf_values;
    const int *iter;       // current CFR iteration (device counter, one per subgame)
    int HS;
    int np;
    int ncomb;
    int sd_span[kSd2Merge];      // most rank positions of 2^lg merged three-way showdown sweep runs
    int deck;              // number of non-board cards (dense card indices 0 .. deck-1)
    int H[SS_MAX_PLAYERS];
    int dup[SS_MAX_PLAYERS];     // range holds some combo more than once
    // root strategy snapshot (batched form: one launch covers many subgames)
    float *snap;
    int root_fe, root_na, root_frozen, root_player;
    // batched form: 0 once the subgame has left the batch; its items stay in
    // the captured launches and their blocks return at once
    int live;
    // best response (FP64 exploitability; set once its buffers exist)
    float *avg_br;            // profile in the output layout [num_dec][8][max_h]
    const int *edge_di;       // [E] decision index of each edge's node
    const int *dec_fe;        // [num_dec] first edge, actions, acting player
    const int *dec_na;
    const int *dec_pl;
    int max_h;
};

// Batched best response: the root sums of one subgame, one block each.
// out[slot] = sum over hands h of the traverser's range weight (reach_d row
// weight_row) x the sum of val_d over rows[0 .. n).
struct alignas(16) RootItem {
    const int *rows;
    int n;
    int sg;
    int trav;
    int weight_row;
    int skip_blocked;         // hands touching the board do not count
    int slot;
};

// Batched average strategy: decision node di of subgame sg.
struct alignas(8) AvgItem {
    int sg;
    int di;
};

// threads per block of the per-hand kernels; each thread covers 4 hands
constexpr int kHandThreads = 64;
constexpr int kHandsPerBlock = kHandThreads * 4;
// threads per block of the value/regret kernel (2 hands each)
constexpr int kCfvThreads = 128;
// warps that share one hand chunk of a value/regret item with a long frontier
constexpr int kCfvSplit = 4;
// threads per block of the per-terminal kernels
constexpr int kTermThreads = 256;

// With ctxs (a device array) every item reads the context of its subgame
// (item.sg) and covers that subgame's hands of `player` / `trav`; without,
// all items use c and cover H hands.  H also sizes the grid (the largest hand
// count of the launch).
cudaError_t launch_reach(const DevCtx &c, const ReachItem *items, int n, int H, cudaStream_t s,
                         const DevCtx *ctxs = nullptr, int player = -1);
// The last n_long items (long frontiers) run with kCfvSplit warps per hand chunk.
cudaError_t launch_cfv(const DevCtx &c, const CfvItem *items, int n, int n_long, int H, cudaStream_t s,
                       const DevCtx *ctxs = nullptr, int trav = -1);
// heads (optional, TK_CR2): the n_heads items that start work (TermItem
// groups and chains); the launch then has one block per head instead of one
// per item (the tensor-core two-opponent form takes every item)
cudaError_t launch_terms(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                         cudaStream_t s, const DevCtx *ctxs = nullptr, const int *heads = nullptr,
                         int n_heads = 0);
cudaError_t launch_terms_fp64(const DevCtx &c, int kind, const TermItem *items, int n, int trav,
                              cudaStream_t s, const DevCtx *ctxs = nullptr);
// Three-way showdowns of many subgames (batches): block b sweeps run group
// bmap[b].y of item bmap[b].x with that item's own merge (kind_detail), so
// each subgame is swept exactly as in its own solve; lg_max sizes the shared
// memory.  FP32 (CFR) or FP64 (best response).
cudaError_t launch_sd2_mapped(const DevCtx &c, const TermItem *items, const int2 *bmap, int nblocks, int lg_max,
                              int trav, cudaStream_t s, const DevCtx *ctxs, bool fp64);
// batched best response: every item reads the context of its subgame (item.sg)
cudaError_t launch_avg_many(const DevCtx *ctxs, const AvgItem *items, int n, int max_h, cudaStream_t s);
cudaError_t launch_br_reach_many(const DevCtx *ctxs, const ReachItem *items, int n, int H, int player,
                                 cudaStream_t s);
cudaError_t launch_br_value_many(const DevCtx *ctxs, const CfvItem *items, int n, int H, int trav, int mode,
                                 cudaStream_t s);
cudaError_t launch_br_root_many(const DevCtx *ctxs, const RootItem *items, int n, double *out, cudaStream_t s);
// Whether two-opponent terminals of a subgame with context c take the
// tensor-core form (tcgen05) rather than the mma.sync form.
bool cr2_tensor_form(const DevCtx &c);
// The device fault word (a bounded tensor-core wait that ran out, or a block
// a kernel was not built for): copied into *code and cleared; synchronizes s.
cudaError_t read_device_fault(unsigned *code, cudaStream_t s);
cudaError_t launch_bump(int *iter, cudaStream_t s);
cudaError_t launch_bump_many(const DevCtx *ctxs, const int *sgs, int n, cudaStream_t s);
cudaError_t launch_snapshot_many(const DevCtx *ctxs, const int *sgs, int n, cudaStream_t s);
cudaError_t launch_br_reach(const DevCtx &c, const ReachItem *items, int n, int H, const float *avg,
                            const int *edge_di, int max_h, cudaStream_t s);
cudaError_t launch_br_value(const DevCtx &c, const CfvItem *items, int n, int H, const float *avg,
                            const int *edge_di, int max_h, int mode, cudaStream_t s);
cudaError_t launch_br_root(const DevCtx &c, const int *rows, int n, int H, int weight_row, int trav,
                           int skip_blocked, double *out, cudaStream_t s);
cudaError_t launch_sum_rows(const DevCtx &c, const int *rows, int n, float *out, int H,
                            cudaStream_t s);
cudaError_t launch_root_strategy(const DevCtx &c, int first_edge, int na, int frozen, int H,
                                 float *out, cudaStream_t s);
cudaError_t launch_avg_strategy(const DevCtx &c, const int *dec_first_edge, const int *dec_na,
                                const int *dec_player, int num_dec, int max_h, float *out,
                                cudaStream_t s);

}  // namespace ssb
