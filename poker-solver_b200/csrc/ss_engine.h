// ss_engine.h -- internal interface of the B200 street solver.
//
// The engine never sees SSTreeData (whose layout depends on SS_MAX_HANDS);
// the ABI layer (ss_abi.cpp, compiled once per SS_MAX_HANDS) turns it into a
// Problem of plain pointers.  SSNode and SSOutput do not depend on
// SS_MAX_HANDS and are shared.
#pragma once

#include "street_solve.h"

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace ssb {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
const char *last_error();

// ---------------------------------------------------------------------------
// host blocks for the largest output array (ss_engine.cu)
// ---------------------------------------------------------------------------
// host_block_take: a block of at least `bytes`, page-locked where the host
// allows it, reused from earlier outputs when one is idle; nullptr when host
// memory is exhausted.  host_block_give: returns a block from host_block_take
// to the pool (or releases it past the pool's cap) and reports true; false
// for any other pointer, which the caller then frees itself.
void *host_block_take(size_t bytes);
bool host_block_give(void *p);

// ---------------------------------------------------------------------------
// tree builder (ss_tree.cpp)
// ---------------------------------------------------------------------------
struct BuiltTree {
    std::vector<SSNode> nodes;
    std::vector<int> children;
    std::vector<int> level_order;
    std::vector<int> node_depth;
    int max_depth = 0;
    int num_leaves = 0;
};

int build_street_tree(const int *board, int num_board, int starting_pot, int effective_stack,
                      const float *bet_sizes, int num_bet_sizes, int num_players,
                      const int *acting_order, int is_river, int use_cont_strats, int max_raises,
                      BuiltTree *out);

// ---------------------------------------------------------------------------
// problem: one subgame as plain pointers
// ---------------------------------------------------------------------------
struct Problem {
    const SSNode *nodes = nullptr;
    const int *children = nullptr;
    int num_nodes = 0;
    int num_children_total = 0;
    int num_players = 0;
    const int *hands[SS_MAX_PLAYERS] = {};     // [num_hands[p]][2]
    const float *weights[SS_MAX_PLAYERS] = {}; // [num_hands[p]]
    int num_hands[SS_MAX_PLAYERS] = {};
    int board[SS_MAX_BOARD] = {};
    int num_board = 0;
    const float *leaf_values = nullptr;        // [num_leaves][num_players][max_hands] or null
    int num_leaves = 0;
    const int *frozen = nullptr;               // [num_nodes] or null
    int starting_pot = 0;
    int is_river = 0;
};

// ---------------------------------------------------------------------------
// device work items (16-byte aligned PODs shared by host planner and kernels)
// ---------------------------------------------------------------------------

// Top-down reach of one player through one of its own decision nodes:
// reach[first_edge + a] = reach[parent_row] * sigma_a.
struct alignas(16) ReachItem {
    int first_edge;
    int na;
    int parent_row;
    int frozen;
    int sg = 0;               // subgame of a batch (0 for a single subgame)
    int pad_[3] = {0, 0, 0};
};

// Bottom-up value and regret update at one traverser decision node; the value
// of edge e is the sum of val[] over frontier(e) = fr_items[fr_off[e] .. fr_off[e+1]).
// A frontier of at most kCfvInline rows in all is also held in the item
// (nfr > 0), so the value kernel reads the rows without the two dependent
// index loads (fr_off, then fr_items).
constexpr int kCfvInline = 8;
struct alignas(16) CfvItem {
    int first_edge;
    int na;
    int frozen;
    int node;
    int sg = 0;               // subgame of a batch (0 for a single subgame)
    float scale = 1.f;        // the node's value row is stored times this (chance weights; 1 on one street)
    int nfr = 0;              // inline frontier: its number of rows (0: not inline)
    int fr_bnd = 0;           // inline frontier: (end of edge a's rows) - 1 at bits 4a .. 4a+3 (15 past the last edge)
    int fr[kCfvInline] = {};  // inline frontier: the rows of all edges, in order
};
// fills the inline frontier of it when the frontier is short enough
void inline_frontier(CfvItem &it, const std::vector<int> &fr_off, const std::vector<int> &fr_items);

// A value/regret item whose edges' frontiers hold at least this many rows in
// total is long: several warps share each of its hand chunks.
constexpr int kCfvLongFrontier = 48;

// Order one level's value/regret items short, then long (stable within each
// class); returns the number of long items.
template <class Item, class FrontierRows>
inline int order_cfv_level(std::vector<Item> &v, FrontierRows rows) {
    auto mid = std::stable_partition(v.begin(), v.end(), [&](const Item &it) { return rows(it) < kCfvLongFrontier; });
    return static_cast<int>(v.end() - mid);
}

// A three-way showdown's rank-order sweep is cut into at most this many runs
// of tie groups, each swept by its own block from a directly computed state.
constexpr int kSd2Chunks = 16;
// sweep cost of a segment, in units of one hand added per opponent: a fixed
// part (its block barriers) plus its hands; a run is cut once it holds about
// kSd2RunCost units (at least a segment), since each run also pays for two
// directly computed states
constexpr int kSd2SegCost = 6;
constexpr int kSd2RunCost = 96;
// sweep blocks resident at once (148 SMs, 4 blocks each): a traverser's runs
// are capped so that its terminals' blocks fit one wave
constexpr int kSd2Slots = 148 * 4;
// A launch may give each block 2^lg consecutive runs (lg < kSd2Merge): many
// terminals in one launch (batches) need fewer, longer sweeps.
constexpr int kSd2Merge = 5;
static_assert(kSd2Chunks == 1 << (kSd2Merge - 1), "runs merge in powers of two");
// a solve's launch of three-way showdowns merges runs (lg > 0) once it would
// exceed this many sweep blocks; the choice belongs to the subgame (its
// TermItem.kind_detail), so a batch sweeps each subgame as a solve alone does
constexpr int kSd2BlocksTarget = 2 * 148 * 4;
inline int sd2_merge_of(int n_terms) {
    int lg = 0;
    while (lg < kSd2Merge - 1 && n_terms * (kSd2Chunks >> lg) > kSd2BlocksTarget) ++lg;
    return lg;
}

// Folds and leaves with three counted opponents use the conditioning closed
// form (TK_CR3) once every counted range holds at least this many hands and
// the first two hold no combo twice; smaller ranges enumerate (TK_ENUM).
constexpr int kCr3MinHands = 16;

// Terminal kinds per traverser.
enum TermKind : int {
    TK_ZERO = 0,     // value 0 (folded traverser at showdown, leaves without leaf values)
    TK_LEAF0 = 1,    // leaf with no live opponent: value = leaf value
    TK_CR1 = 2,      // fold / leaf with one counted opponent: factor * card-removal mass
    TK_CR2 = 3,      // fold / leaf with two counted opponents
    TK_SD1 = 4,      // showdown against one live opponent
    TK_ENUM = 5,     // anything else: exact tuple enumeration (small ranges only)
    TK_SD2 = 6,      // three-way showdown (two live opponents), ranges without repeated combos
    TK_CR1D = 7,     // TK_CR1 against a range that holds some combo more than once
    TK_CR3 = 8,      // fold / leaf with three counted opponents (large ranges; small ones enumerate)
    TK_SD3 = 9,      // four-way showdown (three live opponents), large ranges without repeated combos
    TK_COUNT = 10
};

// One terminal for one traverser.  factor: payoff for folds; leaf_off >= 0
// selects leaf_values[leaf_off + h] instead.  Showdowns use pot / bet.
// Two-opponent terminals whose counted opponents sit on the same reach rows
// (the traverser's own continuation choices below one opponent pair) form a
// group: consecutive items, the first with gextra = number of followers, the
// followers with follow = 1.  A zeroed item is a group of one.  Groups hold
// at most kTermGroupMax items.  Consecutive two-opponent groups on the same
// first-opponent row form a chain of at most kCr2ChainMax groups, computed
// by one block that builds the first opponent's matrix once: the chain's
// first leader has chain = number of groups after it, the other leaders
// chained = 1.  Chains are formed only where a launch keeps at least
// kCr2ChainBlocks blocks (about three waves of the kernel on a B200: with
// fewer, the longer blocks of a chain leave the last wave's SMs idle).
constexpr int kTermGroupMax = 16;
constexpr int kCr2ChainMax = 4;
constexpr int kCr2ChainBlocks = 2048;
struct alignas(16) TermItem {
    int node;
    int kind_detail;          // TK_ENUM: 0 fold, 1 leaf, 2 showdown; TK_SD2: log2 of the runs per block
    int k;                    // number of counted opponents
    int leaf_off;
    float payoff;
    float pot;
    float bet;
    int sg;                   // subgame of a batch (0 for a single subgame)
    int opp_row[SS_MAX_PLAYERS - 1];
    int opp_player[SS_MAX_PLAYERS - 1];
    int gextra;               // group leader: number of following items in its group
    int follow;               // 1: member of the group led by an earlier item
    int chain;                // two-opponent chain head: number of groups after its own
    int chained;              // 1: group leader computed by an earlier chain head
};

// Showdown tables for one board: every non-board 2-card combo ranked by the
// 7-card strength.  pos = rank position (ascending strength), tie group of a
// position = [lo, hi).  card_list[c] = positions of the combos holding card c,
// ascending; for a combo at position q with cards (c1, c2), cl[q] holds the
// number of entries of card_list[c1] below lo, below hi, and the same for c2.
struct alignas(16) SdCombo {
    int lo, hi;
    short c1, c2;
    short l1lo, l1hi, l2lo, l2hi;
    unsigned char d1, d2;     // dense indices of c1, c2 (rank among the non-board cards)
};

// ---------------------------------------------------------------------------
// plan: the flattened tree and every per-traverser work list
// ---------------------------------------------------------------------------
struct Plan {
    int np = 0, N = 0, E = 0;
    int max_h = 0;           // max(num_hands): output stride, leaf_values stride
    int HS = 0;              // device row stride in floats (multiple of 32)
    int H[SS_MAX_PLAYERS] = {};
    int root_player = -1, root_na = 0;
    int num_dec = 0;
    int starting_pot = 0;
    std::vector<int> dec_nodes;        // decision node ids in index order
    std::vector<int> first_edge;       // [N], -1 for terminals
    std::vector<int> edge_node;        // [E]
    // per player: reach levels (top-down)
    std::vector<std::vector<ReachItem>> reach_levels[SS_MAX_PLAYERS];
    // per traverser: cfv levels (bottom-up order); within a level the items
    // with long frontiers come last, cfv_nlong of them
    std::vector<std::vector<CfvItem>> cfv_levels[SS_MAX_PLAYERS];
    std::vector<int> cfv_nlong[SS_MAX_PLAYERS];
    // two-opponent terminals (TK_CR2): the items that start work (group leaders
    // that no chain head computes); the launch gets one block each.  (One block
    // per item, as for every other kind, keeps the one-opponent launches
    // faster: their blocks are short, and reading the head first would add a
    // memory round trip to each.)
    std::vector<int> term_heads[SS_MAX_PLAYERS][TK_COUNT];
    std::vector<int> fr_off;           // [E + 1]
    std::vector<int> fr_items;         // val rows (= node ids)
    std::vector<int> root_fr[SS_MAX_PLAYERS];
    // per traverser, per TermKind: terminal items
    std::vector<TermItem> term[SS_MAX_PLAYERS][TK_COUNT];
    // hand tables, [np][HS]: c0 | c1 << 8 | board_blocked << 16 | d0 << 20 | d1 << 26,
    // d = dense card index (rank among the deck's non-board cards, 63 for a
    // board card); -1 padding
    std::vector<int> hand_code;
    int deck = 0;                      // number of non-board cards
    std::vector<int> pair_idx;         // [np][52][52] range index of each dense-card pair, HS if none
    std::vector<int> cross_idx;        // [np][np][HS] index in o's range of t's hand h, HS if none
    // showdown tables (river only)
    int ncomb = 0;
    std::vector<SdCombo> sd_combo;     // [ncomb]
    std::vector<short> sd_card_list;   // [52][52] rank positions of the combos holding each card
    std::vector<short> sd_card_partner;// [52][52] the other card of each of those combos
    std::vector<int> sd_pos;           // [np][HS], -1 if blocked / padding
    std::vector<int> pos_hand;         // [np][ncomb] hand index at each rank position, -1 if none
    std::vector<int> pos_prefix;       // [np][ncomb + 1] hands of the player below each rank position
    // per player, the rank axis cut into segments for the three-way showdown
    // sweep: {lo, hi, holds a hand of the player, 0}; a segment is one tie
    // group holding some of the player's hands, or a run of groups holding
    // none.  Player p's segments are sd_seg[sd_seg_off[p] .. sd_seg_off[p+1]).
    std::vector<int> sd_seg;           // 4 ints per segment
    int sd_seg_off[SS_MAX_PLAYERS + 1] = {};
    // per player, the segments cut into kSd2Chunks runs swept by separate
    // blocks: run k = segments [sd_chunk[p*(kSd2Chunks+1)+k], ...[k+1]) (empty
    // runs at the end when the player has few segments)
    std::vector<int> sd_chunk;
    int sd_span[kSd2Merge] = {};       // most rank positions covered by 2^lg consecutive runs
    std::vector<uint32_t> strength;    // [np][HS], 0 if blocked / padding
    int dup[SS_MAX_PLAYERS] = {};      // range holds some combo more than once
    double enum_work = 0;              // tuple visits per iteration on TK_ENUM
    double node_hands = 0;             // num_nodes x sum_p H_p
};

int build_plan(const Problem &pb, Plan *plan);

// 7-card rank of board (num_board == 5) plus two hole cards, reference
// encoding (src/hand_eval.h:26-35, 138-156); 0 if any card repeats.
uint32_t rank7_host(const int *board5, int c0, int c1);
int rank7_batch(const int *cards7, int n, unsigned *out);
int rank7_checksum(unsigned long long *checksum, unsigned long long *hist10);

// ---------------------------------------------------------------------------
// solve (ss_engine.cu)
// ---------------------------------------------------------------------------
struct SolveConfig {
    int device = 0;
    int graph_iterations = 10;
    float target_exploitability = -1.f;
    int check_every = 50;
    int compute_exploitability = 0;
    int batch_member = 0;    // the session only runs inside a batch (no launches of its own iterations)
};

int solve(const Problem &pb, int iterations, const SolveConfig &cfg, SSOutput *out,
          SSSolveStats *stats);

// resident sessions (ss_engine.cu)
class Session;
int session_create(const Problem &pb, const SolveConfig &cfg, Session **out);
int session_run(Session *s, int iterations);
int session_sync(Session *s);
int session_reset(Session *s);
int session_iterations(const Session *s);
int session_output(Session *s, SSOutput *out);
int session_profile(Session *s, SSKernelProfile *prof);
int session_profile_launches(const Session *s, SSLaunchRecord *rec, int max_records, int *num_records);
void session_destroy(Session *s);
void *session_stream(Session *s);
int session_exploitability(Session *s, const float *host_avg, double *pct, double *nash, double *br,
                           double *cur, double *z);
// ss_narrow.cu: the reference's range update from the session's average strategy
int session_narrow(Session *s, int player, int node, unsigned action_mask, int n, const int *hand_cards,
                   double *weights, int *applied);

// ss_batch.cu: batched and served forms
int batch_solve(const std::vector<Problem> &pbs, int max_iterations, const SolveConfig &cfg, SSOutput *outs,
                SSSolveStats *stats);
class Server;
int server_create(const SSServerOptions &o, Server **out);
int server_submit(Server *s, const Problem &pb, long long *id);
int server_poll(Server *s, long long id, SSOutput *out, SSSolveStats *stats, double *latency_ms, int wait);
int server_progress(Server *s, long long id, int *state, int *iterations_run);
void server_destroy(Server *s);

// ss_noalloc.cu: solve with all device state in a static device array
int solve_noalloc(const Problem &pb, int iterations, SSOutput *out);

int exploitability(const Problem &pb, const float *avg_strategies, double *expl_pct,
                   double *nashconv, double *br_value, double *cur_value, double *deal_mass);

}  // namespace ssb
