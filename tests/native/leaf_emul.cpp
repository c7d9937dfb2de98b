// Runs the continuation-value producer's per-element functions
// (poker-solver_b200/csrc/ss_leaf.cuh) on the host, phase by phase in the
// order the kernels run them, over the plan the library builds
// (ss_leaf_plan.cpp), for tests/test_leaf_producer.py.  This checks the
// element arithmetic and indexing without a GPU; the GPU tests run the
// kernels themselves.
//   leaf_emul <input.txt> <output.f32> [rows per chunk]
// With a chunk size the value phase runs chunk by chunk into a chunk-sized
// buffer copied into place, as the device driver does with its 256 MiB
// chunks.
// input: np mh num_board nr num_leaves / nh[np] / hand cards [np*mh*2] /
//        board[num_board] / runout cards [nr*(5-num_board)] / leaf_idx[num_leaves] / leaf_pot[num_leaves]
// output: the float32 values [num_leaves*4^np][np][mh], raw bytes.
#include "ss_leaf.cuh"
#include "ss_leaf.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

int main(int argc, char **argv) {
    if (argc != 3 && argc != 4) return 2;
    FILE *f = std::fopen(argv[1], "r");
    if (!f) return 2;
    int np, mh, nb, nr, nl;
    if (std::fscanf(f, "%d %d %d %d %d", &np, &mh, &nb, &nr, &nl) != 5) return 2;
    auto read_ints = [f](size_t n) {
        std::vector<int> v(n);
        for (auto &x : v)
            if (std::fscanf(f, "%d", &x) != 1) x = -1;
        return v;
    };
    std::vector<int> nh = read_ints(static_cast<size_t>(np));
    std::vector<int> cards = read_ints(static_cast<size_t>(np) * mh * 2);
    std::vector<int> board = read_ints(static_cast<size_t>(nb));
    std::vector<int> runs = read_ints(static_cast<size_t>(nr) * (5 - nb));
    std::vector<int> lidx = read_ints(static_cast<size_t>(nl));
    std::vector<double> lpot(static_cast<size_t>(nl));
    for (auto &x : lpot)
        if (std::fscanf(f, "%lf", &x) != 1) x = 0.0;
    std::fclose(f);

    SSLeafValueInput in;
    in.num_players = np;
    in.max_hands = mh;
    in.num_hands = nh.data();
    in.hand_cards = cards.data();
    in.board = board.data();
    in.num_board = nb;
    in.runout_cards = runs.data();
    in.num_runouts = nr;
    in.leaf_idx = lidx.data();
    in.leaf_pot = lpot.data();
    in.num_leaves = nl;

    using namespace ssb::leaf;
    Plan P;
    std::string err;
    if (make_plan(&in, &P, &err) != SS_OK) {
        std::fprintf(stderr, "%s\n", err.c_str());
        return 1;
    }
    const long per_row = static_cast<long>(P.np) * P.mh;
    const long nsh = static_cast<long>(P.nr) * per_row;
    std::vector<unsigned> strength(static_cast<size_t>(nsh));
    std::vector<Digest> digest(P.num_tuples());
    std::vector<double> ratio(static_cast<size_t>(nsh)), equity(static_cast<size_t>(per_row));
    std::vector<float> values(P.num_values());
    Ctx c;
    c.np = P.np;
    c.mh = P.mh;
    c.nr = P.nr;
    c.per = P.per;
    c.num_leaves = P.num_leaves;
    c.nh = P.nh.data();
    c.hand_cards = P.hand_cards.data();
    c.board5 = P.board5.data();
    c.tuple_off = P.tuple_off.data();
    c.tuple_owner = P.tuple_owner.data();
    c.tuple_hand = P.tuple_hand.data();
    c.row_pot = P.row_pot.data();
    c.row_set = P.row_set.data();
    c.strength = strength.data();
    c.digest = digest.data();
    c.ratio = ratio.data();
    c.equity = equity.data();
    for (long i = 0; i < nsh; ++i) strength_at(i, c);
    for (long t = 0; t < static_cast<long>(P.num_tuples()); ++t) digest_at(t, c);
    for (long i = 0; i < nsh; ++i) ratio_at(i, c);
    for (long i = 0; i < per_row; ++i) equity_at(i, c);
    const long rows = static_cast<long>(P.num_rows());
    const long chunk = argc == 4 ? std::max(1L, std::atol(argv[3])) : std::max(1L, rows);
    std::vector<float> buf(static_cast<size_t>(chunk * per_row));
    c.values = buf.data();
    for (long row0 = 0; row0 < rows; row0 += chunk) {
        const long n = std::min(chunk, rows - row0) * per_row;
        for (long i = 0; i < n; ++i) value_at(i, row0, c);
        std::copy(buf.begin(), buf.begin() + n, values.begin() + row0 * per_row);
    }

    FILE *o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    if (!values.empty()) std::fwrite(values.data(), sizeof(float), values.size(), o);
    std::fclose(o);
    return 0;
}
