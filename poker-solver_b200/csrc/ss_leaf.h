// ss_leaf.h -- continuation-value producer, host side (ss_leaf_plan.cpp).
//
// The producer runs the reference's turn / flop leaf-value computation
// (python/leaf_values.py:408-571, 694-816) on the GPU.  Its host part fixes
// everything the reference decides with Python control flow: which hands are
// live on each runout (python/leaf_values.py:771-778), which opponent tuples
// each hero player is scored against (enumerated, or drawn with Python's
// random.Random(42), python/leaf_values.py:615-629), and which output rows
// the leaf descriptors fill (python/leaf_values.py:795-814).  The device part
// (ss_leaf.cuh, ss_leaf.cu) does the arithmetic.  This header and
// ss_leaf_plan.cpp need no CUDA.
#pragma once

#include "street_solve.h"

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace ssb {
namespace leaf {

constexpr int kTupleLimit = SS_LEAF_TUPLE_LIMIT;
constexpr int kMaxHands = 1326;

// Python's random.Random(seed) for a seed in [0, 2^32): the MT19937
// generator of Matsumoto and Nishimura seeded by its init_by_array with the
// one-word key {seed} (CPython's random_seed for a small int), and the two
// draws Random.choice uses: getrandbits(k) for k <= 32 (the top k bits of
// one 32-bit output) and _randbelow(n) (getrandbits(n.bit_length()) until
// the value is below n).
class PyRandom {
  public:
    explicit PyRandom(uint32_t seed);
    uint32_t next32();
    uint32_t below(uint32_t n);   // n >= 1

  private:
    static constexpr int kN = 624;
    uint32_t mt_[kN];
    int i_ = kN;
};

// The reference's tuple rule as positions into the opponents' live-hand
// lists (sizes[k] hands for opponent k): all tuples in itertools.product
// order (last opponent fastest) when the product of the sizes is at most
// kTupleLimit, otherwise kTupleLimit tuples, each drawn opponent by opponent
// with choice() from one PyRandom(42).  Appends nopp positions per tuple to
// *out and returns the tuple count (0 if some list is empty).
int opponent_tuples(int nopp, const int *sizes, std::vector<int> *out);

// Everything the kernels read, flattened.  Runout r's five board cards are
// board5[5r .. 5r+4].  The tuples of hero player p on runout r are
// tuple_off[r*np+p] .. tuple_off[r*np+p+1]-1; tuple t lists the opponents'
// hand indices (players in order, the hero skipped) in
// tuple_hand[t*(np-1) ...] and its owner r*np+p in tuple_owner[t].
struct Plan {
    int np = 0, mh = 0, nr = 0, num_leaves = 0, per = 0;   // per = 4^np
    std::vector<int> nh;                                    // [np]
    std::vector<int> hand_cards;                            // [np][mh][2]
    std::vector<int> board5;                                // [nr][5]
    std::vector<int> tuple_off;                             // [nr*np + 1]
    std::vector<int> tuple_owner;                           // [tuples]
    std::vector<uint16_t> tuple_hand;                       // [tuples][np-1]
    std::vector<double> row_pot;                            // [num_leaves]: pot of output rows leaf*per ..
    std::vector<unsigned char> row_set;                     // [num_leaves]: 1 if a descriptor fills them

    size_t num_tuples() const { return tuple_owner.size(); }
    size_t num_rows() const { return static_cast<size_t>(num_leaves) * per; }
    size_t num_values() const { return num_rows() * np * mh; }
};

// Validates the input and builds the plan.  SS_OK, or SS_ERR_INVALID /
// SS_ERR_NOMEM with a message in *err.
int make_plan(const SSLeafValueInput *in, Plan *plan, std::string *err);

// The whole producer on the current CUDA device (ss_leaf.cu): plan, upload,
// kernels, output rows copied into out[num_values()].  SS_OK or SS_ERR_*
// with the message in last_error().
int leaf_values_gpu(const SSLeafValueInput *in, float *out);

}  // namespace leaf
}  // namespace ssb
