// fs_abi.cpp -- the C ABI of include/flop_solve.h (flop_solve.cuh:128-178).
// The layouts do not depend on SS_MAX_HANDS: one translation unit serves both
// library builds.  Every entry point catches host allocation failures and
// reports them as SS_ERR_NOMEM with a message from ss_last_error().
#include "flop_solve.h"
#include "fs_engine.h"

#include <new>

extern "C" {

int fs_build_tree(const int *flop_board, int starting_pot, int effective_stack, const float *bet_sizes,
                  int num_bet_sizes, FSTreeData *tree_out) {
    if (!tree_out) return SS_ERR_INVALID;
    try {
        return ssb::fs::build_tree(flop_board, starting_pot, effective_stack, bet_sizes, num_bet_sizes, tree_out);
    } catch (const std::bad_alloc &) {
        ssb::fs::free_tree(tree_out);
        ssb::set_error("fs_build_tree: out of host memory");
        return SS_ERR_NOMEM;
    }
}

int fs_solve_gpu(FSTreeData *tree_data, int max_iterations, FSOutput *output) {
    if (!output) return SS_ERR_INVALID;
    try {
        return ssb::fs::solve(tree_data, max_iterations, output, false);
    } catch (const std::bad_alloc &) {
        ssb::set_error("fs_solve_gpu: out of host memory");
        return SS_ERR_NOMEM;
    }
}

int fs_solve_gpu_extract_all(FSTreeData *tree_data, int max_iterations, FSOutput *output) {
    if (!output) return SS_ERR_INVALID;
    try {
        return ssb::fs::solve(tree_data, max_iterations, output, true);
    } catch (const std::bad_alloc &) {
        ssb::set_error("fs_solve_gpu_extract_all: out of host memory");
        return SS_ERR_NOMEM;
    }
}

void fs_free_tree(FSTreeData *tree_data) { ssb::fs::free_tree(tree_data); }

void fs_free_output(FSOutput *output) { ssb::fs::free_output(output); }

}  // extern "C"
