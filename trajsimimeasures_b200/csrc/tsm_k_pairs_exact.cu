// dp_pairs_kernel in exact mode (IEEE sqrt and reciprocal), and the table's entry point
// (tsm_kernels.h).
#include "tsm_tile.cuh"
#include "tsm_pick.cuh"

namespace tsm_k {

const void* dp_pairs(int measure, int R, bool exact) {
    if (!exact) return dp_pairs_fast(measure, R);
    TSM_DP_TABLE(tsm::dp_pairs_kernel, true, measure, R)
}

}  // namespace tsm_k
