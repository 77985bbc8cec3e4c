// dp_matrix_kernel in default mode (hardware sqrt and reciprocal approximations)
// (table: tsm_kernels.h).
#include "tsm_tile.cuh"
#include "tsm_pick.cuh"

namespace tsm_k {

const void* dp_matrix_fast(int measure, int R) {
    TSM_DP_TABLE(tsm::dp_matrix_kernel, false, measure, R)
}

}  // namespace tsm_k
