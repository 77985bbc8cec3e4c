// dp_wave_kernel in default mode (hardware sqrt and reciprocal approximations)
// (table: tsm_kernels.h).
#include "tsm_wave.cuh"
#include "tsm_pick.cuh"

namespace tsm_k {

const void* dp_wave_fast(int measure, int R) {
    TSM_DP_TABLE(tsm::dp_wave_kernel, false, measure, R)
}

}  // namespace tsm_k
