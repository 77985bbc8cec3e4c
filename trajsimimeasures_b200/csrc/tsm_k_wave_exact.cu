// dp_wave_kernel in exact mode (IEEE sqrt and reciprocal), and the table's entry point
// (tsm_kernels.h).
#include "tsm_wave.cuh"
#include "tsm_pick.cuh"

namespace tsm_k {

const void* dp_wave(int measure, int R, bool exact) {
    if (!exact) return dp_wave_fast(measure, R);
    TSM_DP_TABLE(tsm::dp_wave_kernel, true, measure, R)
}

}  // namespace tsm_k
