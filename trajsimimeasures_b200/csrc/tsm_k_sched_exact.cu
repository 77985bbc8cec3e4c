// The scheduled persistent kernel in exact mode, and the table's entry point
// (tsm_kernels.h).
#include "tsm_sched.cuh"
#include "tsm_pick.cuh"

namespace tsm_k {

const void* sched(int R, bool exact) {
    if (!exact) return sched_fast(R);
    return R == 4 ? (const void*)&tsm::dp_sched_kernel<4, true> : R == 8 ? (const void*)&tsm::dp_sched_kernel<8, true> : nullptr;
}

}  // namespace tsm_k
