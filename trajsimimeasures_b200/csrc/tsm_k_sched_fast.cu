// The scheduled persistent kernel in default mode (table: tsm_kernels.h).
#include "tsm_sched.cuh"
#include "tsm_pick.cuh"

namespace tsm_k {

const void* sched_fast(int R) {
    return R == 4 ? (const void*)&tsm::dp_sched_kernel<4, false> : R == 8 ? (const void*)&tsm::dp_sched_kernel<8, false> : nullptr;
}

}  // namespace tsm_k
