// tsm_pairs_sched_noalloc: the scheduled paired batch with its scratch in a
// library-owned, statically allocated device array instead of a caller
// workspace.
//
// Who needs it: callers that cannot allocate device memory at the point of
// the call -- code running where the CUDA allocator must not be touched (a
// host callback or a section that has to stay free of cudaMalloc/cudaFree
// and their implicit synchronisation), plugins whose host application owns
// all device allocations, or C/FFI callers with no device allocator of
// their own.  They still pass their inputs and outputs (device memory they
// were given); the only scratch the scheduled kernel needs -- its task-queue
// head and exit count -- lives in g_sched_scratch below.
//
// The array is kNoallocScratchBytes = 256 bytes, 256-byte aligned, and every
// GPU that loads the library holds it until the process exits.  It is shared
// by every call: calls whose kernels overlap on the GPU (on different
// streams, or from different host threads) race on the same queue and give
// wrong results; serialise them.  The kernel leaves the queue at zero when it
// finishes, so consecutive calls start clean.
//
// Set-up: every call looks up the array's device address in the current
// context with cudaGetSymbolAddress -- the array's name in host code is only a
// host-side stand-in, never a device address.  The first call on each device
// (with that device current) clears the array (cudaMemset, then a device
// synchronisation, so every stream sees the zeros); make that first call
// before any stream capture.  The lookup is not cached: after
// cudaDeviceReset the library's module is loaded again and the array may
// move, and a later call then uses (and clears once more) the new address.
// No call allocates or frees device memory.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "tsm.h"

// Sets the calling thread's tsm_last_error() message (tsm_capi.cu; hidden).
int tsm_internal_fail(int code, const char* msg);

namespace {

constexpr int kNoallocScratchBytes = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) int g_sched_scratch[kNoallocScratchBytes / 4];

std::mutex g_setup_mu;
void* g_cleared_addr[kMaxDevices] = {};  // per device: the address last cleared

int fail_cuda(const char* what, cudaError_t e) {
    char b[256];
    snprintf(b, sizeof(b), "tsm_pairs_sched_noalloc: %s: %s", what, cudaGetErrorString(e));
    return tsm_internal_fail(TSM_ECUDA, b);
}

}  // namespace

extern "C" {

int tsm_pairs_sched_noalloc(const float* pts, const int64_t* off_a, const int32_t* len_a, const int64_t* off_b,
                            const int32_t* len_b, const int32_t* order, const int32_t* tasks, int32_t n_tasks,
                            int32_t max_len, int32_t warp_smem_floats, const tsm_params* params, float* out,
                            int32_t* out_counts, int64_t out_stride, void* stream) {
    const int need = tsm_sched_workspace_bytes();
    if (need > kNoallocScratchBytes) {
        char b[256];
        snprintf(b, sizeof(b), "tsm_pairs_sched_noalloc: the kernel needs %d bytes of scratch, the static array "
                 "holds %d", need, kNoallocScratchBytes);
        return tsm_internal_fail(TSM_ETOOLONG, b);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_cuda("cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices) return tsm_internal_fail(TSM_EINVAL, "tsm_pairs_sched_noalloc: device ordinal out of range");
    void* scratch = nullptr;
    e = cudaGetSymbolAddress(&scratch, g_sched_scratch);  // this context's copy of the array
    if (e != cudaSuccess) return fail_cuda("cudaGetSymbolAddress", e);
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (g_cleared_addr[dev] != scratch) {
            e = cudaMemset(scratch, 0, kNoallocScratchBytes);  // the queue must start at zero
            if (e != cudaSuccess) return fail_cuda("cudaMemset", e);
            e = cudaDeviceSynchronize();  // cleared before any stream's first launch
            if (e != cudaSuccess) return fail_cuda("cudaDeviceSynchronize", e);
            g_cleared_addr[dev] = scratch;
        }
    }
    return tsm_pairs_sched(pts, off_a, len_a, off_b, len_b, order, tasks, n_tasks, max_len, warp_smem_floats,
                           params, out, out_counts, out_stride, scratch, stream);
}

}  // extern "C"
