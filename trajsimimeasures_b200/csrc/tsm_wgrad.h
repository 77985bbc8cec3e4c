// Encoder weight gradients on the tensor cores (tsm_wgrad.cu), called by the
// training backward of tsm_encoder.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Device scratch (bytes, 256-byte aligned start) for a batch of B
// trajectories of at most T steps.
int64_t tsm_wgrad_scratch_bytes(int B, int T);

// d_ih[384][64] += sum over valid (b, t) of G[b][t][:] (x) A[b][t][:],
// d_hh[384][128] += sum of GH[b][t][:] (x) H[b][t][:] (H: T + 1 rows per
// trajectory).  Stream-ordered; a bounded wait that runs out ORs a bit into
// *status (device int) and its CTA adds nothing.
int tsm_wgrad_tc(const float* G, const float* GH, const float* A, const float* H, const int32_t* len, int B, int T,
                 void* scratch, int* status, float* d_ih, float* d_hh, cudaStream_t s);
