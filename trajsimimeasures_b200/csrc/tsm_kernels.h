// Kernel tables of the library: the address of each kernel instantiation,
// by measure, rows per thread and arithmetic mode.  The instantiations live
// in separate translation units (tsm_k_<family>_<mode>.cu), one per kernel
// family and mode, so that they compile in parallel; tsm_capi.cu launches
// them through these addresses.  Every function returns nullptr for an
// unsupported combination (rows per thread other than 4, 8, 16; the
// scheduler: 4, 8).
#pragma once

namespace tsm_k {

// dp_pairs_kernel / dp_matrix_kernel / dp_wave_kernel<M, R, EXACT>, M = TSM_DTW .. TSM_DFRECHET
const void* dp_pairs(int measure, int R, bool exact);
const void* dp_matrix(int measure, int R, bool exact);
const void* dp_wave(int measure, int R, bool exact);
// hausdorff_matrix_kernel (matrix) or hausdorff_pairs_kernel, and hausdorff_wave_kernel <R, EXACT>
const void* haus(bool matrix, int R, bool exact);
const void* haus_wave(int R, bool exact);
// dp_sched_kernel<R, EXACT>
const void* sched(int R, bool exact);

// the default-mode halves (tsm_k_<family>_fast.cu)
const void* dp_pairs_fast(int measure, int R);
const void* dp_matrix_fast(int measure, int R);
const void* dp_wave_fast(int measure, int R);
const void* sched_fast(int R);

}  // namespace tsm_k
