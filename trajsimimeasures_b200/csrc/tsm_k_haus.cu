// Hausdorff kernels, both modes (table: tsm_kernels.h).
#include "tsm_tile.cuh"
#include "tsm_pick.cuh"

namespace tsm_k {

namespace {
template <int R, bool E>
const void* haus_of(bool matrix) {
    return matrix ? (const void*)&tsm::hausdorff_matrix_kernel<R, E> : (const void*)&tsm::hausdorff_pairs_kernel<R, E>;
}
template <bool E>
const void* haus_wave_of(int R) {
    switch (R) {
        case 4: return (const void*)&tsm::hausdorff_wave_kernel<4, E>;
        case 8: return (const void*)&tsm::hausdorff_wave_kernel<8, E>;
        case 16: return (const void*)&tsm::hausdorff_wave_kernel<16, E>;
        default: return nullptr;
    }
}
}  // namespace

const void* haus(bool matrix, int R, bool exact) {
    switch (R) {
        case 4: return exact ? haus_of<4, true>(matrix) : haus_of<4, false>(matrix);
        case 8: return exact ? haus_of<8, true>(matrix) : haus_of<8, false>(matrix);
        case 16: return exact ? haus_of<16, true>(matrix) : haus_of<16, false>(matrix);
        default: return nullptr;
    }
}

const void* haus_wave(int R, bool exact) { return exact ? haus_wave_of<true>(R) : haus_wave_of<false>(R); }

}  // namespace tsm_k
