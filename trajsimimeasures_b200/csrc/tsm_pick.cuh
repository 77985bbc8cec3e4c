// Kernel-address tables for the tsm_k_*.cu units (see tsm_kernels.h).
#pragma once

#include "tsm.h"
#include "tsm_kernels.h"

// the instantiation of KER<M, R, E> for R in {4, 8, 16}, else nullptr
#define TSM_BY_R(KER, M, E, R)                                                       \
    ((R) == 4 ? (const void*)&KER<M, 4, E>                                           \
              : (R) == 8 ? (const void*)&KER<M, 8, E> : (R) == 16 ? (const void*)&KER<M, 16, E> : nullptr)

// the instantiation of KER<measure, R, E> for the five DP measures
#define TSM_DP_TABLE(KER, E, measure, R)                                           \
    switch (measure) {                                                             \
        case TSM_DTW: return TSM_BY_R(KER, tsm::DTW, E, R);                        \
        case TSM_EDR: return TSM_BY_R(KER, tsm::EDR, E, R);                        \
        case TSM_LCSS: return TSM_BY_R(KER, tsm::LCSS, E, R);                      \
        case TSM_ERP: return TSM_BY_R(KER, tsm::ERP, E, R);                        \
        case TSM_DFRECHET: return TSM_BY_R(KER, tsm::DFRECHET, E, R);              \
        default: return nullptr;                                                   \
    }
