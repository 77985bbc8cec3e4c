// Row-wise k-smallest selection (kNN result lists), one CTA per row.
//
// The result for a row is the k smallest (value, column) pairs in
// lexicographic order: smaller value first, ties to the smaller column index,
// i.e. exactly the first k entries of a stable argsort of the row.  NaN sorts
// after +inf.
//
// Method: an exact MSB-first radix select over the 32-bit keys of the values
// (for floats >= 0 the bit pattern orders like the value; negative values and
// NaN are mapped so that the unsigned key order is the float order) finds the
// k-th smallest key T in 4 passes of 8 bits over the row.  Keys < T are
// collected (fewer than k of them), then the keys == T with the smallest
// column indices fill the list; the list is sorted by (key, column) in shared
// memory and written out.  The row is read 5 times; for the kNN shapes
// (1k x 1M) that is a few milliseconds against seconds of DP work.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tsm {

constexpr int kTopkMax = 256;
constexpr int kTopkThreads = 512;

// Order-preserving float -> uint32 (NaN maps to the largest keys).
__device__ __forceinline__ uint32_t fkey(float v) {
    uint32_t b = __float_as_uint(v);
    if (v != v) return 0xffffffffu;
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unkey(uint32_t k) {
    const uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(b);
}

__global__ void __launch_bounds__(kTopkThreads) topk_rows_kernel(const float* __restrict__ d, int64_t n_cols,
                                                                 int64_t ld, int k, float* __restrict__ out_d,
                                                                 int32_t* __restrict__ out_i) {
    __shared__ uint32_t hist[256];
    __shared__ uint32_t s_prefix, s_need, s_nless;
    __shared__ uint64_t cand[kTopkMax];  // (key << 32) | column, sorted at the end
    __shared__ uint32_t ties[kTopkMax];
    const float* row = d + (int64_t)blockIdx.x * ld;
    const int tid = threadIdx.x;
    const int kk = (int)min((int64_t)k, n_cols);

    uint32_t prefix = 0, need = (uint32_t)kk;  // rank (1-based) of the key to find among the matching ones
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const uint32_t hmask = (shift == 24) ? 0u : (0xffffffffu << (shift + 8));
        for (int64_t c = tid; c < n_cols; c += blockDim.x) {
            const uint32_t key = fkey(row[c]);
            if ((key & hmask) == prefix) atomicAdd(&hist[(key >> shift) & 0xffu], 1u);
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t acc = 0;
            int bin = 0;
            for (; bin < 256; ++bin) {
                if (acc + hist[bin] >= need) break;
                acc += hist[bin];
            }
            s_prefix = prefix | ((uint32_t)bin << shift);
            s_need = need - acc;
        }
        __syncthreads();
        prefix = s_prefix;
        need = s_need;
        __syncthreads();
    }
    // prefix = T, the kk-th smallest key; `need` keys equal to T belong to the result
    if (tid == 0) s_nless = 0;
    __syncthreads();
    for (int64_t c = tid; c < n_cols; c += blockDim.x) {
        const uint32_t key = fkey(row[c]);
        if (key < prefix) {
            const uint32_t slot = atomicAdd(&s_nless, 1u);
            cand[slot] = ((uint64_t)key << 32) | (uint32_t)c;
        }
    }
    __syncthreads();
    const uint32_t nless = s_nless;  // = kk - need
    // the `need` smallest column indices with key == T: scan in column order,
    // one chunk of blockDim columns at a time, with a block-wide prefix count
    __shared__ uint32_t warp_cnt[kTopkThreads / 32];
    uint32_t taken = 0;
    for (int64_t base = 0; base < n_cols && taken < need; base += blockDim.x) {
        const int64_t c = base + tid;
        const bool eq = c < n_cols && fkey(row[c]) == prefix;
        const uint32_t bal = __ballot_sync(0xffffffffu, eq);
        if ((tid & 31) == 0) warp_cnt[tid >> 5] = __popc(bal);
        __syncthreads();
        uint32_t before = taken;
        for (int w = 0; w < (tid >> 5); ++w) before += warp_cnt[w];
        before += __popc(bal & ((1u << (tid & 31)) - 1u));
        if (eq && before < need) ties[before] = (uint32_t)c;
        uint32_t tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += warp_cnt[w];
        __syncthreads();
        taken += tot;
    }
    __syncthreads();
    for (uint32_t i = tid; i < need; i += blockDim.x) cand[nless + i] = ((uint64_t)prefix << 32) | ties[i];
    // pad to a power of two and bitonic-sort by (key, column)
    int n2 = 1;
    while (n2 < kk) n2 <<= 1;
    for (int i = kk + tid; i < n2; i += blockDim.x) cand[i] = ~0ull;
    __syncthreads();
    for (int size = 2; size <= n2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = tid; i < n2; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const uint64_t a = cand[i], b = cand[j];
                    if ((a > b) == up) {
                        cand[i] = b;
                        cand[j] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    float* od = out_d + (int64_t)blockIdx.x * k;
    int32_t* oi = out_i + (int64_t)blockIdx.x * k;
    for (int i = tid; i < k; i += blockDim.x) {
        if (i < kk) {
            od[i] = unkey((uint32_t)(cand[i] >> 32));
            oi[i] = (int32_t)(cand[i] & 0xffffffffu);
        } else {
            od[i] = CUDART_INF_F;
            oi[i] = -1;
        }
    }
}

}  // namespace tsm

namespace tsm {

// Unordered k-smallest selection for long candidate lists (any k <= n_cols):
// out_i[row][0..k) receives the column indices of the k smallest values of
// the row (the same set as the first k of a stable argsort), in no particular
// order.  Same radix select as topk_rows_kernel; the keys below the k-th are
// compacted straight to global memory, the ties at the k-th key fill the rest
// in column order.
__global__ void __launch_bounds__(kTopkThreads) select_rows_kernel(const float* __restrict__ d, int64_t n_cols,
                                                                   int64_t ld, int64_t k, int32_t* __restrict__ out_i) {
    __shared__ uint32_t hist[256];
    __shared__ uint32_t s_prefix, s_need, s_nless;
    __shared__ uint32_t warp_cnt[kTopkThreads / 32];
    const float* row = d + (int64_t)blockIdx.x * ld;
    int32_t* oi = out_i + (int64_t)blockIdx.x * k;
    const int tid = threadIdx.x;
    const uint32_t kk = (uint32_t)min(k, n_cols);
    uint32_t prefix = 0, need = kk;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const uint32_t hmask = (shift == 24) ? 0u : (0xffffffffu << (shift + 8));
        for (int64_t c = tid; c < n_cols; c += blockDim.x) {
            const uint32_t key = fkey(row[c]);
            if ((key & hmask) == prefix) atomicAdd(&hist[(key >> shift) & 0xffu], 1u);
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t acc = 0;
            int bin = 0;
            for (; bin < 256; ++bin) {
                if (acc + hist[bin] >= need) break;
                acc += hist[bin];
            }
            s_prefix = prefix | ((uint32_t)bin << shift);
            s_need = need - acc;
        }
        __syncthreads();
        prefix = s_prefix;
        need = s_need;
        __syncthreads();
    }
    if (tid == 0) s_nless = 0;
    __syncthreads();
    for (int64_t c = tid; c < n_cols; c += blockDim.x) {
        if (fkey(row[c]) < prefix) oi[atomicAdd(&s_nless, 1u)] = (int32_t)c;
    }
    __syncthreads();
    const uint32_t nless = s_nless;
    uint32_t taken = 0;
    for (int64_t base = 0; base < n_cols && taken < need; base += blockDim.x) {
        const int64_t c = base + tid;
        const bool eq = c < n_cols && fkey(row[c]) == prefix;
        const uint32_t bal = __ballot_sync(0xffffffffu, eq);
        if ((tid & 31) == 0) warp_cnt[tid >> 5] = __popc(bal);
        __syncthreads();
        uint32_t before = taken;
        for (int w = 0; w < (tid >> 5); ++w) before += warp_cnt[w];
        before += __popc(bal & ((1u << (tid & 31)) - 1u));
        if (eq && before < need) oi[nless + before] = (int32_t)c;
        uint32_t tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += warp_cnt[w];
        __syncthreads();
        taken += tot;
    }
    for (int64_t i = kk + tid; i < k; i += blockDim.x) oi[i] = -1;
}

}  // namespace tsm
