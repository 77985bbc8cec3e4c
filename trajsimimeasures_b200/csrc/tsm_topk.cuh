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

// Unordered k-smallest selection for long candidate lists (any k):
// out_i[row][0..k) receives the column indices of the k smallest values of
// the row (the same set as the first k of a stable argsort), in no particular
// order; entries past n_cols are -1.
//
// Fast path (one read of the row): a sample of up to kSelSamples values, one
// every S columns, gives a key threshold T whose expected count of row keys
// <= T is about 1.25 k plus a margin of several standard deviations of the
// sampling; one pass over the row compacts the (key, column) pairs with key <=
// T into shared memory (warp-aggregated slots), and the exact select runs
// there.  When the compacted list holds fewer than k keys or overflows the
// buffer (kSelCap), or the ties at the k-th key exceed kSelTies, the row is
// selected by the radix path below instead (five reads of the row).  Rows of
// at most kSelCap columns are loaded into shared memory whole.
constexpr int kSelSamples = 16384;
constexpr int kSelCap = 12288;
constexpr int kSelTies = 1024;
// dynamic shared memory of select_rows_kernel: the samples, then reused as
// the candidate keys and columns, plus the tie columns
constexpr size_t kSelSmemBytes = (size_t)2 * kSelCap * 4 + (size_t)kSelTies * 4;

// Adds one to hist[bin] for every lane with want set, one shared atomic per
// distinct bin of the warp (most lanes share a bin in the high-order digits).
// Used on keys in shared memory; on a row streamed from global memory the
// plain atomics measured faster (the match costs more than the contention).
__device__ __forceinline__ void hist_add(uint32_t* hist, bool want, uint32_t bin) {
    const unsigned act = __ballot_sync(0xffffffffu, want);
    if (want) {
        const unsigned peers = __match_any_sync(act, bin);
        if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicAdd(&hist[bin], (uint32_t)__popc(peers));
    }
}

// Values per thread per iteration of a streaming pass over a row: loads
// issued together, so a pass is not bound by one load's latency per value.
constexpr int kSelUnroll = 8;

// Block-wide exact radix select over keys[0..m) in shared memory: the r-th
// smallest key (1-based) -> prefix, and how many of the keys equal to it are
// among the r smallest -> need.  Every thread of the block calls it.
__device__ __forceinline__ void smem_radix_select(const uint32_t* keys, int m, uint32_t r, uint32_t* hist,
                                                  uint32_t* s_pn, uint32_t& prefix, uint32_t& need) {
    const int tid = threadIdx.x;
    prefix = 0;
    need = r;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const uint32_t hmask = (shift == 24) ? 0u : (0xffffffffu << (shift + 8));
        for (int base = 0; base < m; base += blockDim.x) {  // warp-uniform trip count for hist_add
            const int i = base + tid;
            const uint32_t key = i < m ? keys[i] : 0u;
            hist_add(hist, i < m && (key & hmask) == prefix, (key >> shift) & 0xffu);
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t acc = 0;
            int bin = 0;
            for (; bin < 255; ++bin) {
                if (acc + hist[bin] >= need) break;
                acc += hist[bin];
            }
            s_pn[0] = prefix | ((uint32_t)bin << shift);
            s_pn[1] = need - acc;
        }
        __syncthreads();
        prefix = s_pn[0];
        need = s_pn[1];
        __syncthreads();
    }
}

// The radix path: exact selection reading the row from global memory (four
// histogram passes of 8 bits, then the keys below the k-th key, then the ties
// at it in column order).
__device__ __forceinline__ void select_row_radix(const float* __restrict__ row, int64_t n_cols, uint32_t kk,
                                                 int32_t* __restrict__ oi, uint32_t* hist, uint32_t* s_pn,
                                                 uint32_t* warp_cnt) {
    const int tid = threadIdx.x;
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
            for (; bin < 255; ++bin) {
                if (acc + hist[bin] >= need) break;
                acc += hist[bin];
            }
            s_pn[0] = prefix | ((uint32_t)bin << shift);
            s_pn[1] = need - acc;
        }
        __syncthreads();
        prefix = s_pn[0];
        need = s_pn[1];
        __syncthreads();
    }
    if (tid == 0) s_pn[2] = 0;
    __syncthreads();
    for (int64_t c = tid; c < n_cols; c += blockDim.x) {
        if (fkey(row[c]) < prefix) oi[atomicAdd(&s_pn[2], 1u)] = (int32_t)c;
    }
    __syncthreads();
    const uint32_t nless = s_pn[2];
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
}

__global__ void __launch_bounds__(kTopkThreads) select_rows_kernel(const float* __restrict__ d, int64_t n_cols,
                                                                   int64_t ld, int64_t k, int32_t* __restrict__ out_i) {
    extern __shared__ uint32_t sel_smem[];
    uint32_t* keys = sel_smem;                                             // kSelCap keys (samples first)
    int32_t* cols = reinterpret_cast<int32_t*>(sel_smem + kSelCap);        // kSelCap columns
    int32_t* ties = reinterpret_cast<int32_t*>(sel_smem + 2 * kSelCap);    // kSelTies tie columns
    __shared__ uint32_t hist[256];
    __shared__ uint32_t s_pn[4];
    __shared__ uint32_t warp_cnt[kTopkThreads / 32];
    const float* row = d + (int64_t)blockIdx.x * ld;
    int32_t* oi = out_i + (int64_t)blockIdx.x * k;
    const int tid = threadIdx.x;
    const uint32_t kk = (uint32_t)min(k, n_cols);
    for (int64_t i = kk + tid; i < k; i += blockDim.x) oi[i] = -1;
    if (kk == 0) return;
    int count = 0;
    bool fast = true;
    if (n_cols <= kSelCap) {  // the whole row fits
        for (int c = tid; c < (int)n_cols; c += blockDim.x) {
            keys[c] = fkey(row[c]);
            cols[c] = c;
        }
        count = (int)n_cols;
        __syncthreads();
    } else {
        // threshold from a sample: one value every S columns (the samples use
        // the first 2*kSelCap*4 bytes; kSelSamples <= 2*kSelCap)
        const int64_t S = (n_cols + kSelSamples - 1) / kSelSamples;
        const int ns = (int)((n_cols + S - 1) / S);
        const double per = (double)kk * ns / (double)n_cols;  // expected samples below the k-th value
        const double rr = 1.25 * per + 4.0 * sqrt(per) + 16.0;
        const double expect = rr * (double)S;  // expected compacted count
        if (expect > 0.8 * kSelCap) {
            fast = false;
        } else {
            const uint32_t r = (uint32_t)min((double)ns, ceil(rr));
            for (int i0 = 0; i0 < ns; i0 += kSelUnroll * blockDim.x) {
                float v[kSelUnroll];
#pragma unroll
                for (int q = 0; q < kSelUnroll; ++q) {
                    const int i = i0 + q * blockDim.x + tid;
                    v[q] = i < ns ? __ldg(row + (int64_t)i * S) : 0.f;
                }
#pragma unroll
                for (int q = 0; q < kSelUnroll; ++q) {
                    const int i = i0 + q * blockDim.x + tid;
                    if (i < ns) keys[i] = fkey(v[q]);
                }
            }
            __syncthreads();
            uint32_t thr, unused;
            smem_radix_select(keys, ns, r, hist, s_pn, thr, unused);  // ends with a barrier
            if (tid == 0) s_pn[3] = 0;
            __syncthreads();
            const int64_t step = (int64_t)kSelUnroll * blockDim.x;
            for (int64_t base = 0; base < n_cols; base += step) {
                float v[kSelUnroll];
#pragma unroll
                for (int q = 0; q < kSelUnroll; ++q) {
                    const int64_t c = base + q * blockDim.x + tid;
                    v[q] = c < n_cols ? __ldg(row + c) : 0.f;
                }
#pragma unroll
                for (int q = 0; q < kSelUnroll; ++q) {
                    const int64_t c = base + q * blockDim.x + tid;
                    const uint32_t key = fkey(v[q]);
                    const bool pass = c < n_cols && key <= thr;
                    const unsigned bal = __ballot_sync(0xffffffffu, pass);
                    if (bal) {
                        uint32_t slot = 0;
                        if ((tid & 31) == 0) slot = atomicAdd(&s_pn[3], (uint32_t)__popc(bal));
                        slot = __shfl_sync(0xffffffffu, slot, 0) + __popc(bal & ((1u << (tid & 31)) - 1u));
                        if (pass && slot < (uint32_t)kSelCap) {
                            keys[slot] = key;
                            cols[slot] = (int32_t)c;
                        }
                    }
                }
            }
            __syncthreads();
            count = (int)s_pn[3];
            fast = count >= (int)kk && count <= kSelCap;
        }
    }
    if (fast) {
        uint32_t prefix, need;
        smem_radix_select(keys, count, kk, hist, s_pn, prefix, need);
        if (tid == 0) {
            s_pn[2] = 0;  // keys below the k-th
            s_pn[3] = 0;  // ties at it
        }
        __syncthreads();
        for (int i = tid; i < count; i += blockDim.x) {
            const uint32_t key = keys[i];
            if (key < prefix) {
                oi[atomicAdd(&s_pn[2], 1u)] = cols[i];
            } else if (key == prefix) {
                const uint32_t t = atomicAdd(&s_pn[3], 1u);
                if (t < (uint32_t)kSelTies) ties[t] = cols[i];
            }
        }
        __syncthreads();
        const uint32_t nless = s_pn[2], neq = s_pn[3];
        if (neq <= (uint32_t)kSelTies) {
            // the need smallest tie columns: bitonic sort of the ties
            int n2 = 1;
            while (n2 < (int)neq) n2 <<= 1;
            for (int i = (int)neq + tid; i < n2; i += blockDim.x) ties[i] = 0x7fffffff;
            __syncthreads();
            for (int size = 2; size <= n2; size <<= 1) {
                for (int stride = size >> 1; stride > 0; stride >>= 1) {
                    for (int i = tid; i < n2; i += blockDim.x) {
                        const int j = i ^ stride;
                        if (j > i) {
                            const bool up = (i & size) == 0;
                            const int32_t x = ties[i], y = ties[j];
                            if ((x > y) == up) {
                                ties[i] = y;
                                ties[j] = x;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
            for (uint32_t i = tid; i < need; i += blockDim.x) oi[nless + i] = ties[i];
            return;
        }
        // too many ties for the buffer: the radix path rewrites the whole list
    }
    select_row_radix(row, n_cols, kk, oi, hist, s_pn, warp_cnt);
}

}  // namespace tsm
