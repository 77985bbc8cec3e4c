// Candidate scan of the learned kNN filter on the tensor cores (tcgen05).
//
// For queries q and database rows j of the filter's embedding space (160
// values, centred on the database mean), the scan evaluates
//     d(q, j) = |e_j|^2 - 2 e_q . e_j
// (the squared distance less the query's own |e_q|^2, which does not change a
// query's ranking) for every pair, and either writes the dense block (the
// threshold sample) or keeps only the pairs with d <= thr_q, appending them to
// the query's candidate list (database index and d) -- so the [queries x
// database] block is never written.
//
// Precision.  Among a million trajectories the nearest candidates differ in
// d by about 1e-5 of |e|^2, far below TF32 or FP16 rounding of the operands
// (2^-11).  Each operand is split into two FP16 values, x = hi + lo with
// lo = fp16(x - hi), and the tensor cores take
//     e_q . e_j = q_hi . d_hi + q_lo . d_hi + q_hi . d_lo   (+ q_lo . d_lo, dropped)
// as ONE product over K = 3 x 160: queries [q_hi | q_lo | q_hi] against rows
// [d_hi | d_hi | d_lo], accumulated in FP32 -- the split-product method
// (Markidis et al., "NVIDIA Tensor Core Programmability, Performance &
// Precision", IPDPSW 2018), about 2^-21 relative per product.  The squared
// norm enters the same product: three more K columns hold, for the row, the
// FP32 value n_j = |e_j|^2 s^2 / 2^16 split into three FP16 parts (33
// significant bits) and, for the query, 2^15 each, so the accumulator is
//     acc = s^2 (e_q . e_j - |e_j|^2 / 2) = -(s^2 / 2) d(q, j)
// and the epilogue compares raw accumulators (d <= thr  <=>  acc >= -(s^2/2) thr).
// The values are scaled by a power of two s (exact) that keeps every scaled
// value within 2^10 and n_j within FP16's range.  K = 512: the 483 columns
// used, padded with zeros.
//
// Kernel.  One CTA per (query tile of 128, slice of database tiles of 256
// rows).  The query tile's image (128 KB) is copied into shared memory once and
// stays there; the database tiles stream through a five-stage ring, each stage
// a K slice of 32 (16 KB): cp.async.bulk of pre-formatted operand images,
// completion on mbarrier transaction counts.  Warp 0 issues the copies, one
// thread of warp 1 issues the MMAs (M = 128 queries, N = 256 rows, K = 16 per
// instruction, 32 per database tile) into one of two FP32 accumulators of 256
// tensor-memory columns, and warps 2-9 (two per 32-lane quarter of tensor
// memory, each reading half of the columns, 64 per tensor-memory load batch)
// read the other accumulator with tcgen05.ld and apply the threshold -- one
// compare per 64 values against their tree maximum -- while the next tile's
// MMAs run.  A survivor is staged in shared memory (four slots per epilogue
// thread); a warp flushes its staged survivors together (one atomicAdd per
// thread on its query's count, then the stores) when a thread's slots are
// full and at the end, so that the round trip of the atomic is paid about once
// per dozen tiles rather than once per survivor.  Every wait is bounded (about
// 1 s of SM clocks); one that runs out sets a bit of *status and ends that
// role's loop, the CTA waits (bounded) for its own copies and MMAs in flight,
// and frees tensor memory only when no MMA can still write it.
//
// Operand images (tsm_scan_prepare): tiles of R rows (128 for queries, 256
// for the database), each in the K-major core-matrix layout of tsm_umma.cuh
// (8 rows x 16 bytes per core matrix, K chunk stride R * 16 bytes).
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

#include "tsm.h"
#include "tsm_umma.cuh"

int tsm_internal_fail(int code, const char* msg);

namespace tsm {
namespace scan {

constexpr int D = 160;                     // embedding width
constexpr int KE = 3 * D;                  // split-product columns
constexpr int K = 512;                     // + 3 norm columns, zero padding
constexpr int KCH = K / 8;                 // 16-byte K chunks of a row
constexpr int QM = 128;                    // queries per tile (MMA M, tensor-memory lanes)
constexpr int DN = 256;                    // database rows per tile (MMA N)
constexpr int SK = 32;                     // K per pipeline stage: two MMAs of K = 16
constexpr int NSTAGE = 5;
constexpr int STAGES_PER_TILE = K / SK;    // 16
constexpr int A_BYTES = QM * K * 2;        // 131,072: one query tile's image (resident)
constexpr int A_COPY = 8192;               // its copies
constexpr int B_TILE_BYTES = DN * K * 2;   // 262,144: one database tile's image
constexpr int B_STAGE_BYTES = DN * SK * 2; // 16,384
constexpr int EPI_WARPS = 8;               // two per 32-lane quarter of tensor memory, each half the columns
constexpr int EPI_THREADS = 32 * EPI_WARPS;
constexpr int THREADS = 64 + EPI_THREADS;  // warp 0 copies, warp 1 MMAs, warps 2-9 epilogue
constexpr int EPI_COLS = 64;               // accumulator columns per tensor-memory load batch
constexpr int SLOTS = 4;                   // staged survivors per epilogue thread
constexpr uint32_t TMEM_COLS = 2 * DN;     // two accumulators
constexpr int OFF_A = 0;
constexpr int OFF_S = OFF_A + A_BYTES;     // NSTAGE database stages
constexpr int OFF_BAR = OFF_S + NSTAGE * B_STAGE_BYTES;
// mbarriers: full[NSTAGE], empty[NSTAGE], tfull[2], tempty[2], done, a_full; then the tensor-memory slot and flag
constexpr int BAR_FULL = 0, BAR_EMPTY = 8 * NSTAGE, BAR_TFULL = 16 * NSTAGE, BAR_TEMPTY = BAR_TFULL + 16,
              BAR_DONE = BAR_TEMPTY + 16, BAR_AFULL = BAR_DONE + 8, TMEM_SLOT = BAR_AFULL + 8, TMEM_BUSY = TMEM_SLOT + 4;
constexpr int OFF_STG = OFF_BAR + 256;     // SLOTS x EPI_THREADS staged (index, d)
constexpr int SMEM = OFF_STG + SLOTS * EPI_THREADS * 8;  // 221,440 bytes
constexpr long long WAIT_CYCLES = 2000000000LL;
constexpr float NORM_A = 32768.f;          // the query's norm columns (2^15)
constexpr float NORM_SHIFT = 1.f / 65536.f;  // n_j = |e_j|^2 s^2 2^-16
static_assert(K % SK == 0 && SK % 16 == 0 && D % 8 == 0 && KE + 3 <= K && A_BYTES % A_COPY == 0, "sizes");
static_assert(TMEM_BUSY + 4 <= 256, "barrier block");
static_assert(SMEM <= 227 * 1024, "shared memory");

// status bits
constexpr int ERR_COPY = 1;   // a copy (or its stage) did not become available in time
constexpr int ERR_MMA = 2;    // the MMA issuer gave up waiting for an accumulator or a stage
constexpr int ERR_TMEM = 4;   // MMAs still pending at exit: tensor memory left allocated
constexpr int ERR_EPI = 8;    // the epilogue gave up waiting for an accumulator

// Operand image of rows [0, n) of emb (row stride ld floats, D values each,
// times s), padded with rows to whole tiles of R rows.  K columns: queries
// [hi | lo | hi | 2^15 x 3 | 0...]; database rows [hi | hi | lo | -n_j
// as three FP16 parts | 0...] with n_j = |emb_j|^2 s^2 2^-16 (the squared
// norm of the unscaled row, FP32), and for the padding rows of the last tile
// n_j parts at FP16's largest value, so that their accumulator is far below
// any threshold.  norms (nullable): the FP32 |emb_j|^2 of the rows.  One
// thread per (row, 16-byte chunk), consecutive threads on consecutive rows of
// one chunk (coalesced 16-byte stores).
template <bool DB>
__global__ void scan_prepare(const float* __restrict__ emb, int64_t n, int64_t ld, float s, int64_t n_tiles,
                             __half* __restrict__ img, float* __restrict__ norms) {
    constexpr int R = DB ? DN : QM;
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= n_tiles * KCH * R) return;
    const int r = gid % R;
    const int c = (gid / R) % KCH;
    const int64_t t = gid / ((int64_t)R * KCH);
    const int64_t row = t * R + r;
    __align__(16) __half v[8];
    if (8 * c < KE) {
        const int part = (8 * c) / D;  // which third of the split product
        const int k0 = 8 * c - part * D;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const float x = row < n ? s * emb[row * ld + k0 + e] : 0.f;
            const __half h = __float2half_rn(x);
            const __half l = __float2half_rn(x - __half2float(h));
            v[e] = DB ? (part < 2 ? h : l) : (part == 1 ? l : h);
        }
    } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] = __float2half_rn(0.f);
        if (8 * c == KE) {  // the norm columns
            if (!DB) {
                v[0] = v[1] = v[2] = __float2half_rn(NORM_A);
            } else if (row < n) {
                float ss = 0.f;
                for (int k = 0; k < D; ++k) {
                    const float x = emb[row * ld + k];
                    ss = fmaf(x, x, ss);
                }
                if (norms) norms[row] = ss;
                const float nj = ss * (s * s) * NORM_SHIFT;
                const __half h = __float2half_rn(nj);
                const float r1 = nj - __half2float(h);
                const __half m = __float2half_rn(r1);
                const __half l = __float2half_rn(r1 - __half2float(m));
                v[0] = __hneg(h);
                v[1] = __hneg(m);
                v[2] = __hneg(l);
            } else {
                v[0] = v[1] = v[2] = __float2half_rn(-65504.f);
            }
        }
    }
    unsigned char* dst = reinterpret_cast<unsigned char*>(img) + t * ((int64_t)R * K * 2) +
                         (int64_t)c * (R * 16) + (r >> 3) * 128 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(v);
}

// Moves a thread's `n` staged survivors (slots stg[0], stg[EPI_THREADS], ...)
// to its query's list: one atomicAdd on the count, then the stores below cap.
// Kept out of line: it runs about once per dozen tiles, and inlined at every
// staging site it would crowd the instruction cache.
__device__ __noinline__ void flush_staged(const uint2* stg, int n, int32_t* count, int32_t* idx_row, float* d_row,
                                          int cap) {
    const int pos = atomicAdd(count, n);
    for (int e = 0; e < n; ++e) {
        const uint2 v = stg[e * EPI_THREADS];
        if (pos + e < cap) {
            idx_row[pos + e] = (int32_t)v.x;
            d_row[pos + e] = __uint_as_float(v.y);
        }
    }
}

template <bool DENSE>
__global__ void __launch_bounds__(THREADS, 1) scan_kernel(
    const __half* __restrict__ qimg, int64_t nq, const __half* __restrict__ dimg, int64_t nd, float inv_s2,
    const float* __restrict__ thr, int cap, int32_t* __restrict__ cand_idx, float* __restrict__ cand_d,
    int32_t* __restrict__ counts, float* __restrict__ dense, int64_t ld, int nqt, int64_t tiles_per_slice,
    int* __restrict__ status, long long wait_cycles) {
    namespace U = tsm::umma;
    extern __shared__ __align__(1024) unsigned char sm[];
    const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
    const uint32_t bar = sbase + OFF_BAR;
    auto full = [&](int i) { return bar + BAR_FULL + 8 * i; };    // copies landed
    auto empty = [&](int i) { return bar + BAR_EMPTY + 8 * i; };  // stage read by the MMAs
    auto tfull = [&](int b) { return bar + BAR_TFULL + 8 * b; };  // accumulator ready
    auto tempty = [&](int b) { return bar + BAR_TEMPTY + 8 * b; };  // accumulator read
    const uint32_t donebar = bar + BAR_DONE;  // all MMAs done
    const uint32_t afull = bar + BAR_AFULL;   // query tile landed
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(sm + OFF_BAR + TMEM_SLOT);
    volatile int* tmem_busy = reinterpret_cast<volatile int*>(sm + OFF_BAR + TMEM_BUSY);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qt = blockIdx.x % nqt;
    const int64_t sl = blockIdx.x / nqt;
    const int64_t ntiles = (nd + DN - 1) / DN;
    const int64_t t0 = sl * tiles_per_slice;
    const int64_t t1 = min(ntiles, t0 + tiles_per_slice);
    const int64_t ntl = t1 > t0 ? t1 - t0 : 0;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NSTAGE; ++i) {
            U::mbar_init(full(i), 1);
            U::mbar_init(empty(i), 1);
        }
        for (int b = 0; b < 2; ++b) {
            U::mbar_init(tfull(b), 1);
            U::mbar_init(tempty(b), EPI_WARPS);  // one arrival per epilogue warp
        }
        U::mbar_init(donebar, 1);
        U::mbar_init(afull, 1);
        *tmem_busy = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) U::tmem_alloc(sbase + OFF_BAR + TMEM_SLOT, TMEM_COLS);
    U::fence_before_sync();
    __syncthreads();
    U::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0 && ntl > 0) {  // copies
            const unsigned char* asrc = reinterpret_cast<const unsigned char*>(qimg) + (int64_t)qt * A_BYTES;
            U::mbar_arrive_expect_tx(afull, A_BYTES);
            for (int i = 0; i < A_BYTES / A_COPY; ++i)
                U::bulk_load(sbase + OFF_A + i * A_COPY, asrc + i * A_COPY, A_COPY, afull);
            int64_t g = 0;  // stages issued
            bool ok = true;
            for (int64_t t = t0; t < t1 && ok; ++t) {
                const unsigned char* bsrc = reinterpret_cast<const unsigned char*>(dimg) + t * B_TILE_BYTES;
                for (int k = 0; k < STAGES_PER_TILE; ++k) {
                    const int slot = (int)(g % NSTAGE);
                    const uint32_t u = (uint32_t)(g / NSTAGE);
                    if (!U::mbar_wait(empty(slot), (u & 1) ^ 1, wait_cycles)) {
                        atomicOr(status, ERR_COPY);
                        ok = false;
                        break;
                    }
                    U::mbar_arrive_expect_tx(full(slot), B_STAGE_BYTES);
                    U::bulk_load(sbase + OFF_S + slot * B_STAGE_BYTES, bsrc + k * B_STAGE_BYTES, B_STAGE_BYTES,
                                 full(slot));
                    ++g;
                }
            }
            // every copy this CTA issued lands before it exits: the query tile and the last use of each slot
            U::mbar_wait(afull, 0, wait_cycles);
            for (int slot = 0; slot < NSTAGE; ++slot)
                if (slot < g) U::mbar_wait(full(slot), (uint32_t)((g - 1 - slot) / NSTAGE) & 1, wait_cycles);
        }
    } else if (warp == 1) {
        if (lane == 0 && ntl > 0) {  // MMAs
            bool ok = U::mbar_wait(afull, 0, wait_cycles);
            if (!ok) atomicOr(status, ERR_MMA);
            U::fence_after_sync();
            constexpr uint32_t idesc = U::idesc_f16_f32(QM, DN);
            int64_t g = 0;
            for (int64_t t = 0; t < ntl && ok; ++t) {
                const int b = (int)(t & 1);
                const uint32_t v = (uint32_t)(t >> 1);
                if (!U::mbar_wait(tempty(b), (v & 1) ^ 1, wait_cycles)) {
                    atomicOr(status, ERR_MMA);
                    break;
                }
                U::fence_after_sync();
                const uint32_t dt = tmem + (uint32_t)(b * DN);
                for (int k = 0; k < STAGES_PER_TILE; ++k) {
                    const int slot = (int)(g % NSTAGE);
                    const uint32_t u = (uint32_t)(g / NSTAGE);
                    if (!U::mbar_wait(full(slot), u & 1, wait_cycles)) {
                        atomicOr(status, ERR_MMA);
                        ok = false;
                        break;
                    }
                    U::fence_after_sync();
                    const uint32_t st = sbase + OFF_S + slot * B_STAGE_BYTES;
#pragma unroll
                    for (int kk = 0; kk < SK / 16; ++kk) {
                        const int ks = k * (SK / 16) + kk;
                        const uint64_t ad = U::smem_desc(sbase + OFF_A + ks * 2 * (QM * 16), QM * 16, 128);
                        const uint64_t bd = U::smem_desc(st + kk * 2 * (DN * 16), DN * 16, 128);
                        U::mma_bf16(dt, ad, bd, idesc, ks > 0 ? 1u : 0u);  // kind::f16 issue (FP16 idesc)
                    }
                    U::commit(empty(slot));
                    ++g;
                }
                if (!ok) break;
                U::commit(tfull(b));
            }
            // every MMA issued completes before tensor memory is freed
            U::commit(donebar);
            if (!U::mbar_wait(donebar, 0, wait_cycles)) {
                atomicOr(status, ERR_TMEM);
                *tmem_busy = 1;
            }
        }
    } else {  // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. +31, columns half * 128 .. +127
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;
        const int et = threadIdx.x - 64;  // epilogue thread: its staging slots are et, et + 256, ...
        uint2* stg = reinterpret_cast<uint2*>(sm + OFF_STG) + et;
        const int64_t q = (int64_t)qt * QM + 32 * quarter + lane;
        const bool qv = q < nq;
        const float to_d = -2.f * inv_s2;  // d = to_d * acc
        // dense rows start on 16-byte boundaries when the output and its row stride allow
        const bool vec_ok = DENSE && (reinterpret_cast<uintptr_t>(dense) % 16 == 0) && (ld % 4 == 0);
        // d <= thr  <=>  acc >= -(s^2 / 2) thr; padding queries get +inf (never)
        const float at = DENSE ? 0.f : (qv ? -0.5f * thr[q] / inv_s2 : __int_as_float(0x7f800000));
        int staged = 0;
        int32_t* const cnt_q = counts + (qv ? q : 0);
        int32_t* const idx_q = cand_idx + (qv ? q : 0) * cap;
        float* const d_q = cand_d + (qv ? q : 0) * cap;
        auto flush = [&]() {
            flush_staged(stg, staged, cnt_q, idx_q, d_q, cap);
            staged = 0;
        };
        for (int64_t t = 0; t < ntl; ++t) {
            const int b = (int)(t & 1);
            const uint32_t v = (uint32_t)(t >> 1);
            // warp-uniform outcome: the loads below are .sync.aligned and the flush votes over the warp
            if (!__all_sync(0xffffffffu, U::mbar_wait(tfull(b), v & 1, wait_cycles))) {
                if (lane == 0) atomicOr(status, ERR_EPI);
                break;
            }
            U::fence_after_sync();
            const uint32_t ta = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(b * DN + half * (DN / 2));
            const int64_t jh = (t0 + t) * DN + half * (DN / 2);
#pragma unroll 1
            for (int cb = 0; cb < DN / 2; cb += EPI_COLS) {
                uint32_t r[4][16];
                U::ld16(ta + cb, r[0]);
                U::ld16(ta + cb + 16, r[1]);
                U::ld16(ta + cb + 32, r[2]);
                U::ld16(ta + cb + 48, r[3]);
                U::wait_ld(r[0]);
                U::wait_ld(r[1]);
                U::wait_ld(r[2]);
                U::wait_ld(r[3]);
                const int64_t jb = jh + cb;
                if (DENSE) {
                    if (qv) {
                        float* row = dense + q * ld + jb;
                        if (vec_ok && jb + EPI_COLS <= nd) {  // 16-byte stores: a quarter of the L2 transactions
#pragma unroll
                            for (int i = 0; i < EPI_COLS; i += 4)
                                *reinterpret_cast<float4*>(row + i) =
                                    make_float4(to_d * __uint_as_float(r[i >> 4][i & 15]),
                                                to_d * __uint_as_float(r[(i + 1) >> 4][(i + 1) & 15]),
                                                to_d * __uint_as_float(r[(i + 2) >> 4][(i + 2) & 15]),
                                                to_d * __uint_as_float(r[(i + 3) >> 4][(i + 3) & 15]));
                        } else {
#pragma unroll
                            for (int i = 0; i < EPI_COLS; ++i)
                                if (jb + i < nd) row[i] = to_d * __uint_as_float(r[i >> 4][i & 15]);
                        }
                    }
                } else {
                    // tree maximum (depth 6, not a chain of 64); the level of 8 is kept: group g holds
                    // columns 2g + b + 16a (a = 0..3, b = 0..1), i.e. r[a][2g + b]
                    float mx[EPI_COLS / 2], grp[8];
#pragma unroll
                    for (int i = 0; i < EPI_COLS / 2; ++i)
                        mx[i] = fmaxf(__uint_as_float(r[(2 * i) >> 4][(2 * i) & 15]),
                                      __uint_as_float(r[(2 * i + 1) >> 4][(2 * i + 1) & 15]));
#pragma unroll
                    for (int w2 = EPI_COLS / 4; w2 >= 1; w2 >>= 1) {
#pragma unroll
                        for (int i = 0; i < w2; ++i) mx[i] = fmaxf(mx[i], mx[i + w2]);
                        if (w2 == 8) {
#pragma unroll
                            for (int i = 0; i < 8; ++i) grp[i] = mx[i];
                        }
                    }
                    if (mx[0] >= at) {  // rare: visit the groups that hold a survivor (compact code)
                        uint32_t gm = 0;
#pragma unroll
                        for (int g = 0; g < 8; ++g) gm |= (grp[g] >= at ? 1u : 0u) << g;
                        const int64_t lim = nd - jb;
                        while (gm) {
                            const int g = __ffs(gm) - 1;
                            gm &= gm - 1;
                            float vv[8];
#pragma unroll
                            for (int e = 0; e < 8; ++e) vv[e] = 0.f;
#pragma unroll
                            for (int k = 0; k < 8; ++k)
                                if (g == k) {
#pragma unroll
                                    for (int e = 0; e < 8; ++e) vv[e] = __uint_as_float(r[e >> 1][2 * k + (e & 1)]);
                                }
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                const int col = 2 * g + (e & 1) + 16 * (e >> 1);
                                if (vv[e] >= at && col < lim) {
                                    if (staged == SLOTS) flush();
                                    stg[staged * EPI_THREADS] =
                                        make_uint2((uint32_t)(jb + col), __float_as_uint(to_d * vv[e]));
                                    ++staged;
                                }
                            }
                        }
                    }
                }
            }
            U::fence_before_sync();
            __syncwarp();
            if (lane == 0) U::mbar_arrive(tempty(b));
            if (!DENSE && __any_sync(0xffffffffu, staged == SLOTS) && staged > 0) flush();
        }
        if (!DENSE && staged > 0) flush();
    }
    U::fence_before_sync();
    __syncthreads();
    if (warp == 0 && !*tmem_busy) {
        U::fence_after_sync();
        U::tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace scan
}  // namespace tsm

namespace {

int scan_fail(int code, const char* msg) { return tsm_internal_fail(code, msg); }

int scan_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return TSM_OK;
    char b[256];
    snprintf(b, sizeof(b), "%s: %s", what, cudaGetErrorString(e));
    return tsm_internal_fail(TSM_ECUDA, b);
}

}  // namespace

extern "C" {

int32_t tsm_scan_dim(void) { return tsm::scan::D; }

int64_t tsm_scan_image_bytes(int64_t n_rows, int32_t is_db) {
    if (n_rows < 0) return -1;
    const int64_t R = is_db ? tsm::scan::DN : tsm::scan::QM;
    return (n_rows + R - 1) / R * R * tsm::scan::K * 2;
}

int tsm_scan_prepare(const float* emb, int64_t n, int64_t ld, float scale, int32_t is_db, void* img, float* norms,
                     void* stream) {
    using namespace tsm::scan;
    if (n < 0 || ld < D || !(scale > 0.f)) return scan_fail(TSM_EINVAL, "tsm_scan_prepare: bad size or scale");
    if (n == 0) return TSM_OK;
    if (!emb || !img) return scan_fail(TSM_EINVAL, "tsm_scan_prepare: null pointer");
    if (reinterpret_cast<uintptr_t>(img) % 16) return scan_fail(TSM_EINVAL, "tsm_scan_prepare: image not 16-byte aligned");
    const int64_t R = is_db ? DN : QM;
    const int64_t tiles = (n + R - 1) / R;
    const int64_t threads = tiles * KCH * R;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    cudaStream_t s = (cudaStream_t)stream;
    if (is_db)
        scan_prepare<true><<<grid, 256, 0, s>>>(emb, n, ld, scale, tiles, static_cast<__half*>(img), norms);
    else
        scan_prepare<false><<<grid, 256, 0, s>>>(emb, n, ld, scale, tiles, static_cast<__half*>(img), nullptr);
    return scan_cuda(cudaGetLastError(), "tsm_scan_prepare launch");
}

int tsm_scan_opts(const void* q_img, int64_t nq, const void* db_img, int64_t nd, float scale, const float* thresholds,
                  int32_t cap, int32_t* cand_idx, float* cand_d, int32_t* counts, float* dense, int64_t ld_dense,
                  int32_t* status, int64_t wait_cycles, void* stream) {
    using namespace tsm::scan;
    if (nq < 0 || nd < 0) return scan_fail(TSM_EINVAL, "tsm_scan: negative size");
    if (nq == 0 || nd == 0) return TSM_OK;
    if (!q_img || !db_img || !status) return scan_fail(TSM_EINVAL, "tsm_scan: null pointer");
    if (nd > 0x7fffffffLL) return scan_fail(TSM_EINVAL, "tsm_scan: database index exceeds int32");
    if (wait_cycles < 1) return scan_fail(TSM_EINVAL, "tsm_scan: bad wait limit");
    if (!(scale > 0.f)) return scan_fail(TSM_EINVAL, "tsm_scan: bad scale");
    const bool dense_mode = dense != nullptr;
    if (dense_mode == (thresholds != nullptr))
        return scan_fail(TSM_EINVAL, "tsm_scan: give either thresholds (candidate lists) or a dense output");
    if (dense_mode && ld_dense < nd) return scan_fail(TSM_EINVAL, "tsm_scan: ld_dense < nd");
    if (!dense_mode && (cap < 1 || !cand_idx || !cand_d || !counts))
        return scan_fail(TSM_EINVAL, "tsm_scan: candidate lists need cap >= 1 and their three arrays");
    if ((reinterpret_cast<uintptr_t>(q_img) | reinterpret_cast<uintptr_t>(db_img)) % 16)
        return scan_fail(TSM_EINVAL, "tsm_scan: images not 16-byte aligned");
    const float inv_s2 = 1.f / (scale * scale);
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return scan_cuda(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return scan_cuda(e, "cudaDeviceGetAttribute");
    const int64_t nqt = (nq + QM - 1) / QM;
    if (nqt > 0x7fffffffLL / 2) return scan_fail(TSM_EINVAL, "tsm_scan: too many queries");
    const int64_t ntiles = (nd + DN - 1) / DN;
    int64_t slices = sms / nqt;  // one CTA per SM when the query tiles are few
    if (slices < 1) slices = 1;
    if (slices > ntiles) slices = ntiles;
    const int64_t per = (ntiles + slices - 1) / slices;
    slices = (ntiles + per - 1) / per;
    if (nqt * slices > 0x7fffffffLL) return scan_fail(TSM_EINVAL, "tsm_scan: grid too large");
    const void* fn = dense_mode ? (const void*)&scan_kernel<true> : (const void*)&scan_kernel<false>;
    if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM)) != cudaSuccess)
        return scan_cuda(e, "cudaFuncSetAttribute(scan_kernel)");
    int inqt = (int)nqt;
    const __half* qi = static_cast<const __half*>(q_img);
    const __half* di = static_cast<const __half*>(db_img);
    long long wc = (long long)wait_cycles;
    void* args[] = {&qi, &nq, &di, &nd, (void*)&inv_s2, &thresholds, &cap, &cand_idx, &cand_d, &counts, &dense,
                    &ld_dense, &inqt, (void*)&per, &status, &wc};
    e = cudaLaunchKernel(fn, dim3((unsigned)(nqt * slices)), dim3(THREADS), args, (size_t)SMEM, (cudaStream_t)stream);
    return scan_cuda(e, "tsm_scan launch");
}

int tsm_scan(const void* q_img, int64_t nq, const void* db_img, int64_t nd, float scale, const float* thresholds,
             int32_t cap, int32_t* cand_idx, float* cand_d, int32_t* counts, float* dense, int64_t ld_dense,
             int32_t* status, void* stream) {
    return tsm_scan_opts(q_img, nq, db_img, nd, scale, thresholds, cap, cand_idx, cand_d, counts, dense, ld_dense,
                         status, tsm::scan::WAIT_CYCLES, stream);
}

}  // extern "C"
