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
// Precision", IPDPSW 2018), about 2^-21 relative per product.  The values are
// scaled by a power of two s (exact) so that they use FP16's range; the
// squared norms |e_j|^2 are FP32 and enter in the epilogue.
//
// Kernel.  One CTA per (query tile of 128, slice of database tiles of 256
// rows).  Both operands stream through a six-stage ring in shared memory,
// each stage a K slice of 48 of the query tile (12 KB, re-read from L2 for
// every database tile) and of the database tile (24 KB): cp.async.bulk of
// pre-formatted operand images, completion on mbarrier transaction counts.
// (Keeping the query tile resident instead left room for four stages only,
// and the copies' latency held the tensor pipe to a third of its time.)  Warp 0 issues the copies, one thread of warp 1 issues
// the MMAs (M = 128 queries, N = 256 rows, K = 16 per instruction, 30 per
// database tile) into one of two FP32 accumulators of 256 tensor-memory
// columns, and warps 2-9 (two per 32-lane quarter of tensor memory, each
// reading half of the columns, 64 per tensor-memory load batch) read the
// other accumulator with tcgen05.ld, form d and apply the threshold (one
// compare per 64 values against their tree minimum) while the next tile's
// MMAs run.  Every wait is bounded (about 1 s of SM clocks); one
// that runs out sets a bit of *status and ends that role's loop, the CTA
// waits (bounded) for its own copies and MMAs in flight, and frees tensor
// memory only when no MMA can still write it.
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
constexpr int K = 3 * D;                   // split-product K
constexpr int KCH = K / 8;                 // 16-byte K chunks of a row
constexpr int QM = 128;                    // queries per tile (MMA M, tensor-memory lanes)
constexpr int DN = 256;                    // database rows per tile (MMA N)
constexpr int SK = 48;                     // K per pipeline stage: three MMAs of K = 16
constexpr int NSTAGE = 6;
constexpr int STAGES_PER_TILE = K / SK;    // 10
constexpr int A_BYTES = QM * K * 2;        // 122,880: one query tile's image
constexpr int B_TILE_BYTES = DN * K * 2;   // 245,760: one database tile's image
constexpr int A_STAGE_BYTES = QM * SK * 2; // 12,288
constexpr int B_STAGE_BYTES = DN * SK * 2; // 24,576
constexpr int STAGE_BYTES = A_STAGE_BYTES + B_STAGE_BYTES;
constexpr int EPI_WARPS = 8;               // two per 32-lane quarter of tensor memory, each half the columns
constexpr int THREADS = 64 + 32 * EPI_WARPS;  // warp 0 copies, warp 1 MMAs, warps 2-9 epilogue
constexpr int EPI_COLS = 64;               // accumulator columns per tensor-memory load batch
constexpr uint32_t TMEM_COLS = 2 * DN;     // two accumulators
constexpr int NNORM = 4;                   // squared-norm ring: one database tile's norms per slot
constexpr int OFF_S = 0;                   // NSTAGE stages of [A part | B part]
constexpr int OFF_N = OFF_S + NSTAGE * STAGE_BYTES;
constexpr int OFF_BAR = OFF_N + NNORM * DN * 4;
constexpr int SMEM = OFF_BAR + 256;        // 225,536 bytes
constexpr long long WAIT_CYCLES = 2000000000LL;
static_assert(K % SK == 0 && SK % 16 == 0 && D % 8 == 0, "stage and chunk sizes");
static_assert(SMEM <= 227 * 1024, "shared memory");

// status bits
constexpr int ERR_COPY = 1;   // a copy (or its stage) did not become available in time
constexpr int ERR_MMA = 2;    // the MMA issuer gave up waiting for an accumulator or a stage
constexpr int ERR_TMEM = 4;   // MMAs still pending at exit: tensor memory left allocated
constexpr int ERR_EPI = 8;    // the epilogue gave up waiting for an accumulator

// Operand image of rows [0, n) of emb (row stride ld floats, D values each,
// times s), padded with zero rows to whole tiles of R rows.  DB: rows
// [hi | hi | lo] and FP32 squared norms |emb_j|^2 of the unscaled rows, +inf
// for the padding rows of the last tile (their d is then +inf, below no
// threshold); queries: [hi | lo | hi].  One thread per (row, 16-byte chunk),
// consecutive threads on consecutive rows of one chunk (coalesced 16-byte
// stores).
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
    const int part = (8 * c) / D;  // which third of K
    const int k0 = 8 * c - part * D;
    __align__(16) __half v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const float x = row < n ? s * emb[row * ld + k0 + e] : 0.f;
        const __half h = __float2half_rn(x);
        const __half l = __float2half_rn(x - __half2float(h));
        v[e] = DB ? (part < 2 ? h : l) : (part == 1 ? l : h);
    }
    unsigned char* dst = reinterpret_cast<unsigned char*>(img) + t * ((int64_t)R * K * 2) +
                         (int64_t)c * (R * 16) + (r >> 3) * 128 + (r & 7) * 16;
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(v);
    if (DB && norms && c == 0) {
        float ss = __int_as_float(0x7f800000);  // +inf
        if (row < n) {
            ss = 0.f;
            for (int k = 0; k < D; ++k) {
                const float x = emb[row * ld + k];
                ss = fmaf(x, x, ss);
            }
        }
        norms[row] = ss;
    }
}

template <bool DENSE>
__global__ void __launch_bounds__(THREADS, 1) scan_kernel(
    const __half* __restrict__ qimg, int64_t nq, const __half* __restrict__ dimg, const float* __restrict__ norms,
    int64_t nd, float inv_s2, const float* __restrict__ thr, int cap, int32_t* __restrict__ cand_idx,
    float* __restrict__ cand_d, int32_t* __restrict__ counts, float* __restrict__ dense, int64_t ld, int nqt,
    int64_t tiles_per_slice, int* __restrict__ status, long long wait_cycles) {
    namespace U = tsm::umma;
    extern __shared__ __align__(1024) unsigned char sm[];
    const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
    const uint32_t bar = sbase + OFF_BAR;
    // mbarriers: full[4] (copies landed), empty[4] (stage read by the MMAs),
    // tfull[2] (accumulator ready), tempty[2] (accumulator read), all MMAs
    // done, nfull[4] (a tile's norms landed), nempty[4] (norms read)
    auto full = [&](int i) { return bar + 8 * i; };         // i < NSTAGE (6): bytes 0..47
    auto empty = [&](int i) { return bar + 48 + 8 * i; };   // 48..95
    auto tfull = [&](int b) { return bar + 184 + 8 * b; };
    auto tempty = [&](int b) { return bar + 200 + 8 * b; };
    const uint32_t donebar = bar + 104;
    auto nfull = [&](int i) { return bar + 112 + 8 * i; };
    auto nempty = [&](int i) { return bar + 144 + 8 * i; };
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(sm + OFF_BAR + 176);
    volatile int* tmem_busy = reinterpret_cast<volatile int*>(sm + OFF_BAR + 180);
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
        for (int i = 0; i < NNORM; ++i) {
            U::mbar_init(nfull(i), 1);
            U::mbar_init(nempty(i), EPI_WARPS);
        }
        *tmem_busy = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) U::tmem_alloc(sbase + OFF_BAR + 176, TMEM_COLS);
    U::fence_before_sync();
    __syncthreads();
    U::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0 && ntl > 0) {  // copies
            const unsigned char* asrc = reinterpret_cast<const unsigned char*>(qimg) + (int64_t)qt * A_BYTES;
            int64_t g = 0;  // stages issued
            int64_t nt = 0;  // tiles whose norms were issued
            bool ok = true;
            for (int64_t t = t0; t < t1 && ok; ++t) {
                const unsigned char* bsrc = reinterpret_cast<const unsigned char*>(dimg) + t * B_TILE_BYTES;
                {  // the tile's squared norms into the norm ring
                    const int slot = (int)(nt % NNORM);
                    const uint32_t u = (uint32_t)(nt / NNORM);
                    if (!U::mbar_wait(nempty(slot), (u & 1) ^ 1, wait_cycles)) {
                        atomicOr(status, ERR_COPY);
                        break;
                    }
                    U::mbar_arrive_expect_tx(nfull(slot), DN * 4);
                    U::bulk_load(sbase + OFF_N + slot * (DN * 4), norms + t * DN, DN * 4, nfull(slot));
                    ++nt;
                }
                for (int k = 0; k < STAGES_PER_TILE; ++k) {
                    const int slot = (int)(g % NSTAGE);
                    const uint32_t u = (uint32_t)(g / NSTAGE);
                    if (!U::mbar_wait(empty(slot), (u & 1) ^ 1, wait_cycles)) {
                        atomicOr(status, ERR_COPY);
                        ok = false;
                        break;
                    }
                    const uint32_t st = sbase + OFF_S + slot * STAGE_BYTES;
                    U::mbar_arrive_expect_tx(full(slot), STAGE_BYTES);
                    U::bulk_load(st, asrc + k * A_STAGE_BYTES, A_STAGE_BYTES, full(slot));
                    U::bulk_load(st + A_STAGE_BYTES, bsrc + k * B_STAGE_BYTES, B_STAGE_BYTES, full(slot));
                    ++g;
                }
            }
            // every copy this CTA issued lands before it exits: the last use of each slot, and A
            for (int slot = 0; slot < NSTAGE; ++slot)
                if (slot < g) U::mbar_wait(full(slot), (uint32_t)((g - 1 - slot) / NSTAGE) & 1, wait_cycles);
            for (int slot = 0; slot < NNORM; ++slot)
                if (slot < nt) U::mbar_wait(nfull(slot), (uint32_t)((nt - 1 - slot) / NNORM) & 1, wait_cycles);
        }
    } else if (warp == 1) {
        if (lane == 0 && ntl > 0) {  // MMAs
            bool ok = true;
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
                    const uint32_t st = sbase + OFF_S + slot * STAGE_BYTES;
#pragma unroll
                    for (int kk = 0; kk < SK / 16; ++kk) {
                        const int ks = k * (SK / 16) + kk;
                        const uint64_t ad = U::smem_desc(st + kk * 2 * (QM * 16), QM * 16, 128);
                        const uint64_t bd = U::smem_desc(st + A_STAGE_BYTES + kk * 2 * (DN * 16), DN * 16, 128);
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
        const int64_t q = (int64_t)qt * QM + 32 * quarter + lane;
        const bool qv = q < nq;
        // padding queries get -inf: no d (>= finite or +inf) is at or below it
        const float th = DENSE ? 0.f : (qv ? thr[q] : __int_as_float(0xff800000));
        const float m2 = -2.f * inv_s2;
        for (int64_t t = 0; t < ntl; ++t) {
            const int b = (int)(t & 1);
            const uint32_t v = (uint32_t)(t >> 1);
            const int ns = (int)(t % NNORM);
            if (!U::mbar_wait(tfull(b), v & 1, wait_cycles) ||
                !U::mbar_wait(nfull(ns), (uint32_t)(t / NNORM) & 1, wait_cycles)) {
                atomicOr(status, ERR_EPI);
                break;
            }
            U::fence_after_sync();
            const uint32_t ta = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(b * DN + half * (DN / 2));
            const float4* nr = reinterpret_cast<const float4*>(sm + OFF_N + ns * (DN * 4)) + half * (DN / 8);
            const int64_t jh = (t0 + t) * DN + half * (DN / 2);
#pragma unroll 1
            for (int cb = 0; cb < DN / 2; cb += EPI_COLS) {
                uint32_t r0[16], r1[16], r2[16], r3[16];
                U::ld16(ta + cb, r0);
                U::ld16(ta + cb + 16, r1);
                U::ld16(ta + cb + 32, r2);
                U::ld16(ta + cb + 48, r3);
                U::wait_ld(r0);
                U::wait_ld(r1);
                U::wait_ld(r2);
                U::wait_ld(r3);
                float d[EPI_COLS];
#pragma unroll
                for (int i4 = 0; i4 < EPI_COLS / 4; ++i4) {
                    const float4 nv = nr[cb / 4 + i4];  // the same address in every lane: a broadcast
                    const uint32_t* rr = i4 < 4 ? r0 : (i4 < 8 ? r1 : (i4 < 12 ? r2 : r3));
                    const int o = (4 * i4) & 15;
                    d[4 * i4 + 0] = fmaf(m2, __uint_as_float(rr[o + 0]), nv.x);
                    d[4 * i4 + 1] = fmaf(m2, __uint_as_float(rr[o + 1]), nv.y);
                    d[4 * i4 + 2] = fmaf(m2, __uint_as_float(rr[o + 2]), nv.z);
                    d[4 * i4 + 3] = fmaf(m2, __uint_as_float(rr[o + 3]), nv.w);
                }
                const int64_t jb = jh + cb;
                if (DENSE) {
                    if (qv) {
#pragma unroll
                        for (int i = 0; i < EPI_COLS; ++i)
                            if (jb + i < nd) dense[q * ld + jb + i] = d[i];
                    }
                } else {
                    float mn[EPI_COLS / 2];  // tree minimum: depth 6, not a chain of 64
#pragma unroll
                    for (int i = 0; i < EPI_COLS / 2; ++i) mn[i] = fminf(d[2 * i], d[2 * i + 1]);
#pragma unroll
                    for (int w2 = EPI_COLS / 4; w2 >= 1; w2 >>= 1)
#pragma unroll
                        for (int i = 0; i < w2; ++i) mn[i] = fminf(mn[i], mn[i + w2]);
                    if (mn[0] <= th) {  // rare: at least one of the 64 survives (unrolled: d stays in registers)
#pragma unroll
                        for (int i = 0; i < EPI_COLS; ++i) {
                            const int64_t j = jb + i;
                            if (d[i] <= th && j < nd) {
                                const int pos = atomicAdd(counts + q, 1);
                                if (pos < cap) {
                                    cand_idx[q * cap + pos] = (int32_t)j;
                                    cand_d[q * cap + pos] = d[i];
                                }
                            }
                        }
                    }
                }
            }
            U::fence_before_sync();
            __syncwarp();
            if (lane == 0) {
                U::mbar_arrive(tempty(b));
                U::mbar_arrive(nempty(ns));
            }
        }
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

int64_t tsm_scan_norms_count(int64_t n_rows) {
    if (n_rows < 0) return -1;
    return (n_rows + tsm::scan::DN - 1) / tsm::scan::DN * tsm::scan::DN;
}

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
    if (!emb || !img || (is_db && !norms)) return scan_fail(TSM_EINVAL, "tsm_scan_prepare: null pointer");
    if (reinterpret_cast<uintptr_t>(img) % 16) return scan_fail(TSM_EINVAL, "tsm_scan_prepare: image not 16-byte aligned");
    const int64_t R = is_db ? DN : QM;
    const int64_t tiles = (n + R - 1) / R;
    const int64_t threads = tiles * KCH * R;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    cudaStream_t s = (cudaStream_t)stream;
    if (is_db && reinterpret_cast<uintptr_t>(norms) % 16)
        return scan_fail(TSM_EINVAL, "tsm_scan_prepare: norms not 16-byte aligned");
    if (is_db)
        scan_prepare<true><<<grid, 256, 0, s>>>(emb, n, ld, scale, tiles, static_cast<__half*>(img), norms);
    else
        scan_prepare<false><<<grid, 256, 0, s>>>(emb, n, ld, scale, tiles, static_cast<__half*>(img), nullptr);
    return scan_cuda(cudaGetLastError(), "tsm_scan_prepare launch");
}

int tsm_scan_opts(const void* q_img, int64_t nq, const void* db_img, const float* db_norms, int64_t nd, float scale,
                  const float* thresholds, int32_t cap, int32_t* cand_idx, float* cand_d, int32_t* counts,
                  float* dense, int64_t ld_dense, int32_t* status, int64_t wait_cycles, void* stream) {
    using namespace tsm::scan;
    if (nq < 0 || nd < 0) return scan_fail(TSM_EINVAL, "tsm_scan: negative size");
    if (nq == 0 || nd == 0) return TSM_OK;
    if (!q_img || !db_img || !db_norms || !status) return scan_fail(TSM_EINVAL, "tsm_scan: null pointer");
    if (nd > 0x7fffffffLL) return scan_fail(TSM_EINVAL, "tsm_scan: database index exceeds int32");
    if (wait_cycles < 1) return scan_fail(TSM_EINVAL, "tsm_scan: bad wait limit");
    const bool dense_mode = dense != nullptr;
    if (dense_mode == (thresholds != nullptr))
        return scan_fail(TSM_EINVAL, "tsm_scan: give either thresholds (candidate lists) or a dense output");
    if (dense_mode && ld_dense < nd) return scan_fail(TSM_EINVAL, "tsm_scan: ld_dense < nd");
    if (!dense_mode && (cap < 1 || !cand_idx || !cand_d || !counts))
        return scan_fail(TSM_EINVAL, "tsm_scan: candidate lists need cap >= 1 and their three arrays");
    if ((reinterpret_cast<uintptr_t>(q_img) | reinterpret_cast<uintptr_t>(db_img) |
         reinterpret_cast<uintptr_t>(db_norms)) % 16)
        return scan_fail(TSM_EINVAL, "tsm_scan: images or norms not 16-byte aligned");
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
    void* args[] = {&qi, &nq, &di, &db_norms, &nd, (void*)&inv_s2, &thresholds, &cap, &cand_idx, &cand_d, &counts,
                    &dense, &ld_dense, &inqt, (void*)&per, &status, &wc};
    e = cudaLaunchKernel(fn, dim3((unsigned)(nqt * slices)), dim3(THREADS), args, (size_t)SMEM, (cudaStream_t)stream);
    return scan_cuda(e, "tsm_scan launch");
}

int tsm_scan(const void* q_img, int64_t nq, const void* db_img, const float* db_norms, int64_t nd, float scale,
             const float* thresholds, int32_t cap, int32_t* cand_idx, float* cand_d, int32_t* counts, float* dense,
             int64_t ld_dense, int32_t* status, void* stream) {
    return tsm_scan_opts(q_img, nq, db_img, db_norms, nd, scale, thresholds, cap, cand_idx, cand_d, counts, dense,
                         ld_dense, status, tsm::scan::WAIT_CYCLES, stream);
}

}  // extern "C"
