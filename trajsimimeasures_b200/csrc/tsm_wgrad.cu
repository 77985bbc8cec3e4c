// Weight gradients of the encoder's GRU on the tensor cores (tcgen05):
//     dW_ih[j][c]  = sum_(b,t) G [b][t][j] A[b][t][c]       384 x 64
//     dW_hh[j][kk] = sum_(b,t) GH[b][t][j] H[b][t][kk]      384 x 128
// over the valid steps t < len[b] only (the padded steps of a batch, about
// half of b x T for lengths U{20..200}, are skipped), G / GH the gate
// gradients of the input and hidden side written by the BPTT kernel, A the
// conv activations and H the hidden state before step t.
//
// Precision.  The four operands are FP32.  Each is split into BF16 parts,
// x = hi + lo with lo = bf16(x - hi) (BF16 keeps FP32's exponent range, which
// gate gradients of 1e-9 need), and the tensor cores take
//     g . x = g_hi . x_hi + g_lo . x_hi + g_hi . x_lo   (+ g_lo . x_lo, dropped)
// with FP32 accumulation: three MMAs per K step, about 2^-16 relative per
// product (the split-product method of Markidis et al., IPDPSW 2018).
//
// Steps (one stream, no host synchronisation):
//   wg_koff      exclusive scan of the clamped lengths -> koff[B + 1] (K = koff[B])
//   wg_krow      krow[koff[b] + t] = b * T + t for t < len[b] (the compact K order)
//   wg_image     FP32 rows -> BF16 hi and lo operand images, K-major core-matrix
//                layout (tsm_umma.cuh), K rounded up to the stage size with zeros
//   wg_kernel    split-K over the CTAs: CTA (m tile of 128 rows of j, K range)
//                streams both products' operands through a four-stage ring
//                (cp.async.bulk, mbarrier transaction counts), one thread issues
//                six MMAs per K step into two accumulators (64 and 128 columns
//                of tensor memory), and all four warps add the result to the
//                gradient with atomics.  Waits are bounded (about 1 s of SM
//                clocks); one that runs out ORs a bit into *status and the CTA
//                adds nothing.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

#include "tsm.h"
#include "tsm_umma.cuh"
#include "tsm_wgrad.h"

int tsm_internal_fail(int code, const char* msg);

namespace tsm {
namespace wgrad {

constexpr int G3 = 384;   // gate rows j (r, z, n)
constexpr int NA = 64;    // conv channels c
constexpr int NH = 128;   // hidden units kk
constexpr int MT = 128;   // rows of j per CTA (MMA M, tensor-memory lanes)
constexpr int SKW = 32;   // K per stage: two MMAs of K = 16 per product
constexpr int NST = 4;    // stages
constexpr int THREADS = 128;
// one stage: [G hi | G lo | GH hi | GH lo | A hi | A lo | H hi | H lo]
constexpr int M_PART = MT * SKW * 2;   // 8,192
constexpr int A_PART = NA * SKW * 2;   // 4,096
constexpr int H_PART = NH * SKW * 2;   // 8,192
constexpr int S_GHI = 0, S_GLO = M_PART, S_GHHI = 2 * M_PART, S_GHLO = 3 * M_PART, S_AHI = 4 * M_PART,
              S_ALO = S_AHI + A_PART, S_HHI = S_ALO + A_PART, S_HLO = S_HHI + H_PART;
constexpr int STAGE = S_HLO + H_PART;  // 57,344
constexpr int OFF_BAR = NST * STAGE;
constexpr int SMEM = OFF_BAR + 128;    // 229,504
constexpr uint32_t TMEM_COLS = 256;    // acc_ih at column 0 (64 wide), acc_hh at 64 (128 wide)
constexpr long long WAIT_CYCLES = 2000000000LL;
static_assert(SMEM <= 227 * 1024, "shared memory");

// status bits (OR-ed into the caller's word)
constexpr int ERR_COPY = 16, ERR_MMA = 32, ERR_DONE = 64, ERR_TMEM = 128;

// koff[b] = sum_{b' < b} min(max(len[b'], 0), T), koff[B] = K.  One CTA of 1024 threads.
__global__ void __launch_bounds__(1024) wg_koff(const int32_t* __restrict__ len, int B, int T,
                                                 int64_t* __restrict__ koff) {
    __shared__ int64_t warp_tot[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b0 = 0; b0 < B; b0 += 1024) {
        const int b = b0 + threadIdx.x;
        const int64_t v = b < B ? (int64_t)min(max(len[b], 0), T) : 0;
        int64_t x = v;  // inclusive warp scan
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int64_t w = warp_tot[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_tot[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const int64_t before = carry + (warp > 0 ? warp_tot[warp - 1] : 0) + x - v;
        if (b < B) koff[b] = before;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_tot[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) koff[B] = carry;
}

// krow[koff[b] + t] = b * T + t for t < len[b].  One thread per (b, t).
__global__ void wg_krow(const int32_t* __restrict__ len, const int64_t* __restrict__ koff, int B, int T,
                        int64_t* __restrict__ krow) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (int64_t)B * T) return;
    const int b = (int)(g / T), t = (int)(g % T);
    if (t < min(max(len[b], 0), T)) krow[koff[b] + t] = g;
}

// Operand images of a source with `cols` values per row: image row r (of
// cols, in tiles of R rows) holds, along K, the values src[row(k)][r], row(k)
// = krow[k] (+ krow[k] / T when hrows: H keeps T + 1 rows per trajectory).
// Chunks of 8 K values are split into BF16 hi and lo parts and stored in the
// core-matrix layout: tile i at byte i * kp * R * 2, chunk c at c * R * 16,
// row r % R at 16 (r % R).  Chunks up to the end of the last stage hold zeros
// past K; later chunks are not written (the kernel reads only up to there).
// One thread per (chunk, row); consecutive threads take consecutive rows
// (coalesced reads and 16-byte stores).
__global__ void wg_image(const float* __restrict__ src, int cols, int R, const int64_t* __restrict__ krow,
                         const int64_t* __restrict__ koff, int B, int T, int hrows, int64_t kp,
                         __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= kp / 8 * cols) return;
    const int r = (int)(g % cols);
    const int64_t c = g / cols;
    const int64_t K = koff[B];
    const int64_t kend = (K + SKW - 1) / SKW * SKW;
    if (8 * c >= kend) return;
    __align__(16) __nv_bfloat16 vh[8], vl[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int64_t k = 8 * c + e;
        float x = 0.f;
        if (k < K) {
            const int64_t kr = krow[k];
            x = src[(kr + (hrows ? kr / T : 0)) * cols + r];
        }
        vh[e] = __float2bfloat16_rn(x);
        vl[e] = __float2bfloat16_rn(x - __bfloat162float(vh[e]));
    }
    const int64_t o = (int64_t)(r / R) * kp * R * 2 + c * R * 16 + (int64_t)(r % R) * 16;
    *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(hi) + o) = *reinterpret_cast<const uint4*>(vh);
    *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(lo) + o) = *reinterpret_cast<const uint4*>(vl);
}

__global__ void __launch_bounds__(THREADS, 1) wg_kernel(
    const __nv_bfloat16* __restrict__ g_hi, const __nv_bfloat16* __restrict__ g_lo,
    const __nv_bfloat16* __restrict__ gh_hi, const __nv_bfloat16* __restrict__ gh_lo,
    const __nv_bfloat16* __restrict__ a_hi, const __nv_bfloat16* __restrict__ a_lo,
    const __nv_bfloat16* __restrict__ h_hi, const __nv_bfloat16* __restrict__ h_lo, const int64_t* __restrict__ koff,
    int B, int64_t kp, float* __restrict__ d_ih, float* __restrict__ d_hh, int* __restrict__ status,
    long long wait_cycles) {
    namespace U = tsm::umma;
    extern __shared__ __align__(1024) unsigned char sm[];
    const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
    const uint32_t bar = sbase + OFF_BAR;
    auto full = [&](int i) { return bar + 8 * i; };
    auto empty = [&](int i) { return bar + 8 * NST + 8 * i; };
    const uint32_t donebar = bar + 16 * NST;
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(sm + OFF_BAR + 16 * NST + 8);
    volatile int* flags = reinterpret_cast<volatile int*>(sm + OFF_BAR + 16 * NST + 12);  // bit 0 failed, 1 busy
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x;  // tile of j
    // this CTA's stages [s0, s1) of the K range, from the device-side K
    const int64_t K = koff[B];
    const int64_t nst_all = (K + SKW - 1) / SKW;
    const int64_t per = (nst_all + gridDim.y - 1) / gridDim.y;
    const int64_t s0 = (int64_t)blockIdx.y * per;
    const int64_t s1 = min(nst_all, s0 + per);
    const int64_t ns = s1 > s0 ? s1 - s0 : 0;
    if (ns == 0) return;  // uniform over the CTA, before any barrier or allocation

    if (threadIdx.x == 0) {
        for (int i = 0; i < NST; ++i) {
            U::mbar_init(full(i), 1);
            U::mbar_init(empty(i), 1);
        }
        U::mbar_init(donebar, 1);
        *flags = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) U::tmem_alloc(sbase + OFF_BAR + 16 * NST + 8, TMEM_COLS);
    U::fence_before_sync();
    __syncthreads();
    U::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {  // copies
        const int64_t mt_off = (int64_t)mt * kp * MT * 2;  // byte offset of this j tile in the G / GH images
        auto src = [&](const __nv_bfloat16* p, int64_t tile_off, int64_t part, int64_t s) {
            return reinterpret_cast<const unsigned char*>(p) + tile_off + s * part;
        };
        int64_t g = 0;
        for (int64_t s = s0; s < s1; ++s, ++g) {
            const int slot = (int)(g % NST);
            const uint32_t u = (uint32_t)(g / NST);
            if (!U::mbar_wait(empty(slot), (u & 1) ^ 1, wait_cycles)) {
                atomicOr(status, ERR_COPY);
                *flags = 1;
                break;
            }
            const uint32_t st = sbase + slot * STAGE;
            U::mbar_arrive_expect_tx(full(slot), STAGE);
            U::bulk_load(st + S_GHI, src(g_hi, mt_off, M_PART, s), M_PART, full(slot));
            U::bulk_load(st + S_GLO, src(g_lo, mt_off, M_PART, s), M_PART, full(slot));
            U::bulk_load(st + S_GHHI, src(gh_hi, mt_off, M_PART, s), M_PART, full(slot));
            U::bulk_load(st + S_GHLO, src(gh_lo, mt_off, M_PART, s), M_PART, full(slot));
            U::bulk_load(st + S_AHI, src(a_hi, 0, A_PART, s), A_PART, full(slot));
            U::bulk_load(st + S_ALO, src(a_lo, 0, A_PART, s), A_PART, full(slot));
            U::bulk_load(st + S_HHI, src(h_hi, 0, H_PART, s), H_PART, full(slot));
            U::bulk_load(st + S_HLO, src(h_lo, 0, H_PART, s), H_PART, full(slot));
        }
        // every copy issued lands before the CTA exits: the last use of each slot
        for (int slot = 0; slot < NST; ++slot)
            if (slot < g) U::mbar_wait(full(slot), (uint32_t)((g - 1 - slot) / NST) & 1, wait_cycles);
    } else if (warp == 1 && lane == 0) {  // MMAs
        constexpr uint32_t id_ih = U::idesc_bf16_f32(MT, NA), id_hh = U::idesc_bf16_f32(MT, NH);
        const uint32_t t_ih = tmem, t_hh = tmem + NA;
        for (int64_t g = 0; g < ns; ++g) {
            const int slot = (int)(g % NST);
            const uint32_t u = (uint32_t)(g / NST);
            if (!U::mbar_wait(full(slot), u & 1, wait_cycles)) {
                atomicOr(status, ERR_MMA);
                *flags = 1;
                break;
            }
            U::fence_after_sync();
            const uint32_t st = sbase + slot * STAGE;
#pragma unroll
            for (int kk = 0; kk < SKW / 16; ++kk) {
                const uint32_t first = (g == 0 && kk == 0) ? 0u : 1u;
                const uint64_t gd_hi = U::smem_desc(st + S_GHI + kk * 2 * (MT * 16), MT * 16, 128);
                const uint64_t gd_lo = U::smem_desc(st + S_GLO + kk * 2 * (MT * 16), MT * 16, 128);
                const uint64_t ghd_hi = U::smem_desc(st + S_GHHI + kk * 2 * (MT * 16), MT * 16, 128);
                const uint64_t ghd_lo = U::smem_desc(st + S_GHLO + kk * 2 * (MT * 16), MT * 16, 128);
                const uint64_t ad_hi = U::smem_desc(st + S_AHI + kk * 2 * (NA * 16), NA * 16, 128);
                const uint64_t ad_lo = U::smem_desc(st + S_ALO + kk * 2 * (NA * 16), NA * 16, 128);
                const uint64_t hd_hi = U::smem_desc(st + S_HHI + kk * 2 * (NH * 16), NH * 16, 128);
                const uint64_t hd_lo = U::smem_desc(st + S_HLO + kk * 2 * (NH * 16), NH * 16, 128);
                U::mma_bf16(t_ih, gd_hi, ad_hi, id_ih, first);
                U::mma_bf16(t_ih, gd_lo, ad_hi, id_ih, 1u);
                U::mma_bf16(t_ih, gd_hi, ad_lo, id_ih, 1u);
                U::mma_bf16(t_hh, ghd_hi, hd_hi, id_hh, first);
                U::mma_bf16(t_hh, ghd_lo, hd_hi, id_hh, 1u);
                U::mma_bf16(t_hh, ghd_hi, hd_lo, id_hh, 1u);
            }
            U::commit(empty(slot));
        }
        U::commit(donebar);  // completes when every MMA issued above has
    }
    // epilogue: all four warps; warp w reads tensor-memory lanes 32 w .. 32 w + 31 (rows j of the tile)
    __syncwarp();
    const bool done = __all_sync(0xffffffffu, U::mbar_wait(donebar, 0, wait_cycles));
    if (!done) {
        if (lane == 0) atomicOr(status, ERR_DONE);
        if (lane == 0) *flags = 3;  // MMAs may still write tensor memory: keep it allocated
    }
    U::fence_after_sync();
    __syncthreads();
    const int fl = *flags;
    if (fl == 0) {
        const int64_t j = (int64_t)mt * MT + 32 * warp + lane;
        const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16);
        for (int c0 = 0; c0 < NA + NH; c0 += 16) {
            uint32_t r[16];
            U::ld16(ta + c0, r);
            U::wait_ld(r);
            if (c0 < NA) {
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(d_ih + j * NA + c0 + i, __uint_as_float(r[i]));
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(d_hh + j * NH + (c0 - NA) + i, __uint_as_float(r[i]));
            }
        }
    }
    U::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        if (fl & 2) {
            if (lane == 0) atomicOr(status, ERR_TMEM);
        } else {
            U::fence_after_sync();
            U::tmem_dealloc(tmem, TMEM_COLS);
        }
    }
}

}  // namespace wgrad
}  // namespace tsm

namespace {

int64_t al256(int64_t n) { return (n + 255) & ~int64_t(255); }

int wg_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return TSM_OK;
    char b[256];
    snprintf(b, sizeof(b), "%s: %s", what, cudaGetErrorString(e));
    return tsm_internal_fail(TSM_ECUDA, b);
}

struct WgScratch {
    int64_t* koff;
    int64_t* krow;
    __nv_bfloat16 *g_hi, *g_lo, *gh_hi, *gh_lo, *a_hi, *a_lo, *h_hi, *h_lo;
};

// Lays the scratch out (base != NULL) and returns its size in bytes.
int64_t wg_layout(int B, int T, unsigned char* base, WgScratch* w) {
    using namespace tsm::wgrad;
    const int64_t kp = ((int64_t)B * T + SKW - 1) / SKW * SKW;
    int64_t o = 0;
    auto take = [&](int64_t bytes) {
        unsigned char* p = base ? base + o : nullptr;
        o += al256(bytes);
        return p;
    };
    WgScratch tmp;
    WgScratch* x = w ? w : &tmp;
    x->koff = reinterpret_cast<int64_t*>(take((int64_t)(B + 1) * 8));
    x->krow = reinterpret_cast<int64_t*>(take(kp * 8));
    x->g_hi = reinterpret_cast<__nv_bfloat16*>(take(kp * G3 * 2));
    x->g_lo = reinterpret_cast<__nv_bfloat16*>(take(kp * G3 * 2));
    x->gh_hi = reinterpret_cast<__nv_bfloat16*>(take(kp * G3 * 2));
    x->gh_lo = reinterpret_cast<__nv_bfloat16*>(take(kp * G3 * 2));
    x->a_hi = reinterpret_cast<__nv_bfloat16*>(take(kp * NA * 2));
    x->a_lo = reinterpret_cast<__nv_bfloat16*>(take(kp * NA * 2));
    x->h_hi = reinterpret_cast<__nv_bfloat16*>(take(kp * NH * 2));
    x->h_lo = reinterpret_cast<__nv_bfloat16*>(take(kp * NH * 2));
    return o;
}

}  // namespace

int64_t tsm_wgrad_scratch_bytes(int B, int T) { return wg_layout(B, T, nullptr, nullptr); }

int tsm_wgrad_tc(const float* G, const float* GH, const float* A, const float* H, const int32_t* len, int B, int T,
                 void* scratch, int* status, float* d_ih, float* d_hh, cudaStream_t s) {
    using namespace tsm::wgrad;
    if (B < 1 || T < 1 || !scratch || !status) return tsm_internal_fail(TSM_EINVAL, "wgrad: bad arguments");
    if (reinterpret_cast<uintptr_t>(scratch) % 256) return tsm_internal_fail(TSM_EINVAL, "wgrad: scratch alignment");
    WgScratch w;
    wg_layout(B, T, static_cast<unsigned char*>(scratch), &w);
    const int64_t bt = (int64_t)B * T;
    const int64_t kp = (bt + SKW - 1) / SKW * SKW;
    wg_koff<<<1, 1024, 0, s>>>(len, B, T, w.koff);
    wg_krow<<<(unsigned)((bt + 255) / 256), 256, 0, s>>>(len, w.koff, B, T, w.krow);
    auto image = [&](const float* src, int cols, int R, int hrows, __nv_bfloat16* hi, __nv_bfloat16* lo) {
        const int64_t n = kp / 8 * cols;
        wg_image<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, cols, R, w.krow, w.koff, B, T, hrows, kp, hi, lo);
    };
    image(G, G3, MT, 0, w.g_hi, w.g_lo);
    image(GH, G3, MT, 0, w.gh_hi, w.gh_lo);
    image(A, NA, NA, 0, w.a_hi, w.a_lo);
    image(H, NH, NH, 1, w.h_hi, w.h_lo);
    int rc = wg_check(cudaFuncSetAttribute(wg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM),
                      "cudaFuncSetAttribute(wg_kernel)");
    if (rc) return rc;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // K split: one wave of CTAs over the three j tiles, at most the stages there can be
    int64_t ksplit = sms / (G3 / MT);
    const int64_t nst_max = kp / SKW;
    if (ksplit > nst_max) ksplit = nst_max;
    if (ksplit < 1) ksplit = 1;
    wg_kernel<<<dim3(G3 / MT, (unsigned)ksplit), THREADS, SMEM, s>>>(w.g_hi, w.g_lo, w.gh_hi, w.gh_lo, w.a_hi, w.a_lo,
                                                                       w.h_hi, w.h_lo, w.koff, B, kp, d_ih, d_hh,
                                                                       status, WAIT_CYCLES);
    return wg_check(cudaGetLastError(), "wgrad launch");
}
