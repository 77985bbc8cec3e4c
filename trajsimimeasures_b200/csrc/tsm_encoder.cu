// Learned candidate filter: a trajectory encoder trained on DTW distances.
//
// Network (per trajectory of n points, coordinates normalised on the host):
//   conv   a_t = relu(b1 + sum_{k<5, i<2} W1[c][i][k] x_{t+k-2,i})   64 channels, zero padding
//   GRU    r = s(Wir a + bir + Whr h + bhr),  z = s(Wiz a + biz + Whz h + bhz),
//          n = tanh(Win a + bin + r * (Whn h + bhn)),  h' = (1-z) n + z h      hidden 128
//   head   e = [Wo h_n + bo | sc_k * r_k]                                       160-d embedding
//          r_k = point round(k (n - 1) / 15) of the trajectory, k < 16, normalised (32 values):
//          a geometric skip around the recurrent branch, with a learned weight sc_k = exp(u_k)
//          per point (u_k stored: Adam then moves the weights by relative steps)
//   pair   d(a, b) = ||e_a - e_b||_2, trained with MSE against DTW / max DTW.
// Conv and GRU weights are used as BF16 values (rounded from FP32 master
// weights before each forward), all accumulation is FP32; the head and the
// skip are FP32 (a BF16 path cannot hold positions to the ~1e-4 of the box
// that separates DTW neighbours among a million trajectories; the skip
// carries them exactly).
// The reference trains its learned measures the same way (MSE on
// distance / max distance, nn/MLP_trajsimi_train.py:74-84,197-200).
//
// Training recurrences (hand-written, SIMT FP32 FMA): 16 trajectories per CTA,
// the BF16 weights resident in shared memory for all time steps, time stepped
// inside the kernel, FP32 activations, and the caches BPTT needs.  The weight
// gradients of the GRU (reductions over every valid step of the batch) run on
// the tensor cores (tsm_wgrad.cu, BF16 hi/lo split products).  Inference
// (embedding a database or a query batch) runs on the tensor cores instead:
// enc_gru_embed_tc takes 128 trajectories per CTA, so each step's products
// (128 x 384 x 192) are tcgen05 MMA tiles with the accumulators in tensor
// memory.
//
//   enc_round_bf16    FP32 master -> BF16 weights
//   enc_conv_fwd      conv + relu -> A [B][T][64]
//   enc_gru_fwd       persistent GRU over T steps -> H [B][T+1][128] and gate caches
//   enc_head_fwd      e = [Wo h_last + bo | sc_k r_k]
//   enc_pair_loss     distances, MSE loss, dL/de (atomic)
//   enc_head_bwd      dWo, dbo, dh_last; enc_skip_bwd: d sc_k
//   enc_gru_bwd       BPTT: gate gradients G [B][T][384] (input side), dA [B][T][64], bias gradients
//   tsm_wgrad_tc      weight gradients dW_ih, dW_hh on the tensor cores (tsm_wgrad.cu)
//   enc_conv_bwd      dW1, db1
//   enc_adam          Adam step on the FP32 master weights
//   enc_conv_fwd_tc   conv + relu -> BF16 a_t operand images for the tensor-core GRU
//   enc_gru_embed_tc  inference GRU on the tensor cores -> last hidden state
#include <cuda_bf16.h>
#include <cstdio>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tsm.h"
#include "tsm_umma.cuh"
#include "tsm_wgrad.h"

int tsm_internal_fail(int code, const char* msg);

namespace enc {

constexpr int C1 = 64;    // conv channels
constexpr int KW = 5;     // conv width
constexpr int HD = 128;   // hidden
constexpr int G3 = 384;   // 3 gates
constexpr int EO = 128;   // learned head outputs
constexpr int NS = 16;    // resampled points of the geometric skip
constexpr int SK = 2 * NS;  // skip features (x, y of each resampled point)
constexpr int ED = EO + SK; // embedding: [head outputs | skip weights * resampled points]
static_assert(SK == 32, "enc_skip_bwd maps one skip value per lane");
constexpr int S = 16;     // trajectories per GRU CTA
constexpr int GRU_THREADS = 384;
constexpr int SP = S + 4;  // row stride of the backward's trajectory-minor gate gradients (16-byte groups of 4)
constexpr int SPA = S + 4; // row stride of the forward's trajectory-minor h and a_t

// parameter offsets in the flat FP32 master buffer
constexpr int OFF_W1 = 0;                    // [64][2][5]
constexpr int OFF_B1 = OFF_W1 + C1 * 2 * KW; // [64]
constexpr int OFF_WIH = OFF_B1 + C1;         // [384][64]
constexpr int OFF_BIH = OFF_WIH + G3 * C1;   // [384]
constexpr int OFF_WHH = OFF_BIH + G3;        // [384][128]
constexpr int OFF_BHH = OFF_WHH + G3 * HD;   // [384]
constexpr int OFF_WO = OFF_BHH + G3;         // [128][128]
constexpr int OFF_BO = OFF_WO + EO * HD;     // [128]
constexpr int OFF_SC = OFF_BO + EO;          // [16] u_k: log-weights of the resampled points of the skip
constexpr int N_PARAMS = OFF_SC + NS;

__device__ __forceinline__ float sigm(float x) { return 1.f / (1.f + expf(-x)); }

// FP32 master -> BF16 copies of the conv and GRU weights (head stays FP32).
__global__ void enc_round_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < OFF_WO) q[i] = __float2bfloat16_rn(p[i]);
}

// Normalised input coordinate i of point t of trajectory b (0 outside).
__device__ __forceinline__ float xin(const float2* pts, int64_t off, int len, int t, int i, float4 nrm) {
    if (t < 0 || t >= len) return 0.f;
    const float2 v = pts[off + t];
    return i == 0 ? (v.x - nrm.x) * nrm.z : (v.y - nrm.y) * nrm.w;
}

// A[b][t][c] = relu(conv), 0 for t >= len.  One thread per (b, t, c).
__global__ void enc_conv_fwd(const float2* __restrict__ pts, const int64_t* __restrict__ off,
                             const int32_t* __restrict__ len, int B, int T, float4 nrm,
                             const __nv_bfloat16* __restrict__ wq, const float* __restrict__ p,
                             float* __restrict__ A) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (int64_t)B * T * C1) return;
    const int c = gid % C1;
    const int t = (gid / C1) % T;
    const int b = gid / ((int64_t)C1 * T);
    const int n = len[b];
    float a = 0.f;
    if (t < n) {
        float acc = p[OFF_B1 + c];
#pragma unroll
        for (int k = 0; k < KW; ++k)
#pragma unroll
            for (int i = 0; i < 2; ++i)
                acc = fmaf(__bfloat162float(wq[OFF_W1 + (c * 2 + i) * KW + k]), xin(pts, off[b], n, t + k - 2, i, nrm), acc);
        a = fmaxf(acc, 0.f);
    }
    A[gid] = a;
}

// Persistent GRU forward.  CTA = S trajectories, 384 threads (thread j: gate
// rows j % 192 and j % 192 + 192 of trajectories 8 (j / 192) .. +7).  Shared
// memory: Wih and Whh BF16, transposed into (k, k+1) pairs per gate row
// ([k/2][384][2]: a thread reads one 4-byte pair per row, consecutive threads
// consecutive words), h [S][128], a [S][64], gate pre-activations gi, gh
// [S][384].
// Caches for the backward pass (only steps t < len are written):
//   H [B][T+1][128] (H[b][0] = 0), R, Z, N, GHN [B][T][128] with
//   GHN = Whn h + bhn.  hl [B][128] = h after the last valid step.
__global__ void __launch_bounds__(GRU_THREADS, 1) enc_gru_fwd(
    const float* __restrict__ A, const int32_t* __restrict__ len, int B, int T, const __nv_bfloat16* __restrict__ wq,
    const float* __restrict__ p, float* __restrict__ H, float* __restrict__ R, float* __restrict__ Z,
    float* __restrict__ N, float* __restrict__ GHN, float* __restrict__ hl) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __nv_bfloat16* wih = reinterpret_cast<__nv_bfloat16*>(smraw);        // [32][384][2]: (k, k+1) pairs per gate row
    __nv_bfloat16* whh = wih + C1 * G3;                                   // [64][384][2]
    float* hs = reinterpret_cast<float*>(whh + HD * G3);                  // [128][SPA]: h, trajectory-minor
    float* as = hs + HD * SPA;                                            // [64][SPA]: a_t, trajectory-minor
    float* gi = as + C1 * SPA;                                            // [S][384]
    float* gh = gi + S * G3;                                              // [S][384]
    __shared__ int lens[S];
    const int j = threadIdx.x;
    const int b0 = blockIdx.x * S;
    for (int e = j; e < G3 * C1; e += GRU_THREADS) {  // transpose into k-pair-major [k/2][row][k%2]
        const int row = e / C1, col = e % C1;
        wih[((col >> 1) * G3 + row) * 2 + (col & 1)] = wq[OFF_WIH + e];
    }
    for (int e = j; e < G3 * HD; e += GRU_THREADS) {
        const int row = e / HD, col = e % HD;
        whh[((col >> 1) * G3 + row) * 2 + (col & 1)] = wq[OFF_WHH + e];
    }
    for (int e = j; e < HD * SPA; e += GRU_THREADS) hs[e] = 0.f;
    if (j < S) lens[j] = (b0 + j < B) ? len[b0 + j] : 0;
    // the products: thread j takes gate rows jr and jr + 192 for trajectories
    // 8 sh .. 8 sh + 7 as four (s, s + 1) pairs, FP32x2 FMAs of one weight
    // against two trajectories' activations: a 4-byte load of two weights
    // feeds 16 FMAs, a broadcast 16-byte load of four activations 8
    constexpr int SH = S / 2;
    const int jr = j % (G3 / 2), sh = j / (G3 / 2);
    const float bih0 = p[OFF_BIH + jr], bhh0 = p[OFF_BHH + jr];
    const float bih1 = p[OFF_BIH + jr + G3 / 2], bhh1 = p[OFF_BHH + jr + G3 / 2];
    const uint32_t* wih2 = reinterpret_cast<const uint32_t*>(wih);
    const uint32_t* whh2 = reinterpret_cast<const uint32_t*>(whh);
    __syncthreads();
    int tmax = 0;
    for (int s = 0; s < S; ++s) tmax = max(tmax, lens[s]);
    // H[b][0] = 0, and rows past the trajectory's length are zero too (the
    // weight-gradient reduction multiplies every row by a gate gradient, 0
    // past the length; the rows must hold numbers, not stale memory)
    for (int s = 0; s < S; ++s) {
        if (b0 + s >= B) break;
        float* hb = H + (int64_t)(b0 + s) * (T + 1) * HD;
        for (int e = j; e < HD; e += GRU_THREADS) hb[e] = 0.f;
        for (int64_t e = (int64_t)(lens[s] + 1) * HD + j; e < (int64_t)(T + 1) * HD; e += GRU_THREADS) hb[e] = 0.f;
    }
    // this thread's elements e = j + 384 i of a_t, loaded a step ahead (the
    // loads of step t + 1 are in flight during step t's products)
    constexpr int AN = (S * C1 + GRU_THREADS - 1) / GRU_THREADS;
    float an[AN];
    auto load_a = [&](int t) {
#pragma unroll
        for (int i = 0; i < AN; ++i) {
            const int e = j + GRU_THREADS * i;
            const int s = e / C1;
            an[i] = (e < S * C1 && b0 + s < B && t < lens[s]) ? A[((int64_t)(b0 + s) * T + t) * C1 + e % C1] : 0.f;
        }
    };
    // the two BF16 weights of a pair as floats (low half: even k)
    auto lo = [](uint32_t u) { return __uint_as_float(u << 16); };
    auto hi = [](uint32_t u) { return __uint_as_float(u & 0xffff0000u); };
    if (tmax > 0) load_a(0);
    for (int t = 0; t < tmax; ++t) {
#pragma unroll
        for (int i = 0; i < AN; ++i) {
            const int e = j + GRU_THREADS * i;  // element (s, c) = (e / 64, e % 64)
            if (e < S * C1) as[(e % C1) * SPA + e / C1] = an[i];
        }
        __syncthreads();
        if (t + 1 < tmax) load_a(t + 1);
        // accumulator pairs (trajectories 8 sh + 2 q, 8 sh + 2 q + 1) of rows jr and jr + 192
        float2 ai0[SH / 2], ai1[SH / 2], ah0[SH / 2], ah1[SH / 2];
#pragma unroll
        for (int q = 0; q < SH / 2; ++q) {
            ai0[q] = make_float2(bih0, bih0);
            ai1[q] = make_float2(bih1, bih1);
            ah0[q] = make_float2(bhh0, bhh0);
            ah1[q] = make_float2(bhh1, bhh1);
        }
        // k + 3, k + 2, k + 1, k within each group of four: the order of a
        // nested fmaf(w_k, v_k, fmaf(w_k+1, v_k+1, ...)) dot product
        auto prods = [&](const uint32_t* w2, const float* v, int K, float2 (&acc0)[SH / 2], float2 (&acc1)[SH / 2]) {
            for (int k = 0; k < K; k += 4) {
                const uint32_t p01 = w2[(k / 2) * G3 + jr], p23 = w2[(k / 2 + 1) * G3 + jr];
                const uint32_t q01 = w2[(k / 2) * G3 + jr + G3 / 2], q23 = w2[(k / 2 + 1) * G3 + jr + G3 / 2];
                const float wr0[4] = {lo(p01), hi(p01), lo(p23), hi(p23)};
                const float wr1[4] = {lo(q01), hi(q01), lo(q23), hi(q23)};
#pragma unroll
                for (int kk = 3; kk >= 0; --kk) {
                    const float4 va = *reinterpret_cast<const float4*>(v + (k + kk) * SPA + SH * sh);
                    const float4 vb = *reinterpret_cast<const float4*>(v + (k + kk) * SPA + SH * sh + 4);
                    const float2 vv[4] = {make_float2(va.x, va.y), make_float2(va.z, va.w),
                                          make_float2(vb.x, vb.y), make_float2(vb.z, vb.w)};
                    const float2 w0 = make_float2(wr0[kk], wr0[kk]), w1 = make_float2(wr1[kk], wr1[kk]);
#pragma unroll
                    for (int q = 0; q < SH / 2; ++q) {
                        acc0[q] = __ffma2_rn(w0, vv[q], acc0[q]);
                        acc1[q] = __ffma2_rn(w1, vv[q], acc1[q]);
                    }
                }
            }
        };
        prods(wih2, as, C1, ai0, ai1);
        prods(whh2, hs, HD, ah0, ah1);
#pragma unroll
        for (int q = 0; q < SH / 2; ++q) {
            const int s = SH * sh + 2 * q;
            gi[s * G3 + jr] = ai0[q].x;
            gi[(s + 1) * G3 + jr] = ai0[q].y;
            gi[s * G3 + jr + G3 / 2] = ai1[q].x;
            gi[(s + 1) * G3 + jr + G3 / 2] = ai1[q].y;
            gh[s * G3 + jr] = ah0[q].x;
            gh[(s + 1) * G3 + jr] = ah0[q].y;
            gh[s * G3 + jr + G3 / 2] = ah1[q].x;
            gh[(s + 1) * G3 + jr + G3 / 2] = ah1[q].y;
        }
        __syncthreads();
        for (int e = j; e < S * HD; e += GRU_THREADS) {
            const int s = e / HD, k = e % HD;
            if (b0 + s < B && t < lens[s]) {
                const float r = sigm(gi[s * G3 + k] + gh[s * G3 + k]);
                const float z = sigm(gi[s * G3 + HD + k] + gh[s * G3 + HD + k]);
                const float ghn = gh[s * G3 + 2 * HD + k];
                const float n = tanhf(gi[s * G3 + 2 * HD + k] + r * ghn);
                const float hp = hs[k * SPA + s];
                const float hn = (1.f - z) * n + z * hp;
                const int64_t o = ((int64_t)(b0 + s) * T + t) * HD + k;
                R[o] = r;
                Z[o] = z;
                N[o] = n;
                GHN[o] = ghn;
                H[((int64_t)(b0 + s) * (T + 1) + t + 1) * HD + k] = hn;
                hs[k * SPA + s] = hn;
            }
        }
        __syncthreads();
    }
    for (int e = j; e < S * HD; e += GRU_THREADS) {
        const int s = e / HD;
        if (b0 + s < B) hl[(int64_t)(b0 + s) * HD + e % HD] = hs[(e % HD) * SPA + s];
    }
}

// Point index of resampled point k (0 <= k < NS) of a trajectory of n >= 1
// points: round(k (n - 1) / (NS - 1)), halves rounded up, in integers.
__device__ __forceinline__ int skip_index(int k, int n) { return (2 * k * (n - 1) + (NS - 1)) / (2 * (NS - 1)); }

// E[b][o] = bo[o] + sum_k Wo[o][k] hl[b][k] (bias first, k ascending) for
// o < EO; E[b][EO + 2 k + i] = sc_k * coordinate i of resampled point k (the
// normalised input at skip_index(k, n); 0 for an empty trajectory), the
// geometric skip, written unscaled to X[b][2 k + i] too when X is given (the
// training forward keeps it for the gradients of sc_k).  One thread per head
// output o, HEAD_B trajectories per CTA, their hidden states staged in
// shared memory; each W_o row is read once per CTA.
constexpr int HEAD_B = 32;
__global__ void __launch_bounds__(EO) enc_head_fwd(const float* __restrict__ hl, int B, const float* __restrict__ p,
                                                   float* __restrict__ E, const float2* __restrict__ pts,
                                                   const int64_t* __restrict__ off, const int32_t* __restrict__ len,
                                                   float4 nrm, float* __restrict__ X) {
    __shared__ __align__(16) float hs[HEAD_B][HD];
    const int o = threadIdx.x;
    const int64_t b0 = (int64_t)blockIdx.x * HEAD_B;
    for (int e = o; e < HEAD_B * SK; e += EO) {
        const int64_t b = b0 + e / SK;
        const int q = e % SK;
        if (b < B) {
            const int n = len[b];
            const float x = n > 0 ? xin(pts, off[b], n, skip_index(q >> 1, n), q & 1, nrm) : 0.f;
            E[b * ED + EO + q] = expf(p[OFF_SC + (q >> 1)]) * x;
            if (X) X[b * SK + q] = x;
        }
    }
    for (int e = o; e < HEAD_B * HD; e += EO) {
        const int64_t b = b0 + e / HD;
        hs[e / HD][e % HD] = b < B ? hl[b * HD + e % HD] : 0.f;
    }
    __syncthreads();
    float acc[HEAD_B];
    const float bo = p[OFF_BO + o];
#pragma unroll
    for (int j = 0; j < HEAD_B; ++j) acc[j] = bo;
    const float* w = p + OFF_WO + o * HD;  // the caller's buffer: 4-byte alignment only
    for (int k = 0; k < HD; k += 4) {
        const float w0 = __ldg(w + k), w1 = __ldg(w + k + 1), w2 = __ldg(w + k + 2), w3 = __ldg(w + k + 3);
#pragma unroll
        for (int j = 0; j < HEAD_B; ++j) {
            const float4 h = *reinterpret_cast<const float4*>(&hs[j][k]);
            acc[j] = fmaf(w3, h.w, fmaf(w2, h.z, fmaf(w1, h.y, fmaf(w0, h.x, acc[j]))));
        }
    }
#pragma unroll
    for (int j = 0; j < HEAD_B; ++j)
        if (b0 + j < B) E[(b0 + j) * ED + o] = acc[j];
}

// One warp per pair: pred = ||E[ia]-E[ib]|| (all ED embedding values), loss += w (pred-y)^2 / P,
// dE[ia] += 2 w (pred-y)/P * (E[ia]-E[ib])/pred, dE[ib] -= the same; w = wt[p] (1 without weights).
__global__ void enc_pair_loss(const float* __restrict__ E, const int32_t* __restrict__ ia,
                              const int32_t* __restrict__ ib, const float* __restrict__ y,
                              const float* __restrict__ wt, int P, float* __restrict__ pred,
                              float* __restrict__ loss, float* __restrict__ dE) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= P) return;
    const float* ea = E + (int64_t)ia[w] * ED;
    const float* eb = E + (int64_t)ib[w] * ED;
    float d[ED / 32];
    float ss = 0.f;
#pragma unroll
    for (int q = 0; q < ED / 32; ++q) {
        d[q] = ea[lane + 32 * q] - eb[lane + 32 * q];
        ss = fmaf(d[q], d[q], ss);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    const float pr = sqrtf(ss);
    const float err = pr - y[w];
    const float wp = wt ? wt[w] : 1.f;
    if (lane == 0) {
        pred[w] = pr;
        if (loss) atomicAdd(loss, wp * err * err / P);
    }
    if (dE && pr > 0.f) {
        const float g = 2.f * wp * err / (P * pr);
#pragma unroll
        for (int q = 0; q < ED / 32; ++q) {
            atomicAdd(dE + (int64_t)ia[w] * ED + lane + 32 * q, g * d[q]);
            atomicAdd(dE + (int64_t)ib[w] * ED + lane + 32 * q, -g * d[q]);
        }
    }
}

// dWo[o][k] += sum_b dE[b][o] hl[b][k]; dbo[o] += sum_b dE[b][o];
// dhl[b][k] = sum_o Wo[o][k] dE[b][o].
__global__ void enc_head_bwd_w(const float* __restrict__ dE, const float* __restrict__ hl, int B,
                               float* __restrict__ grad) {
    const int o = blockIdx.x;  // EO blocks
    const int k = threadIdx.x; // 128 threads
    float acc = 0.f, accb = 0.f;
    for (int b = 0; b < B; ++b) {
        const float g = dE[(int64_t)b * ED + o];
        acc = fmaf(g, hl[(int64_t)b * HD + k], acc);
        accb += g;
    }
    grad[OFF_WO + o * HD + k] += acc;
    if (k == 0) grad[OFF_BO + o] += accb;
}

__global__ void enc_head_bwd_h(const float* __restrict__ dE, int B, const float* __restrict__ p, float* __restrict__ dhl) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (int64_t)B * HD) return;
    const int k = gid % HD;
    const int64_t b = gid / HD;
    float acc = 0.f;
    for (int o = 0; o < EO; ++o) acc = fmaf(p[OFF_WO + o * HD + k], dE[b * ED + o], acc);
    dhl[gid] = acc;
}

// d u_k += sc_k sum_b sum_i dE[b][EO + 2k + i] X[b][2k + i] (the gradients of
// the skip's log-weights, sc_k = exp(u_k)).  Lane q of every warp takes skip value q of the warp's
// trajectories (blockDim a multiple of 32 = SK); lanes 2k and 2k + 1 are summed
// before one atomic per point and warp.
__global__ void enc_skip_bwd(const float* __restrict__ dE, const float* __restrict__ X, int B,
                             const float* __restrict__ p, float* __restrict__ grad) {
    const int q = threadIdx.x & (SK - 1);
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / SK;
    const int64_t nw = (int64_t)gridDim.x * blockDim.x / SK;
    float acc = 0.f;
    for (int64_t b = wid; b < B; b += nw) acc = fmaf(dE[b * ED + EO + q], X[b * SK + q], acc);
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    if ((q & 1) == 0) atomicAdd(grad + OFF_SC + (q >> 1), expf(p[OFF_SC + (q >> 1)]) * acc);
}

// BPTT.  CTA = S trajectories, 384 threads.  Shared memory: Whh [384][128]
// and Wih [384][64] BF16 (row-major: thread k reads column k of row j),
// dh [S][128], dgi/dgh [S][384].  Writes, for every step t < len:
//   G  [B][T][384]  input-side gate gradients (d pre-activation of r, z, n)
//   GH [B][T][384]  hidden-side (r, z as G; n multiplied by r)
//   dA [B][T][64]   gradient of the conv output
// and zeros for steps t >= len.
__global__ void __launch_bounds__(GRU_THREADS, 1) enc_gru_bwd(
    const float* __restrict__ dhl, const int32_t* __restrict__ len, int B, int T, const __nv_bfloat16* __restrict__ wq,
    const float* __restrict__ H, const float* __restrict__ R, const float* __restrict__ Z, const float* __restrict__ N,
    const float* __restrict__ GHN, float* __restrict__ G, float* __restrict__ GH, float* __restrict__ dA,
    float* __restrict__ gbih, float* __restrict__ gbhh) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __nv_bfloat16* whh = reinterpret_cast<__nv_bfloat16*>(smraw);  // [384][128]
    __nv_bfloat16* wih = whh + G3 * HD;                             // [384][64]
    float* dh = reinterpret_cast<float*>(wih + G3 * C1);            // [S][128]
    float* dhd = dh + S * HD;                                       // [S][128] direct part (dh * z)
    float* dgi = dhd + S * HD;                                      // [384][SP] gate gradients, trajectory-minor
    float* dgh = dgi + G3 * SP;                                     // [384][SP]
    __shared__ int lens[S];
    const int tid = threadIdx.x;
    const int b0 = blockIdx.x * S;
    for (int e = tid; e < G3 * HD; e += GRU_THREADS) whh[e] = wq[OFF_WHH + e];
    for (int e = tid; e < G3 * C1; e += GRU_THREADS) wih[e] = wq[OFF_WIH + e];
    if (tid < S) lens[tid] = (b0 + tid < B) ? len[b0 + tid] : 0;
    for (int e = tid; e < S * HD; e += GRU_THREADS) {
        const int s = e / HD;
        dh[e] = (b0 + s < B) ? dhl[(int64_t)(b0 + s) * HD + e % HD] : 0.f;
    }
    __syncthreads();
    // zero the caches of steps beyond each length
    for (int s = 0; s < S; ++s) {
        if (b0 + s >= B) break;
        const int n0 = lens[s];
        for (int64_t e = (int64_t)n0 * G3 + tid; e < (int64_t)T * G3; e += GRU_THREADS) {
            G[(int64_t)(b0 + s) * T * G3 + e] = 0.f;
            GH[(int64_t)(b0 + s) * T * G3 + e] = 0.f;
        }
        for (int64_t e = (int64_t)n0 * C1 + tid; e < (int64_t)T * C1; e += GRU_THREADS)
            dA[(int64_t)(b0 + s) * T * C1 + e] = 0.f;
    }
    int tmax = 0;
    for (int s = 0; s < S; ++s) tmax = max(tmax, lens[s]);
    // The output products: threads 0..255 take 2 consecutive hidden units
    // (dh) of four trajectories, threads 256..383 2 consecutive channels (dA)
    // of four trajectories; per gate row jj one 4-byte load of 2 BF16 weights
    // and one 16-byte load of the four trajectories' gate gradients feed 8
    // FMAs.  Each sum runs over jj in order from the same start as a dot
    // product per output would, so the values are those of one thread per output.
    float sbi = 0.f, sbh = 0.f;  // this CTA's bias gradients of gate row tid (phase 2 maps e % 384 = tid)
    const bool dh_part = tid < 256;
    const int og = dh_part ? (tid & 63) : ((tid - 256) & 31);  // output pair: units / channels 2 og, 2 og + 1
    const int s0 = 4 * (dh_part ? (tid >> 6) : ((tid - 256) >> 5));  // trajectories s0 .. s0 + 3
    // this thread's cache values (elements e = tid + 384 i of step t), loaded
    // a step ahead: the loads of step t - 1 are in flight during step t's products
    constexpr int EN = (S * HD + GRU_THREADS - 1) / GRU_THREADS;
    float cr[EN], cz[EN], cn[EN], cg[EN], ch[EN];
    auto load_c = [&](int t) {
#pragma unroll
        for (int i = 0; i < EN; ++i) {
            const int e = tid + GRU_THREADS * i;
            const int s = e / HD, k = e % HD;
            if (e < S * HD && b0 + s < B && t < lens[s]) {
                const int64_t o = ((int64_t)(b0 + s) * T + t) * HD + k;
                cr[i] = R[o];
                cz[i] = Z[o];
                cn[i] = N[o];
                cg[i] = GHN[o];
                ch[i] = H[((int64_t)(b0 + s) * (T + 1) + t) * HD + k];
            }
        }
    };
    if (tmax > 0) load_c(tmax - 1);
    for (int t = tmax - 1; t >= 0; --t) {
#pragma unroll
        for (int i = 0; i < EN; ++i) {
            const int e = tid + GRU_THREADS * i;
            if (e >= S * HD) break;
            const int s = e / HD, k = e % HD;
            float gr = 0.f, gz = 0.f, gn = 0.f, gnh = 0.f, d = 0.f;
            if (b0 + s < B && t < lens[s]) {
                const float r = cr[i], z = cz[i], n = cn[i], ghn = cg[i];
                const float hp = ch[i];
                const float g = dh[e];
                const float dn = g * (1.f - z);
                const float dz = g * (hp - n);
                d = g * z;
                gn = dn * (1.f - n * n);
                gr = gn * ghn * r * (1.f - r);
                gz = dz * z * (1.f - z);
                gnh = gn * r;
            } else {
                d = dh[e];  // frozen step: dh passes through unchanged
            }
            dgi[k * SP + s] = gr;
            dgi[(HD + k) * SP + s] = gz;
            dgi[(2 * HD + k) * SP + s] = gn;
            dgh[k * SP + s] = gr;
            dgh[(HD + k) * SP + s] = gz;
            dgh[(2 * HD + k) * SP + s] = gnh;
            dhd[e] = d;
        }
        __syncthreads();
        if (t > 0) load_c(t - 1);
        // gate gradients to global memory; thread tid always holds gate row
        // jj = tid here, so it also sums that row's bias gradients
        for (int e = tid; e < S * G3; e += GRU_THREADS) {
            const int s = e / G3, jj = e % G3;
            if (b0 + s < B && t < lens[s]) {
                const int64_t o = ((int64_t)(b0 + s) * T + t) * G3 + jj;
                const float vi = dgi[jj * SP + s], vh = dgh[jj * SP + s];
                G[o] = vi;
                GH[o] = vh;
                sbi += vi;
                sbh += vh;
            }
        }
        // outputs: 128 dh values and 64 dA values per trajectory, each a dot
        // product over the 384 gate gradients
        bool act[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) act[q] = b0 + s0 + q < B && t < lens[s0 + q];
        if (act[0] || act[1] || act[2] || act[3]) {
            const __nv_bfloat16* w = dh_part ? whh + 2 * og : wih + 2 * og;
            const int wstride = dh_part ? HD : C1;
            const float* dg = (dh_part ? dgh : dgi) + s0;
            float a[4][2];
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int i = 0; i < 2; ++i) a[q][i] = dh_part ? dhd[(s0 + q) * HD + 2 * og + i] : 0.f;
#pragma unroll 4
            for (int jj = 0; jj < G3; ++jj) {
                const uint32_t wv = *reinterpret_cast<const uint32_t*>(w + jj * wstride);
                const float4 g4 = *reinterpret_cast<const float4*>(dg + jj * SP);
                const float w0 = __uint_as_float(wv << 16), w1 = __uint_as_float(wv & 0xffff0000u);
                const float gq[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    a[q][0] = fmaf(w0, gq[q], a[q][0]);
                    a[q][1] = fmaf(w1, gq[q], a[q][1]);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!act[q]) continue;
                if (dh_part) {
                    dhd[(s0 + q) * HD + 2 * og] = a[q][0];
                    dhd[(s0 + q) * HD + 2 * og + 1] = a[q][1];
                } else {
                    *reinterpret_cast<float2*>(dA + ((int64_t)(b0 + s0 + q) * T + t) * C1 + 2 * og) =
                        make_float2(a[q][0], a[q][1]);
                }
            }
        }
        __syncthreads();
        for (int e = tid; e < S * HD; e += GRU_THREADS) dh[e] = dhd[e];
        __syncthreads();
    }
    atomicAdd(gbih + tid, sbi);
    atomicAdd(gbhh + tid, sbh);
}

// Conv weight gradients.  One CTA per trajectory, 704 threads: thread q
// takes weight (c, i, k) = (q / 10, (q / 5) % 2, q % 5) of the 640, or the
// bias of channel q - 640, summed over the trajectory's steps (one atomic per
// thread and trajectory).  The normalised input points are staged in shared
// memory, CBW_T steps (plus the window's two on either side) at a time.
constexpr int CBW_THREADS = C1 * 2 * KW + C1;  // 704
constexpr int CBW_T = 256;
__global__ void __launch_bounds__(CBW_THREADS) enc_conv_bwd(const float2* __restrict__ pts,
                                                           const int64_t* __restrict__ off,
                                                           const int32_t* __restrict__ len, int T, float4 nrm,
                                                           const float* __restrict__ A, const float* __restrict__ dA,
                                                           float* __restrict__ grad) {
    __shared__ float xs[CBW_T + KW - 1][2];  // xs[u][i] = input i at step t0 + u - 2
    const int b = blockIdx.x;
    const int n = len[b];
    if (n <= 0) return;  // uniform per CTA
    const int q = threadIdx.x;
    const bool wt = q < C1 * 2 * KW;
    const int c = wt ? q / (2 * KW) : q - C1 * 2 * KW, i = (q / KW) % 2, k = q % KW;
    const int64_t o0 = off[b];
    float acc = 0.f;
    for (int t0 = 0; t0 < n; t0 += CBW_T) {
        const int t1 = min(n, t0 + CBW_T);
        __syncthreads();  // the previous chunk's readers are done
        for (int e = q; e < (t1 - t0 + KW - 1) * 2; e += CBW_THREADS)
            xs[e / 2][e % 2] = xin(pts, o0, n, t0 + e / 2 - 2, e % 2, nrm);
        __syncthreads();
        for (int t = t0; t < t1; ++t) {
            const int64_t o = ((int64_t)b * T + t) * C1 + c;
            const float g = A[o] > 0.f ? dA[o] : 0.f;
            acc = wt ? fmaf(g, xs[t - t0 + k][i], acc) : acc + g;
        }
    }
    atomicAdd(grad + (wt ? OFF_W1 + q : OFF_B1 + c), acc);
}

__global__ void enc_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                         float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// ---------------------------------------------------------------------------
// Tensor-core GRU forward for inference (tcgen05).  CTA = 128 trajectories
// (the MMA's M), 256 threads.  Per time step the operand [a_t | h_t]
// (128 x 192 BF16, shared memory) is multiplied by the BF16 gate weights,
// resident in shared memory for all steps, into three FP32 accumulators in
// tensor memory (512 columns):
//   columns   0..255  r and z pre-activations  [a_t | h_t] [Wih_rz | Whh_rz]^T  (K = 192)
//   columns 256..383  Win a_t                   a_t Wih_n^T                      (K = 64)
//   columns 384..511  Whn h_t                   h_t Whh_n^T                      (K = 128)
// (n needs Whn h apart from Win a: r multiplies only the hidden part.)  One
// thread issues the 24 MMAs and commits them to an mbarrier; then warp w reads
// lanes 32 (w % 4) .. +31 (its 32 trajectories) and hidden units
// 64 (w / 4) .. +63 (sixteen warps, 32 units each, measured no faster: 1.31 vs
// 1.39 ms for 1,000 queries), applies the gates with the biases in FP32, keeps h in FP32
// registers and writes it back to shared memory as BF16 for the next step.
// The a_t part comes from enc_conv_fwd_tc as one 16 KB BF16 image per step
// already in the operand layout; thread 0 bulk-copies step t+1's image into
// the second of two a-buffers while step t computes (per-buffer mbarriers
// count the bytes).  a_t and h_t enter the products as BF16 (the SIMT training
// kernel multiplies FP32 a and h by the BF16 weights) and the gates use the
// hardware tanh, so the embeddings agree with the training forward to BF16
// rounding of the activations.
constexpr int TC_M = 128;
constexpr int TC_THREADS = 256;  // 8 warps: two per 32-lane quarter of tensor memory
constexpr int TC_HU = HD / (TC_THREADS / 128);  // hidden units per thread (32)
constexpr int TC_K = C1 + HD;                               // 192
constexpr int TC_A_BYTES = TC_M * C1 * 2;                   // one a_t image: 16 KB
constexpr int TC_OFF_A0 = 0;                                // a-buffers [128][64] BF16
constexpr int TC_OFF_A1 = TC_OFF_A0 + TC_A_BYTES;
constexpr int TC_OFF_XH = TC_OFF_A1 + TC_A_BYTES;           // h [128][128] BF16
constexpr int TC_OFF_WRZ = TC_OFF_XH + TC_M * HD * 2;       // W_rz [256][192] BF16
constexpr int TC_OFF_WIN = TC_OFF_WRZ + 2 * HD * TC_K * 2;  // W_in [128][64]
constexpr int TC_OFF_WHN = TC_OFF_WIN + HD * C1 * 2;        // W_hn [128][128]
constexpr int TC_OFF_BIAS = TC_OFF_WHN + HD * HD * 2;       // float b_ih[384], b_hh[384]
constexpr int TC_OFF_BAR = TC_OFF_BIAS + 2 * G3 * 4;        // mbarriers: MMA, a0, a1 (8 B each); TMEM address
constexpr int TC_SMEM = TC_OFF_BAR + 32;
constexpr uint32_t TC_TMEM_COLS = 512;
// a wait for the tensor cores or a copy longer than this many SM clocks (~1 s) is an error
constexpr long long TC_WAIT_CYCLES = 2000000000LL;

// Gate nonlinearities of the inference kernel: the hardware tanh (MUFU,
// about 2^-11 relative error, the size of the BF16 rounding the operands
// already carry) and sigma(x) = (1 + tanh(x / 2)) / 2, one MUFU operation each.
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigm_hw(float x) { return fmaf(0.5f, tanh_hw(0.5f * x), 0.5f); }

// Eight BF16 values as one 16-byte store.
__device__ __forceinline__ uint4 pack8_bf16(const float* v) {
    uint4 u;
    u.x = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[0])) |
          ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[1])) << 16);
    u.y = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2])) |
          ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[3])) << 16);
    u.z = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[4])) |
          ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[5])) << 16);
    u.w = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[6])) |
          ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[7])) << 16);
    return u;
}

// Conv output for the tensor-core GRU (same arithmetic as enc_conv_fwd, then
// rounded to BF16): for block g of 128 trajectories and step t, the 16 KB
// image of the a_t operand (rows = trajectories, k = channels, core-matrix
// layout) at Ab + (g * T + t) * 128 * 64.  Rows past B and steps past a
// trajectory's length are zero.  One thread per (trajectory, step), all 64
// channels, with the conv weights in shared memory; consecutive threads take
// consecutive rows of one image, so a warp's 16-byte stores are contiguous.
// Bp = B rounded up to a multiple of 128; blockDim = 256.
__global__ void __launch_bounds__(256) enc_conv_fwd_tc(const float2* __restrict__ pts, const int64_t* __restrict__ off,
                                                       const int32_t* __restrict__ len, int B, int Bp, int T,
                                                       float4 nrm, const __nv_bfloat16* __restrict__ wq,
                                                       const float* __restrict__ p, __nv_bfloat16* __restrict__ Ab) {
    __shared__ float w1[C1 * 2 * KW], b1[C1];
    for (int e = threadIdx.x; e < C1 * 2 * KW; e += blockDim.x) w1[e] = __bfloat162float(wq[OFF_W1 + e]);
    for (int e = threadIdx.x; e < C1; e += blockDim.x) b1[e] = p[OFF_B1 + e];
    __syncthreads();
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (int64_t)Bp * T) return;
    const int row = gid % TC_M;
    const int t = (gid / TC_M) % T;
    const int g = gid / ((int64_t)TC_M * T);
    const int b = g * TC_M + row;
    const int n = b < B ? len[b] : 0;
    float x[KW][2];  // the window's normalised points
    if (t < n) {
        const int64_t o = off[b];
#pragma unroll
        for (int k = 0; k < KW; ++k)
#pragma unroll
            for (int i = 0; i < 2; ++i) x[k][i] = xin(pts, o, n, t + k - 2, i, nrm);
    }
    unsigned char* img = reinterpret_cast<unsigned char*>(Ab + ((int64_t)g * T + t) * (TC_M * C1));
#pragma unroll 1
    for (int c8 = 0; c8 < C1 / 8; ++c8) {
        float a[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int c = 8 * c8 + q;
            float v = 0.f;
            if (t < n) {
                float acc = b1[c];
#pragma unroll
                for (int k = 0; k < KW; ++k)
#pragma unroll
                    for (int i = 0; i < 2; ++i) acc = fmaf(w1[(c * 2 + i) * KW + k], x[k][i], acc);
                v = fmaxf(acc, 0.f);
            }
            a[q] = v;
        }
        *reinterpret_cast<uint4*>(img + tsm::umma::core_offset(row, 8 * c8, TC_M)) = pack8_bf16(a);
    }
}

// Bits of the embedding status word (the first word of the embed workspace).
constexpr int TC_ERR_COPY = 1;      // an a_t copy did not land within the wait limit (no MMA issued for it)
constexpr int TC_ERR_MMA = 2;       // the MMAs of a step did not complete within the wait limit
constexpr int TC_ERR_TMEM_HELD = 4; // ... nor within a second limit: the CTA exited without freeing tensor memory

// hl[b][128] = h after the last valid step of trajectory b.  Ab: the a_t
// images of enc_conv_fwd_tc (T steps per block of 128).  wq: BF16 weights; p:
// FP32 parameters (biases).  If the tensor cores or a copy do not complete
// within wait_cycles, the CTA ORs a TC_ERR_* bit into *status, writes NaN to
// its rows of hl and stops: after waiting (bounded) for its copy in flight,
// and, if MMAs of the failed step were issued, once more for them; tensor
// memory is freed only when no MMA can still write it.  stall_step >= 0 is a
// test hook: the a_t copy of that step is announced on its mbarrier but never
// issued, so that its wait runs out with no MMA in flight (-1 in normal use).
__global__ void __launch_bounds__(TC_THREADS, 1) enc_gru_embed_tc(const __nv_bfloat16* __restrict__ Ab,
                                                                   const int32_t* __restrict__ len, int B, int T,
                                                                   const __nv_bfloat16* __restrict__ wq,
                                                                   const float* __restrict__ p,
                                                                   float* __restrict__ hl, int* __restrict__ status,
                                                                   long long wait_cycles, int stall_step) {
    namespace U = tsm::umma;
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* XH = sm + TC_OFF_XH;
    float* bias = reinterpret_cast<float*>(sm + TC_OFF_BIAS);
    const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
    const uint32_t mbar = sbase + TC_OFF_BAR, abar0 = mbar + 8, abar1 = mbar + 16;
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(sm + TC_OFF_BAR + 24);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row = 32 * (warp & 3) + lane;  // this thread's trajectory (TMEM lane)
    const int hc = warp >> 2;                // hidden units TC_HU hc .. +TC_HU-1
    const int b = blockIdx.x * TC_M + row;
    const int n = b < B ? len[b] : 0;
    const __nv_bfloat16* img = Ab + (int64_t)blockIdx.x * T * (TC_M * C1);  // this block's a_t images

    // weights -> core-matrix layout (16-byte chunks of 8 consecutive k)
    for (int e = tid; e < 2 * HD * (TC_K / 8); e += TC_THREADS) {  // W_rz: gate rows 0..255, k < 192
        const int r = e / (TC_K / 8), c = e % (TC_K / 8);
        const __nv_bfloat16* src = c < C1 / 8 ? wq + OFF_WIH + r * C1 + 8 * c : wq + OFF_WHH + r * HD + 8 * (c - C1 / 8);
        *reinterpret_cast<uint4*>(sm + TC_OFF_WRZ + U::core_offset(r, 8 * c, 2 * HD)) =
            *reinterpret_cast<const uint4*>(src);
    }
    for (int e = tid; e < HD * (C1 / 8); e += TC_THREADS) {  // W_in: gate rows 256..383, k < 64
        const int r = e / (C1 / 8), c = e % (C1 / 8);
        *reinterpret_cast<uint4*>(sm + TC_OFF_WIN + U::core_offset(r, 8 * c, HD)) =
            *reinterpret_cast<const uint4*>(wq + OFF_WIH + (2 * HD + r) * C1 + 8 * c);
    }
    for (int e = tid; e < HD * (HD / 8); e += TC_THREADS) {  // W_hn: gate rows 256..383, k < 128
        const int r = e / (HD / 8), c = e % (HD / 8);
        *reinterpret_cast<uint4*>(sm + TC_OFF_WHN + U::core_offset(r, 8 * c, HD)) =
            *reinterpret_cast<const uint4*>(wq + OFF_WHH + (2 * HD + r) * HD + 8 * c);
    }
    for (int e = tid; e < 2 * G3; e += TC_THREADS) bias[e] = e < G3 ? p[OFF_BIH + e] : p[OFF_BHH + e - G3];
    {  // h_0 = 0: this thread's 64 hidden units
        const float z8[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int c = 0; c < TC_HU / 8; ++c)
            *reinterpret_cast<uint4*>(XH + U::core_offset(row, TC_HU * hc + 8 * c, TC_M)) = pack8_bf16(z8);
    }
    if (tid == 0) {
        U::mbar_init(mbar, 1);
        U::mbar_init(abar0, 1);
        U::mbar_init(abar1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) U::tmem_alloc(sbase + TC_OFF_BAR + 24, TC_TMEM_COLS);
    U::fence_smem_async();
    U::fence_before_sync();
    __syncthreads();
    U::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t tl = tmem + ((uint32_t)(32 * (warp & 3)) << 16);  // this warp's lane quarter

    int tmax = 0;
    for (int i = 0; i < TC_M; ++i) {
        const int bi = blockIdx.x * TC_M + i;
        if (bi < B) tmax = max(tmax, len[bi]);
    }
    tmax = min(tmax, T);
    int pend = -1;    // thread 0: the step whose a_t copy is issued and not yet waited for
    int issued = -1;  // thread 0: the last step whose MMAs were committed
    if (tid == 0 && tmax > 0) {  // a_0 into buffer 0
        U::mbar_arrive_expect_tx(abar0, TC_A_BYTES);
        if (stall_step != 0) U::bulk_load(sbase + TC_OFF_A0, img, TC_A_BYTES, abar0);
        pend = 0;
    }
    float h[TC_HU];
#pragma unroll
    for (int i = 0; i < TC_HU; ++i) h[i] = 0.f;
    bool failed = false;
    int fail_t = -1;
    for (int t = 0; t < tmax; ++t) {
        const uint32_t abuf = sbase + ((t & 1) ? TC_OFF_A1 : TC_OFF_A0);
        if (tid == 0) {
            // a_t has landed in buffer t % 2 (its (t / 2)-th use)
            if (!U::mbar_wait((t & 1) ? abar1 : abar0, (uint32_t)((t >> 1) & 1), wait_cycles)) {
                atomicOr(status, TC_ERR_COPY);
            } else {
                pend = -1;
                U::fence_after_sync();
                constexpr uint32_t kRZ = U::idesc_bf16_f32(TC_M, 2 * HD), kN = U::idesc_bf16_f32(TC_M, HD);
                constexpr uint32_t kLBO = TC_M * 16;  // K-chunk stride of the 128-row operands
                for (int ks = 0; ks < TC_K / 16; ++ks) {  // r, z: [a_t | h_t] [W_ih | W_hh]^T, K = 192
                    const uint32_t a = ks < C1 / 16 ? abuf + ks * 2 * kLBO : sbase + TC_OFF_XH + (ks - C1 / 16) * 2 * kLBO;
                    U::mma_bf16(tmem, U::smem_desc(a, kLBO, 128),
                                U::smem_desc(sbase + TC_OFF_WRZ + ks * 2 * (2 * HD * 16), 2 * HD * 16, 128), kRZ, ks);
                }
                for (int ks = 0; ks < C1 / 16; ++ks)  // Win a_t
                    U::mma_bf16(tmem + 2 * HD, U::smem_desc(abuf + ks * 2 * kLBO, kLBO, 128),
                                U::smem_desc(sbase + TC_OFF_WIN + ks * 2 * (HD * 16), HD * 16, 128), kN, ks);
                for (int ks = 0; ks < HD / 16; ++ks)  // Whn h_t
                    U::mma_bf16(tmem + 3 * HD, U::smem_desc(sbase + TC_OFF_XH + ks * 2 * kLBO, kLBO, 128),
                                U::smem_desc(sbase + TC_OFF_WHN + ks * 2 * (HD * 16), HD * 16, 128), kN, ks);
                U::commit(mbar);
                issued = t;
                if (t + 1 < tmax) {  // a_{t+1} into the other buffer (its last reader, step t-1, has completed)
                    const uint32_t nb = (t & 1) ? abar0 : abar1;
                    U::mbar_arrive_expect_tx(nb, TC_A_BYTES);
                    if (t + 1 != stall_step)
                        U::bulk_load(sbase + ((t & 1) ? TC_OFF_A0 : TC_OFF_A1), img + (int64_t)(t + 1) * (TC_M * C1),
                                     TC_A_BYTES, nb);
                    pend = t + 1;
                }
            }
        }
        const bool ok = U::mbar_wait(mbar, (uint32_t)(t & 1), wait_cycles);
        if (__syncthreads_or(!ok)) {
            failed = true;
            fail_t = t;
            break;
        }
        U::fence_after_sync();
        const bool live = t < n;
#pragma unroll
        for (int c = 0; c < TC_HU / 16; ++c) {  // 16 hidden units at a time
            const int k0 = TC_HU * hc + 16 * c;
            uint32_t rr[16], zz[16], ii[16], hh[16];
            U::ld16(tl + k0, rr);
            U::ld16(tl + HD + k0, zz);
            U::ld16(tl + 2 * HD + k0, ii);
            U::ld16(tl + 3 * HD + k0, hh);
            U::wait_ld(rr);
            U::wait_ld(zz);
            U::wait_ld(ii);
            U::wait_ld(hh);
            float hv[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int k = k0 + j;
                const float r = sigm_hw(__uint_as_float(rr[j]) + bias[k] + bias[G3 + k]);
                const float z = sigm_hw(__uint_as_float(zz[j]) + bias[HD + k] + bias[G3 + HD + k]);
                const float nn = tanh_hw(__uint_as_float(ii[j]) + bias[2 * HD + k] +
                                         r * (__uint_as_float(hh[j]) + bias[G3 + 2 * HD + k]));
                const float hp = h[16 * c + j];
                hv[j] = live ? (1.f - z) * nn + z * hp : hp;
                h[16 * c + j] = hv[j];
            }
            if (live) {
                *reinterpret_cast<uint4*>(XH + U::core_offset(row, k0, TC_M)) = pack8_bf16(hv);
                *reinterpret_cast<uint4*>(XH + U::core_offset(row, k0 + 8, TC_M)) = pack8_bf16(hv + 8);
            }
        }
        U::fence_smem_async();
        U::fence_before_sync();
        __syncthreads();
    }
    __shared__ int tmem_busy;  // set by thread 0 when MMAs may still write tensor memory
    if (tid == 0) {
        tmem_busy = 0;
        if (pend >= 0)  // after a failure: let this CTA's copy in flight land before exiting
            U::mbar_wait((pend & 1) ? abar1 : abar0, (uint32_t)((pend >> 1) & 1), wait_cycles);
        if (failed && issued == fail_t) {  // the failed step's MMAs were committed: wait for them once more
            atomicOr(status, TC_ERR_MMA);
            if (!U::mbar_wait(mbar, (uint32_t)(fail_t & 1), wait_cycles)) {
                atomicOr(status, TC_ERR_TMEM_HELD);
                tmem_busy = 1;
            }
        }
    }
    if (b < B) {
        float* dst = hl + (int64_t)b * HD + TC_HU * hc;
#pragma unroll
        for (int i = 0; i < TC_HU; ++i) dst[i] = failed ? __int_as_float(0x7fc00000) : h[i];
    }
    U::fence_before_sync();
    __syncthreads();
    if (warp == 0 && !tmem_busy) {
        U::fence_after_sync();
        U::tmem_dealloc(tmem, TC_TMEM_COLS);
    }
}

}  // namespace enc

// ---------------------------------------------------------------------------
// Host orchestration (C ABI, declared in include/tsm.h)
// ---------------------------------------------------------------------------
namespace {

struct EncWs {  // views into the caller's workspace
    int* status;  // first word: bits OR-ed in by the tensor-core weight-gradient kernel (zeroed by the caller)
    float *A, *H, *R, *Z, *N, *GHN, *G, *GH, *dA, *hl, *E, *dE, *dhl, *pred, *loss, *X;
    __nv_bfloat16* wq;
    void* wg;  // scratch of tsm_wgrad_tc
};

int64_t align64(int64_t n) { return (n + 63) & ~int64_t(63); }

// Lays the workspace out (base != NULL) and returns its size in floats.
int64_t ws_layout(int B, int T, int P, float* base, EncWs* w) {
    int64_t o = 0;
    auto take = [&](float** dst, int64_t n) {
        if (base) *dst = base + o;
        o += align64(n);
    };
    EncWs tmp;
    EncWs* x = w ? w : &tmp;
    const int64_t BT = (int64_t)B * T;
    float* st = nullptr;
    take(&st, 1);
    if (base) x->status = reinterpret_cast<int*>(st);
    take(&x->A, BT * enc::C1);
    take(&x->H, (int64_t)B * (T + 1) * enc::HD);
    take(&x->R, BT * enc::HD);
    take(&x->Z, BT * enc::HD);
    take(&x->N, BT * enc::HD);
    take(&x->GHN, BT * enc::HD);
    take(&x->G, BT * enc::G3);
    take(&x->GH, BT * enc::G3);
    take(&x->dA, BT * enc::C1);
    take(&x->hl, (int64_t)B * enc::HD);
    take(&x->E, (int64_t)B * enc::ED);
    take(&x->dE, (int64_t)B * enc::ED);
    take(&x->dhl, (int64_t)B * enc::HD);
    take(&x->X, (int64_t)B * enc::SK);
    take(&x->pred, P > 0 ? P : 1);
    take(&x->loss, 1);
    float* wqf = nullptr;
    take(&wqf, (enc::N_PARAMS + 1) / 2);  // BF16 copy of the weights
    if (base) x->wq = reinterpret_cast<__nv_bfloat16*>(wqf);
    float* wg = nullptr;
    take(&wg, (tsm_wgrad_scratch_bytes(B, T) + 3) / 4);
    if (base) x->wg = wg;
    return o;
}

constexpr int kGruFwdSmem = (enc::C1 * enc::G3 + enc::HD * enc::G3) * 2 +
                            (enc::HD * enc::SPA + enc::C1 * enc::SPA + 2 * enc::S * enc::G3) * 4;
constexpr int kGruBwdSmem = (enc::G3 * enc::HD + enc::G3 * enc::C1) * 2 +
                            (2 * enc::S * enc::HD + 2 * enc::G3 * enc::SP) * 4;
// one CTA per SM: dynamic shared memory plus the kernels' 1 KB of static
// shared memory must fit the 227 KB a CTA may use
static_assert(kGruFwdSmem + 1024 <= 227 * 1024, "enc_gru_fwd shared memory");
static_assert(kGruBwdSmem + 1024 <= 227 * 1024, "enc_gru_bwd shared memory");

int enc_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return TSM_OK;
    char b[256];
    snprintf(b, sizeof(b), "%s: %s", what, cudaGetErrorString(e));
    return tsm_internal_fail(TSM_ECUDA, b);
}

int enc_args(const void* params, const void* pts, const void* off, const void* len, int B, int T, const float* nrm,
             const void* ws) {
    if (!params || !pts || !off || !len || !nrm || !ws) return tsm_internal_fail(TSM_EINVAL, "encoder: null pointer");
    if (B < 1 || T < 1) return tsm_internal_fail(TSM_EINVAL, "encoder: batch and time must be positive");
    if (reinterpret_cast<uintptr_t>(ws) % 256)
        return tsm_internal_fail(TSM_EINVAL, "encoder: workspace must be 256-byte aligned");
    if ((int64_t)B * T * enc::G3 > (int64_t)1 << 40) return tsm_internal_fail(TSM_EINVAL, "encoder: batch too large");
    return TSM_OK;
}

int enc_forward(const float* params, const float* pts, const int64_t* off, const int32_t* len, int B, int T,
                const float* nrm, EncWs& w, cudaStream_t s) {
    using namespace enc;
    const float4 n4 = make_float4(nrm[0], nrm[1], nrm[2], nrm[3]);
    enc_round_bf16<<<(OFF_WO + 255) / 256, 256, 0, s>>>(params, w.wq);
    const int64_t tot = (int64_t)B * T * C1;
    enc_conv_fwd<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(reinterpret_cast<const float2*>(pts), off, len, B, T,
                                                                n4, w.wq, params, w.A);
    int rc = enc_check(cudaFuncSetAttribute(enc_gru_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kGruFwdSmem),
                       "cudaFuncSetAttribute(enc_gru_fwd)");
    if (rc) return rc;
    enc_gru_fwd<<<(B + S - 1) / S, GRU_THREADS, kGruFwdSmem, s>>>(w.A, len, B, T, w.wq, params, w.H, w.R, w.Z, w.N,
                                                                   w.GHN, w.hl);
    enc_head_fwd<<<(unsigned)((B + HEAD_B - 1) / HEAD_B), EO, 0, s>>>(w.hl, B, params, w.E,
                                                                      reinterpret_cast<const float2*>(pts), off, len,
                                                                      n4, w.X);
    return enc_check(cudaGetLastError(), "encoder forward launch");
}

int enc_backward(const float* params, const float* pts, const int64_t* off, const int32_t* len, int B, int T,
                 const float* nrm, EncWs& w, float* grad, cudaStream_t s) {
    using namespace enc;
    const float4 n4 = make_float4(nrm[0], nrm[1], nrm[2], nrm[3]);
    enc_head_bwd_w<<<EO, HD, 0, s>>>(w.dE, w.hl, B, grad);
    enc_skip_bwd<<<(unsigned)(((int64_t)B * SK + 255) / 256 < 256 ? ((int64_t)B * SK + 255) / 256 : 256), 256, 0, s>>>(
        w.dE, w.X, B, params, grad);
    enc_head_bwd_h<<<(unsigned)(((int64_t)B * HD + 255) / 256), 256, 0, s>>>(w.dE, B, params, w.dhl);
    int rc = enc_check(cudaFuncSetAttribute(enc_gru_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kGruBwdSmem),
                       "cudaFuncSetAttribute(enc_gru_bwd)");
    if (rc) return rc;
    // the bias gradients (sums of the gate gradients over the valid (b, t)) come out of the BPTT kernel
    enc_gru_bwd<<<(B + S - 1) / S, GRU_THREADS, kGruBwdSmem, s>>>(w.dhl, len, B, T, w.wq, w.H, w.R, w.Z, w.N,
                                                                   w.GHN, w.G, w.GH, w.dA, grad + OFF_BIH,
                                                                   grad + OFF_BHH);
    // weight gradients dWih[j][c] += G . A, dWhh[j][k] += GH . H[t]: reductions over the valid (b, t) on the
    // tensor cores (tsm_wgrad.cu)
    if ((rc = tsm_wgrad_tc(w.G, w.GH, w.A, w.H, len, B, T, w.wg, w.status, grad + OFF_WIH, grad + OFF_WHH, s)))
        return rc;
    enc_conv_bwd<<<B, CBW_THREADS, 0, s>>>(reinterpret_cast<const float2*>(pts), off, len, T, n4, w.A, w.dA, grad);
    return enc_check(cudaGetLastError(), "encoder backward launch");
}

// Inference workspace: the BF16 a_t images (B rounded up to 128 rows), last
// hidden states, embeddings, BF16 weights.
struct EmbWs {
    int* status;  // first word of the workspace: TC_ERR_* bits of the last call
    __nv_bfloat16* Ab;
    float *hl, *E;
    __nv_bfloat16* wq;
};

int64_t emb_layout(int B, int T, float* base, EmbWs* w) {
    int64_t o = 0;
    auto take = [&](int64_t n) {
        float* q = base ? base + o : nullptr;
        o += align64(n);
        return q;
    };
    float* st = take(1);
    const int64_t Bp = ((int64_t)B + enc::TC_M - 1) / enc::TC_M * enc::TC_M;
    float* Ab = take(Bp * T * enc::C1 / 2);
    float* hl = take((int64_t)B * enc::HD);
    float* E = take((int64_t)B * enc::ED);
    float* wqf = take((enc::N_PARAMS + 1) / 2);
    if (w) {
        w->status = reinterpret_cast<int*>(st);
        w->Ab = reinterpret_cast<__nv_bfloat16*>(Ab);
        w->hl = hl;
        w->E = E;
        w->wq = reinterpret_cast<__nv_bfloat16*>(wqf);
    }
    return o;
}

}  // namespace

extern "C" {

int tsm_enc_param_count(void) { return enc::N_PARAMS; }

int64_t tsm_enc_workspace_bytes(int32_t B, int32_t T, int32_t P) {
    if (B < 1 || T < 1 || P < 0) return -1;
    return ws_layout(B, T, P, nullptr, nullptr) * 4;
}

int tsm_enc_forward(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                    int32_t T, const float* nrm, void* workspace, float* emb, void* stream) {
    int rc = enc_args(params, pts, off, len, B, T, nrm, workspace);
    if (rc) return rc;
    EncWs w;
    ws_layout(B, T, 0, static_cast<float*>(workspace), &w);
    cudaStream_t s = (cudaStream_t)stream;
    rc = enc_forward(params, pts, off, len, B, T, nrm, w, s);
    if (rc) return rc;
    if (emb) rc = enc_check(cudaMemcpyAsync(emb, w.E, (size_t)B * enc::ED * 4, cudaMemcpyDeviceToDevice, s),
                            "copy embeddings");
    return rc;
}

int tsm_enc_loss_grad_w(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                        int32_t T, const float* nrm, const int32_t* ia, const int32_t* ib, const float* y,
                        const float* weights, int32_t P, void* workspace, float* grad, float* loss, float* pred,
                        void* stream) {
    int rc = enc_args(params, pts, off, len, B, T, nrm, workspace);
    if (rc) return rc;
    if (P < 1 || !ia || !ib || !y || !grad) return tsm_internal_fail(TSM_EINVAL, "tsm_enc_loss_grad: bad pairs");
    EncWs w;
    ws_layout(B, T, P, static_cast<float*>(workspace), &w);
    cudaStream_t s = (cudaStream_t)stream;
    rc = enc_forward(params, pts, off, len, B, T, nrm, w, s);
    if (rc) return rc;
    if ((rc = enc_check(cudaMemsetAsync(w.dE, 0, (size_t)B * enc::ED * 4, s), "memset dE"))) return rc;
    if ((rc = enc_check(cudaMemsetAsync(w.loss, 0, 4, s), "memset loss"))) return rc;
    if ((rc = enc_check(cudaMemsetAsync(grad, 0, (size_t)enc::N_PARAMS * 4, s), "memset grad"))) return rc;
    enc::enc_pair_loss<<<(P * 32 + 255) / 256, 256, 0, s>>>(w.E, ia, ib, y, weights, P, w.pred, w.loss, w.dE);
    rc = enc_backward(params, pts, off, len, B, T, nrm, w, grad, s);
    if (rc) return rc;
    if (loss) rc = enc_check(cudaMemcpyAsync(loss, w.loss, 4, cudaMemcpyDeviceToDevice, s), "copy loss");
    if (!rc && pred) rc = enc_check(cudaMemcpyAsync(pred, w.pred, (size_t)P * 4, cudaMemcpyDeviceToDevice, s), "copy pred");
    return rc;
}

int tsm_enc_loss_grad(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                      int32_t T, const float* nrm, const int32_t* ia, const int32_t* ib, const float* y, int32_t P,
                      void* workspace, float* grad, float* loss, float* pred, void* stream) {
    return tsm_enc_loss_grad_w(params, pts, off, len, B, T, nrm, ia, ib, y, nullptr, P, workspace, grad, loss, pred,
                               stream);
}

int tsm_enc_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr, float beta1,
                 float beta2, float eps, void* stream) {
    if (!params || !grad || !m || !v || step < 1) return tsm_internal_fail(TSM_EINVAL, "tsm_enc_adam: bad arguments");
    const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
    enc::enc_adam<<<(enc::N_PARAMS + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, enc::N_PARAMS, lr,
                                                                                 beta1, beta2, eps, bc1, bc2);
    return enc_check(cudaGetLastError(), "enc_adam launch");
}

int64_t tsm_enc_embed_workspace_bytes(int32_t B, int32_t T) {
    if (B < 1 || T < 1) return 0;
    return emb_layout(B, T, nullptr, nullptr) * 4;
}

int tsm_enc_embed_opts(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                       int32_t T, const float* nrm, void* workspace, float* emb, int64_t wait_cycles,
                       int32_t stall_step, void* stream) {
    int rc = enc_args(params, pts, off, len, B, T, nrm, workspace);
    if (rc) return rc;
    if (!emb) return tsm_internal_fail(TSM_EINVAL, "tsm_enc_embed: null output");
    if (wait_cycles < 1 || stall_step < -1) return tsm_internal_fail(TSM_EINVAL, "tsm_enc_embed_opts: bad wait limit or stall step");
    using namespace enc;
    EmbWs w;
    emb_layout(B, T, static_cast<float*>(workspace), &w);
    cudaStream_t s = (cudaStream_t)stream;
    const float4 n4 = make_float4(nrm[0], nrm[1], nrm[2], nrm[3]);
    if ((rc = enc_check(cudaMemsetAsync(w.status, 0, 4, s), "memset embed status"))) return rc;
    enc_round_bf16<<<(OFF_WO + 255) / 256, 256, 0, s>>>(params, w.wq);
    const int Bp = (B + TC_M - 1) / TC_M * TC_M;
    const int64_t tot = (int64_t)Bp * T;
    enc_conv_fwd_tc<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(reinterpret_cast<const float2*>(pts), off, len, B,
                                                                   Bp, T, n4, w.wq, params, w.Ab);
    rc = enc_check(cudaFuncSetAttribute(enc_gru_embed_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM),
                   "cudaFuncSetAttribute(enc_gru_embed_tc)");
    if (rc) return rc;
    enc_gru_embed_tc<<<Bp / TC_M, TC_THREADS, TC_SMEM, s>>>(w.Ab, len, B, T, w.wq, params, w.hl, w.status,
                                                            wait_cycles, stall_step);
    enc_head_fwd<<<(unsigned)((B + HEAD_B - 1) / HEAD_B), EO, 0, s>>>(w.hl, B, params, emb,
                                                                      reinterpret_cast<const float2*>(pts), off, len,
                                                                      n4, nullptr);
    return enc_check(cudaGetLastError(), "tsm_enc_embed launch");
}

int tsm_enc_embed(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                  int32_t T, const float* nrm, void* workspace, float* emb, void* stream) {
    return tsm_enc_embed_opts(params, pts, off, len, B, T, nrm, workspace, emb, enc::TC_WAIT_CYCLES, -1, stream);
}

int tsm_enc_train_status(void* workspace, int32_t* status, void* stream) {
    if (!workspace || !status) return tsm_internal_fail(TSM_EINVAL, "tsm_enc_train_status: null argument");
    int rc = enc_check(cudaStreamSynchronize((cudaStream_t)stream), "tsm_enc_train_status: synchronise");
    if (rc) return rc;
    if ((rc = enc_check(cudaMemcpy(status, workspace, 4, cudaMemcpyDeviceToHost), "tsm_enc_train_status: read")))
        return rc;
    if (*status == 0) return TSM_OK;
    if ((rc = enc_check(cudaMemset(workspace, 0, 4), "tsm_enc_train_status: clear"))) return rc;
    char b[256];
    snprintf(b, sizeof(b), "tsm_enc_loss_grad: a tensor-core wait ran out in the weight gradients (status %d%s); "
             "the gradients of the calls since the last check are incomplete", *status,
             (*status & 128) ? ": tensor memory not freed, reset the device" : "");
    return tsm_internal_fail(TSM_ETIMEOUT, b);
}

int tsm_enc_embed_status(const void* workspace, int32_t* status, void* stream) {
    if (!workspace || !status) return tsm_internal_fail(TSM_EINVAL, "tsm_enc_embed_status: null argument");
    int rc = enc_check(cudaStreamSynchronize((cudaStream_t)stream), "tsm_enc_embed_status: synchronise");
    if (rc) return rc;
    if ((rc = enc_check(cudaMemcpy(status, workspace, 4, cudaMemcpyDeviceToHost), "tsm_enc_embed_status: read")))
        return rc;
    if (*status == 0) return TSM_OK;
    char b[256];
    snprintf(b, sizeof(b), "tsm_enc_embed: a tensor-core wait ran out (status %d: %s%s%s); the affected embeddings are NaN",
             *status, (*status & enc::TC_ERR_COPY) ? "a_t copy " : "", (*status & enc::TC_ERR_MMA) ? "MMA " : "",
             (*status & enc::TC_ERR_TMEM_HELD) ? "tensor memory not freed: reset the device" : "");
    return tsm_internal_fail(TSM_ETIMEOUT, b);
}

}  // extern "C"
