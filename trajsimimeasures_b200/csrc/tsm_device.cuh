// Device-side building blocks shared by the sm_100a kernels: point distances,
// FP32 rounding-controlled arithmetic, and the per-measure DP cell policies.
//
// Every per-cell formula here has a line-for-line FP32 twin in
// oracle/tsm_oracle.c; explicit __f*_rn intrinsics keep nvcc from contracting
// or reassociating, so exact mode reproduces the twin bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace tsm {

enum Measure : int { DTW = 0, EDR = 1, LCSS = 2, ERP = 3, DFRECHET = 4, HAUSDORFF = 5 };

// Square root: IEEE (exact mode) or the hardware approximation.
template <bool EXACT>
__device__ __forceinline__ float tsqrt(float x) {
    if constexpr (EXACT) {
        return __fsqrt_rn(x);
    } else {
        float y;
        asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
        return y;
    }
}

// Reciprocal: IEEE (exact mode) or the hardware approximation.
template <bool EXACT>
__device__ __forceinline__ float trcp(float x) {
    if constexpr (EXACT) {
        return __frcp_rn(x);
    } else {
        float y;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
        return y;
    }
}

// Three-input min/max (PTX ISA 8.8, sm_100+): exact, one instruction.
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Squared point distance, fixed rounding: dx, dy rounded once each, then
// fma(dy, dy, dx*dx).  Symmetric in the two points (dx -> -dx is exact).
__device__ __forceinline__ float d2f(float ax, float ay, float bx, float by) {
    float dx = __fsub_rn(ax, bx);
    float dy = __fsub_rn(ay, by);
    return __fmaf_rn(dy, dy, __fmul_rn(dx, dx));
}

// The same squared distance with the row point held negated, nr = -r: the
// difference c + nr = -(r - c) is exactly the negated scalar difference
// (round-to-nearest is symmetric) and the squares do not see the sign, so
// the value is bit-identical to d2f(r.x, r.y, c.x, c.y).  PACKED: the
// difference is one f32x2 add instead of two scalar adds.  Measured on B200
// (same inputs, same outputs): the packed add is faster for every measure
// with per-lane global columns (paired batches, 5-15 %) and for DTW, EDR,
// LCSS and ERP with columns staged in shared memory (all-pairs, 0.5-4 %);
// discrete Frechet with shared-memory columns is 2 % faster with the scalar
// adds (kPackedSmem in the cell policies).
template <bool PACKED>
__device__ __forceinline__ float d2nr(float2 nr, float2 c) {
    float2 d;
    if constexpr (PACKED) d = __fadd2_rn(nr, c);
    else d = make_float2(__fadd_rn(nr.x, c.x), __fadd_rn(nr.y, c.y));
    return __fmaf_rn(d.y, d.y, __fmul_rn(d.x, d.x));
}

// Pairs mode: a pair whose longer side exceeds kHeavyRows and whose one-lane
// tile loop (passes of 2R rows, nc + 1 steps each) would exceed kTileStepMax
// steps goes to the wave kernel instead: its 32 lanes finish it sooner, and
// one such pair no longer holds a whole tile launch's tail.
constexpr int kHeavyRows = 256;
constexpr int kTileStepMax = 2048;
template <int R>
__host__ __device__ __forceinline__ bool tile_heavy(int nr, int nc) {
    return nr > kHeavyRows && nc > 0 && (int64_t)((nr + 2 * R - 1) / (2 * R)) * (nc + 1) > kTileStepMax;
}

// Kernel parameters (device copy of tsm_params, pre-digested on the host).
struct KParams {
    float eps2;        // (float)(eps*eps)
    float ghx, glx;    // ERP gap point x = ghx + glx (hi/lo split of the FP64 value)
    float ghy, gly;    // ERP gap point y = ghy + gly
};

// Distance of a point to the ERP gap point g = (ghx + glx, ghy + gly): the
// hi part is subtracted first (exact for points near g), then the lo part.
template <bool EXACT>
__device__ __forceinline__ float gapdist(float x, float y, const KParams& p) {
    float dx = __fsub_rn(__fsub_rn(x, p.ghx), p.glx);
    float dy = __fsub_rn(__fsub_rn(y, p.ghy), p.gly);
    return tsqrt<EXACT>(__fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// Total gap distance of a trajectory: FP32 gap distances summed in FP64 in
// index order, rounded once.
template <bool EXACT>
__device__ __forceinline__ float gapsum(const float2* __restrict__ t, int n, const KParams& p) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
        float2 q = t[i];
        s = __dadd_rn(s, (double)gapdist<EXACT>(q.x, q.y, p));
    }
    return (float)s;
}

// ---------------------------------------------------------------------------
// DP cell policies.  A cell (i, j) gets dg = D(i-1, j-1), up = D(i-1, j),
// left = D(i, j-1), the row point r and the column point c.  Borders:
//   corner = D(-1,-1), rowb = D(i,-1), topb = D(-1,j).
// "row"/"col" may be either trajectory of the pair: every policy is symmetric
// under transposition, so the cell values do not depend on the orientation.
// ---------------------------------------------------------------------------

// DTW: D = d + min(dg, up, left)  (core/dtw.py:38-41); borders +inf, corner 0.
template <bool EXACT>
struct DtwCell {
    static constexpr bool kGap = false;
    static constexpr bool kPackedSmem = true;  // f32x2 difference with shared-memory columns (see d2nr)
    __device__ __forceinline__ static float corner() { return 0.f; }
    __device__ __forceinline__ static float rowb(float /*srow*/, int /*i*/) { return CUDART_INF_F; }
    __device__ __forceinline__ static float topb(float /*scol*/, int /*j*/) { return CUDART_INF_F; }
    __device__ __forceinline__ static float cell(float dg, float up, float left, float d2,
                                                 float /*grow*/, float /*gcol*/, float /*eps2*/) {
        return __fadd_rn(tsqrt<EXACT>(d2), min3f(dg, up, left));
    }
    // split form (cell == comb(term(d2))): the local term alone, then the recurrence
    __device__ __forceinline__ static float term(float d2, float) { return tsqrt<EXACT>(d2); }
    __device__ __forceinline__ static float comb(float dg, float up, float left, float t, float, float) {
        return __fadd_rn(t, min3f(dg, up, left));
    }
};

// Discrete Frechet on squared distances: F = max(d2, min(dg, up, left))
// (core/discret_frechet.py:40-42); sqrt once at the end.
template <bool EXACT>
struct FrechetCell {
    static constexpr bool kGap = false;
    static constexpr bool kPackedSmem = false;  // f32x2 difference with shared-memory columns (see d2nr)
    __device__ __forceinline__ static float corner() { return 0.f; }
    __device__ __forceinline__ static float rowb(float, int) { return CUDART_INF_F; }
    __device__ __forceinline__ static float topb(float, int) { return CUDART_INF_F; }
    __device__ __forceinline__ static float cell(float dg, float up, float left, float d2,
                                                 float, float, float) {
        return fmaxf(d2, min3f(dg, up, left));
    }
    __device__ __forceinline__ static float term(float d2, float) { return d2; }
    __device__ __forceinline__ static float comb(float dg, float up, float left, float t, float, float) {
        return fmaxf(t, min3f(dg, up, left));
    }
};

// ERP: D = min(left + g(col), up + g(row), dg + d)  (core/erp.py:80-85);
// D(i,-1) = S(row trajectory), D(-1,j) = S(col trajectory), D(-1,-1) = 0.
template <bool EXACT>
struct ErpCell {
    static constexpr bool kGap = true;
    static constexpr bool kPackedSmem = true;  // f32x2 difference with shared-memory columns (see d2nr)
    __device__ __forceinline__ static float corner() { return 0.f; }
    __device__ __forceinline__ static float rowb(float srow, int) { return srow; }
    __device__ __forceinline__ static float topb(float scol, int) { return scol; }
    __device__ __forceinline__ static float cell(float dg, float up, float left, float d2,
                                                 float grow, float gcol, float) {
        return min3f(__fadd_rn(left, gcol), __fadd_rn(up, grow), __fadd_rn(dg, tsqrt<EXACT>(d2)));
    }
    __device__ __forceinline__ static float term(float d2, float) { return tsqrt<EXACT>(d2); }
    __device__ __forceinline__ static float comb(float dg, float up, float left, float t, float grow, float gcol) {
        return min3f(__fadd_rn(left, gcol), __fadd_rn(up, grow), __fadd_rn(dg, t));
    }
};

// EDR count: C = min(dg + sub, up + 1, left + 1), sub = (d2 < eps2) ? 0 : 1,
// every border 0 (core/edr.py:30,41-44).  The kernels carry the offset value
// F(i,j) = C(i,j) - (i+j) instead of C: then F = min(F_dg + sub - 2, F_up,
// F_left) (two additions fewer per cell), with borders F(i,-1) = 1 - i,
// F(-1,j) = 1 - j, F(-1,-1) = 2, and C(n1-1,n2-1) = F + n1 + n2 - 2.  All
// values are small integers, exact in FP32.
template <bool EXACT>
struct EdrCell {
    static constexpr bool kGap = false;
    static constexpr bool kPackedSmem = true;  // f32x2 difference with shared-memory columns (see d2nr)
    __device__ __forceinline__ static float corner() { return 2.f; }
    __device__ __forceinline__ static float rowb(float, int i) { return (float)(1 - i); }
    __device__ __forceinline__ static float topb(float, int j) { return (float)(1 - j); }
    __device__ __forceinline__ static float cell(float dg, float up, float left, float d2,
                                                 float, float, float eps2) {
        const float s = (d2 < eps2) ? -2.f : -1.f;
        return min3f(__fadd_rn(dg, s), up, left);
    }
    __device__ __forceinline__ static float term(float d2, float eps2) { return (d2 < eps2) ? -2.f : -1.f; }
    __device__ __forceinline__ static float comb(float dg, float up, float left, float t, float, float) {
        return min3f(__fadd_rn(dg, t), up, left);
    }
};

// LCSS count: if d2 < eps2: C = dg + 1 else max(up, left), borders 0
// (core/lcss.py:42-46).  For an LCS table dg + 1 >= max(up, left) and
// dg <= max(up, left), so this equals max(dg + match, up, left).
template <bool EXACT>
struct LcssCell {
    static constexpr bool kGap = false;
    static constexpr bool kPackedSmem = true;  // f32x2 difference with shared-memory columns (see d2nr)
    __device__ __forceinline__ static float corner() { return 0.f; }
    __device__ __forceinline__ static float rowb(float, int) { return 0.f; }
    __device__ __forceinline__ static float topb(float, int) { return 0.f; }
    __device__ __forceinline__ static float cell(float dg, float up, float left, float d2,
                                                 float, float, float eps2) {
        float m = (d2 < eps2) ? 1.f : 0.f;
        return max3f(__fadd_rn(dg, m), up, left);
    }
    __device__ __forceinline__ static float term(float d2, float eps2) { return (d2 < eps2) ? 1.f : 0.f; }
    __device__ __forceinline__ static float comb(float dg, float up, float left, float t, float, float) {
        return max3f(__fadd_rn(dg, t), up, left);
    }
};

template <int M, bool EXACT> struct CellOf;
template <bool E> struct CellOf<DTW, E> { using type = DtwCell<E>; };
template <bool E> struct CellOf<DFRECHET, E> { using type = FrechetCell<E>; };
template <bool E> struct CellOf<ERP, E> { using type = ErpCell<E>; };
template <bool E> struct CellOf<EDR, E> { using type = EdrCell<E>; };
template <bool E> struct CellOf<LCSS, E> { using type = LcssCell<E>; };

// Final value of a pair from D(n1-1, n2-1) (or the degenerate-length rules).
// n1, n2: the pair's lengths.  Writes the float result and the count.
template <int M>
__device__ __forceinline__ void finalize(float dlast, int n1, int n2, float& out, int& count) {
    count = 0;
    if constexpr (M == DTW || M == DFRECHET) {
        float v;
        if (n1 == 0 && n2 == 0) v = 0.f;
        else if (n1 == 0 || n2 == 0) v = CUDART_INF_F;
        else v = dlast;
        out = (M == DFRECHET) ? __fsqrt_rn(v) : v;
    } else if constexpr (M == ERP) {
        out = (n1 == 0 || n2 == 0) ? 0.f : dlast;
    } else if constexpr (M == EDR) {
        count = (n1 == 0 || n2 == 0) ? 0 : __float2int_rn(dlast) + n1 + n2 - 2;  // undo the (i+j) offset
        out = __fdiv_rn((float)count, (float)max(n1, n2));
    } else {  // LCSS
        count = (n1 == 0 || n2 == 0) ? 0 : __float2int_rn(dlast);
        out = __fsub_rn(1.f, __fdiv_rn((float)count, (float)min(n1, n2)));
    }
}

}  // namespace tsm
