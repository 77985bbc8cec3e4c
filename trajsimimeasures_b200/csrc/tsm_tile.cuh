// Tile kernels: one thread per trajectory pair, register-blocked DP.
//
// A thread sweeps its pair's DP matrix in horizontal blocks of R rows.  The R
// row points and the R current DP values live in registers; the block walks
// the columns left to right, one column per step, computing R cells per step.
// The bottom row of a block (one value per column) goes to a per-thread
// boundary row in shared memory, laid out [column][lane] so a warp's 32
// accesses hit 32 banks; the next block reads it as its top border.  Only
// the row points, the column points and this one boundary row are touched per
// step, so a cell costs its arithmetic and ~3/R memory operations.
//
// Pairs mode: every thread has its own pair (rows = longer trajectory,
// columns = shorter, which keeps the boundary row short).  Matrix mode: a CTA
// owns one query trajectory Q_i, staged once in shared memory as the columns,
// and each thread takes one database trajectory D_j as its rows; database
// trajectories are visited in the caller's order (sorted by length, the 32
// lanes of a warp have near-equal row counts and the column loop is uniform).
//
// Reference kernels replaced: core/dtw.py:10-53, core/edr.py:10-52,
// core/lcss.py:12-53, core/erp.py:10-91, core/discret_frechet.py:9-50 (one
// CUDA block per pair, 64 threads, an FP64 3-diagonal ring in global memory
// and a __syncthreads per anti-diagonal), core/hausdorff.py:12-93.
#pragma once

#include "tsm_device.cuh"

namespace tsm {

// Column accessors ----------------------------------------------------------

// Columns read from global memory (pairs mode): per-lane trajectories.
struct GlobalCols {
    const float2* __restrict__ p;
    __device__ __forceinline__ float2 pt(int j) const { return __ldg(p + j); }
};

// Columns staged in shared memory as float4 (x, y, gap distance, 0).
struct SmemCols {
    const float4* p;
    __device__ __forceinline__ float2 pt(int j) const {
        float4 v = p[j];
        return make_float2(v.x, v.y);
    }
    __device__ __forceinline__ float4 pt4(int j) const { return p[j]; }
};

// Gap distance of column j (ERP): staged value, or computed on the fly.
template <bool EXACT>
__device__ __forceinline__ float4 col4(const GlobalCols& c, int j, const KParams& p, bool gap) {
    float2 v = c.pt(j);
    return make_float4(v.x, v.y, gap ? gapdist<EXACT>(v.x, v.y, p) : 0.f, 0.f);
}
template <bool EXACT>
__device__ __forceinline__ float4 col4(const SmemCols& c, int j, const KParams&, bool) {
    return c.pt4(j);
}

// The DP of one pair.  rowp/nr: row trajectory; cols/nc: column trajectory;
// buf: this thread's boundary row (element j at buf[32*j]); srow/scol: ERP
// gap totals of the row/column trajectory.  Returns D(nr-1, nc-1).
template <int M, int R, bool EXACT, class Cols>
__device__ __forceinline__ float dp_pair(const float2* __restrict__ rowp, int nr, const Cols& cols,
                                         int nc, float* buf, const KParams& p, float srow, float scol) {
    using C = typename CellOf<M, EXACT>::type;
    if (nr <= 0 || nc <= 0) return 0.f;
    const float topb = C::topb(scol);
    for (int j = 0; j < nc; ++j) buf[32 * j] = topb;
    float dlast = 0.f;
    for (int rb = 0; rb < nr; rb += R) {
        float rx[R], ry[R], rg[R], D[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = min(rb + r, nr - 1);  // rows past the end repeat the last point
            const float2 q = __ldg(rowp + i);
            rx[r] = q.x;
            ry[r] = q.y;
            rg[r] = C::kGap ? gapdist<EXACT>(q.x, q.y, p) : 0.f;
            D[r] = C::rowb(srow);
        }
        float diag = (rb == 0) ? C::corner() : C::rowb(srow);
        float4 cn = col4<EXACT>(cols, 0, p, C::kGap);
        float tn = buf[0];
        for (int j = 0; j < nc; ++j) {
            const float4 c = cn;
            const float top = tn;
            const int jn = min(j + 1, nc - 1);  // prefetch the next column
            cn = col4<EXACT>(cols, jn, p, C::kGap);
            tn = buf[32 * jn];
            float up = top, dg = diag;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float left = D[r];
                const float d2 = d2f(rx[r], ry[r], c.x, c.y);
                const float nv = C::cell(dg, up, left, d2, rg[r], c.z, p.eps2);
                D[r] = nv;
                dg = left;
                up = nv;
            }
            buf[32 * j] = up;
            diag = top;
        }
        if (rb + R >= nr) {
            const int rr = nr - 1 - rb;
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r == rr) dlast = D[r];
        }
    }
    return dlast;
}

// Pairs mode ------------------------------------------------------------------
// Block = 32*W threads, dynamic shared memory = W*32*cap floats.
template <int M, int R, bool EXACT>
__global__ void __launch_bounds__(128) dp_pairs_kernel(
    const float2* __restrict__ pts, const int64_t* __restrict__ off_a, const int32_t* __restrict__ len_a,
    const int64_t* __restrict__ off_b, const int32_t* __restrict__ len_b, const int32_t* __restrict__ order,
    int64_t n, int cap, int max_len, KParams p, float* __restrict__ out, int32_t* __restrict__ counts) {
    extern __shared__ float smem[];
    float* buf = smem + (threadIdx.x >> 5) * (32 * cap) + (threadIdx.x & 31);
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t k = order ? (int64_t)order[t] : t;
    const int na = len_a[k], nb = len_b[k];
    const bool count = (M == EDR || M == LCSS) && counts != nullptr;
    if (na < 0 || nb < 0 || na > max_len || nb > max_len) {
        out[k] = CUDART_NAN_F;
        if (count) counts[k] = -1;
        return;
    }
    const float2* a = pts + off_a[k];
    const float2* b = pts + off_b[k];
    const bool a_rows = na >= nb;
    const float2* rowp = a_rows ? a : b;
    const float2* colp = a_rows ? b : a;
    const int nr = a_rows ? na : nb, nc = a_rows ? nb : na;
    if (nc > cap) return;  // both trajectories longer than cap: the wave kernel's pair
    float srow = 0.f, scol = 0.f;
    if constexpr (M == ERP) {
        srow = gapsum<EXACT>(rowp, nr, p);
        scol = gapsum<EXACT>(colp, nc, p);
    }
    const float dl = dp_pair<M, R, EXACT>(rowp, nr, GlobalCols{colp}, nc, buf, p, srow, scol);
    float o;
    int c;
    finalize<M>(dl, na, nb, o, c);
    out[k] = o;
    if (count) counts[k] = c;
}

// Matrix mode -----------------------------------------------------------------
// grid.x = nq * chunks; CTA (i, chunk) computes out[i, d_order[chunk*blockDim + t]].
// Dynamic shared memory = cap float4 columns + W*32*cap floats.
template <int M, int R, bool EXACT>
__global__ void __launch_bounds__(128) dp_matrix_kernel(
    const float2* __restrict__ q_pts, const int64_t* __restrict__ q_off, const int32_t* __restrict__ q_len,
    const float2* __restrict__ d_pts, const int64_t* __restrict__ d_off, const int32_t* __restrict__ d_len,
    const int32_t* __restrict__ d_order, int64_t nd, int chunks, int cap, int d_max_len, KParams p,
    float* __restrict__ out, int64_t ld, int32_t* __restrict__ counts) {
    extern __shared__ float smem[];
    __shared__ float s_scol;
    float4* cols = reinterpret_cast<float4*>(smem);
    float* buf = smem + 4 * cap + (threadIdx.x >> 5) * (32 * cap) + (threadIdx.x & 31);
    const int64_t qi = blockIdx.x / chunks;
    const int chunk = blockIdx.x % chunks;
    const int nq = q_len[qi];
    const bool qbad = nq < 0 || nq > cap;
    if (!qbad) {
        const float2* qp = q_pts + q_off[qi];
        for (int j = threadIdx.x; j < nq; j += blockDim.x) {
            const float2 v = __ldg(qp + j);
            cols[j] = make_float4(v.x, v.y, M == ERP ? gapdist<EXACT>(v.x, v.y, p) : 0.f, 0.f);
        }
    }
    __syncthreads();
    if constexpr (M == ERP) {
        if (threadIdx.x == 0 && !qbad) {
            double s = 0.0;
            for (int j = 0; j < nq; ++j) s = __dadd_rn(s, (double)cols[j].z);
            s_scol = (float)s;
        }
        __syncthreads();
    }
    const int64_t slot = (int64_t)chunk * blockDim.x + threadIdx.x;
    if (slot >= nd) return;
    const int64_t dj = d_order ? (int64_t)d_order[slot] : slot;
    const int ndl = d_len[dj];
    const bool count = (M == EDR || M == LCSS) && counts != nullptr;
    const int64_t o_idx = qi * ld + dj;
    if (qbad || ndl < 0 || ndl > d_max_len) {
        out[o_idx] = CUDART_NAN_F;
        if (count) counts[o_idx] = -1;
        return;
    }
    const float2* dp = d_pts + d_off[dj];
    float srow = 0.f, scol = 0.f;
    if constexpr (M == ERP) {
        srow = gapsum<EXACT>(dp, ndl, p);
        scol = s_scol;
    }
    const float dl = dp_pair<M, R, EXACT>(dp, ndl, SmemCols{cols}, nq, buf, p, srow, scol);
    float o;
    int c;
    finalize<M>(dl, nq, ndl, o, c);
    out[o_idx] = o;
    if (count) counts[o_idx] = c;
}

// Hausdorff -------------------------------------------------------------------
// Point-to-segment squared distance (core/hausdorff.py:12-45), restated on
// relative vectors a = p - s1, s = s2 - s1 (no absolute foot point, which
// would cost the FP32 path ~1e-3 relative):
//   u = (a.s) * inv(|s|^2);  t = 0 if u < 1e-5, else min(u, 1);  |a - t s|^2.
// u < 1e-5 -> the reference takes min(|p-s1|^2, |p-s2|^2) = |p-s1|^2 (t = 0);
// u > 1 -> |p-s2|^2 (t = 1).  A zero-length segment has inv = 0, so t = 0 and
// the result is |p - s1|^2 as in hausdorff.py:30-31.  mul.sat clamps u to
// [0, 1] (NaN to 0) in the multiply itself.
__device__ __forceinline__ float p2s(float px, float py, float s1x, float s1y, float sx, float sy,
                                     float inv) {
    const float ax = __fsub_rn(px, s1x), ay = __fsub_rn(py, s1y);
    const float dot = __fmaf_rn(ay, sy, __fmul_rn(ax, sx));
    float u;
    asm("mul.rn.sat.f32 %0, %1, %2;" : "=f"(u) : "f"(dot), "f"(inv));
    const float t = (u < 1e-5f) ? 0.f : u;
    const float ex = __fmaf_rn(-t, sx, ax), ey = __fmaf_rn(-t, sy, ay);
    return __fmaf_rn(ey, ey, __fmul_rn(ex, ex));
}

// max over the points of P of (min over the segments of T): hausdorff.py:48-69
// per point, then the max of the host reduction at :121 over valid points.
// The loop also visits T's last vertex as a zero-length segment (k = nt-1).
// In exact arithmetic that distance is never below the last segment's, so
// the min is the reference's; in FP32 it makes a point that coincides with
// the last vertex come out exactly 0 (u = dot * (1/len2) can round to 1-ulp,
// leaving a ~1e-11 residue), as every other vertex already does as the
// first endpoint of its outgoing segment.
template <int R, bool EXACT, class Segs>
__device__ __forceinline__ float directed_max(const float2* __restrict__ P, int np, const Segs& T, int nt) {
    if (nt < 2 || np <= 0) return 0.f;  // p2t_dist over zero segments is 0.0
    float m = 0.f;
    for (int pb = 0; pb < np; pb += R) {
        float px[R], py[R], best[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float2 q = __ldg(P + min(pb + r, np - 1));
            px[r] = q.x;
            py[r] = q.y;
            best[r] = CUDART_INF_F;
        }
        float2 s1 = T.pt(0);
        float2 s2n = T.pt(1);
        for (int k = 0; k < nt; ++k) {  // nt-1 segments + the last vertex
            const float2 s2 = s2n;
            s2n = T.pt(min(k + 2, nt - 1));
            const float sx = __fsub_rn(s2.x, s1.x), sy = __fsub_rn(s2.y, s1.y);
            const float len2 = __fmaf_rn(sy, sy, __fmul_rn(sx, sx));
            const float inv = (sx == 0.f && sy == 0.f) ? 0.f : trcp<EXACT>(len2);
#pragma unroll
            for (int r = 0; r < R; ++r) best[r] = fminf(best[r], p2s(px[r], py[r], s1.x, s1.y, sx, sy, inv));
            s1 = s2;
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (pb + r < np) m = fmaxf(m, best[r]);
    }
    return m;
}

template <int R, bool EXACT>
__global__ void __launch_bounds__(128) hausdorff_pairs_kernel(
    const float2* __restrict__ pts, const int64_t* __restrict__ off_a, const int32_t* __restrict__ len_a,
    const int64_t* __restrict__ off_b, const int32_t* __restrict__ len_b, const int32_t* __restrict__ order,
    int64_t n, int max_len, float* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t k = order ? (int64_t)order[t] : t;
    const int na = len_a[k], nb = len_b[k];
    if (na < 0 || nb < 0 || na > max_len || nb > max_len) {
        out[k] = CUDART_NAN_F;
        return;
    }
    const float2* a = pts + off_a[k];
    const float2* b = pts + off_b[k];
    const float m1 = directed_max<R, EXACT>(a, na, GlobalCols{b}, nb);
    const float m2 = directed_max<R, EXACT>(b, nb, GlobalCols{a}, na);
    out[k] = __fsqrt_rn(fmaxf(m1, m2));
}

template <int R, bool EXACT>
__global__ void __launch_bounds__(128) hausdorff_matrix_kernel(
    const float2* __restrict__ q_pts, const int64_t* __restrict__ q_off, const int32_t* __restrict__ q_len,
    const float2* __restrict__ d_pts, const int64_t* __restrict__ d_off, const int32_t* __restrict__ d_len,
    const int32_t* __restrict__ d_order, int64_t nd, int chunks, int q_max_len, int d_max_len,
    float* __restrict__ out, int64_t ld) {
    extern __shared__ float smem[];
    float4* cols = reinterpret_cast<float4*>(smem);
    const int64_t qi = blockIdx.x / chunks;
    const int chunk = blockIdx.x % chunks;
    const int nq = q_len[qi];
    const bool qbad = nq < 0 || nq > q_max_len;
    const float2* qp = q_pts + q_off[qi];
    if (!qbad)
        for (int j = threadIdx.x; j < nq; j += blockDim.x) {
            const float2 v = __ldg(qp + j);
            cols[j] = make_float4(v.x, v.y, 0.f, 0.f);
        }
    __syncthreads();
    const int64_t slot = (int64_t)chunk * blockDim.x + threadIdx.x;
    if (slot >= nd) return;
    const int64_t dj = d_order ? (int64_t)d_order[slot] : slot;
    const int ndl = d_len[dj];
    const int64_t o_idx = qi * ld + dj;
    if (qbad || ndl < 0 || ndl > d_max_len) {
        out[o_idx] = CUDART_NAN_F;
        return;
    }
    const float2* dp = d_pts + d_off[dj];
    const float m1 = directed_max<R, EXACT>(dp, ndl, SmemCols{cols}, nq);
    const float m2 = directed_max<R, EXACT>(qp, nq, GlobalCols{dp}, ndl);
    out[o_idx] = __fsqrt_rn(fmaxf(m1, m2));
}

}  // namespace tsm
