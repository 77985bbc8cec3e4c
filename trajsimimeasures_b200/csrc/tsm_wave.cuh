// Wave kernel: one warp per long trajectory pair, a systolic wavefront over
// the warp's 32 lanes.
//
// The pair's rows (the longer trajectory) are cut into strips of R rows.
// Lane l owns strips l, l+32, l+64, ...: strip g = 32*m + l in round m.  Lane l
// computes column j of its round-m strip at step t = m*T + l + j, with the
// round period T = max(ncols, 32).  Within a round, strip g needs the bottom
// row of strip g-1 at the same column, which lane l-1 produced one step
// earlier: it arrives by __shfl_up_sync.  Lane 0 of round m needs the bottom
// row of strip 32m-1 (lane 31, round m-1), produced T-31 >= 1 steps earlier:
// lane 31 writes it to a one-row ring in shared memory and lane 0 reads it
// back, so consecutive rounds overlap with no pipeline drain.  The column
// trajectory is staged in shared memory once per pair; each lane keeps its R
// row points and R DP values in registers and prefetches the points of its
// next strip one round ahead.
//
// Per step and lane: R cells of arithmetic, one shuffle, one shared-memory
// column load, and (lanes 0 and 31) one ring access.  The only idle steps are
// the 31-step ramps at the start and end of a pair, which is why the tile
// kernel (one thread per pair) takes the short pairs and this kernel the
// pairs whose shorter side exceeds the tile kernel's boundary-row capacity.
#pragma once

#include "tsm_device.cuh"

namespace tsm {

// Per-warp shared memory of the wave kernel, in floats, for column capacity cap.
__host__ __device__ constexpr int wave_warp_floats(int cap) { return 4 * cap + cap; }

template <int M, int R, bool EXACT>
__global__ void __launch_bounds__(128) dp_wave_kernel(
    const float2* __restrict__ pts, const int64_t* __restrict__ off_a, const int32_t* __restrict__ len_a,
    const int64_t* __restrict__ off_b, const int32_t* __restrict__ len_b, const int32_t* __restrict__ order,
    int64_t n, int tile_cap, int cap, int max_len, KParams p, float* __restrict__ out,
    int32_t* __restrict__ counts) {
    using C = typename CellOf<M, EXACT>::type;
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    float4* cols = reinterpret_cast<float4*>(smem + w * wave_warp_floats(cap));
    float* ring = smem + w * wave_warp_floats(cap) + 4 * cap;
    const int64_t t_pair = (int64_t)blockIdx.x * (blockDim.x >> 5) + w;
    if (t_pair >= n) return;
    const int64_t k = order ? (int64_t)order[t_pair] : t_pair;
    const int na = len_a[k], nb = len_b[k];
    const bool count = (M == EDR || M == LCSS) && counts != nullptr;
    if (na < 0 || nb < 0 || na > max_len || nb > max_len) {
        if (lane == 0) {
            out[k] = CUDART_NAN_F;
            if (count) counts[k] = -1;
        }
        return;
    }
    const bool a_rows = na >= nb;
    const int nr = a_rows ? na : nb, nc = a_rows ? nb : na;
    if (nc <= tile_cap) return;  // the tile kernel's pair
    const float2* rowp = pts + (a_rows ? off_a[k] : off_b[k]);
    const float2* colp = pts + (a_rows ? off_b[k] : off_a[k]);

    for (int j = lane; j < nc; j += 32) {
        const float2 v = __ldg(colp + j);
        cols[j] = make_float4(v.x, v.y, C::kGap ? gapdist<EXACT>(v.x, v.y, p) : 0.f, 0.f);
    }
    __syncwarp();
    float srow = 0.f, scol = 0.f;
    if constexpr (M == ERP) {
        if (lane == 0) {
            double s = 0.0;
            for (int j = 0; j < nc; ++j) s = __dadd_rn(s, (double)cols[j].z);
            scol = (float)s;
            srow = gapsum<EXACT>(rowp, nr, p);
        }
        srow = __shfl_sync(0xffffffffu, srow, 0);
        scol = __shfl_sync(0xffffffffu, scol, 0);
    }

    const int n_strips = (nr + R - 1) / R;
    const int T = nc > 32 ? nc : 32;
    const int last_strip = n_strips - 1;
    const int total = (last_strip / 32) * T + (last_strip % 32) + nc;  // steps until the last cell
    const int res_lane = last_strip % 32;
    const int res_r = (nr - 1) - last_strip * R;

    float rx[R], ry[R], rg[R], D[R];
    float px[R], py[R];  // prefetched points of this lane's next strip
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const float2 q = __ldg(rowp + min(lane * R + r, nr - 1));
        px[r] = q.x;
        py[r] = q.y;
        rx[r] = ry[r] = rg[r] = D[r] = 0.f;
    }
    float diag = 0.f, bottom = 0.f, dlast = 0.f;
    for (int t = 0; t < total; ++t) {
        const int tau = t - lane;
        const int m = tau >= 0 ? tau / T : 0;
        const int j = tau - m * T;
        const int g = 32 * m + lane;
        const bool act = tau >= 0 && j < nc && g < n_strips;
        const float from_left = __shfl_up_sync(0xffffffffu, bottom, 1);
        if (act) {
            if (j == 0) {  // start strip g: take the prefetched points, prefetch strip g+32
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    rx[r] = px[r];
                    ry[r] = py[r];
                    rg[r] = C::kGap ? gapdist<EXACT>(px[r], py[r], p) : 0.f;
                    D[r] = C::rowb(srow, g * R + r);
                    const float2 q = __ldg(rowp + min((g + 32) * R + r, nr - 1));
                    px[r] = q.x;
                    py[r] = q.y;
                }
                diag = (g == 0) ? C::corner() : C::rowb(srow, g * R - 1);
            }
            float top;
            if (lane == 0) top = (m == 0) ? C::topb(scol, j) : ring[j];
            else top = from_left;
            const float4 c = cols[j];
            float up = top, dg = diag;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float left = D[r];
                const float nv = C::cell(dg, up, left, d2f(rx[r], ry[r], c.x, c.y), rg[r], c.z, p.eps2);
                D[r] = nv;
                dg = left;
                up = nv;
            }
            diag = top;
            bottom = up;
            if (lane == 31) ring[j] = up;
            if (g == last_strip && j == nc - 1) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == res_r) dlast = D[r];
            }
        }
        __syncwarp();
    }
    if (lane == res_lane) {
        float o;
        int c;
        finalize<M>(dlast, na, nb, o, c);
        out[k] = o;
        if (count) counts[k] = c;
    }
}

}  // namespace tsm
