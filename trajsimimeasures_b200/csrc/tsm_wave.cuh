// Wave kernel: one warp per long trajectory pair (pairs mode): the pairs
// whose shorter side exceeds the tile kernel's boundary-row capacity, and the
// pairs whose one-lane tile loop would be very long (tile_heavy).
//
// Persistent: a grid sized to the GPU's resident warps; in round i the nw
// warps take pairs i nw .. i nw + nw - 1 of the processing order, warp w the
// w-th of them in even rounds and the (nw-1-w)-th in odd ones (a snake, so
// that in the largest-first order no warp collects the largest pair of every
// round).  A warp tests 32 of its pairs at once (one per lane), keeps the wave
// pairs by a ballot and runs them one after another; every other pair is the
// tile kernel's.
//
// A pair's rows are swept in super-strips of 32 R rows: lane l holds rows
// l R .. l R + R - 1 of the strip in registers and computes column j at step
// l + j, taking its top value from lane l-1 (one step earlier) by a shuffle;
// lane 0 reads the bottom row of the strip above from a ring in shared
// memory, which lane 31 rewrites 31 steps behind.  The column points come
// through the L1 cache, loaded one step ahead (the warp reads 32 consecutive
// points per step); the ring is the only per-column shared memory.  The step
// loop is unrolled by two with the R values alternating between two register
// arrays, and the rows of the next strip are prefetched one strip ahead.  Per
// step and lane: R cells, one shuffle, one column load, and (lanes 0 and 31)
// one ring access; a strip costs nc + 31 steps.
#pragma once

#include "tsm_device.cuh"

namespace tsm {

// Per-warp shared memory of the wave kernel, in floats, for column capacity
// cap: the ring (one float per point of the longer trajectory, which also
// serves as scratch for the ERP gap sums).
__host__ __device__ constexpr int wave_warp_floats(int cap) { return cap; }

// DP of one wave pair (rows = the longer trajectory, nr >= nc >= 1) by the
// calling warp; writes out[k] (and counts[k]).
template <int M, int R, bool EXACT>
__device__ __forceinline__ void wave_pair(const float2* __restrict__ rowp, const float2* __restrict__ colp, int nr,
                                          int nc, int na, int nb, float* ring, int lane, const KParams& p,
                                          float* __restrict__ out_k, int32_t* __restrict__ count_k) {
    using C = typename CellOf<M, EXACT>::type;
    float srow = 0.f, scol = 0.f;
    if constexpr (M == ERP) {
        // column gap distances into the ring, summed in column order by lane 0
        for (int j = lane; j < nc; j += 32) {
            const float2 v = __ldg(colp + j);
            ring[j] = gapdist<EXACT>(v.x, v.y, p);
        }
        __syncwarp();
        if (lane == 0) {
            double s = 0.0;
            for (int j = 0; j < nc; ++j) s = __dadd_rn(s, (double)ring[j]);
            scol = (float)s;
            srow = gapsum<EXACT>(rowp, nr, p);
        }
        srow = __shfl_sync(0xffffffffu, srow, 0);
        scol = __shfl_sync(0xffffffffu, scol, 0);
        __syncwarp();
    }
    for (int j = lane; j < nc; j += 32) ring[j] = C::topb(scol, j);

    constexpr int SS = 32 * R;
    const int n_ss = (nr + SS - 1) / SS;
    const int span = nc + 31;
    const int last_u = ((nr - 1) % SS) / R, last_r = (nr - 1) % R;
    float px[R], py[R];  // this lane's rows of the next strip
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const float2 q = __ldg(rowp + min(lane * R + r, nr - 1));
        px[r] = q.x;
        py[r] = q.y;
    }
    float dlast = 0.f;
    __syncwarp();
    for (int ss = 0; ss < n_ss; ++ss) {
        const int row0 = ss * SS + lane * R;
        const bool on = row0 < nr;
        float2 rn[R];  // negated row points (d2nr)
        float rg[R], DA[R], DB[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            rn[r] = make_float2(-px[r], -py[r]);
            rg[r] = C::kGap ? gapdist<EXACT>(px[r], py[r], p) : 0.f;
            DA[r] = DB[r] = C::rowb(srow, row0 + r);
        }
        if (on && ss + 1 < n_ss) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float2 q = __ldg(rowp + min(row0 + SS + r, nr - 1));
                px[r] = q.x;
                py[r] = q.y;
            }
        }
        float diag = (row0 == 0) ? C::corner() : C::rowb(srow, row0 - 1);
        float bottom = 0.f;
        float2 cnext = __ldg(colp);  // column of step 0 (lane 0's; the other lanes are idle at step 0)
        auto step = [&](const float (&Din)[R], float (&Dout)[R], int s) {
            const float2 c = cnext;
            cnext = __ldg(colp + min(max(s + 1 - lane, 0), nc - 1));
            const float from_left = __shfl_up_sync(0xffffffffu, bottom, 1);
            const int j = s - lane;
            if (on && (unsigned)j < (unsigned)nc) {
                const float top = (lane == 0) ? ring[j] : from_left;
                const float cg = C::kGap ? gapdist<EXACT>(c.x, c.y, p) : 0.f;
                float up = top, dg = diag;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const float left = Din[r];
                    const float nv = C::cell(dg, up, left, d2nr<C::kPackedSmem>(rn[r], c), rg[r], cg, p.eps2);
                    Dout[r] = nv;
                    dg = left;
                    up = nv;
                }
                diag = top;
                bottom = up;
                if (lane == 31) ring[j] = up;
            }
            __syncwarp();
        };
        int s = 0;
        for (; s + 1 < span; s += 2) {
            step(DA, DB, s);
            step(DB, DA, s + 1);
        }
        if (s < span) step(DA, DB, s);
        if (on && ss == n_ss - 1 && lane == last_u) {
            // the lane's last column nc-1 was step lane + nc - 1: even steps wrote DB, odd ones DA
            const bool in_b = ((lane + nc - 1) & 1) == 0;
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r == last_r) dlast = in_b ? DB[r] : DA[r];
        }
    }
    if (lane == last_u) {
        float o;
        int c;
        finalize<M>(dlast, na, nb, o, c);
        *out_k = o;
        if (count_k) *count_k = c;
    }
    __syncwarp();  // the ring is free for the warp's next pair
}

template <int M, int R, bool EXACT>
__global__ void __launch_bounds__(128) dp_wave_kernel(
    const float2* __restrict__ pts, const int64_t* __restrict__ off_a, const int32_t* __restrict__ len_a,
    const int64_t* __restrict__ off_b, const int32_t* __restrict__ len_b, const int32_t* __restrict__ order,
    int64_t n, int tile_cap, int cap, int max_len, KParams p, float* __restrict__ out,
    int32_t* __restrict__ counts) {
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    float* ring = smem + w * wave_warp_floats(cap);
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + w;
    const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
    const bool count = (M == EDR || M == LCSS) && counts != nullptr;
    for (int64_t i0 = 0; i0 * nw < n; i0 += 32) {
        const int64_t i = i0 + lane;
        const int64_t t = i * nw + ((i & 1) ? nw - 1 - gw : gw);
        int64_t k = 0;
        bool mine = false;
        if (t < n) {
            k = order ? (int64_t)order[t] : t;
            const int na = len_a[k], nb = len_b[k];
            // pairs with bad lengths are flagged by the tile kernel
            if (na >= 0 && nb >= 0 && na <= max_len && nb <= max_len) {
                const int nr = max(na, nb), nc = min(na, nb);
                mine = nc > tile_cap || tile_heavy<R>(nr, nc);
            }
        }
        unsigned todo = __ballot_sync(0xffffffffu, mine);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const int64_t kk = __shfl_sync(0xffffffffu, k, src);
            const int na = len_a[kk], nb = len_b[kk];
            const bool a_rows = na >= nb;
            const float2* rowp = pts + (a_rows ? off_a[kk] : off_b[kk]);
            const float2* colp = pts + (a_rows ? off_b[kk] : off_a[kk]);
            wave_pair<M, R, EXACT>(rowp, colp, a_rows ? na : nb, a_rows ? nb : na, na, nb, ring, lane, p, out + kk,
                                   count ? counts + kk : nullptr);
        }
    }
}

}  // namespace tsm
