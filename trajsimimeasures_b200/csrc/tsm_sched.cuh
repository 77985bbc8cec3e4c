// Persistent, length-bucketed scheduler for uneven paired batches.
//
// One launch processes a list of warp tasks drawn from a device queue:
//
//   kind 0  tile:   up to 32 pairs, one per lane (dp_pair: two skewed row
//                   blocks per thread, boundary row in shared memory); for
//                   pairs whose shorter side fits the tile capacity.
//   kind 1  group8: up to 4 pairs, one per 8-lane group (group wavefront);
//                   medium pairs.
//   kind 2  wave:   1 pair per warp (group wavefront with G = 32); long pairs.
//   kind 3  hausdorff: up to 32 pairs, one per lane (no shared memory).
//   kind 4  hausdorff, 1 pair per warp: the lanes split the points of both
//                   trajectories, a warp max-reduction combines them.
//
// A task is {kind, measure, first, count}: pairs order[first .. first+count)
// of the caller's processing order.  Tasks are sorted by estimated cost,
// largest first, so the longest pairs start first and the short tasks fill
// the tail.  Warps take tasks with an atomicAdd on queue[0]; when a warp finds
// the queue empty it counts itself out on queue[1], and the last warp out
// resets both counters, so the next launch (or CUDA-graph replay) starts from
// zero without a memset.  The queue is the only scratch memory.
//
// Group wavefront (G lanes per pair): the rows of the pair are cut into
// strips of R rows dealt round-robin to the G lanes; local lane u computes
// column j of its round-m strip at local step m*T + u + j (T = max(ncols,
// G)).  The top value comes from lane u-1 by a width-G shuffle, lane 0 of a
// round reads lane G-1's previous round from the group's ring (one row of
// ncols floats in shared memory).  G = 1 would be the tile kernel; G = 32 the
// wave kernel.
#pragma once

#include "tsm_tile.cuh"

namespace tsm {

enum TaskKind : int { TASK_TILE = 0, TASK_GROUP8 = 1, TASK_WAVE = 2, TASK_HAUSDORFF = 3, TASK_HAUSDORFF_WARP = 4 };

// Everything a task needs besides its shared-memory slice.
struct PairsArgs {
    const float2* pts;
    const int64_t* off_a;
    const int32_t* len_a;
    const int64_t* off_b;
    const int32_t* len_b;
    const int32_t* order;
    int max_len;
    KParams p;
    float* out;
    int32_t* counts;
    int64_t out_stride;  // out[measure * out_stride + pair]
};

// One pair per G-lane group; `first` .. `first + count` of the order list,
// group q of the warp takes pair first + q.  ring: this warp's shared
// memory, cap floats per group.
template <int M, int R, int G, bool EXACT>
__device__ __forceinline__ void group_task(const PairsArgs& A, int first, int count, float* ring_base, int cap) {
    using C = typename CellOf<M, EXACT>::type;
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int u = lane % G;
    const KParams& p = A.p;
    bool valid = grp < count;
    int64_t k = 0;
    int na = 0, nb = 0;
    if (valid) {
        k = A.order[first + grp];
        na = A.len_a[k];
        nb = A.len_b[k];
        if (na < 0 || nb < 0 || na > A.max_len || nb > A.max_len || min(na, nb) > cap) {
            if (u == 0) {
                A.out[M * A.out_stride + k] = CUDART_NAN_F;
                if ((M == EDR || M == LCSS) && A.counts) A.counts[M * A.out_stride + k] = -1;
            }
            valid = false;
        }
    }
    const bool a_rows = na >= nb;
    const int nr = valid ? (a_rows ? na : nb) : 0;
    const int nc = valid ? (a_rows ? nb : na) : 0;
    const float2* rowp = valid ? A.pts + (a_rows ? A.off_a[k] : A.off_b[k]) : A.pts;
    const float2* colp = valid ? A.pts + (a_rows ? A.off_b[k] : A.off_a[k]) : A.pts;
    float* ring = ring_base + grp * cap;
    float srow = 0.f, scol = 0.f;
    if constexpr (M == ERP) {
        if (valid && u == 0) {
            srow = gapsum<EXACT>(rowp, nr, p);
            scol = gapsum<EXACT>(colp, nc, p);
        }
        srow = __shfl_sync(0xffffffffu, srow, lane - u);
        scol = __shfl_sync(0xffffffffu, scol, lane - u);
    }
    const int n_strips = (nr + R - 1) / R;
    const int T = nc > G ? nc : G;
    const int last = n_strips - 1;
    const int total = (valid && nr > 0 && nc > 0) ? (last / G) * T + (last % G) + nc : 0;  // live pairs only
    const int steps = __reduce_max_sync(0xffffffffu, total);
    const int res_u = valid && nr > 0 ? last % G : -1;
    const int res_r = (nr - 1) - last * R;

    const bool live = valid && nr > 0 && nc > 0;  // no loads at all for an empty trajectory
    float rx[R], ry[R], rg[R], D[R], px[R], py[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const float2 q = live ? __ldg(rowp + min(u * R + r, nr - 1)) : make_float2(0.f, 0.f);
        px[r] = q.x;
        py[r] = q.y;
        rx[r] = ry[r] = rg[r] = D[r] = 0.f;
    }
    float diag = 0.f, bottom = 0.f, dlast = 0.f;
    int j = -u, m = 0;
    float2 cnext = live ? __ldg(colp) : make_float2(0.f, 0.f);
    for (int t = 0; t < steps; ++t) {
        const float from_left = __shfl_up_sync(0xffffffffu, bottom, 1, G);
        const int g = G * m + u;
        const bool act = j >= 0 && j < nc && g < n_strips;
        if (act) {
            if (j == 0) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    rx[r] = px[r];
                    ry[r] = py[r];
                    rg[r] = C::kGap ? gapdist<EXACT>(px[r], py[r], p) : 0.f;
                    D[r] = C::rowb(srow, g * R + r);
                    const float2 q = __ldg(rowp + min((g + G) * R + r, nr - 1));
                    px[r] = q.x;
                    py[r] = q.y;
                }
                diag = (g == 0) ? C::corner() : C::rowb(srow, g * R - 1);
            }
            const float top = (u == 0) ? ((m == 0) ? C::topb(scol, j) : ring[j]) : from_left;
            const float2 c2 = cnext;
            cnext = __ldg(colp + min(j + 1, nc - 1));
            const float gc = C::kGap ? gapdist<EXACT>(c2.x, c2.y, p) : 0.f;
            float up = top, dg = diag;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float left = D[r];
                const float nv = C::cell(dg, up, left, d2f(rx[r], ry[r], c2.x, c2.y), rg[r], gc, p.eps2);
                D[r] = nv;
                dg = left;
                up = nv;
            }
            diag = top;
            bottom = up;
            if (u == G - 1) ring[j] = up;
            if (g == last && j == nc - 1) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == res_r) dlast = D[r];
            }
            if (j == nc - 1) cnext = __ldg(colp);  // next round restarts at column 0
        }
        if (++j == T) {
            j = 0;
            ++m;
        }
        __syncwarp();
    }
    if (valid && u == res_u) {
        float o;
        int c;
        finalize<M>(dlast, na, nb, o, c);
        A.out[M * A.out_stride + k] = o;
        if ((M == EDR || M == LCSS) && A.counts) A.counts[M * A.out_stride + k] = c;
    }
    // degenerate pairs (a zero length) have no steps: lane 0 of the group writes them
    if (valid && (nr == 0 || nc == 0) && u == 0) {
        float o;
        int c;
        finalize<M>(0.f, na, nb, o, c);
        A.out[M * A.out_stride + k] = o;
        if ((M == EDR || M == LCSS) && A.counts) A.counts[M * A.out_stride + k] = c;
    }
    __syncwarp();
}

// One pair per lane (the tile kernel's per-thread DP).
template <int M, int R, bool EXACT>
__device__ __forceinline__ void tile_task(const PairsArgs& A, int first, int count, float* wsm, int cap) {
    const int lane = threadIdx.x & 31;
    if (lane < count) {
        const int64_t k = A.order[first + lane];
        const int na = A.len_a[k], nb = A.len_b[k];
        const bool cnt = (M == EDR || M == LCSS) && A.counts;
        if (na < 0 || nb < 0 || na > A.max_len || nb > A.max_len || min(na, nb) > cap) {
            A.out[M * A.out_stride + k] = CUDART_NAN_F;
            if (cnt) A.counts[M * A.out_stride + k] = -1;
        } else {
            const bool a_rows = na >= nb;
            const float2* rowp = A.pts + (a_rows ? A.off_a[k] : A.off_b[k]);
            const float2* colp = A.pts + (a_rows ? A.off_b[k] : A.off_a[k]);
            const int nr = a_rows ? na : nb, nc = a_rows ? nb : na;
            float srow = 0.f, scol = 0.f;
            if constexpr (M == ERP) {
                srow = gapsum<EXACT>(rowp, nr, A.p);
                scol = gapsum<EXACT>(colp, nc, A.p);
            }
            const float dl = dp_pair<M, R, EXACT>(rowp, nr, GlobalCols{colp}, nc, wsm + lane, A.p, srow, scol);
            float o;
            int c;
            finalize<M>(dl, na, nb, o, c);
            A.out[M * A.out_stride + k] = o;
            if (cnt) A.counts[M * A.out_stride + k] = c;
        }
    }
    __syncwarp();
}

template <int R, bool EXACT>
__device__ __forceinline__ void hausdorff_task(const PairsArgs& A, int first, int count) {
    const int lane = threadIdx.x & 31;
    if (lane < count) {
        const int64_t k = A.order[first + lane];
        const int na = A.len_a[k], nb = A.len_b[k];
        float o;
        if (na < 0 || nb < 0 || na > A.max_len || nb > A.max_len) {
            o = CUDART_NAN_F;
        } else {
            const float2* a = A.pts + A.off_a[k];
            const float2* b = A.pts + A.off_b[k];
            o = __fsqrt_rn(fmaxf(directed_max2<R, EXACT>(GlobalCols{a}, na, b, nb),
                                 directed_max2<R, EXACT>(GlobalCols{b}, nb, a, na)));
        }
        A.out[HAUSDORFF * A.out_stride + k] = o;
    }
    __syncwarp();
}

// One long pair per warp: lane l takes point blocks l, l+32, ... of both
// directions; max is exact, so the result equals the one-thread result.
template <int R, bool EXACT>
__device__ __forceinline__ void hausdorff_warp_task(const PairsArgs& A, int first) {
    const int lane = threadIdx.x & 31;
    const int64_t k = A.order[first];
    const int na = A.len_a[k], nb = A.len_b[k];
    if (na < 0 || nb < 0 || na > A.max_len || nb > A.max_len) {
        if (lane == 0) A.out[HAUSDORFF * A.out_stride + k] = CUDART_NAN_F;
        __syncwarp();
        return;
    }
    const float2* a = A.pts + A.off_a[k];
    const float2* b = A.pts + A.off_b[k];
    float m = fmaxf(directed_max2<R, EXACT>(GlobalCols{a}, na, b, nb, lane * R, 32 * R),
                    directed_max2<R, EXACT>(GlobalCols{b}, nb, a, na, lane * R, 32 * R));
    // non-negative floats order like their bit patterns
    m = __int_as_float(__reduce_max_sync(0xffffffffu, __float_as_int(m)));
    if (lane == 0) A.out[HAUSDORFF * A.out_stride + k] = __fsqrt_rn(m);
    __syncwarp();
}

template <int R, bool EXACT>
__device__ __forceinline__ void run_task(const int4 task, const PairsArgs& A, float* wsm, int tile_cap, int g8_cap,
                                         int wave_cap) {
    const int kind = task.x, m = task.y, first = task.z, count = task.w;
#define TSM_TASK(MM)                                                                       \
    case MM:                                                                               \
        if (kind == TASK_TILE) tile_task<MM, R, EXACT>(A, first, count, wsm, tile_cap);     \
        else if (kind == TASK_GROUP8) group_task<MM, R, 8, EXACT>(A, first, count, wsm, g8_cap); \
        else group_task<MM, R, 32, EXACT>(A, first, count, wsm, wave_cap);                  \
        break;
    if (kind == TASK_HAUSDORFF) {
        hausdorff_task<R, EXACT>(A, first, count);
        return;
    }
    if (kind == TASK_HAUSDORFF_WARP) {
        hausdorff_warp_task<R, EXACT>(A, first);
        return;
    }
    switch (m) {
        TSM_TASK(DTW)
        TSM_TASK(EDR)
        TSM_TASK(LCSS)
        TSM_TASK(ERP)
        TSM_TASK(DFRECHET)
        default: break;
    }
#undef TSM_TASK
}

// Persistent kernel.  grid = resident CTAs; block = 32*W; dynamic shared
// memory = W * warp_floats floats.  queue: int[2] in global memory, zero
// before the first launch (self-resetting afterwards).
template <int R, bool EXACT>
__global__ void __launch_bounds__(128) dp_sched_kernel(PairsArgs A, const int4* __restrict__ tasks, int n_tasks,
                                                       int* __restrict__ queue, int total_warps, int warp_floats,
                                                       int tile_cap, int g8_cap, int wave_cap) {
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31;
    float* wsm = smem + (threadIdx.x >> 5) * warp_floats;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(queue, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n_tasks) break;
        run_task<R, EXACT>(tasks[t], A, wsm, tile_cap, g8_cap, wave_cap);
    }
    if (lane == 0) {
        // every warp has made its last fetch before it counts itself out, so
        // the last one out may reset the queue for the next launch
        const int done = atomicAdd(queue + 1, 1);
        if (done == total_warps - 1) {
            atomicExch(queue, 0);
            atomicExch(queue + 1, 0);
        }
    }
}

}  // namespace tsm
