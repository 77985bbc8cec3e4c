// Persistent, length-bucketed scheduler for uneven paired batches.
//
// One launch processes a list of warp tasks drawn from a device queue:
//
//   kind 0  tile:   up to 32 pairs, one per lane (dp_pair: two skewed row
//                   blocks per thread, boundary row in shared memory); for
//                   pairs whose shorter side fits the tile capacity.
//   kind 5/1/6/2  group4 / group8 / group16 / wave: up to 32/G pairs, one
//                   per G-lane group (G = 4, 8, 16, 32), super-strip
//                   wavefront (group_task); the planner picks G per pair so
//                   that the longest pairs finish within a step budget.
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
// Group wavefront (G lanes per pair): see group_task.  G = 1 would be the
// tile kernel's one pair per lane.
#pragma once

#include <type_traits>

#include "tsm_tile.cuh"

namespace tsm {

enum TaskKind : int {
    TASK_TILE = 0,
    TASK_GROUP8 = 1,
    TASK_WAVE = 2,  // G = 32
    TASK_HAUSDORFF = 3,
    TASK_HAUSDORFF_WARP = 4,
    TASK_GROUP4 = 5,
    TASK_GROUP16 = 6
};

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

// Group tasks stage their column points in shared memory when they fit.
constexpr bool kGroupStageCols = true;

// One pair per G-lane group (G = 4, 8, 16 or 32); `first` .. `first + count`
// of the order list, group q of the warp takes pair first + q.  ring_base:
// this warp's shared memory, cap floats per group.
//
// Super-strips: the rows go in strips of G*R, lane u holding rows
// u*R .. u*R+R-1 of the strip in registers.  Lane u computes column j of the
// strip at step s = u + j, taking its top value from lane u-1 (computed at
// step s-1) by a width-G shuffle; lane 0 takes it from the ring, which holds
// the bottom row of the strip above (the top border before the first strip)
// and which lane G-1 overwrites column by column, G-1 steps behind lane 0's
// reads.  A strip takes nc + G - 1 steps.  The step loop has no per-lane
// state besides j: it is unrolled by two, with the R values of a lane
// alternating between two register arrays (no copies), and the column points
// are fetched two steps ahead into two registers that alternate the same way.
template <int M, int R, int G, bool EXACT>
__device__ __forceinline__ void group_task(const PairsArgs& A, int first, int count, float* ring_base, int cap) {
    using C = typename CellOf<M, EXACT>::type;
    constexpr unsigned kFull = 0xffffffffu;
    constexpr int SS = G * R;  // rows per super-strip
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
    float* const region = ring_base + grp * cap;
    float srow = 0.f, scol = 0.f;
    if constexpr (M == ERP) {
        if (valid && u == 0) {
            srow = gapsum<EXACT>(rowp, nr, p);
            scol = gapsum<EXACT>(colp, nc, p);
        }
        srow = __shfl_sync(kFull, srow, lane - u);
        scol = __shfl_sync(kFull, scol, lane - u);
    }
    const bool live = valid && nr > 0 && nc > 0;  // no loads at all for an empty trajectory
    // Shared-memory layout of a group's region (cap floats).  The column points
    // are staged there (float2) when every group of the warp has room: the step
    // loop then reads them from shared memory instead of global memory.  The
    // groups' copies start 2*G*grp floats apart modulo 32 banks, so the warp's
    // column loads (G consecutive points per group) take the minimum two
    // wavefronts; the rings (one float per column, read by lane 0 and written
    // by lane G-1 of every group at the same column) start grp floats further
    // apart, so those accesses fall in distinct banks too.
    const int col_skew = (2 * G * grp) & 31;
    const bool staged = kGroupStageCols && __all_sync(kFull, !live || col_skew + 3 * nc + grp <= cap);
    float2* scols = reinterpret_cast<float2*>(region + col_skew);
    float* ring = staged ? region + col_skew + 2 * nc + grp : region + (nc + grp <= cap ? grp : 0);
    const int n_ss = live ? (nr + SS - 1) / SS : 0;
    const int max_ss = __reduce_max_sync(kFull, n_ss);
    const int max_span = __reduce_max_sync(kFull, live ? nc + G - 1 : 0);
    const int last_u = ((nr - 1) % SS) / R;  // the lane and register of row nr-1 in the last strip
    const int last_r = (nr - 1) % R;
    float px[R], py[R];  // this lane's rows of the next strip
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const float2 q = live ? __ldg(rowp + min(u * R + r, nr - 1)) : make_float2(0.f, 0.f);
        px[r] = q.x;
        py[r] = q.y;
    }
    if (staged && live) {
        // asynchronous 8-byte copies, all in flight at once (with the row
        // loads above), then one wait
        for (int j = u; j < nc; j += G) {
            const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(scols + j));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(colp + j) : "memory");
        }
    }
    if (live)
        for (int j = u; j < nc; j += G) ring[j] = C::topb(scol, j);
    if (staged && live) asm volatile("cp.async.wait_all;" ::: "memory");
    float dlast = 0.f;
    __syncwarp();
    auto sweep = [&](auto staged_tag) {
        constexpr bool ST = decltype(staged_tag)::value;
        auto col = [&](int j) -> float2 {
            if constexpr (ST) return scols[j];
            else return __ldg(colp + j);
        };
        for (int ss = 0; ss < max_ss; ++ss) {
            const int row0 = ss * SS + u * R;
            const bool on = live && ss < n_ss && row0 < nr;
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
            // column j is used at step u + j: even steps take cE, odd steps cO
            const int je = u & 1, jo = je ^ 1;
            float2 cE = on ? col(min(je, nc - 1)) : make_float2(0.f, 0.f);
            float2 cO = on ? col(min(jo, nc - 1)) : make_float2(0.f, 0.f);
            auto step = [&](const float (&Din)[R], float (&Dout)[R], float2& cs, int s) {
                const float from_left = __shfl_up_sync(kFull, bottom, 1, G);
                const int j = s - u;
                if (on && (unsigned)j < (unsigned)nc) {
                    const float top = (u == 0) ? ring[j] : from_left;
                    const float2 c = cs;
                    cs = col(min(j + 2, nc - 1));
                    const float gc = C::kGap ? gapdist<EXACT>(c.x, c.y, p) : 0.f;
                    float up = top, dg = diag;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const float left = Din[r];
                        const float nv = C::cell(dg, up, left, d2nr<true>(rn[r], c), rg[r], gc, p.eps2);
                        Dout[r] = nv;
                        dg = left;
                        up = nv;
                    }
                    diag = top;
                    bottom = up;
                    if (u == G - 1) ring[j] = up;
                }
                __syncwarp();
            };
            int s = 0;
            for (; s + 1 < max_span; s += 2) {
                step(DA, DB, cE, s);
                step(DB, DA, cO, s + 1);
            }
            if (s < max_span) step(DA, DB, cE, s);
            if (on && ss == n_ss - 1 && u == last_u) {
                // the lane's last column nc-1 was step u + nc - 1: even steps wrote DB, odd ones DA
                const bool in_b = ((u + nc - 1) & 1) == 0;
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == last_r) dlast = in_b ? DB[r] : DA[r];
            }
        }
    };
    if (staged) sweep(std::true_type{});
    else sweep(std::false_type{});
    if (live && u == last_u) {
        float o;
        int c;
        finalize<M>(dlast, na, nb, o, c);
        A.out[M * A.out_stride + k] = o;
        if ((M == EDR || M == LCSS) && A.counts) A.counts[M * A.out_stride + k] = c;
    }
    // degenerate pairs (a zero length) have no steps: lane 0 of the group writes them
    if (valid && !live && u == 0) {
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
__device__ __forceinline__ void run_task(const int4 task, const PairsArgs& A, float* wsm, int warp_floats) {
    const int kind = task.x, m = task.y, first = task.z, count = task.w;
    // a G-lane group's ring holds warp_floats * G / 32 floats; a tile lane's boundary row warp_floats / 32
#define TSM_TASK(MM)                                                                                     \
    case MM:                                                                                             \
        if (kind == TASK_TILE) tile_task<MM, R, EXACT>(A, first, count, wsm, warp_floats / 32);           \
        else if (kind == TASK_GROUP4) group_task<MM, R, 4, EXACT>(A, first, count, wsm, warp_floats / 8);  \
        else if (kind == TASK_GROUP8) group_task<MM, R, 8, EXACT>(A, first, count, wsm, warp_floats / 4);  \
        else if (kind == TASK_GROUP16) group_task<MM, R, 16, EXACT>(A, first, count, wsm, warp_floats / 2); \
        else group_task<MM, R, 32, EXACT>(A, first, count, wsm, warp_floats);                            \
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
                                                       int* __restrict__ queue, int total_warps, int warp_floats) {
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31;
    float* wsm = smem + (threadIdx.x >> 5) * warp_floats;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(queue, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n_tasks) break;
        run_task<R, EXACT>(tasks[t], A, wsm, warp_floats);
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
