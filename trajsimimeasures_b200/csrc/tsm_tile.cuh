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

#include <type_traits>

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

// R consecutive rows of a pair's DP: their points (negated, for d2nr), their
// ERP gap distances and their current DP values, all in registers.
template <class C, int R, bool EXACT, bool PACKED = true>
struct RowBlock {
    float2 n[R];
    float g[R], D[R];

    // rows i0 .. i0+R-1; rows past the end repeat the last point (their
    // values are never read by a valid cell)
    __device__ __forceinline__ void load(const float2* __restrict__ rowp, int i0, int nr, float srow,
                                         const KParams& p) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float2 q = __ldg(rowp + min(i0 + r, nr - 1));
            n[r] = make_float2(-q.x, -q.y);
            g[r] = C::kGap ? gapdist<EXACT>(q.x, q.y, p) : 0.f;
            D[r] = C::rowb(srow, i0 + r);
        }
    }

    // One column: top = D(i0-1, j), diag = D(i0-1, j-1); D[] holds column j-1
    // on entry and column j on exit.  Returns the block's bottom value.
    __device__ __forceinline__ float step(const float4& c, float top, float diag, float eps2) {
        float up = top, dg = diag;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float left = D[r];
            const float nv = C::cell(dg, up, left, d2nr<PACKED>(n[r], make_float2(c.x, c.y)), g[r], c.z, eps2);
            D[r] = nv;
            dg = left;
            up = nv;
        }
        return up;
    }

    // Same column step, reading the previous column from Din and writing the
    // new one to Dout: alternating two arrays between steps needs no register
    // copies (an in-place update costs one move per row).
    __device__ __forceinline__ float step2(const float (&Din)[R], float (&Dout)[R], const float4& c, float top,
                                           float diag, float eps2) const {
        float up = top, dg = diag;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float left = Din[r];
            const float nv = C::cell(dg, up, left, d2nr<PACKED>(n[r], make_float2(c.x, c.y)), g[r], c.z, eps2);
            Dout[r] = nv;
            dg = left;
            up = nv;
        }
        return up;
    }

    // The local terms of the R cells at column point c (C::term: the square
    // root of the squared distance, or the match value), for step2t.
    __device__ __forceinline__ void terms(const float4& c, float (&T)[R], float eps2) const {
#pragma unroll
        for (int r = 0; r < R; ++r) T[r] = C::term(d2nr<PACKED>(n[r], make_float2(c.x, c.y)), eps2);
    }

    // step2 with the local terms computed beforehand (by terms(), a step
    // ahead): the same cells in the same order, so the same values.
    __device__ __forceinline__ float step2t(const float (&Din)[R], float (&Dout)[R], const float (&T)[R], float gcol,
                                            float top, float diag) const {
        float up = top, dg = diag;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float left = Din[r];
            const float nv = C::comb(dg, up, left, T[r], g[r], gcol);
            Dout[r] = nv;
            dg = left;
            up = nv;
        }
        return up;
    }

    __device__ __forceinline__ float pick(int rr) const {
        float v = 0.f;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (r == rr) v = D[r];
        return v;
    }
};

// The f32x2 form of the cell distance (d2nr): always with per-lane global
// columns, per measure (C::kPackedSmem) with shared-memory columns.
template <class C, class Cols>
constexpr bool kPacked() {
    return std::is_same<Cols, SmemCols>::value ? C::kPackedSmem : true;
}

// Lower-block-first form of the two-block pass (used by dp_pair for EDR and
// LCSS with shared-memory columns, where it was measured 3-5 % faster; the
// sqrt measures lose with it, since their first cells then wait on the
// column load).  At step j the column point and top value of column j are
// loaded first, the lower block computes column j-1 from operands already in
// registers while the load is in flight, then the upper block computes column
// j.  Every carried value then rotates through two registers only, which
// the two-column unrolled loop renames away.
template <int M, int R, bool EXACT, class Cols>
__device__ __forceinline__ float dp_pair_lower_first(const float2* __restrict__ rowp, int nr, const Cols& cols,
                                                     int nc, float* buf, const KParams& p, float srow, float scol) {
    using C = typename CellOf<M, EXACT>::type;
    for (int j = 0; j < nc; ++j) buf[32 * j] = C::topb(scol, j);
    float dlast = 0.f;
    int rb = 0;
    for (; nr - rb > R; rb += 2 * R) {
        RowBlock<C, R, EXACT, kPacked<C, Cols>()> hi, lo;
        hi.load(rowp, rb, nr, srow, p);
        lo.load(rowp, rb + R, nr, srow, p);
        float HA[R], HB[R], LA[R], LB[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            HA[r] = hi.D[r];
            LA[r] = lo.D[r];
        }
        float4 cp = col4<EXACT>(cols, 0, p, C::kGap);  // the lower block's column
        float udiag = buf[0];                          // the upper block's diagonal
        float hb1 = hi.step2(HA, HB, cp, udiag, (rb == 0) ? C::corner() : C::rowb(srow, rb - 1), p.eps2);
        float hb2 = C::rowb(srow, rb + R - 1);  // upper block's bottom values at columns j-1, j-2
        auto st = [&](const float (&Hi)[R], float (&Ho)[R], const float (&Li)[R], float (&Lo)[R], int j) {
            const float4 cj = col4<EXACT>(cols, j, p, C::kGap);
            const float tj = buf[32 * j];
            buf[32 * (j - 1)] = lo.step2(Li, Lo, cp, hb1, hb2, p.eps2);
            const float nb = hi.step2(Hi, Ho, cj, tj, udiag, p.eps2);
            hb2 = hb1;
            hb1 = nb;
            udiag = tj;
            cp = cj;
        };
        int j = 1;
        for (; j + 1 < nc; j += 2) {
            st(HB, HA, LA, LB, j);
            st(HA, HB, LB, LA, j + 1);
        }
        float lb;
        const int rr = nr - 1 - (rb + R);
        if (j < nc) {
            st(HB, HA, LA, LB, j);
            lb = lo.step2(LB, LA, cp, hb1, hb2, p.eps2);
            if (rb + 2 * R >= nr) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == rr) dlast = LA[r];
            }
        } else {
            lb = lo.step2(LA, LB, cp, hb1, hb2, p.eps2);
            if (rb + 2 * R >= nr) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == rr) dlast = LB[r];
            }
        }
        buf[32 * (nc - 1)] = lb;
    }
    if (rb < nr) {  // last rows (at most R): one block, ping-pong over column pairs
        RowBlock<C, R, EXACT, kPacked<C, Cols>()> blk;
        blk.load(rowp, rb, nr, srow, p);
        float DA[R], DB[R];
#pragma unroll
        for (int r = 0; r < R; ++r) DA[r] = blk.D[r];
        float diag = (rb == 0) ? C::corner() : C::rowb(srow, rb - 1);
        int j = 0;
        for (; j + 1 < nc; j += 2) {
            const float4 c0 = col4<EXACT>(cols, j, p, C::kGap);
            const float t0 = buf[32 * j];
            const float4 c1 = col4<EXACT>(cols, j + 1, p, C::kGap);
            const float t1 = buf[32 * (j + 1)];
            blk.step2(DA, DB, c0, t0, diag, p.eps2);
            blk.step2(DB, DA, c1, t1, t0, p.eps2);
            diag = t1;
        }
        const int rr = nr - 1 - rb;
        if (j < nc) {
            const float4 c0 = col4<EXACT>(cols, j, p, C::kGap);
            blk.step2(DA, DB, c0, buf[32 * j], diag, p.eps2);
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r == rr) dlast = DB[r];
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r == rr) dlast = DA[r];
        }
    }
    return dlast;
}

template <int M, class Cols>
struct LowerFirst {
    static constexpr bool value = false;
};
template <>
struct LowerFirst<EDR, SmemCols> {
    static constexpr bool value = true;
};
template <>
struct LowerFirst<LCSS, SmemCols> {
    static constexpr bool value = true;
};

// The DP of one pair, prefetching form (dp_pair's default).  rowp/nr: row
// trajectory; cols/nc: column trajectory; buf: this thread's boundary row
// (element j at buf[32*j]); srow/scol: ERP gap totals of the row/column
// trajectory.  Returns D(nr-1, nc-1).
//
// Rows go in passes of 2R: an upper and a lower block of R rows, the lower
// one column behind the upper.  At step j the upper block computes column j
// from the boundary row, the lower block column j-1 from the upper block's
// bottom values of columns j-1 and j-2 (kept in registers), and writes its
// own bottom value of column j-1 to the boundary row.  The two blocks' cell
// chains are independent within a step (two chains for the scheduler), and
// only one boundary-row load and store are paid per 2R cells.  Each block's
// values alternate between two register arrays, two columns per loop trip,
// so no register copies are needed.  A final pass of at most R rows uses one
// block.  (Packing the two blocks into FP32x2 instructions was measured
// slower: assembling the pairs around the scalar min/max costs more than the
// packed arithmetic saves.  Packing only the squared distances, with the row
// points held as (upper, lower) pairs and one column pair per step, was
// measured too: all-pairs 2000 x 2000 DTW 15.25 -> 19.1 ms, Frechet 12.37 ->
// 17.6 ms, ERP 18.86 -> 23.96 ms on B200, bit-identical results.)
template <int M, int R, bool EXACT, class Cols>
__device__ __forceinline__ float dp_pair_prefetch(const float2* __restrict__ rowp, int nr, const Cols& cols,
                                                  int nc, float* buf, const KParams& p, float srow, float scol,
                                                  int rb0 = 0) {
    using C = typename CellOf<M, EXACT>::type;
    if (rb0 == 0)  // else buf holds row rb0 - 1 (after four-block passes)
        for (int j = 0; j < nc; ++j) buf[32 * j] = C::topb(scol, j);
    float dlast = 0.f;
    int rb = rb0;
    for (; nr - rb > R; rb += 2 * R) {
        RowBlock<C, R, EXACT, kPacked<C, Cols>()> hi, lo;
        hi.load(rowp, rb, nr, srow, p);
        lo.load(rowp, rb + R, nr, srow, p);
        float HA[R], HB[R], LA[R], LB[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            HA[r] = hi.D[r];
            LA[r] = lo.D[r];
        }
        float top = buf[0];
        float4 c = col4<EXACT>(cols, 0, p, C::kGap);
        const int j1 = min(1, nc - 1);
        float4 cn = col4<EXACT>(cols, j1, p, C::kGap);
        float tn = buf[32 * j1];
        // step 0: the upper block's column 0 (HA -> HB); the lower block waits in LA
        float ub1 = hi.step2(HA, HB, c, top, (rb == 0) ? C::corner() : C::rowb(srow, rb - 1), p.eps2);
        float ub2 = C::rowb(srow, rb + R - 1), udiag = top;
        float4 cprev = c;
        // steps 1 .. nc-1: upper column j, lower column j-1
        auto pair_step = [&](const float (&Hi)[R], float (&Ho)[R], const float (&Li)[R], float (&Lo)[R], int j) {
            c = cn;
            top = tn;
            const int jn = min(j + 1, nc - 1);  // prefetch the next column
            cn = col4<EXACT>(cols, jn, p, C::kGap);
            tn = buf[32 * jn];
            const float nb = hi.step2(Hi, Ho, c, top, udiag, p.eps2);
            const float lb = lo.step2(Li, Lo, cprev, ub1, ub2, p.eps2);
            buf[32 * (j - 1)] = lb;
            udiag = top;
            ub2 = ub1;
            ub1 = nb;
            cprev = c;
        };
        int j = 1;
        for (; j + 1 < nc; j += 2) {
            pair_step(HB, HA, LA, LB, j);
            pair_step(HA, HB, LB, LA, j + 1);
        }
        // the lower block's last column; the final arrays depend on nc's parity
        float lb;
        const int rr = nr - 1 - (rb + R);
        if (j < nc) {
            pair_step(HB, HA, LA, LB, j);
            lb = lo.step2(LB, LA, cprev, ub1, ub2, p.eps2);
            if (rb + 2 * R >= nr) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == rr) dlast = LA[r];
            }
        } else {
            lb = lo.step2(LA, LB, cprev, ub1, ub2, p.eps2);
            if (rb + 2 * R >= nr) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == rr) dlast = LB[r];
            }
        }
        buf[32 * (nc - 1)] = lb;
    }
    if (rb < nr) {  // last rows (at most R): one block
        RowBlock<C, R, EXACT, kPacked<C, Cols>()> blk;
        blk.load(rowp, rb, nr, srow, p);
        float diag = (rb == 0) ? C::corner() : C::rowb(srow, rb - 1);
        float4 cn = col4<EXACT>(cols, 0, p, C::kGap);
        float tn = buf[0];
        for (int j = 0; j < nc; ++j) {
            const float4 c = cn;
            const float top = tn;
            const int jn = min(j + 1, nc - 1);
            cn = col4<EXACT>(cols, jn, p, C::kGap);
            tn = buf[32 * jn];
            blk.step(c, top, diag, p.eps2);
            diag = top;
        }
        dlast = blk.pick(nr - 1 - rb);
    }
    return dlast;
}

// The prefetching two-block pass with each cell's local term (C::term: for
// DTW and ERP the MUFU square root of the squared distance) computed one
// column step before the recurrence needs it.  At step j the upper block
// computes column j and the lower block column j - 1 from terms made at step
// j - 1; then the terms of step j + 1 are made: the lower block's at column j
// (point already in registers), the upper block's at column j + 1 (point
// loaded at the start of step j).  A cell's recurrence then no longer waits
// on its own square root.  Term arrays alternate between two per block like
// the value arrays.  The cells and their order along each dependency chain
// are those of dp_pair_prefetch, so the values are identical.
template <int M, int R, bool EXACT, class Cols>
__device__ __forceinline__ float dp_pair_ahead(const float2* __restrict__ rowp, int nr, const Cols& cols, int nc,
                                               float* buf, const KParams& p, float srow, float scol) {
    using C = typename CellOf<M, EXACT>::type;
    constexpr bool PK = kPacked<C, Cols>();
    const float e2 = p.eps2;
    for (int j = 0; j < nc; ++j) buf[32 * j] = C::topb(scol, j);
    float dlast = 0.f;
    int rb = 0;
    for (; nr - rb > R; rb += 2 * R) {
        RowBlock<C, R, EXACT, PK> hi, lo;
        hi.load(rowp, rb, nr, srow, p);
        lo.load(rowp, rb + R, nr, srow, p);
        float HA[R], HB[R], LA[R], LB[R], THA[R], THB[R], TLA[R], TLB[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            HA[r] = hi.D[r];
            LA[r] = lo.D[r];
        }
        float4 c = col4<EXACT>(cols, 0, p, C::kGap);
        float top = buf[0];
        const int j1 = min(1, nc - 1);
        float4 cn = col4<EXACT>(cols, j1, p, C::kGap);
        float tn = buf[32 * j1];
        // step 0: the upper block's column 0; then the terms of step 1
        hi.terms(c, THA, e2);
        float ub1 = hi.step2t(HA, HB, THA, c.z, top, (rb == 0) ? C::corner() : C::rowb(srow, rb - 1));
        lo.terms(c, TLA, e2);
        hi.terms(cn, THA, e2);
        float ub2 = C::rowb(srow, rb + R - 1), udiag = top, gprev = c.z;
        // steps 1 .. nc-1: upper column j, lower column j-1, then the next step's terms
        auto pair_step = [&](const float (&Hi)[R], float (&Ho)[R], const float (&Li)[R], float (&Lo)[R],
                             const float (&THi)[R], float (&THo)[R], const float (&TLi)[R], float (&TLo)[R],
                             int j) {
            c = cn;
            top = tn;
            const int jn = min(j + 1, nc - 1);
            cn = col4<EXACT>(cols, jn, p, C::kGap);
            tn = buf[32 * jn];
            const float nb = hi.step2t(Hi, Ho, THi, c.z, top, udiag);
            const float lb = lo.step2t(Li, Lo, TLi, gprev, ub1, ub2);
            buf[32 * (j - 1)] = lb;
            lo.terms(c, TLo, e2);
            hi.terms(cn, THo, e2);
            udiag = top;
            ub2 = ub1;
            ub1 = nb;
            gprev = c.z;
        };
        int j = 1;
        for (; j + 1 < nc; j += 2) {
            pair_step(HB, HA, LA, LB, THA, THB, TLA, TLB, j);
            pair_step(HA, HB, LB, LA, THB, THA, TLB, TLA, j + 1);
        }
        float lb;
        const int rr = nr - 1 - (rb + R);
        if (j < nc) {
            pair_step(HB, HA, LA, LB, THA, THB, TLA, TLB, j);
            lb = lo.step2t(LB, LA, TLB, gprev, ub1, ub2);
            if (rb + 2 * R >= nr) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == rr) dlast = LA[r];
            }
        } else {
            lb = lo.step2t(LA, LB, TLA, gprev, ub1, ub2);
            if (rb + 2 * R >= nr) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == rr) dlast = LB[r];
            }
        }
        buf[32 * (nc - 1)] = lb;
    }
    if (rb < nr) {  // last rows (at most R): one block, its terms a step ahead too
        RowBlock<C, R, EXACT, PK> blk;
        blk.load(rowp, rb, nr, srow, p);
        float DA[R], DB[R], TA[R], TB[R];
#pragma unroll
        for (int r = 0; r < R; ++r) DA[r] = blk.D[r];
        float diag = (rb == 0) ? C::corner() : C::rowb(srow, rb - 1);
        float4 c = col4<EXACT>(cols, 0, p, C::kGap);
        float top = buf[0];
        blk.terms(c, TA, e2);
        auto st = [&](const float (&Di)[R], float (&Do)[R], const float (&Ti)[R], float (&To)[R], int j) {
            const int jn = min(j + 1, nc - 1);
            const float4 cn = col4<EXACT>(cols, jn, p, C::kGap);
            const float tn = buf[32 * jn];
            blk.step2t(Di, Do, Ti, c.z, top, diag);
            blk.terms(cn, To, e2);
            diag = top;
            top = tn;
            c = cn;
        };
        int j = 0;
        for (; j + 1 < nc; j += 2) {
            st(DA, DB, TA, TB, j);
            st(DB, DA, TB, TA, j + 1);
        }
        const int rr = nr - 1 - rb;
        if (j < nc) {
            st(DA, DB, TA, TB, j);
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r == rr) dlast = DB[r];
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r == rr) dlast = DA[r];
        }
    }
    return dlast;
}

// Four-block pass (used for ERP, whose cells wait on a MUFU square root and a
// three-way min of sums): rows rb .. rb + 4R - 1 as four blocks of R rows, block k
// computing column s - k at step s, so a thread carries four independent
// dependency chains instead of two, and reads and writes the boundary row
// once per 4R rows.  Block k takes its top and diagonal values from the
// bottom values of block k - 1 at the previous two steps; block 0 from the
// boundary row; block 3 writes the boundary row.  Column results alternate
// between two arrays per block (even columns in A, odd in B: no register
// moves).  Needs nc >= 4; the cells and their order along each dependency
// chain are those of the two-block pass, so the values are identical.
// Returns the value of row nr - 1 at column nc - 1 when it lies in this pass.
template <class C, int R, bool EXACT, bool PK, class Cols>
__device__ __forceinline__ float quad_pass(const float2* __restrict__ rowp, int rb, int nr, const Cols& cols,
                                           int nc, float* buf, const KParams& p, float srow) {
    RowBlock<C, R, EXACT, PK> k0, k1, k2, k3;
    k0.load(rowp, rb, nr, srow, p);
    k1.load(rowp, rb + R, nr, srow, p);
    k2.load(rowp, rb + 2 * R, nr, srow, p);
    k3.load(rowp, rb + 3 * R, nr, srow, p);
    float A0[R], B0[R], A1[R], B1[R], A2[R], B2[R], A3[R], B3[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {  // column -1 (the row borders) in the odd arrays
        B0[r] = k0.D[r];
        B1[r] = k1.D[r];
        B2[r] = k2.D[r];
        B3[r] = k3.D[r];
    }
    const float e2 = p.eps2;
    // bottom values of blocks 0..2: at the last column computed (cur) and the one before (prv)
    float c0 = C::rowb(srow, rb + R - 1), p0 = c0;
    float c1 = C::rowb(srow, rb + 2 * R - 1), p1 = c1;
    float c2 = C::rowb(srow, rb + 3 * R - 1), p2 = c2;
    float d0 = (rb == 0) ? C::corner() : C::rowb(srow, rb - 1);  // block 0's diagonal: boundary row, column - 1
    // columns of the four blocks: cs0 = column s, cs1 = s - 1, ...
    float4 cs0 = col4<EXACT>(cols, 0, p, C::kGap), cs1 = cs0, cs2 = cs0, cs3 = cs0;
    float t0 = buf[0];
    // block 0 at column s (its result into O0 from I0); shifts its bottom values
    auto blk0 = [&](const float (&I)[R], float (&O)[R], int s) {
        const float nb = k0.step2(I, O, cs0, t0, d0, e2);
        d0 = t0;
        p0 = c0;
        c0 = nb;
    };
    auto blk1 = [&](const float (&I)[R], float (&O)[R]) {
        const float nb = k1.step2(I, O, cs1, c0, p0, e2);
        p1 = c1;
        c1 = nb;
    };
    auto blk2 = [&](const float (&I)[R], float (&O)[R]) {
        const float nb = k2.step2(I, O, cs2, c1, p1, e2);
        p2 = c2;
        c2 = nb;
    };
    auto blk3 = [&](const float (&I)[R], float (&O)[R], int j) { buf[32 * j] = k3.step2(I, O, cs3, c2, p2, e2); };
    // next step's columns: shift, and load column s for block 0 (and its top value)
    auto advance = [&](int s) {
        cs3 = cs2;
        cs2 = cs1;
        cs1 = cs0;
        if (s < nc) {
            cs0 = col4<EXACT>(cols, s, p, C::kGap);
            t0 = buf[32 * s];
        }
    };
    // prologue: steps 0, 1, 2 (blocks below start one step later each); bottom-up within a step
    blk0(B0, A0, 0);
    advance(1);
    blk1(B1, A1);
    blk0(A0, B0, 1);
    advance(2);
    blk2(B2, A2);
    blk1(A1, B1);
    blk0(B0, A0, 2);
    advance(3);
    // steady state: steps s = 3 .. nc - 1, all four blocks; s odd: blocks 0, 2 write B, blocks 1, 3 write A
    int s = 3;
    for (; s + 1 < nc; s += 2) {
        blk3(B3, A3, s - 3);
        blk2(A2, B2);
        blk1(B1, A1);
        blk0(A0, B0, s);
        advance(s + 1);
        blk3(A3, B3, s - 2);
        blk2(B2, A2);
        blk1(A1, B1);
        blk0(B0, A0, s + 1);
        advance(s + 2);
    }
    const int rr = nr - 1 - (rb + 3 * R);  // the last row's index in block 3 when this pass holds it
    float dlast = 0.f;
    if (s < nc) {  // one more full step (s odd), then the drain from an even step
        blk3(B3, A3, s - 3);
        blk2(A2, B2);
        blk1(B1, A1);
        blk0(A0, B0, s);
        advance(s + 1);
        ++s;
        // drain: s = nc (even): block 3 column nc - 3 (odd -> B), block 2 nc - 2 (even -> A), block 1 nc - 1 (odd -> B)
        blk3(A3, B3, s - 3);
        blk2(B2, A2);
        blk1(A1, B1);
        advance(s + 1);
        blk3(B3, A3, s - 2);  // column nc - 2 (even)
        blk2(A2, B2);         // column nc - 1 (odd)
        advance(s + 2);
        blk3(A3, B3, s - 1);  // column nc - 1 (odd)
        if (rr < R) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r == rr) dlast = B3[r];
        }
    } else {  // s = nc (odd): block 3 column nc - 3 (even -> A), block 2 nc - 2 (odd -> B), block 1 nc - 1 (even -> A)
        blk3(B3, A3, s - 3);
        blk2(A2, B2);
        blk1(B1, A1);
        advance(s + 1);
        blk3(A3, B3, s - 2);  // column nc - 2 (odd)
        blk2(B2, A2);         // column nc - 1 (even)
        advance(s + 2);
        blk3(B3, A3, s - 1);  // column nc - 1 (even)
        if (rr < R) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r == rr) dlast = A3[r];
        }
    }
    return dlast;
}

template <int M, int R, bool EXACT, class Cols>
__device__ __forceinline__ float dp_pair_quad(const float2* __restrict__ rowp, int nr, const Cols& cols, int nc,
                                              float* buf, const KParams& p, float srow, float scol) {
    using C = typename CellOf<M, EXACT>::type;
    if (nc < 4 || nr <= 3 * R) return dp_pair_prefetch<M, R, EXACT>(rowp, nr, cols, nc, buf, p, srow, scol);
    for (int j = 0; j < nc; ++j) buf[32 * j] = C::topb(scol, j);
    int rb = 0;
    float dlast = 0.f;
    for (; nr - rb > 3 * R; rb += 4 * R)
        dlast = quad_pass<C, R, EXACT, kPacked<C, Cols>()>(rowp, rb, nr, cols, nc, buf, p, srow);
    if (rb >= nr) return dlast;
    return dp_pair_prefetch<M, R, EXACT>(rowp, nr, cols, nc, buf, p, srow, scol, rb);
}

// The DP of one pair, with shared-memory columns (the matrix kernels): the
// terms-ahead pass for EDR (kAheadMask), the lower-block-first pass for LCSS,
// the four-block pass for ERP (kQuadPass), else the prefetching one; with
// per-lane global columns (paired and scheduled kernels) the prefetching one.
// Measured on B200, all-pairs 2000 x 2000: ERP 18.84 -> 18.05 ms with four
// blocks of 8 rows; DTW 15.29 -> 15.69 ms (four blocks of 8) and 16.17 ms (of
// 4), so DTW keeps two blocks.  The four-block pass stays out of the scheduled
// kernel: compiled into its ERP tile tasks it raised the whole kernel from 127
// to 190 registers, and the 500k-pair uneven batch from 5.1 to 6.5 ms.
#ifndef TSM_QUAD_PASS
#define TSM_QUAD_PASS 1
#endif
constexpr bool kQuadPass = TSM_QUAD_PASS != 0;
// Measures (bit M) whose matrix kernels run dp_pair_ahead.  Measured on B200,
// all-pairs 2000 x 2000, every measure bit-identical to its default pass:
// EDR 14.79 -> 13.91 ms (its match terms a step ahead beat the lower-first
// pass); slower for the others: DTW 15.17 -> 16.02, LCSS 12.49 -> 12.87, ERP
// 18.05 -> 19.84 (against the four-block pass), Frechet 12.33 -> 12.94 ms,
// and slower still with blocks of 16 rows.
#ifndef TSM_AHEAD_MASK
#define TSM_AHEAD_MASK (1 << EDR)
#endif
constexpr int kAheadMask = TSM_AHEAD_MASK;
template <int M, int R, bool EXACT, class Cols>
__device__ __forceinline__ float dp_pair(const float2* __restrict__ rowp, int nr, const Cols& cols,
                                         int nc, float* buf, const KParams& p, float srow, float scol) {
    if (nr <= 0 || nc <= 0) return 0.f;
    if constexpr (kAheadMask & (1 << M) && std::is_same<Cols, SmemCols>::value) {
        return dp_pair_ahead<M, R, EXACT>(rowp, nr, cols, nc, buf, p, srow, scol);
    } else if constexpr (LowerFirst<M, Cols>::value) {
        return dp_pair_lower_first<M, R, EXACT>(rowp, nr, cols, nc, buf, p, srow, scol);
    } else if constexpr (kQuadPass && M == ERP && R <= 8 && std::is_same<Cols, SmemCols>::value) {
        // (16 rows: four blocks spill)
        return dp_pair_quad<M, R, EXACT>(rowp, nr, cols, nc, buf, p, srow, scol);
    } else {
        return dp_pair_prefetch<M, R, EXACT>(rowp, nr, cols, nc, buf, p, srow, scol);
    }
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
    if (nc > cap || tile_heavy<R>(nr, nc)) return;  // the wave kernel's pair
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
// grid.x = nq * chunks; CTA (s, chunk) computes out[i, d_order[chunk*blockDim + t]]
// for the query i = q_order[s] (i = s without an order).
// Symmetric mode (sym == 1; the query set is the database set and q_order ==
// d_order): only the slots at or after the query's own sorted position s are
// computed (the upper triangle in sorted order), and each value is written to
// out[i, j] and out[j, i]; CTAs wholly below the diagonal exit at once.
// Gather mode (sym == 2): d_order holds one row of nd database indices per
// query i (row i, whatever the processing order q_order), and slot t of query i
// goes to out[i, t].  A database index outside
// 0..d_total-1 gives NaN (count -1).
// Dynamic shared memory = cap float4 columns + W*32*cap floats.

template <int M, int R, bool EXACT>
__global__ void __launch_bounds__(128) dp_matrix_kernel(
    const float2* __restrict__ q_pts, const int64_t* __restrict__ q_off, const int32_t* __restrict__ q_len,
    const int32_t* __restrict__ q_order, const float2* __restrict__ d_pts, const int64_t* __restrict__ d_off,
    const int32_t* __restrict__ d_len, const int32_t* __restrict__ d_order, int64_t nd, int64_t d_total, int chunks,
    int sym, int cap, int d_max_len, KParams p, float* __restrict__ out, int64_t ld, int32_t* __restrict__ counts) {
    extern __shared__ float smem[];
    __shared__ float s_scol;
    float4* cols = reinterpret_cast<float4*>(smem);
    float* buf = smem + 4 * cap + (threadIdx.x >> 5) * (32 * cap) + (threadIdx.x & 31);
    const int64_t qs = blockIdx.x / chunks;
    const int chunk = blockIdx.x % chunks;
    if (sym == 1 && (int64_t)(chunk + 1) * blockDim.x <= qs) return;  // below the diagonal (uniform per CTA)
    const int64_t qi = q_order ? (int64_t)q_order[qs] : qs;
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
    if (slot >= nd || (sym == 1 && slot < qs)) return;
    const int64_t dj = d_order ? (int64_t)d_order[(sym == 2 ? qi * nd : 0) + slot] : slot;
    const bool dbad = dj < 0 || dj >= d_total;
    const int ndl = dbad ? -1 : d_len[dj];
    const bool count = (M == EDR || M == LCSS) && counts != nullptr;
    const int64_t o_idx = qi * ld + (sym == 2 ? slot : dj), t_idx = dj * ld + qi;
    const bool mirror = sym == 1 && dj != qi;
    if (qbad || dbad || ndl < 0 || ndl > d_max_len) {
        out[o_idx] = CUDART_NAN_F;
        if (count) counts[o_idx] = -1;
        if (mirror) {
            out[t_idx] = CUDART_NAN_F;
            if (count) counts[t_idx] = -1;
        }
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
    if (mirror) {
        out[t_idx] = o;
        if (count) counts[t_idx] = c;
    }
}

// Hausdorff -------------------------------------------------------------------
// Point-to-segment squared distance (core/hausdorff.py:12-45), restated on
// relative vectors a = p - s1, s = s2 - s1 (no absolute foot point, which
// would cost the FP32 path ~1e-3 relative):
//   u = (a.s) * inv(|s|^2);  t = 0 if u < 1e-5, else min(u, 1);  |a - t s|^2.
// u < 1e-5 -> the reference takes min(|p-s1|^2, |p-s2|^2) = |p-s1|^2 (t = 0);
// u > 1 -> |p-s2|^2 (t = 1).  A zero-length segment has inv = 0, so t = 0 and
// the result is |p - s1|^2 as in hausdorff.py:30-31.  mul.sat clamps u to
// [0, 1] (NaN to 0) in the multiply itself.  This scalar form is the
// definition (and the oracle twin's formula); the kernels use p2s_pair.
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

// The kernels evaluate p2s two segments at a time in FP32x2: for a point p
// and consecutive segments k, k+1 of one trajectory, the vector quantities
// (a, dot, foot offset, squared distance) are f32x2 pairs, while the clamp
// u -> t and the running min stay scalar (f32x2 has no saturation and no
// min).  Segments are kept negated (-s1, -s, -1/|s|^2), so a - b becomes an
// f32x2 add and the foot a - t s an f32x2 fma: every value is bit-identical
// to p2s above, and min(best, d_k, d_k+1) is one three-input min.  Per two
// evaluations: 8 f32x2 + 2 scalar FMA-pipe and 5 ALU instructions, against
// 18 + 6 for two scalar p2s calls.
struct SegPair {
    float2 n1x, n1y;  // -s1 of segments k, k+1
    float2 nsx, nsy;  // -(s2 - s1)
    float2 ninv;      // -1/|s|^2 (0 for a zero-length segment)
};

// p2s of one point (pair-broadcast px2 = (px, px), py2) against segments
// k and k+1, folded into best.
__device__ __forceinline__ float p2s_pair(float2 px2, float2 py2, const SegPair& g, float best) {
    const float2 ax = __fadd2_rn(px2, g.n1x), ay = __fadd2_rn(py2, g.n1y);
    const float2 ndot = __ffma2_rn(ay, g.nsy, __fmul2_rn(ax, g.nsx));  // -(a.s)
    float u0, u1;
    asm("mul.rn.sat.f32 %0, %1, %2;" : "=f"(u0) : "f"(ndot.x), "f"(g.ninv.x));
    asm("mul.rn.sat.f32 %0, %1, %2;" : "=f"(u1) : "f"(ndot.y), "f"(g.ninv.y));
    const float2 t = make_float2((u0 < 1e-5f) ? 0.f : u0, (u1 < 1e-5f) ? 0.f : u1);
    const float2 ex = __ffma2_rn(t, g.nsx, ax), ey = __ffma2_rn(t, g.nsy, ay);
    const float2 d2 = __ffma2_rn(ey, ey, __fmul2_rn(ex, ex));
    return min3f(best, d2.x, d2.y);
}

// Segment k of trajectory T (k = n-1: the last vertex as a zero-length
// segment), negated, into lane `hi` of a SegPair.
template <bool EXACT>
__device__ __forceinline__ void seg_lane(SegPair& g, int hi, float2 s1, float2 s2) {
    const float sx = __fsub_rn(s2.x, s1.x), sy = __fsub_rn(s2.y, s1.y);
    const float len2 = __fmaf_rn(sy, sy, __fmul_rn(sx, sx));
    const float inv = (sx == 0.f && sy == 0.f) ? 0.f : trcp<EXACT>(len2);
    if (hi) {
        g.n1x.y = -s1.x; g.n1y.y = -s1.y; g.nsx.y = -sx; g.nsy.y = -sy; g.ninv.y = -inv;
    } else {
        g.n1x.x = -s1.x; g.n1y.x = -s1.y; g.nsx.x = -sx; g.nsy.x = -sy; g.ninv.x = -inv;
    }
}

// Staged query segments for the packed matrix kernel: pair j holds segments
// 2j and 2j+1 of the query (the last vertex counted as segment nq-1; an odd
// count repeats it), as float4 (n1x, n1y) + float4 (nsx, nsy) + float2 ninv.
__device__ __forceinline__ SegPair staged_pair(const float4* A, const float4* B, const float2* C, int j) {
    const float4 a = A[j], b = B[j];
    SegPair g;
    g.n1x = make_float2(a.x, a.y);
    g.n1y = make_float2(a.z, a.w);
    g.nsx = make_float2(b.x, b.y);
    g.nsy = make_float2(b.z, b.w);
    g.ninv = C[j];
    return g;
}

// directed_max with P from global memory and T staged as segment pairs.
template <int R>
__device__ __forceinline__ float directed_max_staged2(const float2* __restrict__ P, int np, const float4* A,
                                                      const float4* B, const float2* C, int nq) {
    if (nq < 2 || np <= 0) return 0.f;
    const int npair = (nq + 1) >> 1;
    float m = 0.f;
    for (int pb = 0; pb < np; pb += R) {
        float2 px[R], py[R];
        float best[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float2 q = __ldg(P + min(pb + r, np - 1));
            px[r] = make_float2(q.x, q.x);
            py[r] = make_float2(q.y, q.y);
            best[r] = CUDART_INF_F;
        }
        for (int j = 0; j < npair; ++j) {
            const SegPair g = staged_pair(A, B, C, j);
#pragma unroll
            for (int r = 0; r < R; ++r) best[r] = p2s_pair(px[r], py[r], g, best[r]);
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (pb + r < np) m = fmaxf(m, best[r]);
    }
    return m;
}

// max over the points of P of (min over the segments of T), hausdorff.py:48-69
// per point, then the max of the host reduction at :121 over valid points.
// T's segment pairs are built on the fly from global memory.  The loop also
// visits T's last vertex as a zero-length segment: in exact arithmetic that
// distance is never below the last segment's, so the min is the reference's;
// in FP32 it makes a point that coincides with the last vertex come out
// exactly 0 (u = dot * (1/len2) can round to 1-ulp, leaving a ~1e-11
// residue), as every other vertex already does as the first endpoint of its
// outgoing segment.  Points pb0, pb0 + pstride, ... (blocks of R) of P: a
// thread takes all points (pb0 = 0, pstride = R) or, in a warp-per-pair
// task, every 32nd block.
template <int R, bool EXACT, class Pts>
__device__ __forceinline__ float directed_max2(const Pts& P, int np, const float2* __restrict__ T, int nt,
                                               int pb0 = 0, int pstride = R) {
    if (nt < 2 || np <= 0) return 0.f;  // p2t_dist over zero segments is 0.0
    float m = 0.f;
    for (int pb = pb0; pb < np; pb += pstride) {
        float2 px[R], py[R];
        float best[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float2 q = P.pt(min(pb + r, np - 1));
            px[r] = make_float2(q.x, q.x);
            py[r] = make_float2(q.y, q.y);
            best[r] = CUDART_INF_F;
        }
        float2 v0 = __ldg(T);
        float2 v1 = __ldg(T + 1);
        for (int k = 0; k < nt; k += 2) {  // segments k, k+1 (segment nt-1 is the last vertex)
            const float2 v2 = __ldg(T + min(k + 2, nt - 1));
            SegPair g;
            seg_lane<EXACT>(g, 0, v0, v1);
            if (k + 1 < nt) seg_lane<EXACT>(g, 1, v1, v2);
            else seg_lane<EXACT>(g, 1, v0, v0);  // odd count: repeat the last vertex
#pragma unroll
            for (int r = 0; r < R; ++r) best[r] = p2s_pair(px[r], py[r], g, best[r]);
            v0 = v2;
            v1 = __ldg(T + min(k + 3, nt - 1));
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (pb + r < np) m = fmaxf(m, best[r]);
    }
    return m;
}

// The staged query's points, read back from the negated segment starts.
struct StagedNegPts {
    const float4* A;
    __device__ __forceinline__ float2 pt(int k) const {
        const float4 a = A[k >> 1];
        return make_float2(-((k & 1) ? a.y : a.x), -((k & 1) ? a.w : a.z));
    }
};

// Matrix kernel: CTA (s, chunk) stages query i's segment pairs in shared
// memory once; each thread takes one database trajectory.  Query order,
// symmetric and gather modes as in dp_matrix_kernel.  Dynamic shared memory =
// ceil(q_max_len/2) * 40 bytes.
template <int R, bool EXACT>
__global__ void __launch_bounds__(128) hausdorff_matrix_kernel(
    const float2* __restrict__ q_pts, const int64_t* __restrict__ q_off, const int32_t* __restrict__ q_len,
    const int32_t* __restrict__ q_order, const float2* __restrict__ d_pts, const int64_t* __restrict__ d_off,
    const int32_t* __restrict__ d_len, const int32_t* __restrict__ d_order, int64_t nd, int64_t d_total, int chunks,
    int sym, int q_max_len, int d_max_len, float* __restrict__ out, int64_t ld) {
    extern __shared__ float4 smem4[];
    const int cap_pairs = (q_max_len + 1) >> 1;
    float4* A = smem4;
    float4* B = smem4 + cap_pairs;
    float2* C = reinterpret_cast<float2*>(smem4 + 2 * cap_pairs);
    const int64_t qs = blockIdx.x / chunks;
    const int chunk = blockIdx.x % chunks;
    if (sym == 1 && (int64_t)(chunk + 1) * blockDim.x <= qs) return;
    const int64_t qi = q_order ? (int64_t)q_order[qs] : qs;
    const int nq = q_len[qi];
    const bool qbad = nq < 0 || nq > q_max_len;
    if (!qbad && nq > 0) {
        const float2* qp = q_pts + q_off[qi];
        const int npair = (nq + 1) >> 1;
        for (int j = threadIdx.x; j < npair; j += blockDim.x) {
            SegPair g;
            const int k0 = 2 * j, k1 = min(2 * j + 1, nq - 1);
            seg_lane<EXACT>(g, 0, __ldg(qp + k0), __ldg(qp + min(k0 + 1, nq - 1)));
            seg_lane<EXACT>(g, 1, __ldg(qp + k1), __ldg(qp + min(k1 + 1, nq - 1)));
            A[j] = make_float4(g.n1x.x, g.n1x.y, g.n1y.x, g.n1y.y);
            B[j] = make_float4(g.nsx.x, g.nsx.y, g.nsy.x, g.nsy.y);
            C[j] = g.ninv;
        }
    }
    __syncthreads();
    const int64_t slot = (int64_t)chunk * blockDim.x + threadIdx.x;
    if (slot >= nd || (sym == 1 && slot < qs)) return;
    const int64_t dj = d_order ? (int64_t)d_order[(sym == 2 ? qi * nd : 0) + slot] : slot;
    const bool dbad = dj < 0 || dj >= d_total;
    const int ndl = dbad ? -1 : d_len[dj];
    const int64_t o_idx = qi * ld + (sym == 2 ? slot : dj);
    const bool mirror = sym == 1 && dj != qi;
    float v = CUDART_NAN_F;
    if (!(qbad || dbad || ndl < 0 || ndl > d_max_len)) {
        const float2* dp = d_pts + d_off[dj];
        const float m1 = directed_max_staged2<R>(dp, ndl, A, B, C, nq);
        const float m2 = directed_max2<R, EXACT>(StagedNegPts{A}, nq, dp, ndl);
        v = __fsqrt_rn(fmaxf(m1, m2));
    }
    out[o_idx] = v;
    if (mirror) out[dj * ld + qi] = v;
}

// Pairs mode: a pair with more than kHausWarpCells point products (na * nb)
// runs one warp per pair (hausdorff_wave_kernel): on one thread, a pair of
// two 2000-point trajectories is 8M evaluations and would hold a launch's
// tail for tens of milliseconds.
constexpr int64_t kHausWarpCells = 1 << 17;

// Pairs kernel: one thread per pair, both trajectories from global memory
// (the pairs up to warp_cells point products -- kHausWarpCells, or 0 when a
// small batch runs every non-empty pair on the warp kernel; it also flags
// bad lengths).
template <int R, bool EXACT>
__global__ void __launch_bounds__(128) hausdorff_pairs_kernel(
    const float2* __restrict__ pts, const int64_t* __restrict__ off_a, const int32_t* __restrict__ len_a,
    const int64_t* __restrict__ off_b, const int32_t* __restrict__ len_b, const int32_t* __restrict__ order,
    int64_t n, int max_len, int64_t warp_cells, float* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t k = order ? (int64_t)order[t] : t;
    const int na = len_a[k], nb = len_b[k];
    if (na < 0 || nb < 0 || na > max_len || nb > max_len) {
        out[k] = CUDART_NAN_F;
        return;
    }
    if ((int64_t)na * nb > warp_cells) return;  // the warp kernel's pair
    const float2* a = pts + off_a[k];
    const float2* b = pts + off_b[k];
    const float m1 = directed_max2<R, EXACT>(GlobalCols{a}, na, b, nb);
    const float m2 = directed_max2<R, EXACT>(GlobalCols{b}, nb, a, na);
    out[k] = __fsqrt_rn(fmaxf(m1, m2));
}

// Long pairs (more than warp_cells point products), one warp each.
// Persistent, with the pair assignment of dp_wave_kernel (rounds of nw
// pairs in snake order, a ballot over 32 pairs at a time).  Lane l takes
// point blocks l, l+32, ... of both directions; the lanes' maxima are
// reduced with one warp max (exact), so the result is the one-thread
// kernel's, bit for bit.
template <int R, bool EXACT>
__global__ void __launch_bounds__(128) hausdorff_wave_kernel(
    const float2* __restrict__ pts, const int64_t* __restrict__ off_a, const int32_t* __restrict__ len_a,
    const int64_t* __restrict__ off_b, const int32_t* __restrict__ len_b, const int32_t* __restrict__ order,
    int64_t n, int max_len, int64_t warp_cells, float* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i0 = 0; i0 * nw < n; i0 += 32) {
        const int64_t i = i0 + lane;
        const int64_t t = i * nw + ((i & 1) ? nw - 1 - gw : gw);
        int64_t k = 0;
        bool mine = false;
        if (t < n) {
            k = order ? (int64_t)order[t] : t;
            const int na = len_a[k], nb = len_b[k];
            mine = na >= 0 && nb >= 0 && na <= max_len && nb <= max_len && (int64_t)na * nb > warp_cells;
        }
        unsigned todo = __ballot_sync(0xffffffffu, mine);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const int64_t kk = __shfl_sync(0xffffffffu, k, src);
            const int na = len_a[kk], nb = len_b[kk];
            const float2* a = pts + off_a[kk];
            const float2* b = pts + off_b[kk];
            float m = fmaxf(directed_max2<R, EXACT>(GlobalCols{a}, na, b, nb, lane * R, 32 * R),
                            directed_max2<R, EXACT>(GlobalCols{b}, nb, a, na, lane * R, 32 * R));
            // non-negative floats order like their bit patterns
            m = __int_as_float(__reduce_max_sync(0xffffffffu, __float_as_int(m)));
            if (lane == 0) out[kk] = __fsqrt_rn(m);
        }
    }
}

}  // namespace tsm
