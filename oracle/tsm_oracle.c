/*
 * CPU oracle for the batched pairwise heuristic trajectory measures.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py (its cpu_baseline leg and its
 * `--impl reference` arm) may load it.  The product path
 * (trajsimimeasures_b200) never calls it.
 *
 * Two families of functions, each over the packed layout that the CUDA
 * C-ABI uses (points [n_points][2], per-pair int64 offsets and int32
 * lengths).  The FP64 restatement reads float64 points, the reference's own
 * input type (utilities/data_loader.py:78-79 reads float64 Mercator metres);
 * the FP32 twin reads the float32 points that the kernels see:
 *
 *  1. *_f64: an FP64 restatement of the reference GPU kernels in core/*.py,
 *     following their exact semantics (boundaries, quirks, normalisation):
 *        dtw        core/dtw.py:10-53
 *        edr        core/edr.py:10-52      (all DP borders 0, count/max(n1,n2))
 *        lcss       core/lcss.py:12-53     (borders 0, 1 - count/min(n1,n2))
 *        erp        core/erp.py:10-91      (D(i,-1)=S1, D(-1,j)=S2: TOTAL gap sums)
 *        dfrechet   core/discret_frechet.py:9-50
 *        hausdorff  core/hausdorff.py:12-93 + host sqrt(max) at :121, with the
 *                   max taken over valid points only (the reference's host max
 *                   also reads uninitialised padded slots, hausdorff.py:114,121).
 *     Arithmetic follows the Numba code: (a-b)**2 + (c-d)**2 without FMA,
 *     sqrt in double, serial gap sums.
 *
 *  2. *_f32: an FP32 "same-arithmetic" twin of the CUDA kernels in
 *     trajsimimeasures_b200/csrc: the same per-cell formulas with the same
 *     rounding (explicit fmaf, IEEE sqrtf / division).  A DP cell value is a
 *     pure function of its three neighbours and the two points, so the CUDA
 *     kernels in exact-sqrt mode reproduce these values bit for bit whatever
 *     order they sweep the matrix in.  EDR/LCSS counts from the kernels match
 *     these counts bit for bit in every mode.
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -shared -fPIC (oracle/build.py).
 * -ffp-contract=off matters: fmaf() is the only fused operation allowed.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { M_DTW = 0, M_EDR = 1, M_LCSS = 2, M_ERP = 3, M_DFRECHET = 4, M_HAUSDORFF = 5 };

/* ------------------------------------------------------------------------ */
/* FP64 restatement of the reference                                        */
/* ------------------------------------------------------------------------ */

/* core/utils.py:8-11 squared_dist, :14-17 euc_dist (no FMA in the simulator). */
static double sq64(double ax, double ay, double bx, double by) {
    double dx = ax - bx, dy = ay - by;
    double x2 = dx * dx, y2 = dy * dy;
    return x2 + y2;
}

/* Row-major full DP over (n1+1) x (n2+1); the reference keeps a 3-diagonal
 * ring (dtw.py:35-37) but every cell value is the same. */
static double dtw64(const double* a, int n1, const double* b, int n2) {
    /* dtw.py: D(-1,-1)=0, other borders +inf; empty inputs: both empty -> 0,
     * one empty -> +inf (the ring slot read at :52 keeps its init value). */
    if (n1 == 0 && n2 == 0) return 0.0;
    if (n1 == 0 || n2 == 0) return INFINITY;
    double* prev = (double*)malloc(sizeof(double) * (n2 + 1));
    double* cur = (double*)malloc(sizeof(double) * (n2 + 1));
    for (int j = 0; j <= n2; ++j) prev[j] = INFINITY;
    prev[0] = 0.0;
    for (int i = 0; i < n1; ++i) {
        cur[0] = INFINITY;
        for (int j = 0; j < n2; ++j) {
            double c = sqrt(sq64(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]));
            double m = prev[j];
            if (prev[j + 1] < m) m = prev[j + 1];
            if (cur[j] < m) m = cur[j];
            cur[j + 1] = c + m;
        }
        double* t = prev; prev = cur; cur = t;
    }
    double r = prev[n2];
    free(prev); free(cur);
    return r;
}

static double dfrechet64(const double* a, int n1, const double* b, int n2) {
    /* discret_frechet.py:9-50: max(d, min(three neighbours)), same borders as DTW. */
    if (n1 == 0 && n2 == 0) return 0.0;
    if (n1 == 0 || n2 == 0) return INFINITY;
    double* prev = (double*)malloc(sizeof(double) * (n2 + 1));
    double* cur = (double*)malloc(sizeof(double) * (n2 + 1));
    for (int j = 0; j <= n2; ++j) prev[j] = INFINITY;
    prev[0] = 0.0;
    for (int i = 0; i < n1; ++i) {
        cur[0] = INFINITY;
        for (int j = 0; j < n2; ++j) {
            double c = sqrt(sq64(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]));
            double m = prev[j];
            if (prev[j + 1] < m) m = prev[j + 1];
            if (cur[j] < m) m = cur[j];
            cur[j + 1] = c > m ? c : m;
        }
        double* t = prev; prev = cur; cur = t;
    }
    double r = prev[n2];
    free(prev); free(cur);
    return r;
}

/* edr.py:10-52 / lcss.py:12-53: integer counts with every DP border 0. */
static int64_t edr_count64(const double* a, int n1, const double* b, int n2, double eps) {
    if (n1 == 0 || n2 == 0) return 0;
    double seps = eps * eps;
    int64_t* prev = (int64_t*)calloc(n2 + 1, sizeof(int64_t));
    int64_t* cur = (int64_t*)calloc(n2 + 1, sizeof(int64_t));
    for (int i = 0; i < n1; ++i) {
        cur[0] = 0;
        for (int j = 0; j < n2; ++j) {
            int64_t sub = sq64(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]) < seps ? 0 : 1;
            int64_t v = prev[j] + sub;
            if (cur[j] + 1 < v) v = cur[j] + 1;
            if (prev[j + 1] + 1 < v) v = prev[j + 1] + 1;
            cur[j + 1] = v;
        }
        int64_t* t = prev; prev = cur; cur = t;
    }
    int64_t r = prev[n2];
    free(prev); free(cur);
    return r;
}

static int64_t lcss_count64(const double* a, int n1, const double* b, int n2, double eps) {
    if (n1 == 0 || n2 == 0) return 0;
    double seps = eps * eps;
    int64_t* prev = (int64_t*)calloc(n2 + 1, sizeof(int64_t));
    int64_t* cur = (int64_t*)calloc(n2 + 1, sizeof(int64_t));
    for (int i = 0; i < n1; ++i) {
        cur[0] = 0;
        for (int j = 0; j < n2; ++j) {
            int64_t v;
            if (sq64(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]) < seps)
                v = prev[j] + 1;
            else
                v = prev[j + 1] > cur[j] ? prev[j + 1] : cur[j];
            cur[j + 1] = v;
        }
        int64_t* t = prev; prev = cur; cur = t;
    }
    int64_t r = prev[n2];
    free(prev); free(cur);
    return r;
}

/* erp.py:10-91.  Gap distances to g; S1, S2 are serial sums (:44-49); the
 * borders are the TOTAL sums: D(i,-1)=S1, D(-1,j)=S2, D(-1,-1)=0 (:62-78).
 * With an empty input the reference returns its zero-initialised ring slot. */
static double erp64(const double* a, int n1, const double* b, int n2, double gx, double gy) {
    if (n1 == 0 || n2 == 0) return 0.0;
    double* g1 = (double*)malloc(sizeof(double) * n1);
    double* g2 = (double*)malloc(sizeof(double) * n2);
    double s1 = 0.0, s2 = 0.0;
    for (int i = 0; i < n1; ++i) { g1[i] = sqrt(sq64(gx, gy, a[2 * i], a[2 * i + 1])); }
    for (int j = 0; j < n2; ++j) { g2[j] = sqrt(sq64(gx, gy, b[2 * j], b[2 * j + 1])); }
    for (int i = 0; i < n1; ++i) s1 += g1[i];
    for (int j = 0; j < n2; ++j) s2 += g2[j];
    double* prev = (double*)malloc(sizeof(double) * (n2 + 1));
    double* cur = (double*)malloc(sizeof(double) * (n2 + 1));
    prev[0] = 0.0;
    for (int j = 1; j <= n2; ++j) prev[j] = s2;
    for (int i = 0; i < n1; ++i) {
        cur[0] = s1;
        for (int j = 0; j < n2; ++j) {
            double left = cur[j], upper = prev[j + 1], ul = prev[j];
            if (i == 0 && j > 0) { upper = s2; ul = s2; }
            else if (j == 0 && i > 0) { left = s1; ul = s1; }
            else if (i == 0 && j == 0) { left = s1; upper = s2; ul = 0.0; }
            double cl = left + g2[j];
            double cu = upper + g1[i];
            double cd = ul + sqrt(sq64(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]));
            double m = cl;
            if (cu < m) m = cu;
            if (cd < m) m = cd;
            cur[j + 1] = m;
        }
        double* t = prev; prev = cur; cur = t;
    }
    double r = prev[n2];
    free(prev); free(cur); free(g1); free(g2);
    return r;
}

/* hausdorff.py:12-45 p2s_dist (squared distances, FP64). */
static double p2s64(double px, double py, double p1x, double p1y, double p2x, double p2y,
                    double d1, double d2) {
    if (p1x == p2x && p1y == p2y) return d1;
    double segl = sq64(p1x, p1y, p2x, p2y);
    double xd = p2x - p1x, yd = p2y - p1y;
    double u1 = ((px - p1x) * xd) + ((py - p1y) * yd);
    double u = u1 / segl;
    if (u < 0.00001 || u > 1) return d1 < d2 ? d1 : d2;
    double ix = p1x + u * xd, iy = p1y + u * yd;
    return sq64(px, py, ix, iy);
}

/* hausdorff.py:48-69 p2t_dist: min over the t_len-1 segments, 0.0 if none. */
static double p2t64(double px, double py, const double* t, int n) {
    double dist = 0.0, d1 = 0.0, d2 = 0.0;
    for (int i = 0; i < n - 1; ++i) {
        if (i == 0) {
            d1 = sq64(px, py, t[0], t[1]);
            d2 = sq64(px, py, t[2], t[3]);
        } else {
            d1 = d2;
            d2 = sq64(px, py, t[2 * (i + 1)], t[2 * (i + 1) + 1]);
        }
        double ps = p2s64(px, py, t[2 * i], t[2 * i + 1], t[2 * (i + 1)], t[2 * (i + 1) + 1], d1, d2);
        if (i == 0 || ps < dist) dist = ps;
    }
    return dist;
}

static double hausdorff64(const double* a, int n1, const double* b, int n2) {
    double m = 0.0;
    for (int i = 0; i < n1; ++i) { double d = p2t64(a[2 * i], a[2 * i + 1], b, n2); if (d > m) m = d; }
    for (int j = 0; j < n2; ++j) { double d = p2t64(b[2 * j], b[2 * j + 1], a, n1); if (d > m) m = d; }
    return sqrt(m);
}

/* ------------------------------------------------------------------------ */
/* FP32 same-arithmetic twin of the CUDA kernels                            */
/* ------------------------------------------------------------------------ */

/* dx, dy exact-rounded subtractions, then fma(dy, dy, dx*dx).  Swapping the
 * two points negates dx, dy exactly, so the value is symmetric. */
static inline float d2f(float ax, float ay, float bx, float by) {
    float dx = ax - bx, dy = ay - by;
    return fmaf(dy, dy, dx * dx);
}
static inline float fmin3(float a, float b, float c) { return fminf(fminf(a, b), c); }

float tsm_oracle_dtw_f32(const float* a, int n1, const float* b, int n2) {
    if (n1 == 0 && n2 == 0) return 0.0f;
    if (n1 == 0 || n2 == 0) return INFINITY;
    float* prev = (float*)malloc(sizeof(float) * (n2 + 1));
    float* cur = (float*)malloc(sizeof(float) * (n2 + 1));
    for (int j = 0; j <= n2; ++j) prev[j] = INFINITY;
    prev[0] = 0.0f;
    for (int i = 0; i < n1; ++i) {
        cur[0] = INFINITY;
        for (int j = 0; j < n2; ++j) {
            float c = sqrtf(d2f(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]));
            cur[j + 1] = c + fmin3(prev[j], prev[j + 1], cur[j]);
        }
        float* t = prev; prev = cur; cur = t;
    }
    float r = prev[n2];
    free(prev); free(cur);
    return r;
}

float tsm_oracle_dfrechet_f32(const float* a, int n1, const float* b, int n2) {
    /* max-min DP on squared distances, one sqrt at the end: sqrt is monotone
     * and correctly rounded, so this equals the DP on rounded distances. */
    if (n1 == 0 && n2 == 0) return 0.0f;
    if (n1 == 0 || n2 == 0) return INFINITY;
    float* prev = (float*)malloc(sizeof(float) * (n2 + 1));
    float* cur = (float*)malloc(sizeof(float) * (n2 + 1));
    for (int j = 0; j <= n2; ++j) prev[j] = INFINITY;
    prev[0] = 0.0f;
    for (int i = 0; i < n1; ++i) {
        cur[0] = INFINITY;
        for (int j = 0; j < n2; ++j) {
            float c = d2f(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]);
            cur[j + 1] = fmaxf(c, fmin3(prev[j], prev[j + 1], cur[j]));
        }
        float* t = prev; prev = cur; cur = t;
    }
    float r = sqrtf(prev[n2]);
    free(prev); free(cur);
    return r;
}

int32_t tsm_oracle_edr_count_f32(const float* a, int n1, const float* b, int n2, float eps2) {
    if (n1 == 0 || n2 == 0) return 0;
    int32_t* prev = (int32_t*)calloc(n2 + 1, sizeof(int32_t));
    int32_t* cur = (int32_t*)calloc(n2 + 1, sizeof(int32_t));
    for (int i = 0; i < n1; ++i) {
        cur[0] = 0;
        for (int j = 0; j < n2; ++j) {
            int32_t sub = d2f(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]) < eps2 ? 0 : 1;
            int32_t v = prev[j] + sub;
            int32_t w = (prev[j + 1] < cur[j] ? prev[j + 1] : cur[j]) + 1;
            cur[j + 1] = v < w ? v : w;
        }
        int32_t* t = prev; prev = cur; cur = t;
    }
    int32_t r = prev[n2];
    free(prev); free(cur);
    return r;
}

int32_t tsm_oracle_lcss_count_f32(const float* a, int n1, const float* b, int n2, float eps2) {
    if (n1 == 0 || n2 == 0) return 0;
    int32_t* prev = (int32_t*)calloc(n2 + 1, sizeof(int32_t));
    int32_t* cur = (int32_t*)calloc(n2 + 1, sizeof(int32_t));
    for (int i = 0; i < n1; ++i) {
        cur[0] = 0;
        for (int j = 0; j < n2; ++j) {
            int32_t v;
            if (d2f(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]) < eps2) v = prev[j] + 1;
            else v = prev[j + 1] > cur[j] ? prev[j + 1] : cur[j];
            cur[j + 1] = v;
        }
        int32_t* t = prev; prev = cur; cur = t;
    }
    int32_t r = prev[n2];
    free(prev); free(cur);
    return r;
}

/* ERP gap point as an FP32 hi/lo pair: g = hi + lo.  A gap distance
 * subtracts hi first (exact for points near g), then lo, so an FP64 gap point
 * such as 41.15 costs no FP32 representation error. */
typedef struct { float hx, lx, hy, ly; } gap_pt;

static gap_pt split_gap(double gx, double gy) {
    gap_pt g;
    g.hx = (float)gx; g.lx = (float)(gx - (double)g.hx);
    g.hy = (float)gy; g.ly = (float)(gy - (double)g.hy);
    return g;
}

static inline float gapd_f32(float x, float y, gap_pt g) {
    float dx = (x - g.hx) - g.lx, dy = (y - g.hy) - g.ly;
    return sqrtf(fmaf(dy, dy, dx * dx));
}

/* Gap-distance total: FP32 gap distances summed in FP64 in index order and
 * rounded once to FP32 (the kernels do the same). */
static float gap_sum_f32(const float* t, int n, gap_pt gp, float* g) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
        g[i] = gapd_f32(t[2 * i], t[2 * i + 1], gp);
        s += (double)g[i];
    }
    return (float)s;
}

float tsm_oracle_erp_f32(const float* a, int n1, const float* b, int n2, double gx, double gy) {
    if (n1 == 0 || n2 == 0) return 0.0f;
    gap_pt gp = split_gap(gx, gy);
    float* g1 = (float*)malloc(sizeof(float) * n1);
    float* g2 = (float*)malloc(sizeof(float) * n2);
    float s1 = gap_sum_f32(a, n1, gp, g1);
    float s2 = gap_sum_f32(b, n2, gp, g2);
    float* prev = (float*)malloc(sizeof(float) * (n2 + 1));
    float* cur = (float*)malloc(sizeof(float) * (n2 + 1));
    prev[0] = 0.0f;
    for (int j = 1; j <= n2; ++j) prev[j] = s2;
    for (int i = 0; i < n1; ++i) {
        cur[0] = s1;
        for (int j = 0; j < n2; ++j) {
            float c = sqrtf(d2f(a[2 * i], a[2 * i + 1], b[2 * j], b[2 * j + 1]));
            /* D(-1,-1)=0, D(-1,j)=S2, D(i,-1)=S1 */
            float ul = prev[j];
            if (i == 0) ul = (j == 0) ? 0.0f : s2;
            else if (j == 0) ul = s1;
            float cl = cur[j] + g2[j];
            float cu = prev[j + 1] + g1[i];
            float cd = ul + c;
            cur[j + 1] = fmin3(cl, cu, cd);
        }
        float* t = prev; prev = cur; cur = t;
    }
    float r = prev[n2];
    free(prev); free(cur); free(g1); free(g2);
    return r;
}

/* Point-to-segment squared distance, kernel formulation: relative vectors
 * a = p - s1, s = s2 - s1 (no absolute foot point), t = 0 when u < 1e-5,
 * t = min(u, 1) otherwise, which is the reference rule (hausdorff.py:36-43)
 * restated: u < 1e-5 -> nearer endpoint is s1, u > 1 -> s2.  A zero-length
 * segment gets inv = 0, hence t = 0 and |p - s1|^2 (hausdorff.py:30-31). */
static inline float p2s_f32(float px, float py, float s1x, float s1y, float sx, float sy, float inv) {
    float ax = px - s1x, ay = py - s1y;
    float dot = fmaf(ay, sy, ax * sx);
    float u = dot * inv;
    float t = (u >= 1e-5f) ? fminf(u, 1.0f) : 0.0f; /* NaN -> 0, as mul.sat */
    float ex = fmaf(-t, sx, ax), ey = fmaf(-t, sy, ay);
    return fmaf(ey, ey, ex * ex);
}

static float directed_f32(const float* a, int n1, const float* b, int n2) {
    float m = 0.0f;
    if (n2 < 2) return 0.0f; /* p2t_dist with no segment is 0.0 (hausdorff.py:49-50) */
    for (int i = 0; i < n1; ++i) {
        float px = a[2 * i], py = a[2 * i + 1];
        float best = INFINITY;
        /* the n2-1 segments, then the last vertex as a zero-length segment
         * (never below the last segment's distance in exact arithmetic; makes
         * a point equal to that vertex exactly 0 in FP32) */
        for (int k = 0; k < n2; ++k) {
            int k2 = (k + 1 < n2) ? k + 1 : k;
            float s1x = b[2 * k], s1y = b[2 * k + 1];
            float sx = b[2 * k2] - s1x, sy = b[2 * k2 + 1] - s1y;
            float len2 = fmaf(sy, sy, sx * sx);
            float inv = (sx == 0.0f && sy == 0.0f) ? 0.0f : 1.0f / len2;
            float d = p2s_f32(px, py, s1x, s1y, sx, sy, inv);
            best = fminf(best, d);
        }
        m = fmaxf(m, best);
    }
    return m;
}

float tsm_oracle_hausdorff_f32(const float* a, int n1, const float* b, int n2) {
    float m = fmaxf(directed_f32(a, n1, b, n2), directed_f32(b, n2, a, n1));
    return sqrtf(m);
}

/* ------------------------------------------------------------------------ */
/* Batch entry points (ctypes)                                               */
/* ------------------------------------------------------------------------ */

static int g_threads = 0; /* 0: OpenMP default */

void tsm_oracle_set_threads(int n) { g_threads = n; }
int tsm_oracle_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* FP64 restatement.  out64[k] = distance of pair k; counts (nullable) gets
 * the EDR/LCSS counts. */
int tsm_oracle_pairs_f64(int measure, const double* pts, const int64_t* off_a, const int32_t* len_a,
                         const int64_t* off_b, const int32_t* len_b, int64_t n, double eps,
                         double gx, double gy, double* out64, int64_t* counts) {
    if (measure < 0 || measure > 5) return -1;
    int nt = tsm_oracle_get_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
    for (int64_t k = 0; k < n; ++k) {
        const double* a = pts + 2 * off_a[k];
        const double* b = pts + 2 * off_b[k];
        int n1 = len_a[k], n2 = len_b[k];
        double r = 0.0;
        int64_t c = 0;
        switch (measure) {
            case M_DTW: r = dtw64(a, n1, b, n2); break;
            case M_DFRECHET: r = dfrechet64(a, n1, b, n2); break;
            case M_ERP: r = erp64(a, n1, b, n2, gx, gy); break;
            case M_HAUSDORFF: r = hausdorff64(a, n1, b, n2); break;
            case M_EDR: {
                c = edr_count64(a, n1, b, n2, eps);
                int mx = n1 > n2 ? n1 : n2;
                r = (double)c / (double)mx; /* edr.py:51 (0/0 -> NaN) */
                break;
            }
            case M_LCSS: {
                c = lcss_count64(a, n1, b, n2, eps);
                int mn = n1 < n2 ? n1 : n2;
                r = 1.0 - (double)c / (double)mn; /* lcss.py:52 */
                break;
            }
        }
        out64[k] = r;
        if (counts) counts[k] = c;
    }
    return 0;
}

/* FP32 twin.  out32[k] as the kernels write it; counts (nullable) int32. */
int tsm_oracle_pairs_f32(int measure, const float* pts, const int64_t* off_a, const int32_t* len_a,
                         const int64_t* off_b, const int32_t* len_b, int64_t n, float eps2,
                         double gx, double gy, float* out32, int32_t* counts) {
    if (measure < 0 || measure > 5) return -1;
    int nt = tsm_oracle_get_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
    for (int64_t k = 0; k < n; ++k) {
        const float* a = pts + 2 * off_a[k];
        const float* b = pts + 2 * off_b[k];
        int n1 = len_a[k], n2 = len_b[k];
        float r = 0.0f;
        int32_t c = 0;
        switch (measure) {
            case M_DTW: r = tsm_oracle_dtw_f32(a, n1, b, n2); break;
            case M_DFRECHET: r = tsm_oracle_dfrechet_f32(a, n1, b, n2); break;
            case M_ERP: r = tsm_oracle_erp_f32(a, n1, b, n2, gx, gy); break;
            case M_HAUSDORFF: r = tsm_oracle_hausdorff_f32(a, n1, b, n2); break;
            case M_EDR: {
                c = tsm_oracle_edr_count_f32(a, n1, b, n2, eps2);
                int mx = n1 > n2 ? n1 : n2;
                r = (float)c / (float)mx;
                break;
            }
            case M_LCSS: {
                c = tsm_oracle_lcss_count_f32(a, n1, b, n2, eps2);
                int mn = n1 < n2 ? n1 : n2;
                r = 1.0f - (float)c / (float)mn;
                break;
            }
        }
        out32[k] = r;
        if (counts) counts[k] = c;
    }
    return 0;
}
