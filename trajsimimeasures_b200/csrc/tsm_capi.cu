// C ABI of libtsm_b200.so (declarations and contract: include/tsm.h).
//
// Host-side launch logic only: argument checks, kernel selection by
// (measure, rows-per-thread, exact), shared-memory sizing, launch on the
// caller's stream (tsm_pairs' long-pair kernel on a side stream forked from
// and joined back to it).  No device allocation happens here.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "tsm.h"
#include "tsm_kernels.h"
#include "tsm_sched.cuh"
#include "tsm_tile.cuh"
#include "tsm_topk.cuh"
#include "tsm_wave.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char b[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b, sizeof(b), fmt, ap);
    va_end(ap);
    g_err = b;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(TSM_ECUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

// Pairs mode: pairs whose shorter trajectory has at most kTileCap points run
// on the tile kernel (one thread per pair, a kTileCap-float boundary row per
// thread); longer ones on the wave kernel (one warp per pair).
constexpr int kTileCap = 256;
static_assert(tsm::kHeavyRows >= kTileCap, "a tile-heavy pair must have a side longer than the tile capacity");
// Matrix mode keeps the query as the tile kernel's columns: its boundary
// rows (32 per warp) and staged columns must fit one CTA's shared memory.
constexpr int kMatrixQueryMax = 1400;
// Longest trajectory accepted by the paired kernels: the wave kernel keeps 4
// bytes of shared memory per point of a pair's shorter side for each of its W
// warps (W = 4 up to 8192 points, 2 up to 16384, 1 up to 32768: 128 KB).
constexpr int kMaxLen = 32768;
// A paired batch of at most kSmallBatchPerSm pairs per SM is too small to
// fill the GPU one thread per pair (the tile and Hausdorff pairs kernels
// would then run one pair's whole DP serially on a few warps per SM): every
// non-empty pair runs one warp each on the wave kernels instead, with 4 rows
// per lane unless rows_per_thread says otherwise.
constexpr int kSmallBatchPerSm = 64;
// Shared memory one CTA may use, leaving room for two CTAs per SM at cap 200.
constexpr int kSmemPerCta = 113 * 1024;
constexpr int kSmemMax = 227 * 1024;

tsm::KParams make_kparams(const tsm_params* p) {
    tsm::KParams k{};
    const double eps = p ? p->eps : 0.0;
    const double gx = p ? p->gx : 0.0, gy = p ? p->gy : 0.0;
    k.eps2 = (float)(eps * eps);
    k.ghx = (float)gx;
    k.glx = (float)(gx - (double)k.ghx);
    k.ghy = (float)gy;
    k.gly = (float)(gy - (double)k.ghy);
    return k;
}

// Default rows per thread block: 8 for the DP measures (two packed 8-row
// blocks per pass), 16 for Hausdorff (amortises the per-segment setup).
int rows_of(const tsm_params* p, int measure = TSM_DTW) {
    const int r = p ? p->rows_per_thread : 0;
    return r == 0 ? (measure == TSM_HAUSDORFF ? 16 : 8) : r;
}

bool exact_of(const tsm_params* p) { return p && (p->flags & TSM_FLAG_EXACT); }

// Warps per CTA for a boundary row of `cap` floats per thread.
int warps_for(int cap, int extra_bytes) {
    for (int w = 4; w > 1; --w)
        if (w * 32 * cap * 4 + extra_bytes <= kSmemPerCta) return w;
    return 1;
}

cudaError_t set_smem(const void* fn, int bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

int launch(const void* fn, dim3 grid, dim3 block, int smem, void** args, cudaStream_t s) {
    cudaError_t e = set_smem(fn, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    e = cudaLaunchKernel(fn, grid, block, args, (size_t)smem, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaLaunchKernel");
    return TSM_OK;
}

// The calling thread's side stream (and fork / join events) on device dev,
// created on first use.  nullptr when they cannot be made, and when they do
// not exist yet while the caller's stream is being captured into a graph
// (creating them then could invalidate the capture): the caller then
// launches everything on its own stream.
struct SideStream {
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    bool failed = false;
};
constexpr int kMaxDevices = 64;
thread_local SideStream g_side[kMaxDevices];

SideStream* side_stream(int dev, cudaStream_t caller) {
    if (dev < 0 || dev >= kMaxDevices) return nullptr;
    SideStream& r = g_side[dev];
    if (r.st) return &r;
    if (r.failed) return nullptr;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(caller, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return nullptr;
    }
    SideStream t;
    if (cudaStreamCreateWithFlags(&t.st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&t.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&t.join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (t.join) cudaEventDestroy(t.join);
        if (t.fork) cudaEventDestroy(t.fork);
        if (t.st) cudaStreamDestroy(t.st);
        r.failed = true;
        return nullptr;
    }
    r = t;
    return &r;
}

// Grid of a persistent kernel: the blocks that fit on the device at once
// (at most max_blocks).
int persistent_grid(const char* who, const void* fn, int threads, int smem, int64_t max_blocks, dim3& grid,
                    int& dev) {
    cudaError_t e = set_smem(fn, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    int sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute");
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem)) != cudaSuccess)
        return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) return fail(TSM_ETOOLONG, "%s: the long-pair kernel does not fit on an SM", who);
    int64_t blocks = (int64_t)sms * per_sm;
    if (blocks > max_blocks) blocks = max_blocks;
    grid = dim3((unsigned)blocks);
    return TSM_OK;
}

// tsm_pairs' two kernels, which write disjoint outputs: `main` (the short
// pairs, as a callable taking the stream) on the caller's stream and the
// long-pair kernel on the calling thread's side stream, forked from and
// joined back to the caller's; on the caller's stream one after the other
// when there is no side stream.
template <class Main>
int launch_with_side(Main main, const void* wfn, dim3 w_grid, dim3 w_block, int w_smem, void** w_args,
                     cudaStream_t s, int dev) {
    SideStream* side = side_stream(dev, s);
    if (!side) {
        const int rc = main(s);
        return rc != TSM_OK ? rc : launch(wfn, w_grid, w_block, w_smem, w_args, s);
    }
    cudaError_t e;
    if ((e = cudaEventRecord(side->fork, s)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    if ((e = cudaStreamWaitEvent(side->st, side->fork, 0)) != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");
    const int rc = launch(wfn, w_grid, w_block, w_smem, w_args, side->st);
    const int rc_main = main(s);
    // join even after a failed launch, so that the side stream is not left forked from a capture
    if ((e = cudaEventRecord(side->join, side->st)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    if ((e = cudaStreamWaitEvent(s, side->join, 0)) != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");
    return rc != TSM_OK ? rc : rc_main;
}

}  // namespace

// Internal (hidden, not part of the ABI): lets other translation units of the
// library report through tsm_last_error().
__attribute__((visibility("hidden"))) int tsm_internal_fail(int code, const char* msg) {
    g_err = msg;
    return code;
}

extern "C" {

int tsm_version(void) { return 100; }

const char* tsm_last_error(void) { return g_err.c_str(); }

int32_t tsm_max_supported_len(void) { return kMaxLen; }

int32_t tsm_matrix_query_max(void) { return kMatrixQueryMax; }

int tsm_pairs(int measure, const float* pts, const int64_t* off_a, const int32_t* len_a,
              const int64_t* off_b, const int32_t* len_b, const int32_t* order, int64_t n_pairs,
              int32_t max_len, const tsm_params* params, float* out, int32_t* out_counts, void* stream) {
    g_err.clear();
    if (measure < TSM_DTW || measure > TSM_HAUSDORFF) return fail(TSM_EINVAL, "tsm_pairs: unknown measure %d", measure);
    if (n_pairs < 0) return fail(TSM_EINVAL, "tsm_pairs: n_pairs < 0");
    if (n_pairs == 0) return TSM_OK;
    if (!pts || !off_a || !len_a || !off_b || !len_b || !out) return fail(TSM_EINVAL, "tsm_pairs: null pointer");
    if (max_len < 0) return fail(TSM_EINVAL, "tsm_pairs: max_len < 0");
    if (measure != TSM_HAUSDORFF && max_len > kMaxLen)
        return fail(TSM_ETOOLONG, "tsm_pairs: max_len %d > %d (tsm_max_supported_len)", max_len, kMaxLen);
    const bool exact = exact_of(params);
    cudaStream_t s = (cudaStream_t)stream;
    const tsm::KParams kp = make_kparams(params);
    const float2* p2 = reinterpret_cast<const float2*>(pts);
    int64_t n = n_pairs;
    int ml = max_len;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute");
    const bool small = n <= (int64_t)kSmallBatchPerSm * sms;
    const int R = (small && !(params && params->rows_per_thread)) ? 4 : rows_of(params, measure);
    if (measure == TSM_HAUSDORFF) {
        const void* fn = tsm_k::haus(false, R, exact);
        if (!fn) return fail(TSM_EINVAL, "tsm_pairs: rows_per_thread must be 4, 8 or 16");
        const int threads = 128;
        dim3 grid((unsigned)((n + threads - 1) / threads));
        int64_t warp_cells = small ? 0 : tsm::kHausWarpCells;
        void* args[] = {&p2, &off_a, &len_a, &off_b, &len_b, &order, &n, &ml, &warp_cells, &out};
        if ((int64_t)max_len * max_len <= warp_cells) return launch(fn, grid, dim3(threads), 0, args, s);
        // long pairs (small batch: every non-empty pair): one warp each, persistent
        const void* wfn = tsm_k::haus_wave(R, exact);
        dim3 w_grid;
        int rc = persistent_grid("tsm_pairs", wfn, threads, 0, (n + 3) / 4, w_grid, dev);
        if (rc != TSM_OK) return rc;
        void* w_args[] = {&p2, &off_a, &len_a, &off_b, &len_b, &order, &n, &ml, &warp_cells, &out};
        if (small) {  // the pairs kernel only flags bad lengths and empty pairs: one stream, in order
            rc = launch(fn, grid, dim3(threads), 0, args, s);
            return rc != TSM_OK ? rc : launch(wfn, w_grid, dim3(threads), 0, w_args, s);
        }
        // on the side stream, overlapping the one-thread-per-pair kernel
        return launch_with_side([&](cudaStream_t st) { return launch(fn, grid, dim3(threads), 0, args, st); }, wfn,
                                w_grid, dim3(threads), 0, w_args, s, dev);
    }
    const void* fn = tsm_k::dp_pairs(measure, R, exact);
    if (!fn) return fail(TSM_EINVAL, "tsm_pairs: rows_per_thread must be 4, 8 or 16");
    // small batch: tile capacity 0, so the tile kernel keeps only empty and
    // bad-length pairs and the wave kernel takes every other pair
    int cap = small ? 0 : (max_len < 1 ? 1 : (max_len < kTileCap ? max_len : kTileCap));
    const int tW = warps_for(cap, 0);
    const int t_smem = tW * 32 * cap * 4;
    const dim3 t_grid((unsigned)((n + 32 * tW - 1) / (32 * tW)));
    void* t_args[] = {&p2, &off_a, &len_a, &off_b, &len_b, &order, &n, &cap, &ml, (void*)&kp, &out, &out_counts};
    // (a tile-heavy pair has a side longer than kHeavyRows >= kTileCap)
    if (!small && max_len <= cap) return launch(fn, t_grid, dim3(32 * tW), t_smem, t_args, s);

    // pairs whose shorter side exceeds cap, or whose tile loop would be very
    // long: the persistent wave kernel, one warp per pair
    const void* wfn = tsm_k::dp_wave(measure, R, exact);
    int wcap = (max_len + 3) & ~3;
    const int W = wcap <= 8192 ? 4 : (wcap <= 16384 ? 2 : 1);
    const int w_smem = W * tsm::wave_warp_floats(wcap) * 4;
    if (w_smem > kSmemMax) return fail(TSM_ETOOLONG, "tsm_pairs: wave kernel needs %d bytes", w_smem);
    dim3 w_grid;
    int rc = persistent_grid("tsm_pairs", wfn, 32 * W, w_smem, (n + W - 1) / W, w_grid, dev);
    if (rc != TSM_OK) return rc;
    int tcap = cap;
    void* w_args[] = {&p2, &off_a, &len_a, &off_b, &len_b, &order, &n, &tcap, &wcap, &ml, (void*)&kp, &out, &out_counts};
    if (small) {  // the tile kernel has (almost) nothing to do: one stream, in order
        rc = launch(fn, t_grid, dim3(32 * tW), t_smem, t_args, s);
        return rc != TSM_OK ? rc : launch(wfn, w_grid, dim3(32 * W), w_smem, w_args, s);
    }
    // the wave kernel (few warps with long, uneven loops) on the side stream:
    // the tile kernel's blocks fill the SMs its warps leave idle
    return launch_with_side([&](cudaStream_t st) { return launch(fn, t_grid, dim3(32 * tW), t_smem, t_args, st); },
                            wfn, w_grid, dim3(32 * W), w_smem, w_args, s, dev);
}

namespace {

// One matrix launch: Q x D (q_order == nullptr, sym == 0), the symmetric
// upper triangle of one set in its length order (q_order == d_order, sym ==
// 1), or per-query candidate rows (d_order [nq][nd], sym == 2).  d_total: the
// number of database trajectories (indices from d_order are checked against it).
int matrix_launch(const char* who, int measure, const float* q_pts, const int64_t* q_off, const int32_t* q_len,
                  const int32_t* q_order, int64_t nq, int32_t q_max_len, const float* d_pts, const int64_t* d_off,
                  const int32_t* d_len, const int32_t* d_order, int64_t nd, int64_t d_total, int32_t d_max_len,
                  int sym, const tsm_params* params, float* out, int64_t ld_out, int32_t* out_counts, void* stream) {
    const int R = rows_of(params, measure);
    const bool exact = exact_of(params);
    cudaStream_t s = (cudaStream_t)stream;
    const tsm::KParams kp = make_kparams(params);
    const float2* q2 = reinterpret_cast<const float2*>(q_pts);
    const float2* d2 = reinterpret_cast<const float2*>(d_pts);
    int qcap = q_max_len < 1 ? 1 : q_max_len;
    int dml = d_max_len;
    int64_t ndd = nd, ld = ld_out, dtot = d_total;
    if (measure == TSM_HAUSDORFF) {
        const void* fn = tsm_k::haus(true, R, exact);
        if (!fn) return fail(TSM_EINVAL, "%s: rows_per_thread must be 4, 8 or 16", who);
        const int smem = ((qcap + 1) / 2) * 40;  // staged segment pairs
        if (smem > kSmemMax) return fail(TSM_ETOOLONG, "%s: query length %d too long", who, q_max_len);
        const int threads = 128;
        int chunks = (int)((nd + threads - 1) / threads);
        if ((int64_t)chunks * nq > 0x7fffffffLL) return fail(TSM_EINVAL, "%s: grid too large", who);
        dim3 grid((unsigned)(chunks * nq));
        void* args[] = {&q2,   &q_off,  &q_len, &q_order, &d2,  &d_off, &d_len, &d_order,
                        &ndd,  &dtot,   &chunks, &sym,    &qcap, &dml,  &out,   &ld};
        return launch(fn, grid, dim3(threads), smem, args, s);
    }
    if (q_max_len > kMatrixQueryMax)
        return fail(TSM_ETOOLONG, "%s: q_max_len %d > %d (use the pairs form)", who, q_max_len, kMatrixQueryMax);
    const void* fn = tsm_k::dp_matrix(measure, R, exact);
    if (!fn) return fail(TSM_EINVAL, "%s: rows_per_thread must be 4, 8 or 16", who);
    const int W = warps_for(qcap, qcap * 16);
    const int threads = 32 * W;
    const int smem = qcap * 16 + W * 32 * qcap * 4;
    if (smem > kSmemMax) return fail(TSM_ETOOLONG, "%s: boundary rows need %d bytes", who, smem);
    int chunks = (int)((nd + threads - 1) / threads);
    if ((int64_t)chunks * nq > 0x7fffffffLL) return fail(TSM_EINVAL, "%s: grid too large", who);
    dim3 grid((unsigned)(chunks * nq));
    void* args[] = {&q2,     &q_off, &q_len, &q_order, &d2,        &d_off, &d_len, &d_order, &ndd,
                    &dtot,   &chunks, &sym,  &qcap,    &dml,       (void*)&kp, &out, &ld,     &out_counts};
    return launch(fn, grid, dim3(threads), smem, args, s);
}

}  // namespace

int tsm_matrix(int measure, const float* q_pts, const int64_t* q_off, const int32_t* q_len, int64_t nq,
               int32_t q_max_len, const float* d_pts, const int64_t* d_off, const int32_t* d_len,
               const int32_t* d_order, int64_t nd, int32_t d_max_len, const tsm_params* params,
               float* out, int64_t ld_out, int32_t* out_counts, void* stream) {
    g_err.clear();
    if (measure < TSM_DTW || measure > TSM_HAUSDORFF) return fail(TSM_EINVAL, "tsm_matrix: unknown measure %d", measure);
    if (nq < 0 || nd < 0) return fail(TSM_EINVAL, "tsm_matrix: negative set size");
    if (nq == 0 || nd == 0) return TSM_OK;
    if (!q_pts || !q_off || !q_len || !d_pts || !d_off || !d_len || !out)
        return fail(TSM_EINVAL, "tsm_matrix: null pointer");
    if (ld_out < nd) return fail(TSM_EINVAL, "tsm_matrix: ld_out < nd");
    if (q_max_len < 0 || d_max_len < 0) return fail(TSM_EINVAL, "tsm_matrix: max_len < 0");
    return matrix_launch("tsm_matrix", measure, q_pts, q_off, q_len, nullptr, nq, q_max_len, d_pts, d_off, d_len,
                         d_order, nd, nd, d_max_len, 0, params, out, ld_out, out_counts, stream);
}

int tsm_matrix_rows(int measure, const float* q_pts, const int64_t* q_off, const int32_t* q_len,
                    const int32_t* q_rows, int64_t n_rows, int32_t rows_max_len, const float* d_pts,
                    const int64_t* d_off, const int32_t* d_len, const int32_t* d_order, int64_t nd, int32_t d_max_len,
                    const tsm_params* params, float* out, int64_t ld_out, int32_t* out_counts, void* stream) {
    g_err.clear();
    if (measure < TSM_DTW || measure > TSM_HAUSDORFF) return fail(TSM_EINVAL, "tsm_matrix_rows: unknown measure %d", measure);
    if (n_rows < 0 || nd < 0) return fail(TSM_EINVAL, "tsm_matrix_rows: negative set size");
    if (n_rows == 0 || nd == 0) return TSM_OK;
    if (!q_pts || !q_off || !q_len || !q_rows || !d_pts || !d_off || !d_len || !out)
        return fail(TSM_EINVAL, "tsm_matrix_rows: null pointer");
    if (ld_out < nd) return fail(TSM_EINVAL, "tsm_matrix_rows: ld_out < nd");
    if (rows_max_len < 0 || d_max_len < 0) return fail(TSM_EINVAL, "tsm_matrix_rows: max_len < 0");
    return matrix_launch("tsm_matrix_rows", measure, q_pts, q_off, q_len, q_rows, n_rows, rows_max_len, d_pts, d_off,
                         d_len, d_order, nd, nd, d_max_len, 0, params, out, ld_out, out_counts, stream);
}

int tsm_matrix_gather(int measure, const float* q_pts, const int64_t* q_off, const int32_t* q_len, int64_t nq,
                      int32_t q_max_len, const float* d_pts, const int64_t* d_off, const int32_t* d_len, int64_t nd,
                      int32_t d_max_len, const int32_t* cand, int64_t ncand, const int32_t* q_order,
                      const tsm_params* params, float* out, int64_t ld_out, int32_t* out_counts, void* stream) {
    g_err.clear();
    if (measure < TSM_DTW || measure > TSM_HAUSDORFF)
        return fail(TSM_EINVAL, "tsm_matrix_gather: unknown measure %d", measure);
    if (nq < 0 || nd < 0 || ncand < 0) return fail(TSM_EINVAL, "tsm_matrix_gather: negative size");
    if (nq == 0 || ncand == 0) return TSM_OK;
    if (!q_pts || !q_off || !q_len || !d_pts || !d_off || !d_len || !cand || !out)
        return fail(TSM_EINVAL, "tsm_matrix_gather: null pointer");
    if (ld_out < ncand) return fail(TSM_EINVAL, "tsm_matrix_gather: ld_out < ncand");
    if (q_max_len < 0 || d_max_len < 0) return fail(TSM_EINVAL, "tsm_matrix_gather: max_len < 0");
    return matrix_launch("tsm_matrix_gather", measure, q_pts, q_off, q_len, q_order, nq, q_max_len, d_pts, d_off,
                         d_len, cand, ncand, nd, d_max_len, 2, params, out, ld_out, out_counts, stream);
}

int tsm_allpairs_sym(int measure, const float* pts, const int64_t* off, const int32_t* len, const int32_t* order,
                     int64_t n, int32_t max_len, const tsm_params* params, float* out, int64_t ld_out,
                     int32_t* out_counts, void* stream) {
    g_err.clear();
    if (measure < TSM_DTW || measure > TSM_HAUSDORFF)
        return fail(TSM_EINVAL, "tsm_allpairs_sym: unknown measure %d", measure);
    if (n < 0) return fail(TSM_EINVAL, "tsm_allpairs_sym: negative set size");
    if (n == 0) return TSM_OK;
    if (!pts || !off || !len || !order || !out) return fail(TSM_EINVAL, "tsm_allpairs_sym: null pointer");
    if (ld_out < n) return fail(TSM_EINVAL, "tsm_allpairs_sym: ld_out < n");
    if (max_len < 0) return fail(TSM_EINVAL, "tsm_allpairs_sym: max_len < 0");
    return matrix_launch("tsm_allpairs_sym", measure, pts, off, len, order, n, max_len, pts, off, len, order, n,
                         n, max_len, 1, params, out, ld_out, out_counts, stream);
}

int tsm_topk_rows(const float* d, int64_t n_rows, int64_t n_cols, int64_t ld, int32_t k, float* out_d,
                  int32_t* out_idx, void* stream) {
    g_err.clear();
    if (n_rows < 0 || n_cols < 0) return fail(TSM_EINVAL, "tsm_topk_rows: negative size");
    if (k < 1 || k > tsm::kTopkMax) return fail(TSM_EINVAL, "tsm_topk_rows: k must be in 1..%d", tsm::kTopkMax);
    if (n_rows == 0) return TSM_OK;
    if (n_rows > 0x7fffffffLL) return fail(TSM_EINVAL, "tsm_topk_rows: too many rows");
    if (n_cols > 0x7fffffffLL) return fail(TSM_EINVAL, "tsm_topk_rows: column index exceeds int32");
    if (!d || !out_d || !out_idx) return fail(TSM_EINVAL, "tsm_topk_rows: null pointer");
    if (ld < n_cols) return fail(TSM_EINVAL, "tsm_topk_rows: ld < n_cols");
    tsm::topk_rows_kernel<<<(unsigned)n_rows, tsm::kTopkThreads, 0, (cudaStream_t)stream>>>(d, n_cols, ld, k, out_d,
                                                                                              out_idx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "topk_rows_kernel launch");
    return TSM_OK;
}

int tsm_select_rows(const float* d, int64_t n_rows, int64_t n_cols, int64_t ld, int64_t k, int32_t* out_idx,
                    void* stream) {
    g_err.clear();
    if (n_rows < 0 || n_cols < 0 || k < 1) return fail(TSM_EINVAL, "tsm_select_rows: bad size");
    if (n_rows == 0) return TSM_OK;
    if (n_rows > 0x7fffffffLL || n_cols > 0x7fffffffLL) return fail(TSM_EINVAL, "tsm_select_rows: too large");
    if (!d || !out_idx) return fail(TSM_EINVAL, "tsm_select_rows: null pointer");
    if (ld < n_cols) return fail(TSM_EINVAL, "tsm_select_rows: ld < n_cols");
    cudaError_t e = set_smem((const void*)&tsm::select_rows_kernel, (int)tsm::kSelSmemBytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    tsm::select_rows_kernel<<<(unsigned)n_rows, tsm::kTopkThreads, tsm::kSelSmemBytes, (cudaStream_t)stream>>>(
        d, n_cols, ld, k, out_idx);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "select_rows_kernel launch");
    return TSM_OK;
}

int tsm_sched_workspace_bytes(void) { return 256; }

int tsm_pairs_sched(const float* pts, const int64_t* off_a, const int32_t* len_a, const int64_t* off_b,
                    const int32_t* len_b, const int32_t* order, const int32_t* tasks, int32_t n_tasks,
                    int32_t max_len, int32_t warp_smem_floats, const tsm_params* params, float* out,
                    int32_t* out_counts, int64_t out_stride, void* workspace, void* stream) {
    g_err.clear();
    if (n_tasks < 0) return fail(TSM_EINVAL, "tsm_pairs_sched: n_tasks < 0");
    if (n_tasks == 0) return TSM_OK;
    if (!pts || !off_a || !len_a || !off_b || !len_b || !order || !tasks || !out || !workspace)
        return fail(TSM_EINVAL, "tsm_pairs_sched: null pointer");
    if (max_len < 0 || max_len > kMaxLen) return fail(TSM_EINVAL, "tsm_pairs_sched: max_len out of range");
    if (warp_smem_floats < 32 || warp_smem_floats % 32 != 0)
        return fail(TSM_EINVAL, "tsm_pairs_sched: warp_smem_floats must be a positive multiple of 32");
    if (out_stride < 0) return fail(TSM_EINVAL, "tsm_pairs_sched: out_stride < 0");
    const int R = rows_of(params);
    const bool exact = exact_of(params);
    const void* fn = tsm_k::sched(R, exact);
    if (!fn) return fail(TSM_EINVAL, "tsm_pairs_sched: rows_per_thread must be 4 or 8");
    const int W = 4;
    const int smem = W * warp_smem_floats * 4;
    if (smem > kSmemMax) return fail(TSM_ETOOLONG, "tsm_pairs_sched: %d bytes of shared memory per CTA", smem);
    cudaError_t e = set_smem(fn, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute");
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * W, smem)) != cudaSuccess)
        return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) return fail(TSM_ETOOLONG, "tsm_pairs_sched: the kernel does not fit on an SM");
    int grid = sms * per_sm;
    if ((int64_t)grid * W > (int64_t)n_tasks + 4 * W) grid = (n_tasks + W - 1) / W + 1;  // no more warps than tasks
    tsm::PairsArgs A;
    A.pts = reinterpret_cast<const float2*>(pts);
    A.off_a = off_a;
    A.len_a = len_a;
    A.off_b = off_b;
    A.len_b = len_b;
    A.order = order;
    A.max_len = max_len;
    A.p = make_kparams(params);
    A.out = out;
    A.counts = out_counts;
    A.out_stride = out_stride;
    const int4* t4 = reinterpret_cast<const int4*>(tasks);
    int* queue = static_cast<int*>(workspace);
    int nt = n_tasks, total_warps = grid * W, wf = warp_smem_floats;
    void* args[] = {&A, &t4, &nt, &queue, &total_warps, &wf};
    e = cudaLaunchKernel(fn, dim3(grid), dim3(32 * W), args, (size_t)smem, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaLaunchKernel");
    return TSM_OK;
}

}  // extern "C"
