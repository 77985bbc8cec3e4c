/*
 * tsm.h -- C ABI of the B200 trajectory-similarity library (libtsm_b200.so).
 *
 * Replaces the reference's batched GPU measures, which are Python functions
 * exported by core/__init__.py:1-10 and registered by name in
 * utilities/method_helper.py:32-73 (heuristic_fn_wrapper):
 *
 *   core.dtw(t1, len1, t2, len2, threads_per_traj=64)         core/dtw.py:56-77
 *   core.edr(t1, len1, t2, len2, eps, threads_per_traj=64)    core/edr.py:55-76
 *   core.lcss(t1, len1, t2, len2, eps, threads_per_traj=64)   core/lcss.py:56-77
 *   core.erp(t1, len1, t2, len2, gpoint=None, threads_per_traj=64)  core/erp.py:94-120
 *   core.dfrechet(t1, len1, t2, len2, threads_per_traj=64)    core/discret_frechet.py:53-74
 *   core.hausdorff(t1, len1, t2, len2, threads_per_traj=64)   core/hausdorff.py:97-123
 *
 * The Python package trajsimimeasures_b200 keeps those signatures and calls
 * this ABI through ctypes.
 *
 * Conventions
 *  - Trajectories are packed: one float32 array of (x, y) points, plus per
 *    trajectory an int64 offset (in points) and an int32 length.
 *  - Every pointer argument is DEVICE memory owned by the caller (for example
 *    torch tensors).  `params` is a host pointer.  `stream` is a cudaStream_t
 *    (NULL = legacy default stream).
 *  - Calls only enqueue work on `stream` and return; results are valid after
 *    the stream is synchronised.  The library allocates no device memory in
 *    these calls.  Calls on different streams may run concurrently.
 *  - Return value: 0 on success, a negative TSM_E* code otherwise; nothing is
 *    thrown across the ABI.  tsm_last_error() gives the calling thread's last
 *    message.  Pairs whose lengths are negative or exceed the declared
 *    `max_len` are written as NaN (counts -1) instead of being computed.
 *  - Degenerate lengths follow the reference kernels: DTW/Frechet of two empty
 *    trajectories is 0 and of one empty trajectory +inf; ERP with an empty
 *    trajectory is 0; EDR/LCSS with a zero denominator are NaN; Hausdorff
 *    gives 0 for a direction whose target has fewer than two points.
 */
#ifndef TSM_B200_H
#define TSM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Measures (same numbering as the oracle). */
#define TSM_DTW 0
#define TSM_EDR 1
#define TSM_LCSS 2
#define TSM_ERP 3
#define TSM_DFRECHET 4
#define TSM_HAUSDORFF 5

/* flags */
#define TSM_FLAG_EXACT 1u /* IEEE sqrt/reciprocal per cell: results are bit-identical to the
                             FP32 twin in the oracle (default: hardware approximations,
                             within 1e-6 relative) */

/* error codes */
#define TSM_OK 0
#define TSM_EINVAL -1   /* bad argument */
#define TSM_ECUDA -2    /* a CUDA runtime call failed (message has the CUDA error) */
#define TSM_ETOOLONG -3 /* max_len beyond what the library supports */
#define TSM_ETIMEOUT -4 /* a bounded wait inside a kernel ran out (see tsm_enc_embed_status) */

typedef struct tsm_params {
    double eps;       /* EDR/LCSS match threshold (same units as the points); the
                         kernels compare dx*dx+dy*dy < (float)(eps*eps) in FP32 */
    double gx, gy;    /* ERP gap point (reference default (0, 0), core/erp.py:103) */
    uint32_t flags;   /* TSM_FLAG_* */
    int32_t rows_per_thread; /* 0 = default; else 4, 8 or 16 (register tile height) */
} tsm_params;

/* Library version (major*10000 + minor*100 + patch). */
int tsm_version(void);

/* Last error message of the calling thread ("" if none). */
const char* tsm_last_error(void);

/* Largest trajectory length the paired kernels accept (points): 32768.
 * Longer inputs are rejected with TSM_ETOOLONG (the reference's datasets are
 * cut to 20..200 points, config.py:51-52, and its timing sweep reaches 1,600,
 * test_trajsimi_time.py:109). */
int32_t tsm_max_supported_len(void);

/* Longest query of the matrix forms (tsm_matrix, tsm_matrix_gather,
 * tsm_allpairs_sym; Hausdorff excepted): 1400 points, whose boundary rows and
 * staged columns fill a CTA's shared memory.  Longer queries get
 * TSM_ETOOLONG; the Python layer (core.matrix, core.allpairs,
 * core.matrix_many) computes their rows with tsm_pairs instead. */
int32_t tsm_matrix_query_max(void);

/*
 * Paired batch: out[k] = measure(traj a_k, traj b_k) for k < n_pairs.
 * Replaces core.<measure>(t1, len1, t2, len2, ...) (per-pair batch form, the
 * call made by test_trajsimi_time.py:253).
 *   pts     float32 [n_points][2]
 *   off_a, off_b  int64 [n_pairs]   first point of each trajectory
 *   len_a, len_b  int32 [n_pairs]   lengths; every length <= max_len
 *   order   int32 [n_pairs] or NULL: processing order (a permutation of
 *           0..n_pairs-1 grouping pairs of similar shape), results are still
 *           written at the pair's own index
 *   out     float32 [n_pairs]
 *   out_counts int32 [n_pairs] or NULL: EDR/LCSS edit/match counts before
 *           normalisation (ignored for other measures)
 * When max_len exceeds 256 (Hausdorff: when max_len^2 exceeds 2^17), the
 * long pairs' kernel runs on a stream of the
 * calling thread forked from `stream` (an event record / wait on each side;
 * the side stream and its two events are created once per thread and
 * device).  `stream` waits for it before the call returns, so later work on
 * `stream`, and a graph captured from it, see the complete result.
 */
int tsm_pairs(int measure, const float* pts, const int64_t* off_a, const int32_t* len_a,
              const int64_t* off_b, const int32_t* len_b, const int32_t* order, int64_t n_pairs,
              int32_t max_len, const tsm_params* params, float* out, int32_t* out_counts,
              void* stream);

/*
 * Per-query candidate lists (the refinement step of a kNN query):
 *   out[i*ld_out + s] = measure(Q_i, D_{cand[i*ncand + s]}),  i < nq, s < ncand.
 * Replaces the exact refinement of filtered candidates in the reference's kNN
 * queries (query/cpp/DITA.cpp:276-431, DFT.cpp:89-230, which evaluate the
 * measure on each surviving candidate; and its GPU bridge Traj::TrajSimiGPU,
 * query/cpp/spatial/traj.cpp:242-360, which was meant to batch them).
 *   cand int32 [nq][ncand]: database indices; a query's row is best sorted by
 *        database length (neighbouring threads then get equal loop shapes);
 *        an index outside 0..nd-1 gives NaN (count -1) for that entry
 *   q_order int32 [nq] or NULL: the order in which the queries are processed
 *        (a permutation of 0..nq-1; longest first shortens the tail of the
 *        launch); rows of cand and out stay indexed by query
 *   ld_out >= ncand; the other arguments as in tsm_matrix
 */
int tsm_matrix_gather(int measure, const float* q_pts, const int64_t* q_off, const int32_t* q_len, int64_t nq,
                      int32_t q_max_len, const float* d_pts, const int64_t* d_off, const int32_t* d_len, int64_t nd,
                      int32_t d_max_len, const int32_t* cand, int64_t ncand, const int32_t* q_order,
                      const tsm_params* params, float* out, int64_t ld_out, int32_t* out_counts, void* stream);

/*
 * All pairs of a query set Q and a database set D:
 *   out[i*ld_out + j] = measure(Q_i, D_j),  i < nq, j < nd.
 * Replaces the host-side Q x D pair expansion + batched core.<measure> calls of
 * test_trajsimi_time_DQ.py:147-173 (and, with Q == D, the all-pairs matrix of
 * test_clustering_time.py:219-269).
 *   q_pts/d_pts float32 [.][2]; q_off/d_off int64; q_len/d_len int32
 *   d_order int32 [nd] or NULL: processing order of D (e.g. D sorted by length)
 *   q_max_len, d_max_len: upper bounds of the lengths in Q and D
 *   out float32 [nq][ld_out]; out_counts int32 [nq][ld_out] or NULL (EDR/LCSS)
 */
int tsm_matrix(int measure, const float* q_pts, const int64_t* q_off, const int32_t* q_len, int64_t nq,
               int32_t q_max_len, const float* d_pts, const int64_t* d_off, const int32_t* d_len,
               const int32_t* d_order, int64_t nd, int32_t d_max_len, const tsm_params* params,
               float* out, int64_t ld_out, int32_t* out_counts, void* stream);

/*
 * Selected rows of the Q x D matrix: for r < n_rows, with i = q_rows[r],
 *   out[i*ld_out + j] = measure(Q_i, D_j),  j < nd
 * (the other rows of out are not touched).  rows_max_len bounds the lengths
 * of the selected queries only: launched for a group of queries of similar
 * length, the kernel's shared memory (boundary rows and staged columns of
 * rows_max_len points) admits more CTAs per SM than one launch sized for the
 * longest query of Q.  Same reference call as tsm_matrix.
 */
int tsm_matrix_rows(int measure, const float* q_pts, const int64_t* q_off, const int32_t* q_len,
                    const int32_t* q_rows, int64_t n_rows, int32_t rows_max_len, const float* d_pts,
                    const int64_t* d_off, const int32_t* d_len, const int32_t* d_order, int64_t nd, int32_t d_max_len,
                    const tsm_params* params, float* out, int64_t ld_out, int32_t* out_counts, void* stream);

/*
 * Symmetric all pairs of one set S (the clustering shape):
 *   out[i*ld_out + j] = out[j*ld_out + i] = measure(S_i, S_j),  i, j < n,
 * computing each unordered pair once (every measure here is symmetric, and
 * the kernels' values are bitwise symmetric, so the mirror equals the value
 * computed the other way round).  Replaces the upper-triangle pair
 * enumeration + batched core.<measure> calls of test_clustering_time.py:219-269.
 *   order int32 [n]: a permutation of 0..n-1, S sorted by length (required:
 *         the triangle is taken in this order, so neighbouring threads get
 *         trajectories of similar length)
 *   max_len: upper bound of the lengths in S
 *   out float32 [n][ld_out]; out_counts int32 [n][ld_out] or NULL (EDR/LCSS)
 */
int tsm_allpairs_sym(int measure, const float* pts, const int64_t* off, const int32_t* len, const int32_t* order,
                     int64_t n, int32_t max_len, const tsm_params* params, float* out, int64_t ld_out,
                     int32_t* out_counts, void* stream);

/*
 * Scheduled paired batch: one persistent launch over a task list that the
 * planner (trajsimimeasures_b200.sched) builds from the pair lengths.  It
 * replaces the same reference call as tsm_pairs (core.<measure>(t1, len1,
 * t2, len2), batched 512 pairs at a time by test_trajsimi_time.py:222-276),
 * for batches of very uneven lengths and several measures at once.
 *   tasks      device int32 [n_tasks][4] = {kind, measure, first, count}:
 *              pairs order[first .. first+count) as one warp task; kind 0 =
 *              one pair per lane, 5 / 1 / 6 / 2 = one pair per 4 / 8 / 16 /
 *              32 lanes, 3 = Hausdorff one pair per lane, 4 = Hausdorff one
 *              pair per warp.  Warps take the tasks in this order.
 *   warp_smem_floats  shared memory per warp (floats), a multiple of 32: a
 *              pair's shorter side may be up to warp_smem_floats/32 columns
 *              in kind 0 and warp_smem_floats*G/32 in a G-lane kind; a pair
 *              beyond its kind's capacity gets NaN (count -1)
 *   out        float32 [n_measures_used][out_stride]: out[measure*out_stride + pair]
 *   out_counts int32, same layout (EDR/LCSS), or NULL
 *   workspace  device memory of tsm_sched_workspace_bytes() bytes, zeroed
 *              once by the caller before its first use; the kernel leaves it
 *              zeroed again at exit (a task queue head and an exit count).
 *              Launches that share a workspace must not overlap.
 */
int tsm_sched_workspace_bytes(void);

int tsm_pairs_sched(const float* pts, const int64_t* off_a, const int32_t* len_a, const int64_t* off_b,
                    const int32_t* len_b, const int32_t* order, const int32_t* tasks, int32_t n_tasks,
                    int32_t max_len, int32_t warp_smem_floats, const tsm_params* params, float* out,
                    int32_t* out_counts, int64_t out_stride, void* workspace, void* stream);

/*
 * tsm_pairs_sched without a workspace argument: the same persistent launch,
 * with its scratch (the 8-byte task queue) in a 256-byte array that the
 * library allocates statically on every GPU that loads it.  No counterpart in
 * the reference (its GPU calls allocate per call through Numba).  For callers
 * that cannot allocate device memory where they call (host callbacks,
 * sections that must not touch the CUDA allocator, plugins whose host owns all
 * device memory, FFI callers without an allocator); inputs and outputs are
 * still theirs.  The array is shared by every call: calls that overlap on the
 * GPU race and give wrong results.  The first call on a device sets the array
 * up (symbol lookup + clear + device synchronisation): make it before any
 * stream capture.  Returns TSM_ETOOLONG if the kernel's scratch would exceed
 * the array.
 */
int tsm_pairs_sched_noalloc(const float* pts, const int64_t* off_a, const int32_t* len_a, const int64_t* off_b,
                            const int32_t* len_b, const int32_t* order, const int32_t* tasks, int32_t n_tasks,
                            int32_t max_len, int32_t warp_smem_floats, const tsm_params* params, float* out,
                            int32_t* out_counts, int64_t out_stride, void* stream);

/*
 * Row-wise k smallest (kNN result lists): for each row r < n_rows of the
 * float32 matrix d (row stride ld), the k smallest values in ascending order,
 * ties to the smaller column index (= the first k entries of a stable argsort;
 * NaN after +inf).  out_d float32 [n_rows][k], out_idx int32 [n_rows][k];
 * rows shorter than k are padded with +inf / -1.  k <= 256.
 * The reference's kNN answers queries with CPU index pruning
 * (query/cpp/DITA.cpp:276-431, DFT.cpp:89-230: std::nth_element over refined
 * candidates); this is the selection step of the exhaustive GPU replacement.
 */
int tsm_topk_rows(const float* d, int64_t n_rows, int64_t n_cols, int64_t ld, int32_t k, float* out_d,
                  int32_t* out_idx, void* stream);

/*
 * Unordered selection for long candidate lists: out_idx int32 [n_rows][k]
 * receives, per row, the column indices of the k smallest values (the set of
 * a stable argsort's first k, any order); -1 pads rows shorter than k.  Any k.
 */
int tsm_select_rows(const float* d, int64_t n_rows, int64_t n_cols, int64_t ld, int64_t k, int32_t* out_idx,
                    void* stream);

/*
 * Candidate scan of the learned kNN filter on the tensor cores (tcgen05).
 * Replaces the candidate generation of the reference's filter-and-refine kNN
 * (query/cpp/DITA.cpp:276-431; the learned kNN's embedding scan,
 * test_knn_time.py:138-202).  For embeddings of tsm_scan_dim() values
 * (centred by the caller), d(q, j) = |e_j|^2 - 2 e_q . e_j, computed as one
 * product of FP16 hi/lo splits, [q_hi | q_lo | q_hi] . [d_hi | d_hi | d_lo],
 * with the squared norms (three FP16 parts) folded into the same product and
 * FP32 accumulation (about 2^-21 relative per product).
 *   tsm_scan_prepare: operand image of n rows of emb (row stride ld floats),
 *       scaled by `scale`, a power of two keeping |scale * emb| <= 1024;
 *       is_db = 1: database image (tiles of 256 rows), and norms float32 [n]
 *       (nullable) receives |emb_j|^2; 0: query image (tiles of 128 rows).
 *       img: device memory of tsm_scan_image_bytes(n, is_db) bytes, 16-byte
 *       aligned.
 *   tsm_scan: either dense (thresholds NULL): dense[q * ld_dense + j] = d;
 *       or candidate lists (dense NULL): for each pair with d <= thresholds[q]
 *       a slot of counts[q] (zeroed by the caller) is taken and, below cap,
 *       cand_idx[q * cap + slot] = j, cand_d[q * cap + slot] = d (any order;
 *       counts[q] > cap means the list overflowed).  The same d in both modes.
 *       status: device int, OR-ed with 1/2/8 when a bounded wait inside the
 *       kernel ran out (results then incomplete), 4 when tensor memory was
 *       left allocated because MMAs were still pending (reset the device).
 */
int32_t tsm_scan_dim(void);
int64_t tsm_scan_image_bytes(int64_t n_rows, int32_t is_db);
int tsm_scan_prepare(const float* emb, int64_t n, int64_t ld, float scale, int32_t is_db, void* img, float* norms,
                     void* stream);
int tsm_scan(const void* q_img, int64_t nq, const void* db_img, int64_t nd, float scale, const float* thresholds,
             int32_t cap, int32_t* cand_idx, float* cand_d, int32_t* counts, float* dense, int64_t ld_dense,
             int32_t* status, void* stream);
/* tsm_scan with its wait limit in SM clocks (tsm_scan uses about 1 s). */
int tsm_scan_opts(const void* q_img, int64_t nq, const void* db_img, int64_t nd, float scale, const float* thresholds,
                  int32_t cap, int32_t* cand_idx, float* cand_d, int32_t* counts, float* dense, int64_t ld_dense,
                  int32_t* status, int64_t wait_cycles, void* stream);

/*
 * Learned candidate filter (trajectory encoder).  The reference's learned
 * measures embed trajectories and train on heuristic distances normalised by
 * their maximum with an MSE loss (nn/MLP_trajsimi_train.py:74-84,197-200); this
 * encoder (conv 2->64 k=5 + GRU 64->128 + linear 128->128, BF16 weights, FP32
 * accumulation, plus a geometric skip: the trajectory's 16 points at indices
 * round(k (n-1) / 15), normalised, each times its learned weight exp(u_k),
 * appended as 32 more embedding values) is trained the same way on DTW labels from
 * tsm_pairs and serves as a kNN filter.  Embeddings are 160 floats.
 *   params  float32 [tsm_enc_param_count()] master weights (layout: conv W
 *           [64][2][5], b [64]; W_ih [384][64], b_ih [384]; W_hh [384][128],
 *           b_hh [384]; W_o [128][128], b_o [128]; skip log-weights u [16];
 *           gate order r, z, n)
 *   pts/off/len  a packed batch of B trajectories, T = max length in it
 *   nrm     HOST float[4] = (mean_x, mean_y, 1/s_x, 1/s_y) input scaling (the
 *           Python encoder uses one scale for both axes, s_x = s_y)
 *   workspace  device memory of tsm_enc_workspace_bytes(B, T, P) bytes, 256-byte
 *           aligned; its first 4 bytes are the training status word
 *           (tsm_enc_train_status): zero them once after allocating it
 */
int tsm_enc_param_count(void);
int64_t tsm_enc_workspace_bytes(int32_t B, int32_t T, int32_t P);
/* emb float32 [B][160] (device) */
int tsm_enc_forward(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                    int32_t T, const float* nrm, void* workspace, float* emb, void* stream);
/* Inference-only forward on the tensor cores (tcgen05): 128 trajectories per
 * CTA, each GRU step one set of BF16 x BF16 -> FP32 MMAs into tensor memory,
 * with a_t and h_t entering the products as BF16 (the training forward above
 * keeps them FP32), and no training caches.  Used to embed the kNN database
 * and the queries: the test-time embedding of the reference's learned
 * measures (nn/MLP_trajsimi_train.py).  emb float32 [B][160] (device);
 * workspace of tsm_enc_embed_workspace_bytes(B, T) bytes, 256-byte aligned.  Batches of similar
 * lengths waste fewer steps (a CTA runs its longest trajectory's length). */
int64_t tsm_enc_embed_workspace_bytes(int32_t B, int32_t T);
int tsm_enc_embed(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                  int32_t T, const float* nrm, void* workspace, float* emb, void* stream);
/* Status of the last tsm_enc_embed call on this workspace: synchronises
 * `stream`, copies the status word (the first 4 bytes of the workspace, set to
 * 0 by each call) into *status and returns TSM_OK if it is 0.  The kernel's
 * waits on its own copies and tensor-core MMAs are bounded (about 1 s of SM
 * clocks); a wait that runs out sets a bit (1: an a_t copy, 2: an MMA step,
 * 4: tensor memory left allocated because MMAs were still pending -- the
 * context should then be reset), writes NaN for that CTA's trajectories and
 * makes this call return TSM_ETIMEOUT with a message. */
int tsm_enc_embed_status(const void* workspace, int32_t* status, void* stream);
/* Status of the training calls (tsm_enc_loss_grad*) made with this
 * workspace since the last check: synchronises the stream, reads the
 * workspace's first word into *status and clears it.  The word holds bits
 * OR-ed in by the tensor-core weight-gradient kernel when one of its bounded
 * waits ran out (16 copy, 32 MMA, 64 completion, 128 tensor memory left
 * allocated); the gradients are then incomplete.  Zero the word once when the
 * workspace is allocated.  Returns TSM_ETIMEOUT when it was nonzero. */
int tsm_enc_train_status(void* workspace, int32_t* status, void* stream);
/* tsm_enc_embed with its wait limit (SM clocks, >= 1) and a failure-path test
 * hook: stall_step >= 0 announces that step's a_t copy on its mbarrier but
 * never issues it, so that every CTA's wait for it runs out with no MMA in
 * flight; -1 in normal use.  tsm_enc_embed = (wait limit ~1 s, -1). */
int tsm_enc_embed_opts(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                       int32_t T, const float* nrm, void* workspace, float* emb, int64_t wait_cycles,
                       int32_t stall_step, void* stream);
/* Forward + pair loss + backward.  Pairs (ia[p], ib[p]) index the batch,
 * y[p] the target distances; loss = mean_p (||e_ia - e_ib|| - y)^2.
 * grad float32 [param_count] (overwritten), loss float32 [1], pred [P]
 * (both device, nullable). */
int tsm_enc_loss_grad(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                      int32_t T, const float* nrm, const int32_t* ia, const int32_t* ib, const float* y, int32_t P,
                      void* workspace, float* grad, float* loss, float* pred, void* stream);
/* The same with per-pair weights (device float32 [P], nullable = all 1):
 * loss = mean_p w_p (||e_ia - e_ib|| - y_p)^2.  Weights 1 / y_p^2 give the
 * relative error, which keeps the near pairs (the ones a kNN filter must
 * order) from vanishing next to the far ones. */
int tsm_enc_loss_grad_w(const float* params, const float* pts, const int64_t* off, const int32_t* len, int32_t B,
                        int32_t T, const float* nrm, const int32_t* ia, const int32_t* ib, const float* y,
                        const float* weights, int32_t P, void* workspace, float* grad, float* loss, float* pred,
                        void* stream);
/* One Adam step on params with moments m, v (device, param_count each). */
int tsm_enc_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr, float beta1,
                 float beta2, float eps, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TSM_B200_H */
