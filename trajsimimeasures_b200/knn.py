"""kNN queries over a trajectory database on the GPU.

The reference answers kNN queries with CPU indices that prune by lower
bounds and refine with exact measures (DITA for DTW/ERP,
query/cpp/DITA.cpp:276-431; DFT for Hausdorff/Frechet, query/cpp/DFT.cpp:89-230;
its GPU refinement bridge Traj::TrajSimiGPU is broken as shipped).  Here:

* ``knn_exhaustive``: exact top-k by evaluating every (query, database) pair
  with the all-pairs kernel, chunk by chunk over the length-sorted database,
  and selecting with the top-k kernel (tsm_topk_rows); per chunk the k best
  are kept, then merged.
* ``knn_rerank``: exact top-k among given candidates (e.g. a learned filter's
  top-200): each query's candidates are evaluated by the matrix kernel in
  gather mode (tsm_matrix_gather: the query staged once, the candidates in
  database-length order), and the best k selected.  ``recall_at_k`` compares
  two answers.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import (DEFAULT_ROWS, MATRIX_QUERY_MAX, TrajSet, _ptr, _stream_ptr, matrix_gather_raw, matrix_raw,
                     measure_id, pairs_raw, same_origin, shift_gpoint)


def topk_rows(d: torch.Tensor, k: int, stream=None):
    """k smallest per row of a float32 CUDA matrix -> (values [n, k], int32 columns [n, k]),
    ascending, ties to the smaller column (a stable argsort's first k)."""
    if d.dtype != torch.float32 or not d.is_cuda or d.dim() != 2 or d.stride(1) != 1:
        raise ValueError("expected a row-major float32 CUDA matrix")
    n, m = d.shape
    vals = torch.empty((n, k), dtype=torch.float32, device=d.device)
    idx = torch.empty((n, k), dtype=torch.int32, device=d.device)
    rc = _lib.load().tsm_topk_rows(_ptr(d), n, m, d.stride(0), int(k), _ptr(vals), _ptr(idx), _stream_ptr(stream))
    _lib.check(rc, "tsm_topk_rows")
    return vals, idx


def _subset(s: TrajSet, idx: torch.Tensor) -> TrajSet:
    """A view of trajectories idx of s (same point pool)."""
    lens_h = s.lens_host[idx.cpu().numpy()] if s.lens_host is not None else None
    out = TrajSet(s.pts, s.off[idx], s.lens[idx], int(lens_h.max()) if lens_h is not None and lens_h.size
                  else int(s.lens[idx].max().item()), lens_h, origin=s.origin)
    out._order = torch.arange(idx.shape[0], dtype=torch.int32, device=s.device)  # idx is length-sorted
    return out


def knn_exhaustive(Q: TrajSet, D: TrajSet, k=10, measure="dtw", *, chunk=1 << 18, eps=0.0, gpoint=(0.0, 0.0),
                   exact=False, stream=None):
    """Exact k nearest database trajectories of every query: (dist float32
    [nq, k], index int64 [nq, k]) ascending, ties to the smaller index."""
    m = measure_id(measure)
    order = D.order_by_length().long()
    best_d, best_i = [], []
    buf = torch.empty((Q.n, min(chunk, D.n)), dtype=torch.float32, device=Q.device)
    for s in range(0, D.n, chunk):
        ids = order[s:s + chunk]
        sub = _subset(D, ids)
        out = buf[:, :sub.n]
        matrix_raw(m, Q, sub, out=out, eps=eps, gpoint=gpoint, exact=exact, stream=stream)
        v, j = topk_rows(out, min(k, sub.n), stream=stream)
        best_d.append(v)
        best_i.append(ids[j.long()])
    dcat = torch.cat(best_d, dim=1)
    icat = torch.cat(best_i, dim=1)
    if len(best_d) == 1:
        return dcat, icat
    # merge the per-chunk lists; ties to the smaller database index: order the
    # concatenated candidates by index first, then a stable top-k by value
    o = torch.argsort(icat, dim=1)
    dcat = torch.gather(dcat, 1, o).contiguous()
    icat = torch.gather(icat, 1, o)
    v, j = topk_rows(dcat, k, stream=stream)
    return v, torch.gather(icat, 1, j.long())


def knn_rerank(Q: TrajSet, D: TrajSet, cand: torch.Tensor, k=10, measure="dtw", *, eps=0.0, gpoint=(0.0, 0.0),
               exact=False, stream=None):
    """Exact top-k among candidate database indices cand [nq, c] (int64):
    (dist [nq, k], index [nq, k])."""
    m = measure_id(measure)
    nq, c = cand.shape
    if Q.max_len <= MATRIX_QUERY_MAX:
        # each query's candidates in database-length order: the query is staged
        # once per CTA (tsm_matrix_gather) and a warp's lanes get equal loop shapes
        o = torch.argsort(D.lens[cand], dim=1, stable=True)
        cs = torch.gather(cand, 1, o).to(torch.int32).contiguous()
        dd = torch.empty((nq, c), dtype=torch.float32, device=Q.device)
        matrix_gather_raw(m, Q, D, cs, out=dd, eps=eps, gpoint=gpoint, exact=exact, stream=stream)
        cand = cs.long()
    else:  # queries too long for the matrix form: the paired kernel, in loop-shape order
        shift = D.pts.shape[0]
        pool = torch.cat([D.pts, Q.pts])  # one point pool for the paired kernel
        qi = torch.arange(nq, device=Q.device).repeat_interleave(c)
        di = cand.reshape(-1).long()
        off_a, len_a = Q.off[qi] + shift, Q.lens[qi]
        off_b, len_b = D.off[di], D.lens[di]
        dd = torch.empty(nq * c, dtype=torch.float32, device=Q.device)
        pairs_raw(m, pool, off_a, len_a, off_b, len_b, max(Q.max_len, D.max_len), out=dd, eps=eps,
                  gpoint=shift_gpoint(gpoint, same_origin(Q, D)), exact=exact, stream=stream,
                  order=shape_order(len_a, len_b))
        dd = dd.view(nq, c)
    # ties to the smaller database index, as in knn_exhaustive
    o = torch.argsort(cand, dim=1)
    dd = torch.gather(dd, 1, o).contiguous()
    ci = torch.gather(cand, 1, o)
    v, j = topk_rows(dd, k, stream=stream)
    return v, torch.gather(ci, 1, j.long())


def shape_order(len_a: torch.Tensor, len_b: torch.Tensor, rows=DEFAULT_ROWS) -> torch.Tensor:
    """engine.pair_order on the device: the pairs ordered by (row blocks,
    columns) of their DP, the largest first, so a warp's 32 lanes run loops of
    equal trip counts (int32 processing order for tsm_pairs)."""
    la, lb = len_a.long(), len_b.long()
    nr, nc = torch.maximum(la, lb), torch.minimum(la, lb)
    key = ((nr + rows - 1) // rows) * 65536 + nc
    return torch.argsort(-key, stable=True).to(torch.int32)


def recall_at_k(approx_idx, exact_idx) -> float:
    """Mean |approx top-k  intersect  exact top-k| / k over the queries."""
    a = np.asarray(approx_idx.cpu() if isinstance(approx_idx, torch.Tensor) else approx_idx)
    e = np.asarray(exact_idx.cpu() if isinstance(exact_idx, torch.Tensor) else exact_idx)
    k = e.shape[1]
    return float(np.mean([len(np.intersect1d(a[i], e[i])) / k for i in range(e.shape[0])]))


def select_rows(d: torch.Tensor, k: int, stream=None) -> torch.Tensor:
    """Column indices (int32 [n, k], any order) of the k smallest values of
    each row of a float32 CUDA matrix (the set of a stable argsort's first k)."""
    if d.dtype != torch.float32 or not d.is_cuda or d.dim() != 2 or d.stride(1) != 1:
        raise ValueError("expected a row-major float32 CUDA matrix")
    n, m = d.shape
    idx = torch.empty((n, k), dtype=torch.int32, device=d.device)
    rc = _lib.load().tsm_select_rows(_ptr(d), n, m, d.stride(0), int(k), _ptr(idx), _stream_ptr(stream))
    _lib.check(rc, "tsm_select_rows")
    return idx


class SurrogateIndex:
    """Database embeddings of a trained encoder, used to pick kNN candidates:
    the c database trajectories nearest to a query in embedding space
    (squared L2 via one TF32 matrix product on mean-centred embeddings with
    the squared norms folded in, then the sampled-threshold selection kernel),
    then reranked by exact DP.

    The candidate count is calibrated, not guessed: ``calibrate`` runs the
    exhaustive search on a sample of queries and takes the smallest count of
    a ladder whose recall@k reaches the target; if none does within the
    speed budget, queries fall back to the exhaustive search."""

    LADDER = (200, 500, 1000, 1500, 2000, 2500, 3000, 4000, 5000, 7000, 10000, 20000, 50000)

    # embedding width + 1 (the squared norm), padded to a multiple of 4 floats
    AUG = 132

    def __init__(self, encoder, D: TrajSet, batch=None):
        self.enc = encoder
        self.D = D
        emb = encoder.embed(D, batch=batch)
        w = emb.shape[1]
        # Embeddings are centred on the database mean mu (distances do not
        # change): a TF32 product rounds its inputs to 11 significant bits,
        # relative to their size, and a trained network's embeddings share a
        # large common offset.  Measured on the trained encoder (1,000 queries
        # x 1M, recall@10 at 200 / 5,000 candidates): FP32 0.463 / 0.9998,
        # TF32 0.202 / 0.998, centred TF32 0.437 / 0.9998.
        self.mu = emb.mean(0)
        emb = emb - self.mu
        # augmented rows [e_j, |e_j|^2, 0...]: one product with [-2 e_q, 1, 0...]
        # gives |e_j|^2 - 2 e_q.e_j, the squared distance less the query's own
        # |e_q|^2, which does not change a query's ranking
        self.aug = torch.zeros((emb.shape[0], max(self.AUG, (w + 4) // 4 * 4)), dtype=torch.float32,
                               device=emb.device)
        self.aug[:, :w] = emb
        self.aug[:, w] = (emb * emb).sum(1)
        self.width = w
        self.c = None

    @property
    def emb(self) -> torch.Tensor:
        """Database embeddings [n, width]."""
        return self.aug[:, :self.width] + self.mu

    def scan(self, e: torch.Tensor) -> torch.Tensor:
        """Embedding-space distances (less |e_q - mu|^2) of queries e [b, width]
        to every database trajectory: one TF32 tensor-core product, FP32
        accumulation and output ([b, n] float32)."""
        q = torch.zeros((e.shape[0], self.aug.shape[1]), dtype=torch.float32, device=e.device)
        q[:, :self.width] = -2.0 * (e - self.mu)
        q[:, self.width] = 1.0
        mm = torch.backends.cuda.matmul
        prev = mm.allow_tf32
        mm.allow_tf32 = True
        try:
            return q @ self.aug.T
        finally:
            mm.allow_tf32 = prev

    def candidates(self, Q: TrajSet, c: int, chunk=1024) -> torch.Tensor:
        """Candidate indices [nq, c] (int64, any order).  chunk queries per
        scan: one [chunk, n] float32 distance block (4 GB at 1024 x 1M); 1,000
        queries x 1M on B200, ms: 4.76 at 256, 4.56 at 512, 4.23 at 1024."""
        eq = self.enc.embed(Q)
        out = torch.empty((Q.n, c), dtype=torch.int64, device=Q.device)
        for q0 in range(0, Q.n, chunk):
            d = self.scan(eq[q0:q0 + chunk])
            out[q0:q0 + d.shape[0]] = select_rows(d, c).long()
        return out

    def query(self, Q: TrajSet, k=10, c=None, measure="dtw", **kw):
        c = c or self.c
        if c is None:  # not calibrated, or the filter could not reach the target: exhaustive
            return knn_exhaustive(Q, self.D, k, measure, **kw)
        cand = self.candidates(Q, min(c, self.D.n))
        return knn_rerank(Q, self.D, cand, k, measure, **kw)

    def calibrate(self, Q_sample: TrajSet, k=10, target=0.99, max_fraction=0.05, margin=None, measure="dtw",
                  **kw):
        """-> (chosen count or None, {count: recall}) on the sample.

        A count is chosen only if its sample recall clears the target by a
        margin of two standard errors of a recall measured on n*k answers
        (default), so that the recall on the full query set does not fall
        below the target by sampling noise."""
        _, exact = knn_exhaustive(Q_sample, self.D, k, measure, **kw)
        if margin is None:
            margin = 2.0 * float(np.sqrt(target * (1.0 - target) / (Q_sample.n * k)))
        rec = {}
        self.c = None
        for c in self.LADDER:
            if c > max_fraction * self.D.n and c > self.LADDER[0]:
                break
            _, got = self.query(Q_sample, k, c=c, measure=measure, **kw)
            rec[c] = recall_at_k(got, exact)
            if rec[c] >= min(target + margin, 1.0):
                self.c = c
                break
        return self.c, rec


def merge_topk(dists: torch.Tensor, idx: torch.Tensor, k: int):
    """Merge candidate lists [nq, m] (values, global indices) into the k
    smallest per row, ties to the smaller index (the order of a stable
    argsort over the whole database).  Device-agnostic tensor ops."""
    o = torch.argsort(idx, dim=1, stable=True)
    d = torch.gather(dists, 1, o)
    i = torch.gather(idx, 1, o)
    o2 = torch.argsort(d, dim=1, stable=True)[:, :k]
    return torch.gather(d, 1, o2), torch.gather(i, 1, o2)


def shard_range(n: int, rank: int, world: int):
    """Contiguous database shard [start, end) of a rank (sizes differ by <= 1)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def knn_sharded(local_topk, Q_n: int, k: int, shard_start: int, group=None):
    """Multi-GPU kNN merge.  local_topk = (dist [nq, k], index [nq, k]) of this
    rank's database shard, indices local to the shard; returns the global
    (dist, index) on every rank after one all-gather of the lists (the only
    exchange: nq * k * 12 bytes per rank)."""
    import torch.distributed as dist
    d, i = local_topk
    i = i.long() + shard_start
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return merge_topk(d, i, k)
    w = dist.get_world_size(group)
    ds = [torch.empty_like(d) for _ in range(w)]
    is_ = [torch.empty_like(i) for _ in range(w)]
    dist.all_gather(ds, d.contiguous(), group=group)
    dist.all_gather(is_, i.contiguous(), group=group)
    return merge_topk(torch.cat(ds, 1), torch.cat(is_, 1), k)
