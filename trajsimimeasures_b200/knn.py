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
import math

import numpy as np
import torch

from . import _lib
from .engine import (DEFAULT_ROWS, MATRIX_QUERY_MAX, TrajSet, _ptr, _stream_ptr, matrix_gather_raw, matrix_raw,
                     measure_id, pair_order_dev, pairs_raw, same_origin, shift_gpoint)


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
               exact=False, stream=None, gather_lpt=True):
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
        # longest queries first: their CTAs run longest, so the launch ends with short ones
        qo = torch.argsort(Q.lens, descending=True, stable=True).to(torch.int32) if gather_lpt else None
        matrix_gather_raw(m, Q, D, cs, out=dd, eps=eps, gpoint=gpoint, exact=exact, stream=stream, q_order=qo)
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
    return pair_order_dev(len_a, len_b, rows)


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
    the c database trajectories nearest to a query in embedding space, then
    reranked by exact DP.

    Candidate scan (tsm_scan, tensor cores): embeddings centred on the
    database mean, split into FP16 hi/lo pairs, |e_j|^2 - 2 e_q.e_j from one
    split product in FP32 accumulation (about 2^-21 relative per product: a
    TF32 product, at 2^-11, cannot separate the nearest of a million
    trajectories).  A threshold per query comes from a dense scan of a fixed
    sample of SAMPLE database rows (the order statistic whose expected count
    in the full database is 1.25 c plus four standard deviations); the full
    scan keeps only the pairs under it, in per-query lists, and the exact c
    smallest are selected from those.  A query whose list holds fewer than c
    or overflowed is scanned densely instead.

    Two things are calibrated, not guessed: the weight of the recurrent
    branch against the geometric skip in the scan's distance (BRANCH_WEIGHTS;
    the training objective, a regression on distances, does not set the
    balance that ranks the nearest few best) and the candidate count (LADDER).
    ``calibrate`` runs the exhaustive search on a sample of queries and takes
    the smallest count, over the weights, whose recall@k reaches the target;
    if none does within the speed budget, queries fall back to the
    exhaustive search."""

    LADDER = (100, 200, 300, 500, 700, 1000, 1500, 2000, 3000, 5000, 7000, 10000, 20000, 50000)
    BRANCH_WEIGHTS = (1.0, 0.5, 0.3, 0.1)
    SAMPLE = 16384
    SCALED_TOP = 1024.0  # largest scaled magnitude of an operand value (tsm_scan_prepare)

    def __init__(self, encoder, D: TrajSet, batch=None, branch_weight=1.0):
        self.enc = encoder
        self.D = D
        emb = encoder.embed(D, batch=batch)
        self.width = emb.shape[1]
        if self.width != _lib.load().tsm_scan_dim():
            raise ValueError(f"the scan takes {_lib.load().tsm_scan_dim()}-value embeddings, got {self.width}")
        self.mu = emb.double().mean(0).float()
        self.E = emb - self.mu  # centred (distances do not change)
        n = self.E.shape[0]
        self.sample = torch.arange(0, n, max(1, n // self.SAMPLE), device=emb.device)[:self.SAMPLE]
        self.status = torch.zeros(1, dtype=torch.int32, device=emb.device)
        self.c = None
        self.set_branch_weight(branch_weight)

    # -- operand images ------------------------------------------------------
    def set_branch_weight(self, beta: float):
        """Re-weights the recurrent branch (the first width - 32 values) in the
        scan's distance and rebuilds the database operand images."""
        self.beta = float(beta)
        self.wt = torch.ones(self.width, dtype=torch.float32, device=self.E.device)
        self.wt[:self.width - 32] = self.beta
        X = self.E * self.wt
        top = float(X.abs().max()) if X.numel() else 1.0
        self.scale = float(2.0 ** math.floor(math.log2(self.SCALED_TOP / max(top, 1e-30))))
        self.img = self._image(X, True)
        self.s_img = self._image(X[self.sample].contiguous(), True)

    def _image(self, X, is_db):
        lib = _lib.load()
        n = X.shape[0]
        img = torch.empty(max(lib.tsm_scan_image_bytes(n, int(is_db)), 16), dtype=torch.uint8, device=X.device)
        rc = lib.tsm_scan_prepare(_ptr(X), n, X.stride(0), self.scale, int(is_db), _ptr(img), None,
                                  _stream_ptr(None))
        _lib.check(rc, "tsm_scan_prepare")
        return img

    def _query_image(self, e):
        X = ((e - self.mu) * self.wt).contiguous()
        return self._image(X, False)

    @property
    def emb(self) -> torch.Tensor:
        """Database embeddings [n, width]."""
        return self.E + self.mu

    # -- scans ------------------------------------------------------------------
    def _dense(self, qimg, nq, img, nd):
        out = torch.empty((nq, nd), dtype=torch.float32, device=self.E.device)
        rc = _lib.load().tsm_scan(_ptr(qimg), nq, _ptr(img), nd, self.scale, None, 0, None, None, None, _ptr(out), nd,
                                  _ptr(self.status), _stream_ptr(None))
        _lib.check(rc, "tsm_scan")
        return out

    def scan(self, e: torch.Tensor) -> torch.Tensor:
        """Embedding-space distances (less |e_q - mu|^2 in the weighted
        space) of queries e [b, width] to every database trajectory
        ([b, n] float32, dense)."""
        return self._dense(self._query_image(e), e.shape[0], self.img, self.E.shape[0])

    def _check_status(self):
        st = int(self.status.item())
        if st:
            self.status.zero_()
            raise _lib.TsmError(f"tsm_scan: a tensor-core wait ran out (status {st})")

    def candidates(self, Q: TrajSet, c: int, chunk=4096, scan_events=None) -> torch.Tensor:
        """Candidate indices [nq, c] (int64, any order).  scan_events: a list
        to which (start, end, queries, rows) CUDA events are appended around
        each main scan launch (for timing it on its stream).  The host waits
        on the device once per chunk, for the status words and the overflow
        count together."""
        lib = _lib.load()
        n = self.E.shape[0]
        c = min(int(c), n)
        enc_status = torch.zeros(1, dtype=torch.int32, device=Q.device)
        eq = self.enc.embed(Q, status_out=enc_status)
        dense_only = False
        out = torch.empty((Q.n, c), dtype=torch.int64, device=Q.device)
        S = int(self.sample.shape[0])
        exp = c * S / n
        ks = int(min(S, max(1, math.ceil(1.25 * exp + 4.0 * math.sqrt(exp)))))
        expect = ks * n / S  # expected list length at the threshold
        cap = int(min(n, math.ceil(expect + 6.0 * expect / math.sqrt(ks)) + 64))
        for q0 in range(0, Q.n, chunk):
            e = eq[q0:q0 + chunk]
            b = e.shape[0]
            qimg = self._query_image(e)
            if ks >= S or cap >= n:  # the list would hold most of the database: dense
                out[q0:q0 + b] = select_rows(self._dense(qimg, b, self.img, n), c).long()
                dense_only = True
                continue
            ds = self._dense(qimg, b, self.s_img, S)
            thr = torch.topk(ds, ks, dim=1, largest=False, sorted=True).values[:, -1].contiguous()
            idx = torch.empty((b, cap), dtype=torch.int32, device=Q.device)
            dd = torch.full((b, cap), float("inf"), dtype=torch.float32, device=Q.device)
            cnt = torch.zeros(b, dtype=torch.int32, device=Q.device)
            if scan_events is not None:
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                ev[0].record()
            rc = lib.tsm_scan(_ptr(qimg), b, _ptr(self.img), n, self.scale, _ptr(thr), cap, _ptr(idx), _ptr(dd),
                              _ptr(cnt), None, 0, _ptr(self.status), _stream_ptr(None))
            _lib.check(rc, "tsm_scan")
            if scan_events is not None:
                ev[1].record()
                scan_events.append((ev[0], ev[1], b, n))
            pos = select_rows(dd, c).long()
            res = torch.gather(idx, 1, pos).long()
            badm = (cnt < c) | (cnt > cap)
            # one host wait: embedding status, scan status and the number of lists to redo
            flags = torch.stack([enc_status[0], self.status[0], badm.sum().to(torch.int32)]).cpu()
            if int(flags[0]):
                raise _lib.TsmError(f"tsm_enc_embed: a tensor-core wait ran out (status {int(flags[0])})")
            if int(flags[1]):
                self._check_status()
            if int(flags[2]):  # threshold too tight or list overflowed: those queries densely
                bad = torch.nonzero(badm).flatten()
                eb = e[bad]
                res[bad] = select_rows(self._dense(self._query_image(eb), eb.shape[0], self.img, n), c).long()
            out[q0:q0 + b] = res
        if dense_only:  # chunks without the combined wait above
            if int(enc_status.item()):
                raise _lib.TsmError(f"tsm_enc_embed: a tensor-core wait ran out (status {int(enc_status.item())})")
            self._check_status()
        return out

    def query(self, Q: TrajSet, k=10, c=None, measure="dtw", **kw):
        c = c or self.c
        if c is None:  # not calibrated, or the filter could not reach the target: exhaustive
            return knn_exhaustive(Q, self.D, k, measure, **kw)
        cand = self.candidates(Q, min(c, self.D.n))
        return knn_rerank(Q, self.D, cand, k, measure, **kw)

    def calibrate(self, Q_sample: TrajSet, k=10, target=0.99, max_fraction=0.05, margin=None, measure="dtw",
                  weights=None, **kw):
        """-> (chosen count or None, {count: recall} at the chosen branch
        weight) on the sample; sets self.c and the branch weight.

        For each branch weight (``weights``, default BRANCH_WEIGHTS) the
        smallest count of the ladder whose sample recall clears the target by
        a margin of two standard errors of a recall measured on n*k answers
        (default) -- so that the recall on the full query set does not fall
        below the target by sampling noise -- and the weight with the
        smallest such count.  Recalls are judged on the candidate sets (the
        exact rerank keeps every true answer a set contains)."""
        _, exact = knn_exhaustive(Q_sample, self.D, k, measure, **kw)
        ex = exact.cpu().numpy()
        if margin is None:
            margin = 2.0 * float(np.sqrt(target * (1.0 - target) / (Q_sample.n * k)))
        best, table = None, {}
        for beta in (self.BRANCH_WEIGHTS if weights is None else weights):
            self.set_branch_weight(beta)
            rec = {}
            for c in self.LADDER:
                if (c > max_fraction * self.D.n and c > self.LADDER[0]) or (best is not None and c >= best[1]):
                    break
                got = self.candidates(Q_sample, c).cpu().numpy()
                rec[c] = float(np.mean([len(np.intersect1d(got[i], ex[i])) / k for i in range(ex.shape[0])]))
                if rec[c] >= min(target + margin, 1.0):
                    best = (beta, c)
                    break
            table[beta] = rec
        if best is None:
            self.c = None
            self.set_branch_weight(self.BRANCH_WEIGHTS[0] if weights is None else weights[0])
            return None, table[next(iter(table))]
        self.set_branch_weight(best[0])
        self.c = best[1]
        self.calibration = table
        return self.c, table[best[0]]


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
