"""Learned DTW surrogate: a trajectory encoder trained on GPU-computed DTW
distances, used as a kNN candidate filter.

Network and kernels: see the C ABI (tsm_enc_* in include/tsm.h).  Training
follows the reference's learned-measure protocol (nn/MLP_trajsimi_train.py:
random pairs from a trajectory pool, targets = heuristic distance / max
distance, MSE loss, Adam), with the labels computed by this library's own DTW
kernel (tsm_pairs) on the GPU.

    enc = Encoder.init(pool)                       # normalisation from the pool
    hist = enc.fit(pool, pa, pb, labels, epochs=…)  # labels already normalised
    emb = enc.embed(pool)                          # [n, 160] float32 on the device
"""
from __future__ import annotations

import contextlib
import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .engine import TrajSet, _ptr, _stream_ptr, pairs_in_set

EMB = 160  # 128 head outputs + the geometric skip (16 resampled points x 2)
# (fan_in, count) of the parameter blocks in layout order; PyTorch-style
# uniform(-1/sqrt(k), 1/sqrt(k)) init with k = fan_in (conv: 2*5, GRU: 128,
# head: 128); the 16 skip weights (one per resampled point, stored as their
# logarithms) start at 1/sqrt(32) (fan-in of the 32 skip values) before the
# data-dependent balance
_BLOCKS = [("conv_w", 10, 64 * 2 * 5), ("conv_b", 10, 64), ("w_ih", 128, 384 * 64), ("b_ih", 128, 384),
           ("w_hh", 128, 384 * 128), ("b_hh", 128, 384), ("w_o", 128, 128 * 128), ("b_o", 128, 128),
           ("skip_scale", 32, 16)]
NSKIP = 16  # resampled points of the geometric skip (one learned weight each)


def spearman(a, b) -> float:
    """Spearman rank correlation (average ranks for ties)."""
    def ranks(x):
        x = np.asarray(x, dtype=np.float64)
        o = np.argsort(x, kind="stable")
        r = np.empty(len(x))
        r[o] = np.arange(len(x))
        _, inv, cnt = np.unique(x, return_inverse=True, return_counts=True)
        sums = np.bincount(inv, weights=r)
        return sums[inv] / cnt[inv]
    ra, rb = ranks(a), ranks(b)
    ra -= ra.mean()
    rb -= rb.mean()
    return float((ra * rb).sum() / math.sqrt((ra * ra).sum() * (rb * rb).sum()))


@dataclass
class Encoder:
    params: torch.Tensor                  # float32 [n_params] master weights (device)
    nrm: np.ndarray                       # (mean_x, mean_y, 1/s, 1/s), s: RMS of the axes' std
    m: torch.Tensor = None
    v: torch.Tensor = None
    step: int = 0
    _ws: torch.Tensor = field(default=None, repr=False)
    _ws_key: tuple = field(default=(0, 0, 0), repr=False)
    _ews: torch.Tensor = field(default=None, repr=False)  # inference workspace (tsm_enc_embed)
    # failure-path test hook: (wait limit in SM clocks, stalled step) for tsm_enc_embed_opts; None in use
    _wait_override: tuple = field(default=None, repr=False)

    @staticmethod
    def n_params() -> int:
        return _lib.load().tsm_enc_param_count()

    @classmethod
    def init(cls, pool: TrajSet, seed=0, device=None):
        dev = device or pool.device
        g = np.random.Generator(np.random.PCG64(seed))
        chunks = [g.uniform(-1 / math.sqrt(k), 1 / math.sqrt(k), n).astype(np.float32) for _, k, n in _BLOCKS]
        chunks[-1][:] = math.log(1 / math.sqrt(32))
        p = np.concatenate(chunks)
        assert p.size == cls.n_params()
        pts = pool.pts.double()
        mean = pts.mean(0).cpu().numpy()
        # one scale for both axes (the RMS of their standard deviations): the
        # measures are isotropic, and so must the normalised coordinates be
        sd = float(np.sqrt((pts.var(0).cpu().numpy()).mean()))
        nrm = np.array([mean[0], mean[1], 1.0 / max(sd, 1e-12), 1.0 / max(sd, 1e-12)], dtype=np.float32)
        t = torch.from_numpy(p).to(dev)
        enc = cls(t, nrm, torch.zeros_like(t), torch.zeros_like(t))
        enc._balance_skip(pool, seed)
        return enc

    @staticmethod
    def skip_prior():
        """Initial profile of the skip weights over the 16 resampled points:
        1 + |2k/15 - 1|, twice the weight at the two ends as in the middle.
        DTW matches the first points and the last points of the two
        trajectories in every warping path, so their offsets count in full,
        while the inner points can be re-aligned; a uniform weighting
        under-states the ends.  (On 1,000 queries x 1M random walks, recall@10
        of the resampled points alone at 200 candidates: uniform 0.9927, this
        profile 0.9985.)"""
        k = np.arange(NSKIP, dtype=np.float64)
        return 1.0 + np.abs(2.0 * k / (NSKIP - 1) - 1.0)

    def _balance_skip(self, pool: TrajSet, seed=0, n=4096):
        """Data-dependent initial skip weights: the prior profile (skip_prior)
        times one scale chosen so that the embedding's two paths (the
        recurrent branch's 128 outputs and the 32 resampled-point values)
        contribute equal mean squared distances over random pairs of the pool,
        the way weight-normalised networks set their scales from data at
        initialisation (Salimans and Kingma, NeurIPS 2016).  Training then
        decides how much of each path the distances use."""
        g = np.random.Generator(np.random.PCG64(seed + 1))
        idx = g.choice(pool.n, size=min(n, pool.n), replace=False)
        prior = torch.as_tensor(np.log(self.skip_prior()), dtype=torch.float32, device=self.params.device)
        self.params[-NSKIP:] = prior
        e = self.embed(pool, idx).double()
        a, b = torch.from_numpy(g.permutation(len(idx))).to(e.device), torch.from_numpy(g.permutation(len(idx))).to(e.device)
        d = e[a] - e[b]
        fb = float((d[:, :EMB - 32] ** 2).sum(1).mean())
        fs = float((d[:, EMB - 32:] ** 2).sum(1).mean())
        self.params[-NSKIP:] = prior + (0.5 * math.log(fb / fs) if fs > 0 and fb > 0 else math.log(1.0 / math.sqrt(32)))

    # -- device buffers ---------------------------------------------------------
    def _workspace(self, B, T, P):
        key = (B, T, P)
        if self._ws is None or any(k > h for k, h in zip(key, self._ws_key)):
            nb = _lib.load().tsm_enc_workspace_bytes(*[max(k, h) for k, h in zip(key, self._ws_key)])
            if nb < 0:
                raise ValueError("bad encoder batch shape")
            if self._ws is not None:
                self.check_training()  # the old workspace's status word goes with it
            self._ws = torch.empty(nb // 4 + 64, dtype=torch.float32, device=self.params.device)
            self._ws[:1].zero_()  # the training status word (tsm_enc_train_status)
            self._ws_key = tuple(max(k, h) for k, h in zip(key, self._ws_key))
        return self._ws

    def check_training(self, stream=None):
        """Raises TsmError if a bounded wait of the tensor-core weight-gradient
        kernel ran out in a loss_grad call since the last check (the gradients
        of those calls are incomplete).  Synchronises the stream; fit() calls
        it once per epoch."""
        if self._ws is None:
            return
        st = ctypes.c_int32(0)
        rc = _lib.load().tsm_enc_train_status(_ptr(self._ws), ctypes.byref(st), _stream_ptr(stream))
        _lib.check(rc, "tsm_enc_train_status")

    def _nrm_ptr(self):
        return (ctypes.c_float * 4)(*[float(x) for x in self.nrm])

    # -- inference ----------------------------------------------------------------
    # trajectories per tensor-core embedding launch: 296 CTAs of 128, two waves over a B200's 148 SMs
    TC_BATCH = 296 * 128

    def embed(self, s: TrajSet, idx=None, batch=None, stream=None, tensor_cores=True,
              status_out=None) -> torch.Tensor:
        """Embeddings [n, 160] of trajectories idx (default all) of s.

        tensor_cores=True: the tcgen05 inference kernel (tsm_enc_embed; a_t
        and h_t enter the gate products as BF16), over batches of similar
        lengths.  False: the training forward (tsm_enc_forward, FP32 a_t and h_t).
        status_out: a device int32 [1] into which the kernels' status bits are
        OR-ed, for a caller that checks it later (no host synchronisation
        here); None: checked here, TsmError on a wait that ran out."""
        lib = _lib.load()
        batch = batch or (self.TC_BATCH if tensor_cores else 4096)
        idx_given = idx is not None
        idx = torch.arange(s.n, device=s.device) if idx is None else torch.as_tensor(idx, device=s.device).long()
        n = int(idx.shape[0])
        out = torch.empty((n, EMB), dtype=torch.float32, device=s.device)
        if n == 0:
            return out
        # length order on the device: a kernel CTA runs as many steps as its longest trajectory
        lens_d = s.lens[idx]
        perm = torch.argsort(lens_d, stable=True) if tensor_cores else torch.arange(n, device=s.device)
        sel_all = idx[perm]
        off_all, ln_all = s.off[sel_all].contiguous(), s.lens[sel_all].contiguous()
        starts = list(range(0, n, batch))
        ends = [min(b0 + batch, n) for b0 in starts]
        if tensor_cores and len(starts) == 1 and idx_given is False:  # the whole set: its max length is known
            tmax = np.array([s.max_len])
        elif tensor_cores:  # sorted: a batch's longest trajectory is its last
            tmax = ln_all[torch.tensor([e - 1 for e in ends], device=s.device)].cpu().numpy()
        else:
            tmax = torch.stack([ln_all[b0:e].max() for b0, e in zip(starts, ends)]).cpu().numpy()
        res = torch.empty((n, EMB), dtype=torch.float32, device=s.device)  # in processing order
        if tensor_cores:  # one workspace for the largest batch
            need = max(lib.tsm_enc_embed_workspace_bytes(e - b0, max(int(t), 1))
                       for b0, e, t in zip(starts, ends, tmax))
            if self._ews is None or self._ews.numel() * 4 < need:
                self._ews = torch.empty(need // 4 + 64, dtype=torch.float32, device=self.params.device)
        status = None
        if tensor_cores:
            status = status_out if status_out is not None else torch.zeros(1, dtype=torch.int32, device=s.device)
        for b0, e, t in zip(starts, ends, tmax):
            B, T = e - b0, max(int(t), 1)
            off, ln, r = off_all[b0:e], ln_all[b0:e], res[b0:e]
            if tensor_cores:
                if self._wait_override is None:
                    rc = lib.tsm_enc_embed(_ptr(self.params), _ptr(s.pts), _ptr(off), _ptr(ln), B, T,
                                           self._nrm_ptr(), _ptr(self._ews), _ptr(r), _stream_ptr(stream))
                else:  # failure-path test hook (wait limit, stalled step)
                    rc = lib.tsm_enc_embed_opts(_ptr(self.params), _ptr(s.pts), _ptr(off), _ptr(ln), B, T,
                                                self._nrm_ptr(), _ptr(self._ews), _ptr(r), *self._wait_override,
                                                _stream_ptr(stream))
                _lib.check(rc, "tsm_enc_embed")
                with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
                    status.bitwise_or_(self._ews[:1].view(torch.int32))  # the batch's status word, no sync
            else:
                ws = self._workspace(B, T, 1)
                rc = lib.tsm_enc_forward(_ptr(self.params), _ptr(s.pts), _ptr(off), _ptr(ln), B, T,
                                         self._nrm_ptr(), _ptr(ws), _ptr(r), _stream_ptr(stream))
                _lib.check(rc, "tsm_enc_forward")
        out[perm] = res
        if status is not None and status_out is None and int(status.item()):
            raise _lib.TsmError(f"tsm_enc_embed: a tensor-core wait ran out (status {int(status.item())}); "
                                "the affected embeddings are NaN")
        return out

    # -- training -----------------------------------------------------------------
    def loss_grad(self, s: TrajSet, tidx, ia, ib, y, w=None, stream=None):
        """Loss, gradient and predictions for pairs (ia, ib) over the batch of
        trajectories tidx of s; w: per-pair loss weights (None = 1).
        -> (loss tensor [1], grad [n_params], pred [P])."""
        lib = _lib.load()
        tidx = torch.as_tensor(tidx, device=s.device).long()
        B = int(tidx.shape[0])
        lens_h = s.lens_host if s.lens_host is not None else s.lens.cpu().numpy()
        T = max(int(lens_h[tidx.cpu().numpy()].max()), 1)
        off, ln = s.off[tidx].contiguous(), s.lens[tidx].contiguous()
        ia = torch.as_tensor(ia, device=s.device).int().contiguous()
        ib = torch.as_tensor(ib, device=s.device).int().contiguous()
        y = torch.as_tensor(y, device=s.device).float().contiguous()
        P = int(ia.shape[0])
        grad = torch.empty_like(self.params)
        loss = torch.empty(1, dtype=torch.float32, device=s.device)
        pred = torch.empty(P, dtype=torch.float32, device=s.device)
        ws = self._workspace(B, T, P)
        w = None if w is None else torch.as_tensor(w, device=s.device).float().contiguous()
        rc = lib.tsm_enc_loss_grad_w(_ptr(self.params), _ptr(s.pts), _ptr(off), _ptr(ln), B, T, self._nrm_ptr(),
                                     _ptr(ia), _ptr(ib), _ptr(y), _ptr(w), P, _ptr(ws), _ptr(grad), _ptr(loss),
                                     _ptr(pred), _stream_ptr(stream))
        _lib.check(rc, "tsm_enc_loss_grad")
        return loss, grad, pred

    def adam(self, grad, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, stream=None):
        self.step += 1
        rc = _lib.load().tsm_enc_adam(_ptr(self.params), _ptr(grad), _ptr(self.m), _ptr(self.v), self.step,
                                      float(lr), float(betas[0]), float(betas[1]), float(eps), _stream_ptr(stream))
        _lib.check(rc, "tsm_enc_adam")

    def fit(self, s: TrajSet, pa, pb, y, *, epochs=5, batch_pairs=1024, lr=1e-3, seed=0, log=None,
            relative=False, floor=1e-3, train_skip=True, group=None):
        """Trains on pairs (pa[i], pb[i]) of s with targets y (normalised
        distances).  relative=True weights each pair by 1 / max(y, floor)^2
        (relative squared error: near pairs count as much as far ones).
        Every step encodes the 2*batch_pairs endpoints.  The loss is summed
        on the device and read once per epoch (the host does not wait for
        each step).  -> mean loss per epoch.

        Data-parallel with `group`, a torch.distributed process group
        (torch.distributed.group.WORLD for all ranks), called on every rank
        of it: every rank holds the same pool,
        pairs, targets and initial parameters; a step takes one global batch
        of batch_pairs * world pairs from the permutation that every rank
        draws from `seed`, rank r computes the gradient of pairs r, r + world,
        ... of it, and one all-reduce forms the pair-weighted mean gradient,
        so every rank applies the same Adam step and the replicas stay equal.
        One process trains exactly as before."""
        import torch.distributed as dist
        world = dist.get_world_size(group) if group is not None else 1
        rank = dist.get_rank(group) if world > 1 else 0
        pa, pb, y = np.asarray(pa), np.asarray(pb), np.asarray(y, dtype=np.float32)
        wts = (1.0 / np.maximum(y, floor) ** 2).astype(np.float32) if relative else None
        rng = np.random.Generator(np.random.PCG64(seed))
        hist = []
        n = len(pa)
        for ep in range(epochs):
            perm = rng.permutation(n)
            tot = torch.zeros(1, dtype=torch.float64, device=s.device)
            for b0 in range(0, n, batch_pairs * world):
                sel_all = perm[b0:b0 + batch_pairs * world]
                sel = sel_all[rank::world]
                P = len(sel)
                if P:
                    tidx = np.concatenate([pa[sel], pb[sel]])
                    loss, grad, _ = self.loss_grad(s, tidx, np.arange(P), P + np.arange(P), y[sel],
                                                   None if wts is None else wts[sel])
                else:  # a final global batch smaller than the world: this rank adds nothing
                    loss, grad = torch.zeros(1, device=s.device), torch.zeros_like(self.params)
                if world > 1:  # per-rank means -> the mean over the global batch
                    grad.mul_(P)
                    dist.all_reduce(grad, group=group)
                    grad.div_(len(sel_all))
                if not train_skip:
                    grad[-NSKIP:] = 0.0  # the skip weights keep their initial values
                self.adam(grad, lr=lr * 0.5 * (1 + math.cos(math.pi * (ep + b0 / n) / epochs)))
                tot += loss.double() * P
            if world > 1:
                dist.all_reduce(tot, group=group)
            hist.append(float(tot.item()) / n)
            self.check_training()
            if log:
                log(f"epoch {ep}: mse {hist[-1]:.3e}")
        return hist

    def predict_pairs(self, s: TrajSet, pa, pb, batch=None) -> np.ndarray:
        """||e_a - e_b|| for pairs of s (normalised-distance units)."""
        pa = np.asarray(pa)
        pb = np.asarray(pb)
        uniq, inv = np.unique(np.concatenate([pa, pb]), return_inverse=True)
        e = self.embed(s, uniq, batch=batch)
        ea = e[torch.from_numpy(inv[:len(pa)]).to(e.device)]
        eb = e[torch.from_numpy(inv[len(pa):]).to(e.device)]
        return torch.linalg.vector_norm(ea - eb, dim=1).cpu().numpy()


def neighbour_pairs(s: TrajSet, n_anchors, k=20, seed=0, chunk=4096):
    """Training pairs from the neighbourhoods that a kNN filter must order:
    n_anchors trajectories of s drawn at random, each paired with its k
    nearest trajectories of s by exact GPU DTW (itself excluded).  The
    reference's learned baselines sample training pairs by distance for the
    same reason (nn/NEUTRAJ_trajsimi_train.py:59,282-319).
    -> (anchors int64 [n_anchors * k], neighbours int64 [n_anchors * k])."""
    from .knn import _subset, knn_exhaustive
    rng = np.random.Generator(np.random.PCG64(seed))
    anc = np.sort(rng.choice(s.n, size=min(n_anchors, s.n), replace=False))
    pa, pb = [], []
    for a0 in range(0, len(anc), chunk):
        a = anc[a0:a0 + chunk]
        _, nb = knn_exhaustive(_subset(s, torch.as_tensor(a, device=s.device)), s, k + 1)
        nb = nb.cpu().numpy()
        for i, ai in enumerate(a):
            row = nb[i][nb[i] != ai][:k]
            pa.append(np.full(row.shape[0], ai, dtype=np.int64))
            pb.append(row.astype(np.int64))
    return np.concatenate(pa), np.concatenate(pb)


def dtw_labels(s: TrajSet, pa, pb, batch=1 << 20):
    """GPU DTW of pairs (pa, pb) of s (float32, the library's paired kernel)."""
    out = []
    for b0 in range(0, len(pa), batch):
        d, _ = pairs_in_set("dtw", s, pa[b0:b0 + batch], pb[b0:b0 + batch])
        out.append(d.cpu().numpy())
    return np.concatenate(out) if out else np.zeros(0, np.float32)
