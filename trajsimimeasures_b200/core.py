"""Drop-in replacements for the reference's batched GPU measures (core/*.py).

Same call surface as the reference:

    dtw(t1, len1, t2, len2, threads_per_traj=64)            core/dtw.py:56-77
    edr(t1, len1, t2, len2, eps, threads_per_traj=64)       core/edr.py:55-76
    lcss(t1, len1, t2, len2, eps, threads_per_traj=64)      core/lcss.py:56-77
    erp(t1, len1, t2, len2, gpoint=None, threads_per_traj=64)  core/erp.py:94-120
    dfrechet(t1, len1, t2, len2, threads_per_traj=64)       core/discret_frechet.py:53-74
    hausdorff(t1, len1, t2, len2, threads_per_traj=64)      core/hausdorff.py:97-123

t1, t2: padded [batch, seq, 2] arrays (float64 in the reference; any float
dtype is accepted and rounded to float32, the arithmetic type of the B200
kernels) or lists of [n_i, 2] trajectories; len1, len2: lengths.  The result
is a float64 NumPy array [batch] computed synchronously, like the reference.
CUDA torch tensors in give a CUDA float64 tensor out without host copies.

Differences from the reference, all deliberate:
  * threads_per_traj is accepted and validated but does not set the launch
    shape (the reference runs one 64-thread block per pair; the B200 kernels
    pick their own tiling).
  * erp accepts the gap point as a list, tuple or ndarray (the reference's
    `gpoint == None` test raises for an ndarray, core/erp.py:103).
  * hausdorff takes the max over valid points only (the reference's host
    reduction also reads uninitialised padded slots, core/hausdorff.py:114,121).
  * EDR/LCSS normalise the exact integer counts in float64 exactly as the
    reference does (count / max(n1, n2), 1 - count / min(n1, n2)).

Extra entry points for the Q x D and all-pairs shapes (the reference expands
them into pair batches on the host, test_trajsimi_time_DQ.py:147-173 and
test_clustering_time.py:219-269): ``matrix(measure, Q, lenQ, D, lenD, ...)``
and ``<measure>_matrix(...)``.
"""
from __future__ import annotations

import threading

import numpy as np
import torch

from . import _lib, engine
from .engine import (MATRIX_QUERY_MAX, TrajSet, allpairs_sym_raw, first_points_lists, matrix_raw, measure_id, needs_origin,
                     origin_of_points, pack_lists, pair_order, pairs_raw, shift_gpoint, sub_origin_f32)

__all__ = ["dtw", "edr", "lcss", "erp", "dfrechet", "hausdorff", "matrix", "dtw_matrix", "edr_matrix",
           "lcss_matrix", "erp_matrix", "dfrechet_matrix", "hausdorff_matrix", "pairs", "allpairs", "matrix_many",
           "matrix_sharded", "pair_origins", "set_origin"]


def _check_tpt(threads_per_traj):
    if not isinstance(threads_per_traj, (int, np.integer)) or threads_per_traj <= 0:
        raise ValueError(f"threads_per_traj must be a positive int, got {threads_per_traj!r}")


def _lens_np(lens, n):
    if isinstance(lens, torch.Tensor):
        lens = lens.detach().cpu().numpy()
    a = np.asarray(lens, dtype=np.int64).reshape(-1)
    if a.shape[0] != n:
        raise ValueError(f"{a.shape[0]} lengths for {n} trajectories")
    return a


def _as_points(t):
    """padded array/tensor -> (its [N, L, 2] coordinates in their own dtype, N, L); list -> None."""
    if isinstance(t, torch.Tensor):
        if t.dim() != 3 or t.shape[-1] < 2:
            raise ValueError("expected a padded [batch, seq, 2] tensor")
        return t[..., :2], t.shape[0], t.shape[1]
    if isinstance(t, np.ndarray):
        if t.ndim != 3 or t.shape[-1] < 2:
            raise ValueError("expected a padded [batch, seq, 2] array")
        return t[..., :2], t.shape[0], t.shape[1]
    return None


def _to_f32(a, origin):
    """[N, L, 2] host array or tensor -> float32, translated by origin (None,
    [2] or per-trajectory [N, 2]) in FP64 first."""
    if isinstance(a, torch.Tensor):
        if origin is None:
            return a.to(torch.float32).contiguous()
        o = torch.as_tensor(np.asarray(origin, dtype=np.float64).reshape(-1, 1, 2), device=a.device)
        return (a.to(torch.float64) - o).to(torch.float32).contiguous()
    if origin is None:
        return np.ascontiguousarray(a, dtype=np.float32)
    return sub_origin_f32(a, np.asarray(origin, dtype=np.float64).reshape(-1, 1, 2), np.empty(a.shape, np.float32))


def _first_points(a, lens):
    """[N, 2] float64 first point of each padded trajectory (rows of empty ones are unused)."""
    if isinstance(a, torch.Tensor):
        return a[:, 0, :2].detach().to(torch.float64).cpu().numpy() if a.shape[1] else np.zeros((a.shape[0], 2))
    return np.asarray(a[:, 0, :2], dtype=np.float64) if a.shape[1] else np.zeros((a.shape[0], 2))


def _dtype_of(t):
    if isinstance(t, (torch.Tensor, np.ndarray)):
        return t.dtype
    for x in t:
        if len(x):
            return np.asarray(x).dtype
    return np.dtype(np.float32)


def pair_origins(measure, t1, len1, t2, len2):
    """The FP64 origin(s) a paired batch is translated by before rounding to
    float32: None for float32 input; else one origin per pair, the pair's
    first point rounded to FP32 (every measure but ERP), or one for the whole
    call (ERP, whose gap point is one per call), the FP32-rounded midpoint of
    the bounding box of the trajectories' first points.
    -> None, float64 [n, 2] or float64 [2]."""
    if not (needs_origin(_dtype_of(t1)) or needs_origin(_dtype_of(t2))):
        return None
    p1, p2 = _as_points(t1), _as_points(t2)
    n = len(t1)
    if p1 is None or p2 is None:
        la = _lens_np(len1, n) if len1 is not None else np.array([len(x) for x in t1])
        lb = _lens_np(len2, n) if len2 is not None else np.array([len(x) for x in t2])
        f1, f2 = np.zeros((n, 2)), np.zeros((n, 2))
        for k in range(n):
            if la[k]:
                f1[k] = np.asarray(t1[k], dtype=np.float64).reshape(-1, np.shape(t1[k])[-1])[0, :2]
            if lb[k]:
                f2[k] = np.asarray(t2[k], dtype=np.float64).reshape(-1, np.shape(t2[k])[-1])[0, :2]
    else:
        la, lb = _lens_np(len1, n), _lens_np(len2, n)
        f1, f2 = _first_points(p1[0], la), _first_points(p2[0], lb)
    if measure_id(measure) == _lib.ERP:
        return np.asarray(origin_of_points(np.concatenate([f1[la > 0], f2[lb > 0]])), dtype=np.float64)
    o = np.where((la > 0)[:, None], f1, np.where((lb > 0)[:, None], f2, 0.0))
    o = o.astype(np.float32).astype(np.float64)
    o[~np.isfinite(o).all(axis=1)] = 0.0
    return o


def set_origin(*sets):
    """The FP64 origin that the sets of one Q x D or all-pairs call share:
    a TrajSet's own origin if one is given; None if every set is float32;
    else the FP32-rounded midpoint of the bounding box of all first points."""
    firsts = []
    for t, lens in sets:
        if isinstance(t, TrajSet):
            return None if tuple(t.origin) == (0.0, 0.0) else t.origin
    if not any(needs_origin(_dtype_of(t)) for t, _ in sets):
        return None
    for t, lens in sets:
        p = _as_points(t)
        if p is None:
            tl = list(t) if lens is None else [np.asarray(x)[:l] for x, l in zip(t, _lens_np(lens, len(t)))]
            firsts.append(first_points_lists(tl))
        else:
            la = _lens_np(lens, p[1])
            firsts.append(_first_points(p[0], la)[la > 0])
    return origin_of_points(np.concatenate(firsts) if firsts else np.zeros((0, 2)))


_tls = threading.local()


PINNED_KEEP_BYTES = 64 << 20  # largest staging buffer a thread keeps between calls


def _pinned(nbytes):
    """A pinned host staging buffer (uint8, at least nbytes).  Up to
    PINNED_KEEP_BYTES the calling thread's buffer is reused (grown by
    doubling); a larger request gets a buffer of its own, released with the
    call.  A call that uploads from it synchronises before returning, so the
    next call may overwrite it."""
    if nbytes > PINNED_KEEP_BYTES:
        return torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    b = getattr(_tls, "pinned", None)
    if b is None or b.numel() < nbytes:
        size = min(max(nbytes, 2 * (b.numel() if b is not None else 0), 1 << 20), PINNED_KEEP_BYTES)
        b = torch.empty(size, dtype=torch.uint8, pin_memory=True)
        _tls.pinned = b
    return b


def release_staging():
    """Frees the calling thread's pinned staging buffer."""
    _tls.pinned = None


def _stage_padded(a1, a2, la, lb, order, dev, origin=None):
    """Padded host pair arrays [n, L, >=2] to the device through one pinned
    buffer and one copy: the points are rounded to float32 straight into the
    buffer (the rounding of astype; with an origin, [2] or per pair [n, 2],
    after an FP64 translation by it), followed by the int32 lengths and
    processing order; the offsets are made on the device.
    -> (pts [n*L1 + n*L2, 2] float32, len_a, len_b, order int32, off_a, off_b int64)."""
    n, L1, L2 = a1.shape[0], a1.shape[1], a2.shape[1]
    nf1, nf2 = n * L1 * 2, n * L2 * 2
    pts_bytes = 4 * (nf1 + nf2)  # a multiple of 8: nf1 and nf2 are even
    nbytes = pts_bytes + 12 * n
    pin = _pinned(nbytes)
    host = pin.numpy()
    f = host[:pts_bytes].view(np.float32)
    if origin is None:
        np.copyto(f[:nf1].reshape(n, L1, 2), a1[..., :2], casting="unsafe")
        np.copyto(f[nf1:].reshape(n, L2, 2), a2[..., :2], casting="unsafe")
    else:
        o = np.asarray(origin, dtype=np.float64).reshape(-1, 1, 2)
        sub_origin_f32(a1[..., :2], o, f[:nf1].reshape(n, L1, 2))
        sub_origin_f32(a2[..., :2], o, f[nf1:].reshape(n, L2, 2))
    ints = host[pts_bytes:nbytes].view(np.int32)
    ints[:n] = la
    ints[n:2 * n] = lb
    ints[2 * n:] = order
    d = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    d.copy_(pin[:nbytes], non_blocking=True)
    di = d[pts_bytes:].view(torch.int32)
    ar = torch.arange(n, dtype=torch.int64, device=dev)
    return d[:pts_bytes].view(torch.float32).view(-1, 2), di[:n], di[n:2 * n], di[2 * n:], ar * L1, n * L1 + ar * L2


def _normalise_counts(m, counts, la, lb):
    """Reference normalisation in float64 (edr.py:51, lcss.py:52)."""
    c = counts.astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        if m == _lib.EDR:
            return c / np.maximum(la, lb)
        return 1.0 - c / np.minimum(la, lb)


def pairs(measure, t1, len1, t2, len2, *, eps=0.0, gpoint=(0.0, 0.0), exact=False, rows=0, counts=False):
    """Paired batch: result[k] = measure(t1[k][:len1[k]], t2[k][:len2[k]]).

    Returns float64 (NumPy for host inputs, CUDA tensor for CUDA inputs); with
    counts=True also the int32 EDR/LCSS counts.  Inputs that are not float32
    are translated by an FP64 origin before rounding (``pair_origins``)."""
    m = measure_id(measure)
    if (isinstance(t1, np.ndarray) and isinstance(t2, np.ndarray) and t1.ndim == 3 and t2.ndim == 3
            and t1.shape[-1] >= 2 and t2.shape[-1] >= 2 and t1.shape[0] == t2.shape[0] and t1.shape[0] > 0
            and t1.shape[1] > 0 and t2.shape[1] > 0):
        # padded host arrays (the reference's input): one staged upload
        n, L1, L2 = t1.shape[0], t1.shape[1], t2.shape[1]
        la, lb = _lens_np(len1, n), _lens_np(len2, n)
        if la.min() < 0 or lb.min() < 0 or la.max() > L1 or lb.max() > L2:
            raise ValueError("a length is negative or exceeds the padded width")
        dev = torch.device("cuda")
        max_len = int(max(la.max(), lb.max()))
        origin = pair_origins(m, t1, la, t2, lb)
        if origin is not None and origin.ndim == 1:
            gpoint = shift_gpoint(gpoint, origin)
        pts_t, la_t, lb_t, order_t, off_a_t, off_b_t = _stage_padded(t1, t2, la, lb, pair_order(la, lb), dev,
                                                                     origin)
        out = torch.empty(n, dtype=torch.float32, device=dev)
        cnt = torch.empty(n, dtype=torch.int32, device=dev) if m in (_lib.EDR, _lib.LCSS) else None
        pairs_raw(m, pts_t, off_a_t, la_t, off_b_t, lb_t, max_len, out=out, counts=cnt, order=order_t, eps=eps,
                  gpoint=gpoint, exact=exact, rows=rows)
        return _host_result(m, out, cnt, la, lb, counts)
    p1, p2 = _as_points(t1), _as_points(t2)
    if p1 is None or p2 is None:  # lists of trajectories
        n = len(t1)
        if len(t2) != n:
            raise ValueError("t1 and t2 hold different numbers of trajectories")
        la = _lens_np(len1, n) if len1 is not None else np.array([len(x) for x in t1])
        lb = _lens_np(len2, n) if len2 is not None else np.array([len(x) for x in t2])
        origin = pair_origins(m, t1, la, t2, lb)
        if origin is not None and origin.ndim == 2:
            origin = np.concatenate([origin, origin])  # per trajectory: t1's, then t2's
        pts, off, lens = pack_lists([np.asarray(x)[:l] for x, l in zip(list(t1) + list(t2), np.concatenate([la, lb]))],
                                    origin)
        off_a, off_b = off[:n], off[n:]
        on_device = False
        dev = torch.device("cuda")
    else:
        (a1, n, L1), (a2, n2, L2) = p1, p2
        if n2 != n:
            raise ValueError("t1 and t2 hold different numbers of trajectories")
        la, lb = _lens_np(len1, n), _lens_np(len2, n)
        if n and (la.min() < 0 or lb.min() < 0 or la.max() > L1 or lb.max() > L2):
            raise ValueError("a length is negative or exceeds the padded width")
        origin = pair_origins(m, t1, la, t2, lb) if n else None
        on_device = isinstance(a1, torch.Tensor) and a1.is_cuda
        dev = a1.device if on_device else torch.device("cuda")
        off_a = np.arange(n, dtype=np.int64) * L1
        off_b = n * L1 + np.arange(n, dtype=np.int64) * L2
        a1, a2 = _to_f32(a1, origin), _to_f32(a2.to(dev) if on_device else a2, origin)
        if on_device:
            pts = torch.cat([a1.reshape(-1, 2), a2.reshape(-1, 2)])
        else:
            a1 = a1.numpy() if isinstance(a1, torch.Tensor) else a1
            a2 = a2.numpy() if isinstance(a2, torch.Tensor) else a2
            pts = np.concatenate([a1.reshape(-1, 2), a2.reshape(-1, 2)])
    if origin is not None and origin.ndim == 1:
        gpoint = shift_gpoint(gpoint, origin)
    max_len = int(max(la.max(initial=0), lb.max(initial=0)))
    order = pair_order(la, lb)

    def up(x, dt):
        if isinstance(x, torch.Tensor):
            return x.to(dev)
        return torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).to(dev)

    pts_t = up(pts, np.float32)
    la_t, lb_t = up(la, np.int32), up(lb, np.int32)
    out = torch.empty(n, dtype=torch.float32, device=dev)
    cnt = torch.empty(n, dtype=torch.int32, device=dev) if m in (_lib.EDR, _lib.LCSS) else None
    pairs_raw(m, pts_t, up(off_a, np.int64), la_t, up(off_b, np.int64), lb_t, max_len, out=out, counts=cnt,
              order=up(order, np.int32), eps=eps, gpoint=gpoint, exact=exact, rows=rows)
    if on_device:
        if cnt is not None:
            c = cnt.double()
            lat, lbt = la_t.double(), lb_t.double()
            res = c / torch.maximum(lat, lbt) if m == _lib.EDR else 1.0 - c / torch.minimum(lat, lbt)
        else:
            res = out.double()
        return (res, cnt) if counts else res
    return _host_result(m, out, cnt, la, lb, counts)


def _host_result(m, out, cnt, la, lb, counts):
    """float64 host result of a pair batch (EDR/LCSS: the normalised counts)."""
    if cnt is not None:
        c_h = cnt.cpu().numpy()
        res = _normalise_counts(m, c_h, la, lb)
        return (res, c_h) if counts else res
    res = out.cpu().numpy().astype(np.float64)
    return (res, None) if counts else res


def dtw(t1, len1, t2, len2, threads_per_traj=64):
    """core/dtw.py:56-77 (asserts t1.shape == t2.shape as the reference does, :60)."""
    _check_tpt(threads_per_traj)
    assert np.shape(t1) == np.shape(t2) if not isinstance(t1, list) else len(t1) == len(t2)
    return pairs(_lib.DTW, t1, len1, t2, len2)


def edr(t1, len1, t2, len2, eps, threads_per_traj=64):
    """core/edr.py:55-76: count / max(n1, n2), match iff dx^2 + dy^2 < eps^2."""
    _check_tpt(threads_per_traj)
    assert len(t1) == len(t2)
    return pairs(_lib.EDR, t1, len1, t2, len2, eps=eps)


def lcss(t1, len1, t2, len2, eps, threads_per_traj=64):
    """core/lcss.py:56-77: 1 - count / min(n1, n2)."""
    _check_tpt(threads_per_traj)
    assert len(t1) == len(t2)
    return pairs(_lib.LCSS, t1, len1, t2, len2, eps=eps)


def _gpoint(gpoint):
    if gpoint is None:
        return (0.0, 0.0)  # core/erp.py:103
    g = np.asarray(gpoint, dtype=np.float64).reshape(-1)
    if g.shape[0] < 2:
        raise ValueError("gpoint must have two coordinates")
    return (float(g[0]), float(g[1]))


def erp(t1, len1, t2, len2, gpoint=None, threads_per_traj=64):
    """core/erp.py:94-120 (gap point default (0, 0))."""
    _check_tpt(threads_per_traj)
    assert len(t1) == len(t2)
    return pairs(_lib.ERP, t1, len1, t2, len2, gpoint=_gpoint(gpoint))


def dfrechet(t1, len1, t2, len2, threads_per_traj=64):
    """core/discret_frechet.py:53-74."""
    _check_tpt(threads_per_traj)
    assert len(t1) == len(t2)
    return pairs(_lib.DFRECHET, t1, len1, t2, len2)


def hausdorff(t1, len1, t2, len2, threads_per_traj=64):
    """core/hausdorff.py:97-123 (max over valid points only)."""
    _check_tpt(threads_per_traj)
    assert len(t1) == len(t2)
    return pairs(_lib.HAUSDORFF, t1, len1, t2, len2)


# ---------------------------------------------------------------------------
# Q x D / all-pairs
# ---------------------------------------------------------------------------

def _set_of(t, lens, device, origin=None):
    """A device TrajSet of host/device input (translated by origin, if any)."""
    if isinstance(t, TrajSet):
        return t
    p = _as_points(t)
    o = (0.0, 0.0) if origin is None else origin
    if p is None:
        trajs = list(t) if lens is None else [np.asarray(x)[:l] for x, l in zip(t, _lens_np(lens, len(t)))]
        return TrajSet.from_lists(trajs, device=device, origin=o)
    a, n, L = p
    la = _lens_np(lens, n)
    if isinstance(a, torch.Tensor) and a.is_cuda:
        off = torch.arange(n, dtype=torch.int64, device=a.device) * L
        lens_t = torch.as_tensor(la, dtype=torch.int32).to(a.device)
        a = _to_f32(a, origin)
        return TrajSet(a.reshape(-1, 2), off, lens_t, int(la.max(initial=0)), la.astype(np.int32), origin=o)
    a = a.numpy() if isinstance(a, torch.Tensor) else a
    return TrajSet.from_padded(a, la, device=device, origin=o)


def _matrix_into(m, qs, ds, out, cnt, *, eps, gpoint, exact, rows, stream=None):
    """out (and cnt) [qs.n, ds.n] = measure over Q x D.  Queries up to the
    matrix forms' limit (MATRIX_QUERY_MAX points; Hausdorff: any) in one
    tsm_matrix launch; the rows of longer queries with tsm_pairs over
    (query, every database trajectory) pairs, whose kernels take any length
    up to tsm_max_supported_len.  Both give the same values bit for bit."""
    lq = qs.lens_host if qs.lens_host is not None else qs.lens.cpu().numpy()
    if m == _lib.HAUSDORFF or qs.max_len <= MATRIX_QUERY_MAX:
        matrix_raw(m, qs, ds, out=out, counts=cnt, eps=eps, gpoint=gpoint, exact=exact, rows=rows, stream=stream)
        return
    dev = qs.device
    long_i = np.nonzero(np.asarray(lq) > MATRIX_QUERY_MAX)[0]
    short_i = np.nonzero(np.asarray(lq) <= MATRIX_QUERY_MAX)[0]
    if short_i.size:
        si = torch.as_tensor(short_i, device=dev)
        sub = TrajSet(qs.pts, qs.off[si], qs.lens[si], int(np.asarray(lq)[short_i].max()),
                      np.asarray(lq)[short_i].astype(np.int32), origin=qs.origin)
        o = torch.empty((sub.n, ds.n), dtype=torch.float32, device=dev)
        c = torch.empty((sub.n, ds.n), dtype=torch.int32, device=dev) if cnt is not None else None
        matrix_raw(m, sub, ds, out=o, counts=c, eps=eps, gpoint=gpoint, exact=exact, rows=rows, stream=stream)
        out[si] = o
        if cnt is not None:
            cnt[si] = c
    origin = engine.same_origin(qs, ds)
    shift = ds.pts.shape[0]
    pool = torch.cat([ds.pts, qs.pts])  # one point pool for the paired kernels
    nd = ds.n
    for i in long_i:
        ia = torch.full((nd,), int(i), dtype=torch.int64, device=dev)
        off_a, len_a = qs.off[ia] + shift, qs.lens[ia]
        o = torch.empty(nd, dtype=torch.float32, device=dev)
        c = torch.empty(nd, dtype=torch.int32, device=dev) if cnt is not None else None
        pairs_raw(m, pool, off_a, len_a, ds.off, ds.lens, max(qs.max_len, ds.max_len), out=o, counts=c,
                  order=engine.pair_order_dev(len_a, ds.lens), eps=eps, gpoint=shift_gpoint(gpoint, origin),
                  exact=exact, rows=rows, stream=stream)
        out[int(i)] = o
        if cnt is not None:
            cnt[int(i)] = c


def matrix(measure, Q, lenQ, D, lenD, *, eps=0.0, gpoint=None, exact=False, rows=0, counts=False):
    """result[i, j] = measure(Q_i, D_j) for all pairs, one launch.

    Q, D: padded arrays/tensors with lengths, lists of trajectories (lengths
    optional), or TrajSet objects already on the device.  Returns float64
    [nq, nd] (NumPy for host inputs, CUDA tensor for device inputs)."""
    m = measure_id(measure)
    dev = torch.device("cuda")
    on_device = isinstance(Q, TrajSet) or (isinstance(Q, torch.Tensor) and Q.is_cuda)
    origin = set_origin((Q, lenQ), (D, lenD))
    qs = _set_of(Q, lenQ, dev, origin)
    ds = _set_of(D, lenD, qs.device, origin)
    out = torch.empty((qs.n, ds.n), dtype=torch.float32, device=qs.device)
    cnt = torch.empty((qs.n, ds.n), dtype=torch.int32, device=qs.device) if m in (_lib.EDR, _lib.LCSS) else None
    _matrix_into(m, qs, ds, out, cnt, eps=eps, gpoint=_gpoint(gpoint), exact=exact, rows=rows)
    return _finish_matrix(m, out, cnt, qs, ds, on_device, counts)


def _finish_matrix(m, out, cnt, qs, ds, on_device, counts):
    """float64 results of a float32 matrix (EDR/LCSS: from the counts)."""
    lq = qs.lens_host if qs.lens_host is not None else qs.lens.cpu().numpy()
    ld = ds.lens_host if ds.lens_host is not None else ds.lens.cpu().numpy()
    if on_device:
        if cnt is not None:
            c = cnt.double()
            a = qs.lens.double()[:, None]
            b = ds.lens.double()[None, :]
            res = c / torch.maximum(a, b) if m == _lib.EDR else 1.0 - c / torch.minimum(a, b)
        else:
            res = out.double()
        return (res, cnt) if counts else res
    if cnt is not None:
        c_h = cnt.cpu().numpy()
        res = _normalise_counts(m, c_h, lq.astype(np.int64)[:, None], ld.astype(np.int64)[None, :])
        return (res, c_h) if counts else res
    res = out.cpu().numpy().astype(np.float64)
    return (res, None) if counts else res


def allpairs(measure, S, lenS=None, *, eps=0.0, gpoint=None, exact=False, rows=0, counts=False):
    """result[i, j] = measure(S_i, S_j) for all pairs of one set, computing
    each unordered pair once and mirroring it (the clustering driver's upper
    triangle, test_clustering_time.py:219-269, as one launch).  Same inputs
    and return types as ``matrix``; equal to ``matrix(measure, S, lenS, S,
    lenS)`` bit for bit."""
    m = measure_id(measure)
    dev = torch.device("cuda")
    on_device = isinstance(S, TrajSet) or (isinstance(S, torch.Tensor) and S.is_cuda)
    ss = _set_of(S, lenS, dev, set_origin((S, lenS)))
    out = torch.empty((ss.n, ss.n), dtype=torch.float32, device=ss.device)
    cnt = torch.empty((ss.n, ss.n), dtype=torch.int32, device=ss.device) if m in (_lib.EDR, _lib.LCSS) else None
    if m != _lib.HAUSDORFF and ss.max_len > MATRIX_QUERY_MAX:  # the full matrix, long rows by tsm_pairs
        _matrix_into(m, ss, ss, out, cnt, eps=eps, gpoint=_gpoint(gpoint), exact=exact, rows=rows)
    else:
        allpairs_sym_raw(m, ss, out=out, counts=cnt, eps=eps, gpoint=_gpoint(gpoint), exact=exact, rows=rows)
    return _finish_matrix(m, out, cnt, ss, ss, on_device, counts)


def matrix_many(measures, Q, lenQ, D, lenD, *, eps=0.0, gpoint=None, exact=False, rows=0, stream=None):
    """Several measures over the same Q x D, one upload of each set:
    {name: float64 [nq, nd] NumPy array}.  Host inputs (padded arrays with
    lengths, or lists) or TrajSets.

    The float64 results are formed on the GPU as each measure finishes (EDR/LCSS
    counts normalised in float64 exactly as on the host: count / max(n1, n2),
    1 - count / min(n1, n2)) and copied into pinned host memory on a side
    stream, overlapping the next measure's kernel."""
    dev = torch.device("cuda")
    origin = set_origin((Q, lenQ), (D, lenD))
    qs = _set_of(Q, lenQ, dev, origin)
    ds = qs if (D is Q and lenD is lenQ) else _set_of(D, lenD, dev, origin)
    g = _gpoint(gpoint)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    copy = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(s):
        lq = qs.lens.double()[:, None]
        ld = ds.lens.double()[None, :]
    host = {}
    for meas in measures:
        m = measure_id(meas)
        out = torch.empty((qs.n, ds.n), dtype=torch.float32, device=dev)
        cnt = torch.empty((qs.n, ds.n), dtype=torch.int32, device=dev) if m in (_lib.EDR, _lib.LCSS) else None
        _matrix_into(m, qs, ds, out, cnt, eps=eps, gpoint=g, exact=exact, rows=rows, stream=s)
        with torch.cuda.stream(s):
            if m == _lib.EDR:
                res = cnt.double() / torch.maximum(lq, ld)
            elif m == _lib.LCSS:
                res = 1.0 - cnt.double() / torch.minimum(lq, ld)
            else:
                res = out.double()
        done = torch.cuda.Event()
        done.record(s)
        h = torch.empty(res.shape, dtype=torch.float64, pin_memory=True)
        copy.wait_event(done)
        with torch.cuda.stream(copy):
            h.copy_(res, non_blocking=True)
        res.record_stream(copy)
        host[_lib.MEASURE_NAMES[m]] = h
    copy.synchronize()
    return {k: v.numpy() for k, v in host.items()}


def _rows_of(t, lens, s, e):
    """Rows s..e of a padded array/tensor or list of trajectories, with their lengths."""
    if isinstance(t, TrajSet):
        raise ValueError("matrix_sharded takes host inputs (padded arrays or lists), not a TrajSet")
    p = _as_points(t)
    if p is None:
        tl = list(t)
        ln = np.array([len(x) for x in tl]) if lens is None else _lens_np(lens, len(tl))
        return tl[s:e], ln[s:e], ln
    ln = _lens_np(lens, p[1])
    return t[s:e], ln[s:e], ln


def matrix_sharded(measures, Q, lenQ, D, lenD, *, eps=0.0, gpoint=None, exact=False, rows=0, group=None,
                   block_fn=None):
    """Q x D for several measures over the ranks of a torch.distributed group
    (one process per GPU): {name: float64 [nq, nd] NumPy array} on every rank.

    The rows of the matrix are split into contiguous blocks of near-equal work
    (shard.row_shards, by query length); each rank computes its block of
    every measure on its own GPU with no exchange of intermediate data, and
    one all-gather per measure (float32 values, int32 EDR/LCSS counts)
    assembles the matrix.  EDR/LCSS are normalised in float64 as the
    reference does.  Q and D must be the same host inputs on every rank; they
    share one FP64 origin (set_origin), so every rank rounds identically.
    Without an initialised group, or with one rank, this is matrix_many.

    block_fn(measure_ids, Q_rows, len_rows, D, lenD, origin) -> {m: (values
    float32 [r, nd], counts int32 [r, nd] or None)} replaces the GPU block
    computation (the tensors' device must suit the group's backend); None =
    the CUDA kernels on the current device."""
    import torch.distributed as dist
    from .shard import row_shards
    g = _gpoint(gpoint)
    ids = [measure_id(m) for m in measures]
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    if world == 1 and block_fn is None:
        return matrix_many(measures, Q, lenQ, D, lenD, eps=eps, gpoint=gpoint, exact=exact, rows=rows)
    rank = dist.get_rank(group) if world > 1 else 0
    lq_all = _rows_of(Q, lenQ, 0, 0)[2]
    shards = row_shards(lq_all, world)
    s, e = shards[rank]
    q_rows, l_rows, _ = _rows_of(Q, lenQ, s, e)
    origin = set_origin((Q, lenQ), (D, lenD))
    if block_fn is None:
        dev = torch.device("cuda", torch.cuda.current_device())
        ds = _set_of(D, lenD, dev, origin)
        qs = _set_of(q_rows, l_rows, dev, origin)
        blocks = {}
        for m in ids:
            out = torch.empty((qs.n, ds.n), dtype=torch.float32, device=dev)
            cnt = torch.empty((qs.n, ds.n), dtype=torch.int32, device=dev) if m in (_lib.EDR, _lib.LCSS) else None
            if qs.n:
                _matrix_into(m, qs, ds, out, cnt, eps=eps, gpoint=g, exact=exact, rows=rows)
            blocks[m] = (out, cnt)
        ld_all = ds.lens_host if ds.lens_host is not None else ds.lens.cpu().numpy()
    else:
        blocks = block_fn(ids, q_rows, l_rows, D, lenD, origin)
        ld_all = _rows_of(D, lenD, 0, 0)[2]
    nq, nd = int(lq_all.shape[0]), int(len(ld_all))
    maxr = max(b - a for a, b in shards)

    def gather(t):
        pad = torch.zeros((maxr, nd), dtype=t.dtype, device=t.device)
        pad[:t.shape[0]] = t
        parts = [torch.empty_like(pad) for _ in range(world)]
        if world > 1:
            dist.all_gather(parts, pad, group=group)
        else:
            parts = [pad]
        return torch.cat([p[:b - a] for p, (a, b) in zip(parts, shards)]).cpu().numpy()

    res = {}
    lq64, ld64 = lq_all.astype(np.int64)[:, None], np.asarray(ld_all, dtype=np.int64)[None, :]
    for m in ids:
        out, cnt = blocks[m]
        if cnt is not None:
            res[_lib.MEASURE_NAMES[m]] = _normalise_counts(m, gather(cnt), lq64, ld64)
        else:
            res[_lib.MEASURE_NAMES[m]] = gather(out).astype(np.float64)
    return res


def dtw_matrix(Q, lenQ, D, lenD, **kw):
    return matrix(_lib.DTW, Q, lenQ, D, lenD, **kw)


def edr_matrix(Q, lenQ, D, lenD, eps, **kw):
    return matrix(_lib.EDR, Q, lenQ, D, lenD, eps=eps, **kw)


def lcss_matrix(Q, lenQ, D, lenD, eps, **kw):
    return matrix(_lib.LCSS, Q, lenQ, D, lenD, eps=eps, **kw)


def erp_matrix(Q, lenQ, D, lenD, gpoint=None, **kw):
    return matrix(_lib.ERP, Q, lenQ, D, lenD, gpoint=gpoint, **kw)


def dfrechet_matrix(Q, lenQ, D, lenD, **kw):
    return matrix(_lib.DFRECHET, Q, lenQ, D, lenD, **kw)


def hausdorff_matrix(Q, lenQ, D, lenD, **kw):
    return matrix(_lib.HAUSDORFF, Q, lenQ, D, lenD, **kw)
