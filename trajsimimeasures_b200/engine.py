"""Device-side engine: packed trajectory sets in HBM and the calls into the
CUDA library.  PyTorch tensors are only the device buffers and the stream.

HBM layout of a trajectory set (``TrajSet``):
    pts   float32 [n_points, 2]  all points back to back (x = lon, y = lat)
    off   int64   [n]            first point of trajectory k
    lens  int32   [n]            number of points of trajectory k
    order int32   [n]            trajectories sorted by length (stable), used as
                                 the processing order of a database in matrix
                                 mode so that the 32 lanes of a warp get
                                 near-equal lengths
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib

DEFAULT_ROWS = 8


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream_ptr(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def measure_id(measure) -> int:
    if isinstance(measure, str):
        try:
            return _lib.MEASURES[measure.lower()]
        except KeyError:
            raise ValueError(f"unknown measure {measure!r}") from None
    m = int(measure)
    if m not in _lib.MEASURE_NAMES:
        raise ValueError(f"unknown measure {measure!r}")
    return m


# ---------------------------------------------------------------------------
# host packing
# ---------------------------------------------------------------------------

def pack_lists(trajs):
    """List of [n_i, 2] sequences -> (pts float32 [P,2], off int64 [N], lens int32 [N])."""
    lens = np.fromiter((len(t) for t in trajs), dtype=np.int32, count=len(trajs))
    off = np.zeros(len(trajs), dtype=np.int64)
    if len(trajs) > 1:
        np.cumsum(lens[:-1], out=off[1:])
    total = int(lens.sum()) if len(trajs) else 0
    pts = np.empty((total, 2), dtype=np.float32)
    for k, t in enumerate(trajs):
        if lens[k]:
            pts[off[k]:off[k] + lens[k]] = np.asarray(t, dtype=np.float32).reshape(-1, 2)[:, :2]
    return pts, off, lens


def pack_padded(arr, lens):
    """Padded [N, L, 2] (+ lengths) -> packed views without moving points:
    trajectory k starts at point k*L of the flattened array."""
    a = np.ascontiguousarray(np.asarray(arr)[..., :2], dtype=np.float32)
    n, L = a.shape[0], a.shape[1]
    lens = np.asarray(lens, dtype=np.int64).reshape(-1)
    if lens.shape[0] != n:
        raise ValueError(f"{lens.shape[0]} lengths for {n} trajectories")
    if n and (lens.min() < 0 or lens.max() > L):
        raise ValueError("a length exceeds the padded width")
    off = np.arange(n, dtype=np.int64) * L
    return a.reshape(-1, 2), off, lens.astype(np.int32)


@dataclass
class TrajSet:
    """Packed trajectories resident on one CUDA device."""
    pts: torch.Tensor
    off: torch.Tensor
    lens: torch.Tensor
    max_len: int
    lens_host: np.ndarray = field(repr=False, default=None)
    _order: torch.Tensor = field(repr=False, default=None)

    @property
    def n(self) -> int:
        return int(self.off.shape[0])

    @property
    def device(self):
        return self.pts.device

    @classmethod
    def from_packed(cls, pts, off, lens, device="cuda", non_blocking=False):
        lens_h = np.asarray(lens, dtype=np.int32)
        dev = torch.device(device)

        def up(x, dt):
            t = torch.as_tensor(np.ascontiguousarray(x, dtype=dt))
            if non_blocking:
                t = t.pin_memory()
            return t.to(dev, non_blocking=non_blocking)

        pts_t = up(np.asarray(pts, dtype=np.float32).reshape(-1, 2), np.float32)
        return cls(pts_t, up(off, np.int64), up(lens_h, np.int32),
                   int(lens_h.max()) if lens_h.size else 0, lens_h)

    @classmethod
    def from_lists(cls, trajs, device="cuda"):
        return cls.from_packed(*pack_lists(trajs), device=device)

    @classmethod
    def from_padded(cls, arr, lens, device="cuda"):
        return cls.from_packed(*pack_padded(arr, lens), device=device)

    def order_by_length(self) -> torch.Tensor:
        if self._order is None:
            if self.lens_host is not None:
                o = np.argsort(self.lens_host, kind="stable").astype(np.int32)
                self._order = torch.as_tensor(o).to(self.device)
            else:
                self._order = torch.argsort(self.lens, stable=True).to(torch.int32)
        return self._order


def pair_order(len_a: np.ndarray, len_b: np.ndarray, rows=DEFAULT_ROWS) -> np.ndarray:
    """Processing order for a paired batch: pairs grouped by (row blocks,
    columns) of their DP so that a warp's 32 threads run loops of near-equal
    trip counts, the largest first (the longest loops start at once instead of
    forming the launch's tail).  Rows are the longer trajectory, columns the
    shorter."""
    la = np.asarray(len_a, dtype=np.int64)
    lb = np.asarray(len_b, dtype=np.int64)
    nr, nc = np.maximum(la, lb), np.minimum(la, lb)
    key = ((nr + rows - 1) // rows) * 65536 + nc
    return np.argsort(-key, kind="stable").astype(np.int32)


# ---------------------------------------------------------------------------
# launches
# ---------------------------------------------------------------------------

def pairs_raw(measure, pts, off_a, len_a, off_b, len_b, max_len, *, out, counts=None, order=None,
              eps=0.0, gpoint=(0.0, 0.0), exact=False, rows=0, stream=None):
    """tsm_pairs on device tensors (no copies, no sync)."""
    m = measure_id(measure)
    lib = _lib.load()
    p = _lib.params(eps, gpoint, exact, rows)
    n = int(off_a.shape[0])
    rc = lib.tsm_pairs(m, _ptr(pts), _ptr(off_a), _ptr(len_a), _ptr(off_b), _ptr(len_b), _ptr(order),
                       n, int(max_len), ctypes.byref(p), _ptr(out), _ptr(counts), _stream_ptr(stream))
    _lib.check(rc, "tsm_pairs")
    return out


def matrix_raw(measure, q: TrajSet, d: TrajSet, *, out, counts=None, d_order=None, eps=0.0,
               gpoint=(0.0, 0.0), exact=False, rows=0, stream=None):
    """tsm_matrix on two device-resident sets (no copies, no sync)."""
    m = measure_id(measure)
    lib = _lib.load()
    p = _lib.params(eps, gpoint, exact, rows)
    if d_order is None:
        d_order = d.order_by_length()
    rc = lib.tsm_matrix(m, _ptr(q.pts), _ptr(q.off), _ptr(q.lens), q.n, q.max_len,
                        _ptr(d.pts), _ptr(d.off), _ptr(d.lens), _ptr(d_order), d.n, d.max_len,
                        ctypes.byref(p), _ptr(out), int(out.stride(0)), _ptr(counts), _stream_ptr(stream))
    _lib.check(rc, "tsm_matrix")
    return out


MATRIX_QUERY_MAX = 1400  # longest query of the matrix forms (kMatrixQueryMax in the library)


def matrix_gather_raw(measure, q: TrajSet, d: TrajSet, cand: torch.Tensor, *, out, counts=None, eps=0.0,
                      gpoint=(0.0, 0.0), exact=False, rows=0, stream=None):
    """tsm_matrix_gather: out[i, s] = measure(Q_i, D_cand[i, s]) for an int32
    candidate matrix cand [nq, c] on the device (no copies, no sync)."""
    m = measure_id(measure)
    lib = _lib.load()
    p = _lib.params(eps, gpoint, exact, rows)
    if cand.dtype != torch.int32 or cand.dim() != 2 or not cand.is_contiguous():
        raise ValueError("cand must be a contiguous int32 [nq, c] tensor")
    rc = lib.tsm_matrix_gather(m, _ptr(q.pts), _ptr(q.off), _ptr(q.lens), q.n, q.max_len, _ptr(d.pts), _ptr(d.off),
                               _ptr(d.lens), d.n, d.max_len, _ptr(cand), int(cand.shape[1]), ctypes.byref(p),
                               _ptr(out), int(out.stride(0)), _ptr(counts), _stream_ptr(stream))
    _lib.check(rc, "tsm_matrix_gather")
    return out


def allpairs_sym_raw(measure, s: TrajSet, *, out, counts=None, eps=0.0, gpoint=(0.0, 0.0), exact=False, rows=0,
                     stream=None):
    """tsm_allpairs_sym on a device-resident set: the full symmetric n x n
    matrix from the upper triangle (no copies, no sync)."""
    m = measure_id(measure)
    lib = _lib.load()
    p = _lib.params(eps, gpoint, exact, rows)
    rc = lib.tsm_allpairs_sym(m, _ptr(s.pts), _ptr(s.off), _ptr(s.lens), _ptr(s.order_by_length()), s.n, s.max_len,
                              ctypes.byref(p), _ptr(out), int(out.stride(0)), _ptr(counts), _stream_ptr(stream))
    _lib.check(rc, "tsm_allpairs_sym")
    return out


def matrix(measure, q: TrajSet, d: TrajSet, *, eps=0.0, gpoint=(0.0, 0.0), exact=False, rows=0,
           stream=None, with_counts=None):
    """All pairs Q x D on the device -> (out float32 [nq, nd], counts int32 or None)."""
    m = measure_id(measure)
    out = torch.empty((q.n, d.n), dtype=torch.float32, device=q.device)
    want = (m in (_lib.EDR, _lib.LCSS)) if with_counts is None else with_counts
    counts = torch.empty((q.n, d.n), dtype=torch.int32, device=q.device) if want else None
    matrix_raw(m, q, d, out=out, counts=counts, eps=eps, gpoint=gpoint, exact=exact, rows=rows, stream=stream)
    return out, counts


def pairs_in_set(measure, s: TrajSet, idx_a, idx_b, *, eps=0.0, gpoint=(0.0, 0.0), exact=False, rows=0,
                 stream=None, order=None, with_counts=None):
    """Pairs (idx_a[k], idx_b[k]) of one device set -> (out float32 [n], counts)."""
    m = measure_id(measure)
    ia = torch.as_tensor(idx_a, device=s.device).long()
    ib = torch.as_tensor(idx_b, device=s.device).long()
    off_a, len_a = s.off[ia], s.lens[ia]
    off_b, len_b = s.off[ib], s.lens[ib]
    n = ia.shape[0]
    out = torch.empty(n, dtype=torch.float32, device=s.device)
    want = (m in (_lib.EDR, _lib.LCSS)) if with_counts is None else with_counts
    counts = torch.empty(n, dtype=torch.int32, device=s.device) if want else None
    pairs_raw(m, s.pts, off_a, len_a, off_b, len_b, s.max_len, out=out, counts=counts, order=order,
              eps=eps, gpoint=gpoint, exact=exact, rows=rows, stream=stream)
    return out, counts
