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
# float64 inputs: one FP64 origin per call
# ---------------------------------------------------------------------------
#
# The reference computes in FP64 on float64 inputs, e.g. Mercator metres read
# by utilities/data_loader.py:78-79 (x ~ -9.7e5, y ~ 5.0e6 m in Porto, where
# FP32 spacing is 0.5 m) with eps = 200 m (config.py:52).  Every measure here
# depends on point differences only (and ERP on differences to the gap point),
# so the points are translated by an FP64 origin before they are rounded to
# FP32 and the gap point is translated with them: the rounding error of a
# coordinate is then half an FP32 ulp of its distance to the origin instead of
# half an ulp of its absolute value.
#
# The origin is rounded to FP32 itself.  x - o is then exact in FP64, rounded
# once to FP32, and for FP32-representable inputs within a factor of two of o
# it is exact (Sterbenz), so the kernels see the same point differences as
# without the translation.  float32 (and float16/bfloat16) inputs are taken
# as they are: rounding them again could only add error.

_EXACT_IN_F32 = {np.dtype(np.float32), np.dtype(np.float16)}


def needs_origin(dtype) -> bool:
    """True if coordinates of this dtype lose precision when rounded to FP32."""
    if isinstance(dtype, torch.dtype):
        return dtype not in (torch.float32, torch.float16, torch.bfloat16)
    return np.dtype(dtype) not in _EXACT_IN_F32


def origin_of_points(first_pts) -> tuple:
    """Origin of one call: the FP32-rounded midpoint of the bounding box of the
    given points (one per non-empty trajectory, [k, 2]); (0, 0) for none."""
    p = np.asarray(first_pts, dtype=np.float64).reshape(-1, 2)
    if p.shape[0] == 0:
        return (0.0, 0.0)
    mid = 0.5 * (p.min(axis=0) + p.max(axis=0))
    m32 = mid.astype(np.float32)
    if not np.all(np.isfinite(m32)):
        return (0.0, 0.0)
    return (float(m32[0]), float(m32[1]))


def first_points_padded(arr, lens) -> np.ndarray:
    """First point of every non-empty trajectory of a padded [N, L, >=2] array."""
    a = np.asarray(arr)
    lens = np.asarray(lens).reshape(-1)
    return np.asarray(a[lens > 0, 0, :2], dtype=np.float64)


def first_points_lists(trajs) -> np.ndarray:
    firsts = [np.asarray(t, dtype=np.float64).reshape(-1, np.shape(t)[-1])[0, :2] for t in trajs if len(t)]
    return np.array(firsts, dtype=np.float64).reshape(-1, 2)


def sub_origin_f32(src, origin, out):
    """out (float32 ndarray) = src - origin, computed in FP64 and rounded once.
    origin broadcasts against src (e.g. [2], or [n, 1, 2] per trajectory).
    Runs as one multithreaded torch CPU op: NumPy's broadcast subtract with a
    float32 destination is several times slower on [n, L, 2] arrays."""
    a = torch.from_numpy(np.asarray(src, dtype=np.float64))
    o = torch.from_numpy(np.ascontiguousarray(origin, dtype=np.float64))
    torch.from_numpy(out).copy_(a - o)
    return out


def _nonzero(origin):
    return None if origin is None or tuple(float(v) for v in origin) == (0.0, 0.0) else origin


def shift_gpoint(gpoint, origin) -> tuple:
    """The ERP gap point in the coordinates of a set translated by origin."""
    return (float(gpoint[0]) - float(origin[0]), float(gpoint[1]) - float(origin[1]))


# ---------------------------------------------------------------------------
# host packing
# ---------------------------------------------------------------------------

def pack_lists(trajs, origin=None):
    """List of [n_i, 2] sequences -> (pts float32 [P,2], off int64 [N], lens int32 [N]).
    With an origin ([2], or [N, 2] per trajectory) the points are translated
    by it in FP64 and then rounded to float32."""
    lens = np.fromiter((len(t) for t in trajs), dtype=np.int32, count=len(trajs))
    off = np.zeros(len(trajs), dtype=np.int64)
    if len(trajs) > 1:
        np.cumsum(lens[:-1], out=off[1:])
    total = int(lens.sum()) if len(trajs) else 0
    pts = np.empty((total, 2), dtype=np.float32)
    o = None if origin is None else np.broadcast_to(np.asarray(origin, dtype=np.float64).reshape(-1, 2),
                                                    (len(trajs), 2))
    for k, t in enumerate(trajs):
        if lens[k]:
            a = np.asarray(t)
            a = a.reshape(-1, a.shape[-1])[:, :2]
            if o is None:
                pts[off[k]:off[k] + lens[k]] = a
            else:
                pts[off[k]:off[k] + lens[k]] = np.asarray(a, dtype=np.float64) - o[k]
    return pts, off, lens


def pack_padded(arr, lens, origin=None):
    """Padded [N, L, 2] (+ lengths) -> packed views without moving points:
    trajectory k starts at point k*L of the flattened array.  With an origin
    the points are translated by it in FP64 before rounding to float32."""
    src = np.asarray(arr)
    n, L = src.shape[0], src.shape[1]
    lens = np.asarray(lens, dtype=np.int64).reshape(-1)
    if lens.shape[0] != n:
        raise ValueError(f"{lens.shape[0]} lengths for {n} trajectories")
    if n and (lens.min() < 0 or lens.max() > L):
        raise ValueError("a length exceeds the padded width")
    if origin is None:
        a = np.ascontiguousarray(src[..., :2], dtype=np.float32)
    else:
        a = np.empty((n, L, 2), dtype=np.float32)
        sub_origin_f32(src[..., :2], np.asarray(origin, dtype=np.float64).reshape(-1, 1, 2), a)
    off = np.arange(n, dtype=np.int64) * L
    return a.reshape(-1, 2), off, lens.astype(np.int32)


@dataclass
class TrajSet:
    """Packed trajectories resident on one CUDA device.  ``origin`` is the FP64
    point the float32 coordinates are relative to ((0, 0) unless the set was
    built from float64 input); sets used together in one call must share it."""
    pts: torch.Tensor
    off: torch.Tensor
    lens: torch.Tensor
    max_len: int
    lens_host: np.ndarray = field(repr=False, default=None)
    _order: torch.Tensor = field(repr=False, default=None)
    origin: tuple = (0.0, 0.0)

    @property
    def n(self) -> int:
        return int(self.off.shape[0])

    @property
    def device(self):
        return self.pts.device

    @classmethod
    def from_packed(cls, pts, off, lens, device="cuda", non_blocking=False, origin=None):
        """origin: None = the set's own (see origin_of_points) when pts is not
        float32, else (0, 0); or an explicit (x, y), for sets that will be
        used together."""
        lens_h = np.asarray(lens, dtype=np.int32)
        dev = torch.device(device)
        off_h = np.asarray(off, dtype=np.int64).reshape(-1)
        src = np.asarray(pts)
        src = src.reshape(-1, src.shape[-1]) if src.size else src.reshape(-1, 2)

        def up(x, dt):
            t = torch.as_tensor(np.ascontiguousarray(x, dtype=dt))
            if non_blocking:
                t = t.pin_memory()
            return t.to(dev, non_blocking=non_blocking)

        if origin is None and needs_origin(src.dtype):
            origin = origin_of_points(src[off_h[lens_h > 0], :2] if src.shape[0] else src[:0, :2])
        if origin is None or tuple(origin) == (0.0, 0.0):
            f32 = np.asarray(src[:, :2], dtype=np.float32)
            origin = (0.0, 0.0)
        else:
            origin = (float(origin[0]), float(origin[1]))
            f32 = np.empty((src.shape[0], 2), dtype=np.float32)
            sub_origin_f32(src[:, :2], np.asarray(origin, dtype=np.float64), f32)
        return cls(up(f32, np.float32), up(off_h, np.int64), up(lens_h, np.int32),
                   int(lens_h.max()) if lens_h.size else 0, lens_h, origin=origin)

    @classmethod
    def from_lists(cls, trajs, device="cuda", origin=None):
        """origin as in from_packed."""
        trajs = list(trajs)
        if origin is None and any(needs_origin(np.asarray(t).dtype) for t in trajs if len(t)):
            origin = origin_of_points(first_points_lists(trajs))
        pts, off, lens = pack_lists(trajs, _nonzero(origin))
        return cls.from_packed(pts, off, lens, device=device, origin=(0.0, 0.0))._with_origin(origin)

    @classmethod
    def from_padded(cls, arr, lens, device="cuda", origin=None):
        """origin as in from_packed."""
        a = np.asarray(arr)
        if origin is None and needs_origin(a.dtype):
            origin = origin_of_points(first_points_padded(a, lens))
        pts, off, ln = pack_padded(a, lens, _nonzero(origin))
        return cls.from_packed(pts, off, ln, device=device, origin=(0.0, 0.0))._with_origin(origin)

    def _with_origin(self, origin):
        self.origin = (0.0, 0.0) if origin is None else (float(origin[0]), float(origin[1]))
        return self

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


def same_origin(q: TrajSet, d: TrajSet) -> tuple:
    """The common origin of two sets used in one call (raises if they differ:
    their float32 coordinates would not be comparable)."""
    if tuple(q.origin) != tuple(d.origin):
        raise ValueError(f"the two trajectory sets are relative to different origins ({q.origin} vs {d.origin}); "
                         "build them with the same origin=")
    return q.origin


MATRIX_BUCKETS = 4          # query-length groups of one Q x D product, when asked for (buckets=)


def length_buckets(s: TrajSet, n_buckets=MATRIX_BUCKETS):
    """The set's trajectories in length order, cut into n_buckets groups of
    equal count: [(rows int32 tensor on the device, longest length)].  Cached
    on the set."""
    key = ("_buckets", n_buckets)
    cache = s.__dict__.setdefault("_bucket_cache", {})
    if key not in cache:
        lh = s.lens_host if s.lens_host is not None else s.lens.cpu().numpy()
        o = np.argsort(lh, kind="stable")
        parts = [p for p in np.array_split(o, n_buckets) if p.size]
        cache[key] = [(torch.as_tensor(p.astype(np.int32)).to(s.device), int(lh[p].max())) for p in parts]
    return cache[key]


def matrix_raw(measure, q: TrajSet, d: TrajSet, *, out, counts=None, d_order=None, eps=0.0,
               gpoint=(0.0, 0.0), exact=False, rows=0, stream=None, buckets=None):
    """tsm_matrix on two device-resident sets (no copies, no sync).  gpoint is
    in the sets' original coordinates (translated here by their origin).

    With buckets > 1 the queries go in groups of similar length
    (length_buckets), one tsm_matrix_rows launch each: a group's shared
    memory is sized for its own longest query, so its launch fits more CTAs
    per SM than one sized for the longest of Q.  Every value is the one
    tsm_matrix gives.  Measured on B200 (2000 x 2000, lengths U{20..200},
    four groups): no gain -- DTW 15.26 -> 15.25 ms, ERP 18.85 -> 18.87,
    Hausdorff 39.9 -> 42.0: the long queries, which hold most of the cells,
    keep two CTAs per SM, and each launch adds its own tail -- so one launch
    is the default."""
    m = measure_id(measure)
    lib = _lib.load()
    p = _lib.params(eps, shift_gpoint(gpoint, same_origin(q, d)), exact, rows)
    if d_order is None:
        d_order = d.order_by_length()
    nb = buckets if buckets is not None else 1
    if nb <= 1:
        rc = lib.tsm_matrix(m, _ptr(q.pts), _ptr(q.off), _ptr(q.lens), q.n, q.max_len,
                            _ptr(d.pts), _ptr(d.off), _ptr(d.lens), _ptr(d_order), d.n, d.max_len,
                            ctypes.byref(p), _ptr(out), int(out.stride(0)), _ptr(counts), _stream_ptr(stream))
        _lib.check(rc, "tsm_matrix")
        return out
    for rows_t, ml in length_buckets(q, nb):
        rc = lib.tsm_matrix_rows(m, _ptr(q.pts), _ptr(q.off), _ptr(q.lens), _ptr(rows_t), int(rows_t.shape[0]), ml,
                                 _ptr(d.pts), _ptr(d.off), _ptr(d.lens), _ptr(d_order), d.n, d.max_len,
                                 ctypes.byref(p), _ptr(out), int(out.stride(0)), _ptr(counts), _stream_ptr(stream))
        _lib.check(rc, "tsm_matrix_rows")
    return out


MATRIX_QUERY_MAX = 1400  # longest query of the matrix forms (tsm_matrix_query_max() of the library)


def pair_order_dev(len_a: torch.Tensor, len_b: torch.Tensor, rows=DEFAULT_ROWS) -> torch.Tensor:
    """pair_order on the device (int32 processing order for tsm_pairs)."""
    la, lb = len_a.long(), len_b.long()
    nr, nc = torch.maximum(la, lb), torch.minimum(la, lb)
    key = ((nr + rows - 1) // rows) * 65536 + nc
    return torch.argsort(-key, stable=True).to(torch.int32)


def matrix_gather_raw(measure, q: TrajSet, d: TrajSet, cand: torch.Tensor, *, out, counts=None, eps=0.0,
                      gpoint=(0.0, 0.0), exact=False, rows=0, stream=None, q_order=None):
    """tsm_matrix_gather: out[i, s] = measure(Q_i, D_cand[i, s]) for an int32
    candidate matrix cand [nq, c] on the device (no copies, no sync).
    q_order: int32 [nq] device processing order of the queries (None: 0..nq-1)."""
    m = measure_id(measure)
    lib = _lib.load()
    p = _lib.params(eps, shift_gpoint(gpoint, same_origin(q, d)), exact, rows)
    if cand.dtype != torch.int32 or cand.dim() != 2 or not cand.is_contiguous():
        raise ValueError("cand must be a contiguous int32 [nq, c] tensor")
    rc = lib.tsm_matrix_gather(m, _ptr(q.pts), _ptr(q.off), _ptr(q.lens), q.n, q.max_len, _ptr(d.pts), _ptr(d.off),
                               _ptr(d.lens), d.n, d.max_len, _ptr(cand), int(cand.shape[1]), _ptr(q_order),
                               ctypes.byref(p),
                               _ptr(out), int(out.stride(0)), _ptr(counts), _stream_ptr(stream))
    _lib.check(rc, "tsm_matrix_gather")
    return out


def allpairs_sym_raw(measure, s: TrajSet, *, out, counts=None, eps=0.0, gpoint=(0.0, 0.0), exact=False, rows=0,
                     stream=None):
    """tsm_allpairs_sym on a device-resident set: the full symmetric n x n
    matrix from the upper triangle (no copies, no sync)."""
    m = measure_id(measure)
    lib = _lib.load()
    p = _lib.params(eps, shift_gpoint(gpoint, s.origin), exact, rows)
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
              eps=eps, gpoint=shift_gpoint(gpoint, s.origin), exact=exact, rows=rows, stream=stream)
    return out, counts
