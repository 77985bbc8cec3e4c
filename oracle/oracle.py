"""ctypes wrappers of the oracle (TEST INFRASTRUCTURE ONLY).

* ``pairs_f64``: FP64 restatement of the reference kernels (core/*.py).
* ``pairs_f32``: FP32 same-arithmetic twin of the CUDA kernels.
* ``RefSet``: the reference's own C++ measures (query/cpp/spatial/traj.cpp),
  compiled from the reference sources into oracle/_ref/libtsm_ref.so.

Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and the
--impl reference arm) import this module.  The product package
trajsimimeasures_b200 never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import ORACLE_SO, REF_SO, build_oracle

DTW, EDR, LCSS, ERP, DFRECHET, HAUSDORFF = 0, 1, 2, 3, 4, 5

_vp, _i32, _i64, _dbl, _flt = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_float
_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        build_oracle()  # (re)builds only when missing or older than its source
        L = ctypes.CDLL(ORACLE_SO)
        L.tsm_oracle_pairs_f64.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _i64, _dbl, _dbl, _dbl, _vp, _vp]
        L.tsm_oracle_pairs_f32.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _i64, _flt, _dbl, _dbl, _vp, _vp]
        L.tsm_oracle_set_threads.argtypes = [ctypes.c_int]
        L.tsm_oracle_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def set_threads(n: int):
    lib().tsm_oracle_set_threads(int(n))


def get_threads() -> int:
    return lib().tsm_oracle_get_threads()


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _p(a):
    return a.ctypes.data_as(_vp)


def _pairs_args(pts, off_a, len_a, off_b, len_b, dt=np.float32):
    pts = _c(pts, dt).reshape(-1, 2)
    return (pts, _c(off_a, np.int64), _c(len_a, np.int32), _c(off_b, np.int64), _c(len_b, np.int32))


def pairs_f64(measure, pts, off_a, len_a, off_b, len_b, eps=0.0, gpoint=(0.0, 0.0)):
    """FP64 restatement -> (dist float64 [n], counts int64 [n]).  The points
    are read as float64 (float32 inputs convert exactly)."""
    pts, oa, la, ob, lb = _pairs_args(pts, off_a, len_a, off_b, len_b, np.float64)
    n = oa.shape[0]
    out = np.empty(n, dtype=np.float64)
    cnt = np.zeros(n, dtype=np.int64)
    rc = lib().tsm_oracle_pairs_f64(int(measure), _p(pts), _p(oa), _p(la), _p(ob), _p(lb), n, float(eps),
                                    float(gpoint[0]), float(gpoint[1]), _p(out), _p(cnt))
    assert rc == 0
    return out, cnt


def eps2_f32(eps) -> np.float32:
    """FP32 threshold of the kernels: (float)(eps*eps), the square taken in FP64."""
    return np.float32(float(eps) * float(eps))


def pairs_f32(measure, pts, off_a, len_a, off_b, len_b, eps=0.0, gpoint=(0.0, 0.0)):
    """FP32 same-arithmetic twin -> (dist float32 [n], counts int32 [n])."""
    pts, oa, la, ob, lb = _pairs_args(pts, off_a, len_a, off_b, len_b)
    n = oa.shape[0]
    out = np.empty(n, dtype=np.float32)
    cnt = np.zeros(n, dtype=np.int32)
    rc = lib().tsm_oracle_pairs_f32(int(measure), _p(pts), _p(oa), _p(la), _p(ob), _p(lb), n,
                                    float(eps2_f32(eps)), float(gpoint[0]), float(gpoint[1]), _p(out), _p(cnt))
    assert rc == 0
    return out, cnt


def pairs_idx(fn, measure, pts, off, lens, ia, ib, **kw):
    """Pairs given as trajectory indices into one packed set."""
    ia = np.asarray(ia, dtype=np.int64)
    ib = np.asarray(ib, dtype=np.int64)
    return fn(measure, pts, off[ia], lens[ia], off[ib], lens[ib], **kw)


def matrix_idx(fn, measure, pts_q, off_q, len_q, pts_d, off_d, len_d, **kw):
    """All pairs Q x D through the pair form -> ([nq, nd] dist, [nq, nd] counts)."""
    nq, nd = len(off_q), len(off_d)
    dt = np.result_type(np.asarray(pts_q).dtype, np.asarray(pts_d).dtype, np.float32)
    pts = np.concatenate([np.asarray(pts_q, dt).reshape(-1, 2), np.asarray(pts_d, dt).reshape(-1, 2)])
    shift = np.asarray(pts_q).reshape(-1, 2).shape[0]
    qi = np.repeat(np.arange(nq), nd)
    di = np.tile(np.arange(nd), nq)
    out, cnt = fn(measure, pts, np.asarray(off_q)[qi], np.asarray(len_q)[qi], np.asarray(off_d)[di] + shift,
                  np.asarray(len_d)[di], **kw)
    return out.reshape(nq, nd), cnt.reshape(nq, nd)


class RefSet:
    """The reference's C++ Traj objects for one packed set (oracle/_ref)."""

    def __init__(self, pts, off, lens):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference checkout)")
        global _ref
        if _ref is None:
            R = ctypes.CDLL(REF_SO)
            R.tsm_ref_build.restype = _vp
            R.tsm_ref_build.argtypes = [_vp, _vp, _vp, _i64]
            R.tsm_ref_free.argtypes = [_vp]
            R.tsm_ref_pairs.argtypes = [_vp, ctypes.c_int, _vp, _vp, _i64, _flt, _flt, _vp, ctypes.c_int]
            _ref = R
        self._pts = _c(pts, np.float32).reshape(-1, 2)
        self._off = _c(off, np.int64)
        self._len = _c(lens, np.int32)
        self.h = _ref.tsm_ref_build(_p(self._pts), _p(self._off), _p(self._len), self._off.shape[0])

    def pairs(self, measure, ia, ib, gpoint=(0.0, 0.0), threads=1):
        """FP32 distances from Traj::DTW / ERP / Frechet / HausdorffDistance."""
        ia, ib = _c(ia, np.int32), _c(ib, np.int32)
        out = np.empty(ia.shape[0], dtype=np.float32)
        rc = _ref.tsm_ref_pairs(self.h, int(measure), _p(ia), _p(ib), ia.shape[0], float(gpoint[0]),
                                float(gpoint[1]), _p(out), int(threads))
        if rc == -2:
            raise ValueError("the reference has no C++ code for this measure")
        assert rc == 0
        return out

    def close(self):
        if self.h:
            _ref.tsm_ref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_available() -> bool:
    return os.path.exists(REF_SO)
