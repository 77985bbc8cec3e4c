"""ctypes binding of libtsm_b200.so (C ABI declared in include/tsm.h).

The library is the only compute path: if it is missing or a call fails, the
functions here raise.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libtsm_b200.so")

DTW, EDR, LCSS, ERP, DFRECHET, HAUSDORFF = 0, 1, 2, 3, 4, 5
MEASURES = {"dtw": DTW, "edr": EDR, "lcss": LCSS, "erp": ERP, "dfrechet": DFRECHET,
            "frechet": DFRECHET, "hausdorff": HAUSDORFF}
MEASURE_NAMES = {DTW: "dtw", EDR: "edr", LCSS: "lcss", ERP: "erp", DFRECHET: "dfrechet",
                 HAUSDORFF: "hausdorff"}
FLAG_EXACT = 1

# Every symbol include/tsm.h declares (checked by the test suite).
EXPORTS = ("tsm_version", "tsm_last_error", "tsm_max_supported_len", "tsm_matrix_query_max", "tsm_pairs", "tsm_matrix",
           "tsm_matrix_rows",
           "tsm_sched_workspace_bytes", "tsm_pairs_sched", "tsm_topk_rows", "tsm_pairs_sched_noalloc",
           "tsm_enc_param_count", "tsm_enc_workspace_bytes", "tsm_enc_forward", "tsm_enc_loss_grad", "tsm_enc_adam",
           "tsm_select_rows", "tsm_allpairs_sym", "tsm_matrix_gather", "tsm_enc_embed_workspace_bytes",
           "tsm_enc_embed", "tsm_enc_embed_status", "tsm_enc_train_status", "tsm_enc_embed_opts",
           "tsm_enc_loss_grad_w", "tsm_scan_dim",
           "tsm_scan_image_bytes", "tsm_scan_prepare", "tsm_scan", "tsm_scan_opts")


class TsmParams(ctypes.Structure):
    _fields_ = [("eps", ctypes.c_double), ("gx", ctypes.c_double), ("gy", ctypes.c_double),
                ("flags", ctypes.c_uint32), ("rows_per_thread", ctypes.c_int32)]


class TsmError(RuntimeError):
    pass


_lock = threading.Lock()
_lib = None

_vp, _i32, _i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64


def load():
    """Loads the CUDA library once; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise TsmError(f"{LIB_PATH} is missing: build it with `python -m trajsimimeasures_b200.build` "
                           "(the CUDA library is the only compute path)")
        lib = ctypes.CDLL(LIB_PATH)
        lib.tsm_version.restype = ctypes.c_int
        lib.tsm_last_error.restype = ctypes.c_char_p
        lib.tsm_max_supported_len.restype = _i32
        lib.tsm_matrix_query_max.restype = _i32
        lib.tsm_pairs.restype = ctypes.c_int
        lib.tsm_pairs.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i32,
                                  ctypes.POINTER(TsmParams), _vp, _vp, _vp]
        lib.tsm_matrix.restype = ctypes.c_int
        lib.tsm_matrix.argtypes = [ctypes.c_int, _vp, _vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp, _i64, _i32,
                                   ctypes.POINTER(TsmParams), _vp, _i64, _vp, _vp]
        lib.tsm_matrix_rows.restype = ctypes.c_int
        lib.tsm_matrix_rows.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp, _i64, _i32,
                                        ctypes.POINTER(TsmParams), _vp, _i64, _vp, _vp]
        lib.tsm_matrix_gather.restype = ctypes.c_int
        lib.tsm_matrix_gather.argtypes = [ctypes.c_int, _vp, _vp, _vp, _i64, _i32, _vp, _vp, _vp, _i64, _i32, _vp, _i64,
                                          _vp, ctypes.POINTER(TsmParams), _vp, _i64, _vp, _vp]
        lib.tsm_allpairs_sym.restype = ctypes.c_int
        lib.tsm_allpairs_sym.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp, _i64, _i32, ctypes.POINTER(TsmParams), _vp,
                                         _i64, _vp, _vp]
        lib.tsm_sched_workspace_bytes.restype = ctypes.c_int
        lib.tsm_pairs_sched.restype = ctypes.c_int
        lib.tsm_pairs_sched.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32,
                                        ctypes.POINTER(TsmParams), _vp, _vp, _i64, _vp, _vp]
        lib.tsm_pairs_sched_noalloc.restype = ctypes.c_int
        lib.tsm_pairs_sched_noalloc.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32,
                                                ctypes.POINTER(TsmParams), _vp, _vp, _i64, _vp]
        lib.tsm_enc_param_count.restype = ctypes.c_int
        lib.tsm_enc_workspace_bytes.restype = _i64
        lib.tsm_enc_workspace_bytes.argtypes = [_i32, _i32, _i32]
        _fp = ctypes.POINTER(ctypes.c_float)
        lib.tsm_enc_forward.restype = ctypes.c_int
        lib.tsm_enc_forward.argtypes = [_vp, _vp, _vp, _vp, _i32, _i32, _fp, _vp, _vp, _vp]
        lib.tsm_enc_embed_workspace_bytes.restype = _i64
        lib.tsm_enc_embed_workspace_bytes.argtypes = [_i32, _i32]
        lib.tsm_enc_embed.restype = ctypes.c_int
        lib.tsm_enc_embed.argtypes = [_vp, _vp, _vp, _vp, _i32, _i32, _fp, _vp, _vp, _vp]
        lib.tsm_enc_embed_opts.restype = ctypes.c_int
        lib.tsm_enc_embed_opts.argtypes = [_vp, _vp, _vp, _vp, _i32, _i32, _fp, _vp, _vp, _i64, _i32, _vp]
        lib.tsm_enc_train_status.restype = ctypes.c_int
        lib.tsm_enc_train_status.argtypes = [_vp, _vp, _vp]
        lib.tsm_enc_embed_status.restype = ctypes.c_int
        lib.tsm_enc_embed_status.argtypes = [_vp, ctypes.POINTER(_i32), _vp]
        lib.tsm_enc_loss_grad.restype = ctypes.c_int
        lib.tsm_enc_loss_grad.argtypes = [_vp, _vp, _vp, _vp, _i32, _i32, _fp, _vp, _vp, _vp, _i32, _vp, _vp, _vp,
                                          _vp, _vp]
        lib.tsm_enc_loss_grad_w.restype = ctypes.c_int
        lib.tsm_enc_loss_grad_w.argtypes = [_vp, _vp, _vp, _vp, _i32, _i32, _fp, _vp, _vp, _vp, _vp, _i32, _vp, _vp,
                                            _vp, _vp, _vp]
        lib.tsm_enc_adam.restype = ctypes.c_int
        lib.tsm_enc_adam.argtypes = [_vp, _vp, _vp, _vp, _i32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_float, _vp]
        lib.tsm_scan_dim.restype = _i32
        lib.tsm_scan_image_bytes.restype = _i64
        lib.tsm_scan_image_bytes.argtypes = [_i64, _i32]
        lib.tsm_scan_prepare.restype = ctypes.c_int
        lib.tsm_scan_prepare.argtypes = [_vp, _i64, _i64, ctypes.c_float, _i32, _vp, _vp, _vp]
        lib.tsm_scan.restype = ctypes.c_int
        lib.tsm_scan.argtypes = [_vp, _i64, _vp, _i64, ctypes.c_float, _vp, _i32, _vp, _vp, _vp, _vp, _i64, _vp, _vp]
        lib.tsm_scan_opts.restype = ctypes.c_int
        lib.tsm_scan_opts.argtypes = [_vp, _i64, _vp, _i64, ctypes.c_float, _vp, _i32, _vp, _vp, _vp, _vp, _i64, _vp,
                                      _i64, _vp]
        lib.tsm_select_rows.restype = ctypes.c_int
        lib.tsm_select_rows.argtypes = [_vp, _i64, _i64, _i64, _i64, _vp, _vp]
        lib.tsm_topk_rows.restype = ctypes.c_int
        lib.tsm_topk_rows.argtypes = [_vp, _i64, _i64, _i64, _i32, _vp, _vp, _vp]
        _lib = lib
    return _lib


def check(rc: int, what: str):
    if rc != 0:
        msg = load().tsm_last_error().decode(errors="replace")
        raise TsmError(f"{what} failed ({rc}): {msg}")


def params(eps=0.0, gpoint=(0.0, 0.0), exact=False, rows_per_thread=0) -> TsmParams:
    gx, gy = float(gpoint[0]), float(gpoint[1])
    return TsmParams(float(eps), gx, gy, FLAG_EXACT if exact else 0, int(rows_per_thread))
