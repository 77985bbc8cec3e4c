"""Name-based dispatch and collation for the heuristic measures, mirroring
the heuristic part of the reference's utilities/method_helper.py
(is_heuristic :27-29, heuristic_fn_wrapper :32-73, heuristic_colllate_fn
:142-153) and the hot-path knobs of config.py.

The reference's "<name>_cpu" entries call the third-party traj_dist package
(CPU); they are not part of this GPU library and raise NotImplementedError.
The spatio-temporal measures (cdds, stedr, stlcss, sar) are outside this
library's scope and raise the same way.
"""
from __future__ import annotations

from functools import partial

import numpy as np

from . import core


class Config:
    """Hot-path subset of the reference's config.py (:40-52)."""
    effi_gpu_threads_per_traj = 64   # config.py:45
    effi_batch_size_gpu = 512        # config.py:43
    effi_cpu_method_num_cores = 8    # config.py:40
    trajsimi_edr_lcss_eps = 200      # config.py:52 (metres, Mercator coordinates)
    erp_gpoint = (0.0, 0.0)          # core/erp.py:103 default


_HEURISTICS = ["dtw", "erp", "frechet", "hausdorff", "edr", "lcss", "sar", "cdds"]
_GPU = {"dtw": core.dtw, "edr": core.edr, "erp": core.erp, "frechet": core.dfrechet,
        "hausdorff": core.hausdorff, "lcss": core.lcss}
_OUT_OF_SCOPE = {"cdds", "stedr", "stlcss", "sar"}


def is_heuristic(fn_name: str) -> bool:
    """utilities/method_helper.py:27-29."""
    return any(h in fn_name for h in _HEURISTICS)


def heuristic_fn_wrapper(fn_name: str):
    """utilities/method_helper.py:32-73: the measure function with eps and
    threads_per_traj bound from Config."""
    base = fn_name[:-4] if fn_name.endswith("_cpu") else fn_name
    if fn_name.endswith("_cpu") and (base in _GPU or base in _OUT_OF_SCOPE):
        raise NotImplementedError(f"{fn_name}: the reference's CPU path (traj_dist / core_cpu) is not part of "
                                  "this GPU library")
    if base in _OUT_OF_SCOPE:
        raise NotImplementedError(f"{fn_name}: spatio-temporal measures are outside this library")
    fn = _GPU.get(fn_name)
    assert fn is not None, f"unknown measure {fn_name!r}"
    if fn_name in ("edr", "lcss"):
        fn = partial(fn, eps=Config.trajsimi_edr_lcss_eps)
    return partial(fn, threads_per_traj=Config.effi_gpu_threads_per_traj)


def pad_lists_to_array(lst):
    """Zero-pad a list of [n_i, d] trajectories to float64 [N, max n_i, d]
    (utilities/tool_funcs.py:230-234, core/utils.py:21-27)."""
    dim2 = len(lst[0][0]) if len(lst) and len(lst[0]) else 2
    width = max((len(t) for t in lst), default=0)
    arr = np.zeros((len(lst), width, dim2), dtype=np.float64)
    for i, t in enumerate(lst):
        if len(t):
            arr[i, :len(t)] = t
    return arr


def heuristic_colllate_fn(batch, is_pad):
    """utilities/method_helper.py:142-153: pads t1 and t2 jointly so both share
    one width (is_pad=True, GPU) or returns the lists unchanged (CPU)."""
    lst_trajs, lst_trajs2 = zip(*batch)
    trajs_len = list(map(len, lst_trajs))
    trajs_len2 = list(map(len, lst_trajs2))
    if is_pad:
        arr = pad_lists_to_array(lst_trajs + lst_trajs2)
        t2 = np.copy(arr[-len(trajs_len2):])
        t1 = np.copy(arr[:len(trajs_len)])
        return t1, trajs_len, t2, trajs_len2
    return lst_trajs, trajs_len, lst_trajs2, trajs_len2
