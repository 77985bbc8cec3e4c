"""The allocation-free scheduled entry point, tsm_pairs_sched_noalloc.

Some callers cannot allocate device memory where they call the library (host
callbacks, code that must not touch the CUDA allocator, plugins whose host
application owns every device allocation, FFI callers without an allocator).
For them the scheduled kernel's scratch -- its task queue -- lives in a small
array the library allocates statically.  This test calls that entry point
through the C ABI twice in a row and checks each result against the
workspace entry point (tsm_pairs_sched) on the same inputs.  The file sorts
last so that a run stopping at its first failure has run every other test
already; it must pass alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _dev(x, dt):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).cuda()


def test_noalloc_matches_workspace_entry_point_twice():
    from trajsimimeasures_b200 import _lib, datagen as D
    from trajsimimeasures_b200.sched import PairsScheduler

    lib = _lib.load()
    pts, off, lens, ia, ib = D.pairs_lognormal(6000, seed=31)
    args = (_dev(pts, np.float32), _dev(off[ia], np.int64), _dev(lens[ia], np.int32), _dev(off[ib], np.int64),
            _dev(lens[ib], np.int32))
    measures = ["dtw", "edr", "dfrechet", "hausdorff"]
    ref = PairsScheduler(*args, measures, eps=3e-4, len_a_host=lens[ia], len_b_host=lens[ib])
    ref.run()
    torch.cuda.synchronize()
    rows = [0, 1, 4, 5]
    n = ref.n
    p = ctypes.c_void_p
    for call in range(2):
        out = torch.full((6, n), -1.0, device="cuda")
        cnt = torch.full((6, n), -1, dtype=torch.int32, device="cuda")
        rc = lib.tsm_pairs_sched_noalloc(p(args[0].data_ptr()), p(args[1].data_ptr()), p(args[2].data_ptr()),
                                         p(args[3].data_ptr()), p(args[4].data_ptr()), p(ref.order.data_ptr()),
                                         p(ref.tasks.data_ptr()), ref.plan.n_tasks, ref.plan.max_len,
                                         ref.plan.warp_floats, ctypes.byref(ref.params), p(out.data_ptr()),
                                         p(cnt.data_ptr()), n, p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, lib.tsm_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out[rows], ref.out[rows]), f"call {call}"
        assert torch.equal(cnt[1], ref.counts[1]), f"call {call}"
