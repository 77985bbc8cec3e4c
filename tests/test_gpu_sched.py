"""GPU tests of the persistent length-bucketed scheduler (tsm_pairs_sched):
mixed measures in one launch, every bucket kind, bit-identical to the FP32
twin in exact mode; CUDA-graph replay; queue self-reset; autotuner."""
import numpy as np
import pytest
import torch

from conftest import REL_TOL, rel_err

pytestmark = pytest.mark.gpu

EPS = 3e-4
G = (-8.625, 41.15)
ALL = ["dtw", "edr", "lcss", "erp", "dfrechet", "hausdorff"]


def _batch(n, seed):
    """n lognormal pairs plus a few long ones, so every bucket kind occurs."""
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import pack_lists
    pts, off, lens, ia, ib = D.pairs_lognormal(n, seed=seed)
    extra_a = [1500, 2000, 1300, 1100, 600, 700, 3, 0]
    extra_b = [1800, 1200, 1300, 1999, 650, 2, 2000, 900]
    xp, xo, xl = D._walks(np.random.default_rng(seed), np.array(extra_a + extra_b), D.STEP_SIGMA)
    trajs = D.unpack(pts, off, lens) + D.unpack(xp, xo, xl)
    pts, off, lens = pack_lists(trajs)
    m = len(extra_a)
    base = 2 * n
    ia = np.concatenate([ia, base + np.arange(m)])
    ib = np.concatenate([ib, base + m + np.arange(m)])
    dev = lambda x, dt: torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).cuda()  # noqa: E731
    t = (dev(pts, np.float32), dev(off[ia], np.int64), dev(lens[ia], np.int32), dev(off[ib], np.int64),
         dev(lens[ib], np.int32))
    return (pts, off, lens, ia, ib), t


@pytest.mark.parametrize("rows,wf,max_steps", [(8, 4096, 8192), (4, 2048, 8192), (8, 8192, 8192), (8, 2048, 1024),
                                               (8, 4096, 1 << 20)])
def test_sched_mixed_measures_bit_identical(oracle_mod, rows, wf, max_steps):
    O = oracle_mod
    from trajsimimeasures_b200 import sched
    (pts, off, lens, ia, ib), t = _batch(20_000, seed=21)
    s = sched.PairsScheduler(*t, ALL, eps=EPS, gpoint=G, exact=True, rows=rows, warp_floats=wf,
                             max_steps=max_steps, len_a_host=lens[ia], len_b_host=lens[ib])
    kinds = set(s.plan.tasks[:, 0].tolist())
    assert {sched.KIND_TILE, sched.KIND_HAUSDORFF, sched.KIND_HAUSDORFF_WARP} <= kinds
    assert len(kinds & set(sched.GROUP_KIND.values())) >= 2
    s.run()
    torch.cuda.synchronize()
    out = s.out.cpu().numpy()
    cnt = s.counts.cpu().numpy()
    for m in range(6):
        want, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        np.testing.assert_array_equal(out[m], want, err_msg=str(m))
        if m in (1, 2):
            np.testing.assert_array_equal(cnt[m], wcnt)


def test_sched_default_mode_tolerance(oracle_mod):
    O = oracle_mod
    from trajsimimeasures_b200.sched import PairsScheduler
    (pts, off, lens, ia, ib), t = _batch(10_000, seed=22)
    s = PairsScheduler(*t, ["dtw", "dfrechet", "edr"], eps=EPS, gpoint=G, len_a_host=lens[ia], len_b_host=lens[ib])
    s.run()
    torch.cuda.synchronize()
    out = s.out.cpu().numpy()
    for m in (0, 4):
        d64, _ = O.pairs_idx(O.pairs_f64, m, pts, off, lens, ia, ib)
        assert rel_err(out[m], d64).max() <= REL_TOL
    _, wcnt = O.pairs_idx(O.pairs_f32, 1, pts, off, lens, ia, ib, eps=EPS)
    np.testing.assert_array_equal(s.counts.cpu().numpy()[1], wcnt)


def test_sched_graph_replay_and_queue_reset():
    from trajsimimeasures_b200.sched import PairsScheduler
    (pts, off, lens, ia, ib), t = _batch(5_000, seed=23)
    s = PairsScheduler(*t, ["dtw", "edr", "dfrechet"], eps=EPS, len_a_host=lens[ia], len_b_host=lens[ib])
    s.run()
    torch.cuda.synchronize()
    ref = s.out.clone()
    assert int(s.workspace.abs().sum().item()) == 0  # the last warp out reset the queue
    s.capture()
    rows = [0, 1, 4]  # the planned measures' result rows
    for _ in range(3):
        s.out.fill_(-1.0)
        s.replay()
        torch.cuda.synchronize()
        assert torch.equal(s.out[rows], ref[rows])
        assert int(s.workspace.abs().sum().item()) == 0


def test_autotune_picks_a_candidate(tmp_path, monkeypatch):
    monkeypatch.setenv("TSM_CACHE_DIR", str(tmp_path))
    from trajsimimeasures_b200 import sched
    (pts, off, lens, ia, ib), t = _batch(5_000, seed=24)
    best, times = sched.autotune(*t, ["dtw", "dfrechet", "edr"], eps=EPS, len_a_host=lens[ia],
                                 len_b_host=lens[ib])
    assert len(best) == 3 and ",".join(map(str, best)) in times and all(v > 0 for v in times.values())
    best2, _ = sched.autotune(*t, ["dtw", "dfrechet", "edr"], eps=EPS, len_a_host=lens[ia], len_b_host=lens[ib])
    assert best2 == best  # from the cache
