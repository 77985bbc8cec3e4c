"""Multi-process (world_size 2, gloo, CPU) tests of the sharding and
result-assembly logic of the multi-GPU path.  The oracle stands in for the
kernels inside these CPU ranks (test-only use)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from trajsimimeasures_b200 import shard


def test_pair_shards_partition_and_balance():
    from trajsimimeasures_b200 import datagen as D
    _, _, lens, ia, ib = D.pairs_lognormal(50_000, seed=9)
    la, lb = lens[ia], lens[ib]
    for world in (1, 2, 3, 4, 8):
        sh = shard.pair_shards(la, lb, world)
        allidx = np.sort(np.concatenate(sh))
        np.testing.assert_array_equal(allidx, np.arange(len(la)))
        if world > 1:
            assert shard.imbalance(shard.pair_cost(la, lb), sh) < 0.02


def test_row_shards_cover_rows():
    q = np.random.default_rng(0).integers(20, 201, 2000)
    for world in (1, 2, 4, 8):
        rs = shard.row_shards(q, world)
        assert rs[0][0] == 0 and rs[-1][1] == 2000
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        loads = [q[s:e].sum() for s, e in rs]
        assert max(loads) / (sum(loads) / world) < 1.02


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from trajsimimeasures_b200 import datagen as D
        O.set_threads(1)
        # paired batch, equal-work shards, gathered back in pair order
        pts, off, lens, ia, ib = D.pairs_lognormal(2000, seed=3)
        la, lb = lens[ia], lens[ib]
        mine = shard.pair_shards(la, lb, world)[rank]
        d, _ = O.pairs_f32(0, pts, off[ia[mine]], la[mine], off[ib[mine]], lb[mine])
        parts = [None] * world
        dist.all_gather_object(parts, (mine, d))
        # matrix rows
        p, o, l = D.trajectory_set(40, seed=5)
        (s, e) = shard.row_shards(l, world)[rank]
        blk, _ = O.matrix_idx(O.pairs_f32, 4, p, o[s:e], l[s:e], p, o, l)
        full = shard.gather_rows(blk, (s, e), len(l))
        tmax = shard.max_over_ranks(10.0 + rank)
        if rank == 0:
            res = np.empty(len(la), dtype=np.float32)
            for idx, vals in parts:
                res[idx] = vals
            q.put((res, full, tmax))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_gloo_shards_match_single_process():
    from oracle import oracle as O
    from trajsimimeasures_b200 import datagen as D
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res, full, tmax = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pts, off, lens, ia, ib = D.pairs_lognormal(2000, seed=3)
    want, _ = O.pairs_idx(O.pairs_f32, 0, pts, off, lens, ia, ib)
    np.testing.assert_array_equal(res, want)
    p, o, l = D.trajectory_set(40, seed=5)
    wfull, _ = O.matrix_idx(O.pairs_f32, 4, p, o, l, p, o, l)
    np.testing.assert_array_equal(full, wfull)
    assert tmax == 11.0


def _knn_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch
        from oracle import oracle as O
        from trajsimimeasures_b200 import datagen as D
        from trajsimimeasures_b200.knn import knn_sharded, shard_range
        O.set_threads(1)
        qp, qo, ql = D.trajectory_set(6, seed=41)
        dp, do, dl = D.trajectory_set(401, seed=42)
        s, e = shard_range(401, rank, world)
        # the oracle stands in for this rank's kernels: local distances, local top-k
        m, _ = O.matrix_idx(O.pairs_f32, 0, qp, qo, ql, dp, do[s:e], dl[s:e])
        o = np.argsort(m, axis=1, kind="stable")[:, :10]
        local = (torch.from_numpy(np.take_along_axis(m, o, 1)), torch.from_numpy(o))
        gd, gi = knn_sharded(local, 6, 10, s)
        if rank == 0:
            q.put((gd.numpy(), gi.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_gloo_knn_merge_matches_single_process():
    from oracle import oracle as O
    from trajsimimeasures_b200 import datagen as D
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_knn_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gd, gi = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    qp, qo, ql = D.trajectory_set(6, seed=41)
    dp, do, dl = D.trajectory_set(401, seed=42)
    m, _ = O.matrix_idx(O.pairs_f32, 0, qp, qo, ql, dp, do, dl)
    o = np.argsort(m, axis=1, kind="stable")[:, :10]
    np.testing.assert_array_equal(gi, o)
    np.testing.assert_array_equal(gd, np.take_along_axis(m, o, 1))


def test_shard_range_covers():
    from trajsimimeasures_b200.knn import shard_range
    for n in (0, 1, 7, 401, 1000):
        for w in (1, 2, 3, 8):
            rs = [shard_range(n, r, w) for r in range(w)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))


def _oracle_blocks(ids, q_rows, l_rows, D, lenD, origin):
    """CPU stand-in for the GPU block of core.matrix_sharded: the FP32 twin on
    the same translated float32 points the kernels would get."""
    import torch
    from oracle import oracle as O
    from trajsimimeasures_b200.engine import pack_padded, shift_gpoint
    from trajsimimeasures_b200 import datagen as DG
    o = None if origin is None else origin
    qp, qo, ql = pack_padded(q_rows, l_rows, o)
    dp, do, dl = pack_padded(D, lenD, o)
    g = shift_gpoint(DG.BOX_CENTRE, origin or (0.0, 0.0))
    out = {}
    for m in ids:
        v, c = O.matrix_idx(O.pairs_f32, m, qp, qo, ql, dp, do, dl, eps=DG.EPS_DEG, gpoint=g)
        out[m] = (torch.from_numpy(v), torch.from_numpy(c) if m in (1, 2) else None)
    return out


def _sharded_case():
    from trajsimimeasures_b200 import datagen as D
    p, o, l, ia, ib = D.near_pairs_f64(30, lo=5, hi=40, seed=77, units="deg")
    t = D.unpack(p, o, l)
    P = D.pad(t)
    return P[:37], l[:37], P, l


def _sharded_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from trajsimimeasures_b200 import core, datagen as D
        O.set_threads(1)
        Q, lq, S, ls = _sharded_case()
        res = core.matrix_sharded(["dtw", "edr", "lcss", "erp", "dfrechet", "hausdorff"], Q, lq, S, ls,
                                  eps=D.EPS_DEG, gpoint=D.BOX_CENTRE, block_fn=_oracle_blocks)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_gloo_matrix_sharded_matches_single_process():
    """core.matrix_sharded's real code path (row shards, one all-gather per
    measure, float64 assembly on every rank) over 2 gloo ranks, the oracle
    standing in for the kernels: both ranks get the single-process matrix."""
    from oracle import oracle as O
    from trajsimimeasures_b200 import core, datagen as D
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=240) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    Q, lq, S, ls = _sharded_case()
    O.set_threads(1)
    want = core.matrix_sharded(["dtw", "edr", "lcss", "erp", "dfrechet", "hausdorff"], Q, lq, S, ls, eps=D.EPS_DEG,
                               gpoint=D.BOX_CENTRE, block_fn=_oracle_blocks)
    assert set(got) == {0, 1}
    for r in (0, 1):
        for name, v in want.items():
            assert v.shape == (37, 60) and v.dtype == np.float64
            np.testing.assert_array_equal(got[r][name], v, err_msg=name)
    # and against the FP64 restatement on the original float64 inputs
    qp = np.concatenate([Q[i, :lq[i]] for i in range(37)])
    sp = np.concatenate([S[i, :ls[i]] for i in range(60)])
    qo = np.concatenate([[0], np.cumsum(lq)[:-1]])
    so = np.concatenate([[0], np.cumsum(ls)[:-1]])
    d64, _ = O.matrix_idx(O.pairs_f64, 0, qp, qo, lq, sp, so, ls)
    assert np.all(np.abs(want["dtw"] - d64) <= 1e-5 * d64)


# -- data-parallel encoder training -------------------------------------------------
# Encoder.fit's data-parallel loop (shares of one global batch per rank, one
# all-reduce of the pair-weighted gradients per step) around a CPU stand-in
# for the kernels: a linear model of the pair's feature difference, plain
# gradient steps.  Two gloo ranks with batch_pairs = B must end where one
# process with batch_pairs = 2B ends.

class _FakeSet:
    def __init__(self, feat):
        import torch
        self.feat = feat
        self.device = torch.device("cpu")


def _linear_encoder():
    import torch
    from trajsimimeasures_b200.surrogate import Encoder

    class _Linear(Encoder):
        def loss_grad(self, s, tidx, ia, ib, y, w=None, stream=None):
            t = torch.as_tensor(np.asarray(tidx))
            d = s.feat[t[torch.as_tensor(ia)]] - s.feat[t[torch.as_tensor(ib)]]
            err = d @ self.params - torch.as_tensor(np.asarray(y), dtype=torch.float64)
            wp = torch.ones_like(err) if w is None else torch.as_tensor(np.asarray(w), dtype=torch.float64)
            loss = (wp * err * err).mean().reshape(1)
            grad = 2.0 * ((wp * err)[:, None] * d).mean(0)
            return loss, grad, None

        def adam(self, grad, lr=1e-3, **kw):
            self.params -= lr * grad

        def check_training(self, stream=None):
            pass

    return _Linear(params=torch.zeros(24, dtype=torch.float64), nrm=np.zeros(4))


def _dp_case():
    import torch
    rng = np.random.default_rng(9)
    feat = torch.as_tensor(rng.normal(size=(300, 24)))
    pa, pb = rng.integers(0, 300, 257), rng.integers(0, 300, 257)  # 257: a last global batch of one pair
    theta = rng.normal(size=24)
    y = np.abs((feat.numpy()[pa] - feat.numpy()[pb]) @ theta) + 0.1
    return _FakeSet(feat), pa, pb, y


def _dp_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s, pa, pb, y = _dp_case()
        enc = _linear_encoder()
        hist = enc.fit(s, pa, pb, y, epochs=3, batch_pairs=64, lr=0.002, seed=4, relative=True,
                       group=dist.group.WORLD)
        q.put((rank, enc.params.numpy().copy(), hist))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_gloo_data_parallel_fit_matches_one_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict((r, (th, h)) for r, th, h in (q.get(timeout=240) for _ in range(2)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    s, pa, pb, y = _dp_case()
    one = _linear_encoder()
    hist = one.fit(s, pa, pb, y, epochs=3, batch_pairs=128, lr=0.002, seed=4, relative=True)
    np.testing.assert_array_equal(got[0][0], got[1][0])  # the replicas stay equal
    np.testing.assert_allclose(got[0][0], one.params.numpy(), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(got[0][1], hist, rtol=1e-10)
    assert hist[-1] < hist[0]  # it trains
