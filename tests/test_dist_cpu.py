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
