"""CPU tests: the C-ABI library loads and exports what include/tsm.h declares,
argument checks that return before any CUDA call, and the host-side logic
(packing, ordering, generators, reference-signature validation)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "tsm.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tsm_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from trajsimimeasures_b200 import _lib
    from trajsimimeasures_b200.build import build
    build()
    return _lib.load()


def test_header_declares_python_exports():
    from trajsimimeasures_b200 import _lib
    assert set(_declared()) == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in _declared():
        assert hasattr(lib, name), name


def test_library_is_sm100a_only():
    from trajsimimeasures_b200.build import ARCH
    assert ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_version_and_limits(lib):
    assert lib.tsm_version() >= 100
    assert lib.tsm_max_supported_len() == 32768
    from trajsimimeasures_b200.engine import MATRIX_QUERY_MAX
    assert lib.tsm_matrix_query_max() == MATRIX_QUERY_MAX
    assert lib.tsm_last_error() == b""


def test_invalid_arguments_fail_before_cuda(lib):
    from trajsimimeasures_b200 import _lib
    p = _lib.params()
    nul = ctypes.c_void_p(0)
    rc = lib.tsm_pairs(9, nul, nul, nul, nul, nul, nul, 1, 10, ctypes.byref(p), nul, nul, nul)
    assert rc == -1 and b"unknown measure" in lib.tsm_last_error()
    rc = lib.tsm_pairs(0, nul, nul, nul, nul, nul, nul, 4, 10, ctypes.byref(p), nul, nul, nul)
    assert rc == -1 and b"null pointer" in lib.tsm_last_error()
    assert lib.tsm_pairs(0, nul, nul, nul, nul, nul, nul, 0, 10, ctypes.byref(p), nul, nul, nul) == 0
    rc = lib.tsm_pairs(0, nul, nul, nul, nul, nul, nul, -1, 10, ctypes.byref(p), nul, nul, nul)
    assert rc == -1
    rc = lib.tsm_matrix(0, nul, nul, nul, 3, 10, nul, nul, nul, nul, 3, 10, ctypes.byref(p), nul, 3, nul, nul)
    assert rc == -1
    dummy = ctypes.c_void_p(16)
    rc = lib.tsm_matrix(0, dummy, dummy, dummy, 3, 10, dummy, dummy, dummy, nul, 3, 10, ctypes.byref(p), dummy, 2,
                        nul, nul)
    assert rc == -1 and b"ld_out" in lib.tsm_last_error()
    rc = lib.tsm_allpairs_sym(0, dummy, dummy, dummy, nul, 3, 10, ctypes.byref(p), dummy, 3, nul, nul)
    assert rc == -1 and b"null pointer" in lib.tsm_last_error()
    rc = lib.tsm_allpairs_sym(0, dummy, dummy, dummy, dummy, 3, 10, ctypes.byref(p), dummy, 2, nul, nul)
    assert rc == -1 and b"ld_out" in lib.tsm_last_error()
    rc = lib.tsm_allpairs_sym(7, dummy, dummy, dummy, dummy, 3, 10, ctypes.byref(p), dummy, 3, nul, nul)
    assert rc == -1 and b"unknown measure" in lib.tsm_last_error()
    assert lib.tsm_allpairs_sym(0, nul, nul, nul, nul, 0, 10, ctypes.byref(p), nul, 0, nul, nul) == 0
    rc = lib.tsm_pairs(0, dummy, dummy, dummy, dummy, dummy, nul, 4, 40000, ctypes.byref(p), dummy, nul, nul)
    assert rc == -3 and b"max_len 40000 > 32768" in lib.tsm_last_error()
    st = ctypes.c_int32(0)
    assert lib.tsm_enc_embed_status(nul, ctypes.byref(st), nul) == -1
    rc = lib.tsm_enc_embed_opts(dummy, dummy, dummy, dummy, 4, 8, (ctypes.c_float * 4)(0, 0, 1, 1),
                                ctypes.c_void_p(256), dummy, 0, -1, nul)
    assert rc == -1 and b"wait limit" in lib.tsm_last_error()
    assert lib.tsm_enc_train_status(nul, ctypes.byref(st), nul) == -1
    rc = lib.tsm_enc_embed(dummy, dummy, dummy, dummy, 4, 8, (ctypes.c_float * 4)(0, 0, 1, 1), ctypes.c_void_p(272),
                           dummy, nul)
    assert rc == -1 and b"256-byte aligned" in lib.tsm_last_error()
    with pytest.raises(_lib.TsmError):
        _lib.check(-1, "x")


def test_float64_inputs_get_an_fp64_origin():
    """Host logic of the FP64 origin: float32 input is taken as is; float64
    input is translated per pair (ERP: per call, with the gap point) by an
    FP32-rounded origin, in FP64, and rounded once; for FP32 values near the
    origin the translation is exact (Sterbenz)."""
    from trajsimimeasures_b200 import core
    from trajsimimeasures_b200.engine import TrajSet, origin_of_points, pack_lists, pack_padded, shift_gpoint
    rng = np.random.default_rng(1)
    t1 = np.stack([rng.uniform(-9.7e5, -9.6e5, (5, 7)), rng.uniform(5.03e6, 5.04e6, (5, 7))], axis=-1)
    t2 = t1 + rng.normal(0, 100.0, t1.shape)
    l1, l2 = np.array([7, 0, 3, 7, 1]), np.array([7, 4, 0, 2, 7])
    assert core.pair_origins(0, t1.astype(np.float32), l1, t2.astype(np.float32), l2) is None
    o = core.pair_origins(0, t1, l1, t2, l2)
    assert o.shape == (5, 2) and np.array_equal(o[0], t1[0, 0].astype(np.float32))
    assert np.array_equal(o[1], t2[1, 0].astype(np.float32))  # empty t1: t2's first point
    assert np.all(o.astype(np.float32) == o)
    g = core.pair_origins(3, t1, l1, t2, l2)
    assert g.shape == (2,) and np.all(np.float32(g) == g)
    f = np.concatenate([t1[l1 > 0, 0], t2[l2 > 0, 0]])
    assert np.allclose(g, 0.5 * (f.min(0) + f.max(0)), rtol=1e-7)
    assert shift_gpoint((0.0, 0.0), g) == (-g[0], -g[1])
    # one rounding of the FP64 difference
    pts, off, lens = pack_lists([t1[0]], origin=o[0])
    assert np.array_equal(pts, (t1[0] - o[0]).astype(np.float32))
    p2, _, _ = pack_padded(t1[:2], [7, 7], origin=o[:2])
    assert np.array_equal(p2.reshape(2, 7, 2), (t1[:2] - o[:2, None, :]).astype(np.float32))
    # FP32 values near the origin: exact
    x = t1.astype(np.float32).astype(np.float64)
    ox = core.pair_origins(0, x, l1, x, l1)
    assert np.array_equal((x - ox[:, None, :]).astype(np.float32).astype(np.float64), x - ox[:, None, :])
    # a set origin is shared by Q and D; no origin for float32 sets or none given
    t2f = t2.astype(np.float32)
    assert core.set_origin((t1, l1), (t2f, l2)) == origin_of_points(np.concatenate([t1[l1 > 0, 0], t2f[l2 > 0, 0]]))
    assert core.set_origin((t1.astype(np.float32), l1)) is None
    assert origin_of_points(np.zeros((0, 2))) == (0.0, 0.0)
    # TrajSet records the origin it was built with; TrajSet.from_packed picks its own for float64
    from trajsimimeasures_b200.engine import same_origin
    a = TrajSet.__new__(TrajSet)
    a.origin = (1.0, 2.0)
    b = TrajSet.__new__(TrajSet)
    b.origin = (1.0, 2.5)
    with pytest.raises(ValueError, match="different origins"):
        same_origin(a, b)


def test_pack_lists_and_padded():
    from trajsimimeasures_b200.engine import pack_lists, pack_padded
    trajs = [np.arange(6, dtype=np.float64).reshape(3, 2), np.zeros((0, 2)), np.ones((2, 2))]
    pts, off, lens = pack_lists(trajs)
    assert pts.dtype == np.float32 and pts.shape == (5, 2)
    assert off.tolist() == [0, 3, 3] and lens.tolist() == [3, 0, 2]
    arr = np.zeros((2, 4, 2))
    p2, o2, l2 = pack_padded(arr, [4, 1])
    assert p2.shape == (8, 2) and o2.tolist() == [0, 4] and l2.tolist() == [4, 1]
    with pytest.raises(ValueError):
        pack_padded(arr, [5, 1])


def test_pair_order_groups_shapes():
    from trajsimimeasures_b200.engine import pair_order
    rng = np.random.default_rng(0)
    la, lb = rng.integers(1, 300, 1000), rng.integers(1, 300, 1000)
    o = pair_order(la, lb, rows=8)
    assert sorted(o.tolist()) == list(range(1000))
    nr = np.maximum(la, lb)[o]
    blocks = (nr + 7) // 8
    assert np.all(np.diff(blocks) <= 0)  # largest first
    nc = np.minimum(la, lb)[o]
    same = np.diff(blocks) == 0
    assert np.all(np.diff(nc)[same] <= 0)


def test_generators_are_seeded_and_shaped():
    from trajsimimeasures_b200 import datagen as G
    a = G.trajectory_set(50)
    b = G.trajectory_set(50)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    pts, off, lens = a
    assert pts.dtype == np.float32 and lens.min() >= 20 and lens.max() <= 200
    assert pts[:, 0].min() > -8.9 and pts[:, 0].max() < -8.3
    _, _, ll, _, _ = G.pairs_lognormal(5000)
    assert ll.min() >= 10 and ll.max() <= 2000 and 40 <= np.median(ll) <= 80


def test_reference_signature_validation():
    from trajsimimeasures_b200 import core
    t = np.zeros((2, 5, 2))
    with pytest.raises(AssertionError):
        core.dtw(t, [5, 5], np.zeros((2, 6, 2)), [5, 5])  # dtw.py:60 asserts equal shapes
    with pytest.raises(ValueError):
        core.dtw(t, [5, 5], t, [5, 5], threads_per_traj=0)
    with pytest.raises(AssertionError):
        core.edr(t, [5, 5], np.zeros((3, 5, 2)), [5, 5, 5], 0.1)


def test_heuristic_dispatch_names():
    from trajsimimeasures_b200 import method_helper as mh
    assert mh.is_heuristic("dtw") and mh.is_heuristic("hausdorff_cpu") and not mh.is_heuristic("T3S")
    fn = mh.heuristic_fn_wrapper("edr")
    assert fn.keywords["eps"] == mh.Config.trajsimi_edr_lcss_eps
    assert fn.keywords["threads_per_traj"] == mh.Config.effi_gpu_threads_per_traj
    with pytest.raises(NotImplementedError):
        mh.heuristic_fn_wrapper("dtw_cpu")
    with pytest.raises(AssertionError):
        mh.heuristic_fn_wrapper("nope")


def test_collate_pads_jointly():
    from trajsimimeasures_b200 import method_helper as mh
    batch = [([[0, 0], [1, 1], [2, 2]], [[5, 5]]), ([[1, 0]], [[3, 3], [4, 4]])]
    t1, l1, t2, l2 = mh.heuristic_colllate_fn(batch, True)
    assert t1.shape == t2.shape == (2, 3, 2) and t1.dtype == np.float64
    assert l1 == [3, 1] and l2 == [1, 2]
    u1, ul1, u2, ul2 = mh.heuristic_colllate_fn(batch, False)
    assert ul1 == [3, 1] and len(u1) == 2


def test_sched_plan_covers_every_item_once():
    from trajsimimeasures_b200 import datagen as D, sched
    _, _, lens, ia, ib = D.pairs_lognormal(20_000, seed=2)
    la, lb = lens[ia], lens[ib]
    for rows, wf in [(8, 4096), (4, 2048), (8, 8192)]:
        pl = sched.plan_pairs(la, lb, ["dtw", "dfrechet", "edr", "hausdorff"], rows=rows, warp_floats=wf)
        t = pl.tasks
        assert t.dtype == np.int32 and t.shape[1] == 4
        # long tasks first, largest first; then one measure after the other, each largest first
        long = pl.cost > pl.cost.sum() / sched.WARPS / 4
        n_long = int(long.sum())
        assert np.all(long[:n_long]) and not np.any(long[n_long:])
        assert np.all(np.diff(pl.cost[:n_long]) <= 0)
        rest_m = t[n_long:, 1]
        assert np.sum(np.diff(rest_m) != 0) == len(set(rest_m.tolist())) - 1  # contiguous measure blocks
        for m in set(rest_m.tolist()):
            assert np.all(np.diff(pl.cost[n_long:][rest_m == m]) <= 0)
        nc = np.minimum(la, lb)
        seen = {m: np.zeros(len(la), np.int64) for m in (0, 4, 1, 5)}
        for kind, m, first, cnt in t:
            idx = pl.order[first:first + cnt]
            seen[m][idx] += 1
            cap = {0: wf // 32, 5: wf // 8, 1: wf // 4, 6: wf // 2, 2: wf, 3: 1 << 30, 4: 1 << 30}[kind]
            assert cnt <= {0: 32, 5: 8, 1: 4, 6: 2, 2: 1, 3: 32, 4: 1}[kind]
            assert nc[idx].max() <= cap
            assert (kind in (3, 4)) == (m == 5)
        for m, v in seen.items():
            assert np.all(v == 1), m
        # a pair keeps its lanes for at most max_steps steps unless even a whole warp cannot do that
        nr = np.maximum(la, lb)
        for kind, m, first, cnt in t:
            idx = pl.order[first:first + cnt]
            if kind == 0:
                assert np.all(2 * sched.tile_steps(nr[idx], nc[idx], rows) <= sched.MAX_STEPS)
            elif kind in (5, 1, 6):
                G = {5: 4, 1: 8, 6: 16}[kind]
                assert np.all(sched.group_steps(nr[idx], nc[idx], rows, G) <= sched.MAX_STEPS)


def test_sched_plan_rejects_pairs_beyond_capacity():
    from trajsimimeasures_b200 import sched
    with pytest.raises(ValueError):
        sched.plan_pairs([5000], [5000], ["dtw"], warp_floats=4096)
    pl = sched.plan_pairs([5000], [5000], ["hausdorff"], warp_floats=4096)  # no shared memory needed
    assert pl.n_tasks == 1


def test_autotune_signature_and_cache(tmp_path, monkeypatch):
    from trajsimimeasures_b200 import sched
    monkeypatch.setenv("TSM_CACHE_DIR", str(tmp_path))
    a = sched.signature([10, 20, 300], [40, 50, 60], ["dtw", "edr"])
    b = sched.signature([10, 20, 300], [40, 50, 60], ["edr", "dtw"])
    assert a == b
    sched.save_cache({"k": {"best": [8, 4096, 8192]}})
    assert sched.load_cache()["k"]["best"] == [8, 4096, 8192]
