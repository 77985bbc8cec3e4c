"""GPU parity tests: the CUDA library (through its C ABI) against the oracle.

  * exact mode (IEEE sqrt/reciprocal): every measure bit-identical to the
    FP32 same-arithmetic twin;
  * default mode: DTW/ERP/Frechet/Hausdorff within REL_TOL (1e-5) of the FP64
    restatement of the reference, EDR/LCSS counts bit-identical to the twin
    (the threshold test runs in the same FP32 arithmetic) in every mode;
  * the golden fixtures (outputs of the reference's own kernels) through the
    reference-signature API;
  * size-independent properties at the full 2000 x 2000 all-pairs size.
"""
import numpy as np
import pytest
import torch

from conftest import REL_TOL, golden_cases, rel_err

pytestmark = pytest.mark.gpu

MEAS = [0, 1, 2, 3, 4, 5]
NAMES = {0: "dtw", 1: "edr", 2: "lcss", 3: "erp", 4: "dfrechet", 5: "hausdorff"}
EPS = 3e-4
G = (-8.625, 41.15)


def _dev(x, dt):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).cuda()


def run_pairs(m, pts, off, lens, ia, ib, exact=False, rows=0, order=True, eps=EPS, gpoint=G):
    from trajsimimeasures_b200.engine import pairs_raw, pair_order
    ia, ib = np.asarray(ia), np.asarray(ib)
    la, lb = lens[ia], lens[ib]
    n = len(ia)
    out = torch.full((n,), -7.0, device="cuda")
    cnt = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    o = _dev(pair_order(la, lb), np.int32) if order else None
    pairs_raw(m, _dev(pts, np.float32), _dev(off[ia], np.int64), _dev(la, np.int32), _dev(off[ib], np.int64),
              _dev(lb, np.int32), int(max(la.max(initial=0), lb.max(initial=0))), out=out, counts=cnt, order=o,
              eps=eps, gpoint=gpoint, exact=exact, rows=rows)
    torch.cuda.synchronize()
    return out.cpu().numpy(), cnt.cpu().numpy()


@pytest.fixture(scope="module")
def cfg_pairs():
    from trajsimimeasures_b200 import datagen as D
    return D.pairs_uniform(1000)


@pytest.fixture(scope="module")
def near():
    from trajsimimeasures_b200 import datagen as D
    return D.near_pairs(300)


@pytest.mark.parametrize("m", MEAS)
@pytest.mark.parametrize("rows", [4, 8, 16])
def test_exact_mode_bit_identical_to_twin(oracle_mod, cfg_pairs, m, rows):
    O = oracle_mod
    pts, off, lens, ia, ib = cfg_pairs
    got, cnt = run_pairs(m, pts, off, lens, ia, ib, exact=True, rows=rows)
    want, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
    np.testing.assert_array_equal(got, want)
    if m in (1, 2):
        np.testing.assert_array_equal(cnt, wcnt)


@pytest.mark.parametrize("m", MEAS)
def test_exact_mode_large_batch_bit_identical_to_twin(oracle_mod, cfg_pairs, m):
    """A batch too large for the small-batch path (more than 64 pairs per SM):
    one thread per pair (tile and Hausdorff pairs kernels) for the short
    pairs; bit-identical to the twin as the warp-per-pair path is."""
    O = oracle_mod
    pts, off, lens, ia, ib = cfg_pairs
    sm = torch.cuda.get_device_properties(0).multi_processor_count
    reps = 64 * sm // len(ia) + 2
    ja, jb = np.tile(ia, reps), np.tile(ib, reps)
    got, cnt = run_pairs(m, pts, off, lens, ja, jb, exact=True, rows=8)
    want, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
    np.testing.assert_array_equal(got, np.tile(want, reps))
    if m in (1, 2):
        np.testing.assert_array_equal(cnt, np.tile(wcnt, reps))


@pytest.mark.parametrize("m", MEAS)
def test_default_mode_within_tolerance_of_fp64(oracle_mod, cfg_pairs, m):
    O = oracle_mod
    pts, off, lens, ia, ib = cfg_pairs
    got, cnt = run_pairs(m, pts, off, lens, ia, ib)
    d64, c64 = O.pairs_idx(O.pairs_f64, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
    if m in (1, 2):
        _, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        np.testing.assert_array_equal(cnt, wcnt)
        np.testing.assert_array_equal(cnt, c64)
    else:
        assert rel_err(got, d64).max() <= REL_TOL


@pytest.mark.parametrize("m", [1, 2, 0, 5])
def test_near_pairs_threshold_counts(oracle_mod, near, m):
    O = oracle_mod
    pts, off, lens, ia, ib = near
    for exact in (False, True):
        got, cnt = run_pairs(m, pts, off, lens, ia, ib, exact=exact)
        want, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        if m in (1, 2):
            np.testing.assert_array_equal(cnt, wcnt)
            assert np.mean(wcnt > 0) > 0.5  # the threshold actually fires
        elif exact:
            np.testing.assert_array_equal(got, want)


def test_edge_lengths_follow_reference_rules(oracle_mod):
    """Lengths 0, 1, 2 and 31..33 (tile boundaries), in one batch."""
    O = oracle_mod
    from trajsimimeasures_b200 import datagen as D
    ls = [0, 1, 2, 3, 7, 8, 9, 15, 16, 17, 31, 32, 33, 64, 65, 200]
    la = np.repeat(ls, len(ls))
    lb = np.tile(ls, len(ls))
    pts, off, lens = D._walks(np.random.default_rng(5), np.concatenate([la, lb]), D.STEP_SIGMA)
    n = len(la)
    ia, ib = np.arange(n), np.arange(n) + n
    for m in MEAS:
        got, cnt = run_pairs(m, pts, off, lens, ia, ib, exact=True)
        want, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        np.testing.assert_array_equal(got, want, err_msg=NAMES[m])
        if m in (1, 2):
            np.testing.assert_array_equal(cnt, wcnt)


def test_overlong_pairs_are_flagged_not_computed():
    from trajsimimeasures_b200.engine import pairs_raw
    pts = torch.zeros((10, 2), device="cuda")
    off = torch.zeros(2, dtype=torch.int64, device="cuda")
    la = torch.tensor([5, 9], dtype=torch.int32, device="cuda")
    lb = torch.tensor([5, 5], dtype=torch.int32, device="cuda")
    out = torch.zeros(2, device="cuda")
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    pairs_raw(1, pts, off, la, off, lb, 6, out=out, counts=cnt, eps=0.1)
    torch.cuda.synchronize()
    assert out[0].item() == 0.0 and cnt[0].item() == 0
    assert np.isnan(out[1].item()) and cnt[1].item() == -1


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: p.rsplit("/", 1)[-1][:-4])
def test_golden_through_reference_signature(path):
    """The reference's own outputs, reproduced through core.<measure>(t1, len1, t2, len2, ...)."""
    from trajsimimeasures_b200 import core, datagen as D
    z = np.load(path)
    pts, off, lens, ia, ib = z["pts"], z["off"], z["lens"], z["ia"], z["ib"]
    ta = D.unpack(pts, off, lens, ia)
    tb = D.unpack(pts, off, lens, ib)
    w = int(lens.max())
    t1, t2 = D.pad(ta, w), D.pad(tb, w)
    l1, l2 = lens[ia], lens[ib]
    eps, g = float(z["eps"]), list(z["gpoint"])
    got = {
        "dtw": core.dtw(t1, l1, t2, l2), "edr": core.edr(t1, l1, t2, l2, eps),
        "lcss": core.lcss(t1, l1, t2, l2, eps), "erp": core.erp(t1, l1, t2, l2, g),
        "dfrechet": core.dfrechet(t1, l1, t2, l2), "hausdorff": core.hausdorff(t1, l1, t2, l2),
    }
    for k, v in got.items():
        assert v.dtype == np.float64 and v.shape == (len(ia),)
        if k in ("edr", "lcss"):
            np.testing.assert_array_equal(v, z[k], err_msg=k)
        else:
            assert rel_err(v, z[k]).max() <= REL_TOL, k


def test_list_inputs_and_device_tensors_agree():
    from trajsimimeasures_b200 import core, datagen as D
    pts, off, lens, ia, ib = D.pairs_uniform(64, seed=11)
    ta, tb = D.unpack(pts, off, lens, ia), D.unpack(pts, off, lens, ib)
    w = int(lens.max())
    t1, t2 = D.pad(ta, w), D.pad(tb, w)
    a = core.dtw(t1, lens[ia], t2, lens[ib])
    b = core.pairs(0, ta, None, tb, None)
    c = core.dtw(torch.from_numpy(t1).cuda(), lens[ia], torch.from_numpy(t2).cuda(), lens[ib])
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c.cpu().numpy())
    # host padded arrays go through one pinned staging buffer, reused and grown
    # by later calls: calls in a row of other sizes and measures still agree
    for n, m in ((300, 1), (2000, 0), (40, 1)):
        pts, off, lens, ia, ib = D.pairs_uniform(n, seed=12 + n)
        ta, tb = D.unpack(pts, off, lens, ia), D.unpack(pts, off, lens, ib)
        w = int(lens.max())
        t1, t2 = D.pad(ta, w), D.pad(tb, w)
        kw = dict(eps=D.EPS_DEG) if m == 1 else {}
        a, ca = core.pairs(m, t1, lens[ia], t2, lens[ib], counts=True, **kw)
        b, cb = core.pairs(m, ta, None, tb, None, counts=True, **kw)
        np.testing.assert_array_equal(a, b)
        if m == 1:
            np.testing.assert_array_equal(ca, cb)


@pytest.mark.parametrize("m", MEAS)
def test_matrix_equals_pairs_and_oracle(oracle_mod, m):
    O = oracle_mod
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet, matrix
    qp, qo, ql = D.trajectory_set(37, seed=D.SEED_QUERY)
    dp, do, dl = D.trajectory_set(301)
    qs, ds = TrajSet.from_packed(qp, qo, ql), TrajSet.from_packed(dp, do, dl)
    for exact in (True, False):
        out, cnt = matrix(m, qs, ds, eps=EPS, gpoint=G, exact=exact)
        out = out.cpu().numpy()
        if exact:
            want, wcnt = O.matrix_idx(O.pairs_f32, m, qp, qo, ql, dp, do, dl, eps=EPS, gpoint=G)
            np.testing.assert_array_equal(out, want)
        else:
            d64, c64 = O.matrix_idx(O.pairs_f64, m, qp, qo, ql, dp, do, dl, eps=EPS, gpoint=G)
            if m in (1, 2):
                np.testing.assert_array_equal(cnt.cpu().numpy(), c64)
            else:
                assert rel_err(out, d64).max() <= REL_TOL


@pytest.fixture(scope="module")
def full_set():
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet
    p, o, l = D.trajectory_set(2000)
    return (p, o, l), TrajSet.from_packed(p, o, l)


@pytest.mark.parametrize("m", MEAS)
def test_full_size_all_pairs_properties(oracle_mod, full_set, m):
    """2000 x 2000 (the all-pairs benchmark size): exact symmetry, zero
    self-distance, and 16 sampled rows against the oracle."""
    O = oracle_mod
    (p, o, l), s = full_set
    from trajsimimeasures_b200.engine import matrix
    out, cnt = matrix(m, s, s, eps=EPS, gpoint=G)
    M = out.cpu().numpy()
    assert np.array_equal(M, M.T)
    np.testing.assert_array_equal(np.diag(M), np.zeros(2000, np.float32))
    rows = np.random.default_rng(m).choice(2000, 16, replace=False)
    d64, c64 = O.matrix_idx(O.pairs_f64, m, p, o[rows], l[rows], p, o, l, eps=EPS, gpoint=G)
    if m in (1, 2):
        np.testing.assert_array_equal(cnt.cpu().numpy()[rows], c64)
    else:
        assert rel_err(M[rows], d64).max() <= REL_TOL


@pytest.mark.parametrize("rows", [4, 8, 16])
def test_long_pairs_wave_kernel_exact(oracle_mod, rows):
    """Pairs whose shorter side exceeds the tile kernel's boundary row
    (256 points), and pairs longer than 256 points whose one-lane tile loop
    would exceed 2048 steps (e.g. 2000 x 256 and 600 x 200 at every
    rows_per_thread, 2000 x 33 at 4 and 8), run one warp per pair; so do the
    Hausdorff pairs of more than 2^17 point products.  Mixed in one batch with
    short pairs, in the given order and the shape order."""
    O = oracle_mod
    from trajsimimeasures_b200 import datagen as D
    la = np.array([257, 300, 513, 1000, 2000, 2000, 40, 700, 256, 999, 1, 2000,
                   2000, 600, 513, 1999, 1500, 2000, 33, 2000])
    lb = np.array([300, 257, 600, 1000, 2000, 31, 2000, 1500, 257, 1001, 2000, 1999,
                   256, 200, 100, 2, 64, 33, 2000, 3])
    pts, off, lens = D._walks(np.random.default_rng(rows), np.concatenate([la, lb]), D.STEP_SIGMA)
    n = len(la)
    ia, ib = np.arange(n), np.arange(n) + n
    for m in (0, 1, 2, 3, 4, 5):
        want, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        for order in (True, False):
            got, cnt = run_pairs(m, pts, off, lens, ia, ib, exact=True, rows=rows, order=order)
            np.testing.assert_array_equal(got, want, err_msg=NAMES[m])
            if m in (1, 2):
                np.testing.assert_array_equal(cnt, wcnt)


def _long_batch(seed, n=600):
    from trajsimimeasures_b200 import datagen as D
    rng = np.random.default_rng(seed)
    la = rng.integers(1, 1200, n)
    lb = rng.integers(1, 300, n)
    pts, off, lens = D._walks(rng, np.concatenate([la, lb]), D.STEP_SIGMA)
    return pts, off, lens, np.arange(n), np.arange(n) + n


def _pairs_dev(pts, off, lens, ia, ib):
    from trajsimimeasures_b200.engine import pair_order
    la, lb = lens[ia], lens[ib]
    return (_dev(pts, np.float32), _dev(off[ia], np.int64), _dev(la, np.int32), _dev(off[ib], np.int64),
            _dev(lb, np.int32)), int(max(la.max(), lb.max())), _dev(pair_order(la, lb), np.int32)


def test_long_pairs_stream_order(oracle_mod):
    """The long-pair kernel runs on a forked side stream: work enqueued on the
    caller's stream right after tsm_pairs (no host sync) sees every result."""
    from trajsimimeasures_b200.engine import pairs_raw
    pts, off, lens, ia, ib = _long_batch(11)
    T, mx, o = _pairs_dev(pts, off, lens, ia, ib)
    st = torch.cuda.Stream()
    for m in (0, 5):  # DTW; Hausdorff (its own long-pair kernel)
        want, _ = oracle_mod.pairs_idx(oracle_mod.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        with torch.cuda.stream(st):
            for rep in range(3):
                out = torch.full((len(ia),), -7.0, device="cuda")
                pairs_raw(m, *T, mx, out=out, order=o, exact=True, stream=st)
                snap = out.clone()  # on st, ordered after tsm_pairs
                snap_host = snap.cpu()
                np.testing.assert_array_equal(snap_host.numpy(), want)
    torch.cuda.synchronize()


@pytest.mark.parametrize("fresh_thread", [False, True])
def test_long_pairs_graph_capture(oracle_mod, fresh_thread):
    """tsm_pairs with long pairs inside a CUDA graph capture: on a thread that
    already has its side stream (fork / join captured into the graph), and on
    a new thread whose first call is the captured one (everything on the
    captured stream)."""
    import threading
    from trajsimimeasures_b200.engine import pairs_raw
    pts, off, lens, ia, ib = _long_batch(12)
    T, mx, o = _pairs_dev(pts, off, lens, ia, ib)
    want, wcnt = oracle_mod.pairs_idx(oracle_mod.pairs_f32, 1, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
    res = {}

    def body():
        out = torch.full((len(ia),), -7.0, device="cuda")
        cnt = torch.full((len(ia),), -7, dtype=torch.int32, device="cuda")
        if not fresh_thread:  # creates this thread's side stream outside the capture
            pairs_raw(1, *T, mx, out=out, counts=cnt, order=o, eps=EPS, exact=True)
            torch.cuda.synchronize()
        s = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                pairs_raw(1, *T, mx, out=out, counts=cnt, order=o, eps=EPS, exact=True, stream=s)
        for _ in range(2):
            out.fill_(-7.0)
            cnt.fill_(-7)
            g.replay()
            torch.cuda.synchronize()
            res.setdefault("out", []).append(out.cpu().numpy().copy())
            res.setdefault("cnt", []).append(cnt.cpu().numpy().copy())
        del g

    if fresh_thread:
        err = []

        def run():
            try:
                body()
            except BaseException as e:  # surfaced in the test thread
                err.append(e)
        t = threading.Thread(target=run)
        t.start()
        t.join()
        if err:
            raise err[0]
    else:
        body()
    for got, cnt in zip(res["out"], res["cnt"]):
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(cnt, wcnt)


def test_lognormal_batch(oracle_mod):
    """20k pairs of the uneven (lognormal, clipped to [10, 2000]) workload."""
    O = oracle_mod
    from trajsimimeasures_b200 import datagen as D
    pts, off, lens, ia, ib = D.pairs_lognormal(20_000, seed=4)
    assert np.minimum(lens[ia], lens[ib]).max() > 256  # the wave kernel runs too
    for m in MEAS:
        got, cnt = run_pairs(m, pts, off, lens, ia, ib, exact=True)
        want, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        np.testing.assert_array_equal(got, want, err_msg=NAMES[m])
        got, cnt = run_pairs(m, pts, off, lens, ia, ib)
        d64, c64 = O.pairs_idx(O.pairs_f64, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        if m in (1, 2):
            np.testing.assert_array_equal(cnt, wcnt)
        else:
            assert rel_err(got, d64).max() <= REL_TOL, NAMES[m]


def test_matrix_many_equals_per_measure_matrix():
    """The e2e API (host arrays in, float64 out, results formed on the GPU and
    copied on a side stream) gives exactly the per-measure results."""
    from trajsimimeasures_b200 import core, datagen as D
    t = D.unpack(*D.trajectory_set(90, seed=21))
    P = D.pad(t)
    L = np.array([len(x) for x in t])
    many = core.matrix_many(["dtw", "edr", "lcss", "erp", "dfrechet", "hausdorff"], P, L, P, L, eps=EPS, gpoint=G)
    for name, m in many.items():
        one = core.matrix(name, P, L, P, L, eps=EPS, gpoint=G)
        assert m.dtype == np.float64
        np.testing.assert_array_equal(m, one, err_msg=name)


@pytest.mark.parametrize("m", MEAS)
def test_allpairs_sym_equals_full_matrix(m):
    """The symmetric driver (upper triangle in length order, mirrored) gives
    the full Q == D matrix bit for bit, counts included, in both modes, on a
    ragged set (lengths 1..400, near-duplicates for EDR/LCSS matches) that
    spans several 128-trajectory chunks."""
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet, allpairs_sym_raw, matrix
    rng = np.random.default_rng(40 + m)
    lens = np.concatenate([[1, 2, 3, 1, 400], rng.integers(1, 260, 296)])
    lens[11:41:2] = lens[10:40:2]
    pts, off, _ = D._walks(rng, lens, D.STEP_SIGMA)
    for k in range(10, 40, 2):  # near-duplicates: copy k into k+1 with ~1e-4 deg noise
        a, b, n_k = off[k], off[k + 1], lens[k]
        pts[b:b + n_k] = pts[a:a + n_k] + rng.normal(0, 1e-4, (n_k, 2)).astype(np.float32)
    s = TrajSet.from_packed(pts, off, lens)
    n = s.n
    for exact in (True, False):
        full, fcnt = matrix(m, s, s, eps=EPS, gpoint=G, exact=exact)
        out = torch.full((n, n), -7.0, device="cuda")
        cnt = torch.full((n, n), -7, dtype=torch.int32, device="cuda") if m in (1, 2) else None
        allpairs_sym_raw(m, s, out=out, counts=cnt, eps=EPS, gpoint=G, exact=exact)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), full.cpu().numpy())
        if cnt is not None:
            np.testing.assert_array_equal(cnt.cpu().numpy(), fcnt.cpu().numpy())


def test_allpairs_sym_reference_signature_full_size(full_set):
    """core.allpairs on host padded arrays at 2000 trajectories equals
    core.matrix(S, S) (float64 results, EDR/LCSS normalised)."""
    from trajsimimeasures_b200 import core, datagen as D
    (p, o, l), _ = full_set
    P = D.pad(D.unpack(p, o, l))
    for name in ("dtw", "edr", "hausdorff"):
        a = core.allpairs(name, P, l, eps=EPS, gpoint=G)
        b = core.matrix(name, P, l, P, l, eps=EPS, gpoint=G)
        assert a.dtype == np.float64 and a.shape == (2000, 2000)
        np.testing.assert_array_equal(a, b, err_msg=name)


@pytest.mark.parametrize("m", [0, 1, 3])
def test_long_lengths_through_matrix_allpairs_and_pairs(oracle_mod, m):
    """Lengths 801..1,600 (the reference's timing sweep, test_trajsimi_time.py:109)
    with some short ones: core.matrix (the rows of queries longer than the
    matrix forms' 1,400-point limit computed by tsm_pairs), core.allpairs and
    core.pairs, exact mode, bit-identical to the FP32 twin (float32 inputs)."""
    from trajsimimeasures_b200 import core, datagen as D
    O = oracle_mod
    rng = np.random.default_rng(70 + m)
    lens = np.concatenate([rng.integers(801, 1601, 14), rng.integers(20, 201, 6), [1400, 1401]])
    pts, off, lens = D._walks(rng, lens, D.STEP_SIGMA)
    t = D.unpack(pts, off, lens)
    P = D.pad(t, dtype=np.float32)
    kw = dict(eps=EPS, gpoint=G, exact=True)
    got, cnt = core.matrix(m, P, lens, P, lens, counts=True, **kw)
    want, wcnt = O.matrix_idx(O.pairs_f32, m, pts, off, lens, pts, off, lens, eps=EPS, gpoint=G)
    if m in (1, 2):
        np.testing.assert_array_equal(cnt, wcnt)
    else:
        np.testing.assert_array_equal(got.astype(np.float32), want)
    sym = core.allpairs(m, P, lens, **kw)
    np.testing.assert_array_equal(sym, got)
    ia, ib = np.arange(0, 21), np.arange(1, 22)
    pr = core.pairs(m, P[ia], lens[ia], P[ib], lens[ib], **kw)
    np.testing.assert_array_equal(pr, got[ia, ib])


def test_pairs_beyond_8192_points(oracle_mod):
    """Pairs longer than 8,192 points (the wave kernel with fewer warps per
    CTA) up to 12,000: exact mode bit-identical to the twin; above
    tsm_max_supported_len (32,768) the call is refused with TSM_ETOOLONG."""
    from trajsimimeasures_b200 import _lib, datagen as D
    O = oracle_mod
    rng = np.random.default_rng(81)
    lens = np.array([12000, 9000, 8193, 300, 10000, 16])
    pts, off, lens = D._walks(rng, lens, D.STEP_SIGMA)
    ia, ib = np.array([0, 1, 2, 4]), np.array([1, 3, 4, 5])
    for m in (0, 1):
        got, cnt = run_pairs(m, pts, off, lens, ia, ib, exact=True)
        want, wcnt = O.pairs_idx(O.pairs_f32, m, pts, off, lens, ia, ib, eps=EPS, gpoint=G)
        np.testing.assert_array_equal(got, want)
        if m == 1:
            np.testing.assert_array_equal(cnt, wcnt)
    with pytest.raises(_lib.TsmError, match="TSM_ETOOLONG|-3"):
        run_pairs(0, np.zeros((33000, 2), np.float32), np.array([0]), np.array([33000]), np.array([0]), np.array([0]))


@pytest.mark.parametrize("m", MEAS)
def test_matrix_rows_and_length_buckets(m):
    """tsm_matrix_rows writes exactly the selected rows, with tsm_matrix's
    values; matrix_raw's length-bucketed launches (one per query-length
    group) give the one-launch matrix bit for bit, counts included."""
    import ctypes
    from trajsimimeasures_b200 import _lib, datagen as D
    from trajsimimeasures_b200.engine import TrajSet, _ptr, matrix_raw
    rng = np.random.default_rng(90 + m)
    pts, off, lens = D._walks(rng, rng.integers(1, 260, 400), D.STEP_SIGMA)
    s = TrajSet.from_packed(pts, off, lens)
    n = s.n
    ref = torch.empty((n, n), device="cuda")
    rc = torch.empty((n, n), dtype=torch.int32, device="cuda") if m in (1, 2) else None
    matrix_raw(m, s, s, out=ref, counts=rc, eps=EPS, gpoint=G, buckets=1)
    got = torch.full((n, n), -7.0, device="cuda")
    gc = torch.full((n, n), -7, dtype=torch.int32, device="cuda") if m in (1, 2) else None
    matrix_raw(m, s, s, out=got, counts=gc, eps=EPS, gpoint=G, buckets=4)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)
    if rc is not None:
        assert torch.equal(gc, rc)
    rows = torch.as_tensor(np.sort(rng.choice(n, 37, replace=False)).astype(np.int32)).cuda()
    sel = torch.full((n, n), -7.0, device="cuda")
    lib = _lib.load()
    p = _lib.params(EPS, G, False, 0)
    assert lib.tsm_matrix_rows(m, _ptr(s.pts), _ptr(s.off), _ptr(s.lens), _ptr(rows), 37,
                               int(s.lens[rows.long()].max()), _ptr(s.pts), _ptr(s.off), _ptr(s.lens),
                               _ptr(s.order_by_length()), n, s.max_len, ctypes.byref(p), _ptr(sel), n, None,
                               None) == 0
    torch.cuda.synchronize()
    mask = torch.zeros(n, dtype=torch.bool, device="cuda")
    mask[rows.long()] = True
    assert torch.equal(sel[mask], ref[mask])
    assert bool((sel[~mask] == -7.0).all())
