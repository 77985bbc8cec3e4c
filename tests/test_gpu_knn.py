"""GPU tests of the kNN selection (tsm_topk_rows) and the kNN drivers."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _stable_topk(a, k):
    o = np.argsort(a, axis=1, kind="stable")[:, :k]
    return np.take_along_axis(a, o, axis=1), o


@pytest.mark.parametrize("k", [1, 10, 64, 256])
def test_topk_rows_matches_stable_argsort(k):
    from trajsimimeasures_b200.knn import topk_rows
    rng = np.random.default_rng(k)
    a = rng.random((37, 5000)).astype(np.float32)
    a[:, ::7] = np.round(a[:, ::7], 2)  # many ties
    a[0, :] = 0.5                     # a row of equal values
    a[1, 100:200] = np.inf
    a[2, 5] = np.nan
    a[3, :50] = -1.0 - a[3, :50]        # negative values
    v, i = topk_rows(torch.from_numpy(a).cuda(), k)
    wv, wi = _stable_topk(a, k)
    np.testing.assert_array_equal(i.cpu().numpy(), wi)
    np.testing.assert_array_equal(v.cpu().numpy(), wv)


def test_topk_rows_short_rows_are_padded():
    from trajsimimeasures_b200.knn import topk_rows
    a = torch.tensor([[3.0, 1.0, 2.0]], device="cuda")
    v, i = topk_rows(a, 5)
    assert i.cpu().tolist() == [[1, 2, 0, -1, -1]]
    assert v.cpu().numpy()[0, 3] == np.inf


def test_knn_exhaustive_and_rerank(oracle_mod):
    O = oracle_mod
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet
    from trajsimimeasures_b200.knn import knn_exhaustive, knn_rerank, recall_at_k
    qp, qo, ql = D.trajectory_set(12, seed=D.SEED_QUERY)
    dp, do, dl = D.trajectory_set(3000)
    Q, Dset = TrajSet.from_packed(qp, qo, ql), TrajSet.from_packed(dp, do, dl)
    want, _ = O.matrix_idx(O.pairs_f32, 0, qp, qo, ql, dp, do, dl)
    wv, wi = _stable_topk(want, 10)
    v, i = knn_exhaustive(Q, Dset, k=10, chunk=700, exact=True)  # several chunks, merged
    np.testing.assert_array_equal(i.cpu().numpy(), wi)
    np.testing.assert_array_equal(v.cpu().numpy(), wv)
    # rerank from a candidate superset that contains the answer
    rng = np.random.default_rng(0)
    cand = np.stack([np.concatenate([wi[q], rng.choice(3000, 190, replace=False)]) for q in range(12)])
    cand = np.array([np.unique(c)[:200] if len(np.unique(c)) >= 200 else np.unique(c) for c in cand], dtype=object)
    width = min(len(c) for c in cand)
    cand = np.stack([np.concatenate([wi[q], np.setdiff1d(c, wi[q])])[:width] for q, c in enumerate(cand)])
    rv, ri = knn_rerank(Q, Dset, torch.from_numpy(cand).cuda(), k=10, exact=True)
    np.testing.assert_array_equal(ri.cpu().numpy(), wi)
    np.testing.assert_array_equal(rv.cpu().numpy(), wv)
    assert recall_at_k(ri, i) == 1.0


@pytest.mark.parametrize("k", [1, 300, 5000])
def test_select_rows_is_the_stable_argsort_set(k):
    from trajsimimeasures_b200.knn import select_rows
    rng = np.random.default_rng(k)
    a = rng.random((9, 20000)).astype(np.float32)
    a[:, ::3] = np.round(a[:, ::3], 3)  # ties at the cut
    a[0, :] = 1.0
    i = select_rows(torch.from_numpy(a).cuda(), k).cpu().numpy()
    want = np.argsort(a, axis=1, kind="stable")[:, :k]
    for r in range(a.shape[0]):
        assert set(i[r].tolist()) == set(want[r].tolist())
    short = select_rows(torch.from_numpy(a[:, :50].copy()).cuda(), 60).cpu().numpy()
    assert (short[:, 50:] == -1).all() and all(set(row[:50]) == set(range(50)) for row in short)


@pytest.mark.parametrize("k", [1, 64, 5000, 20000])
def test_select_rows_sampled_threshold_and_fallbacks(k):
    """Long rows (the sampled-threshold path, its radix fallback for large k),
    a row whose k-th value repeats more often than the tie buffer holds, a row
    of one value, negative values, +-inf and NaN: always the stable argsort's
    first-k set."""
    from trajsimimeasures_b200.knn import select_rows
    rng = np.random.default_rng(100 + k)
    n = 300_000
    a = rng.standard_normal((6, n)).astype(np.float32)
    a[1] = np.abs(a[1])
    a[2, rng.choice(n, 5000, replace=False)] = np.nan
    a[2, :3] = -np.inf
    a[2, 3:6] = np.inf
    srt = np.sort(a[3])
    a[3, rng.choice(n, 3000, replace=False)] = srt[min(k, n - 1)]  # > 1024 ties at the cut
    a[4] = 0.5
    a[5] = np.round(a[5], 2)  # heavy ties everywhere
    i = select_rows(torch.from_numpy(a).cuda(), k).cpu().numpy()
    want = np.argsort(a, axis=1, kind="stable")[:, :k]
    for r in range(a.shape[0]):
        assert set(i[r].tolist()) == set(want[r].tolist()), r
    # rows that fit the shared-memory buffer whole
    b = np.round(rng.random((3, 10_000)), 3).astype(np.float32)
    j = select_rows(torch.from_numpy(b).cuda(), min(k, 10_000)).cpu().numpy()
    wb = np.argsort(b, axis=1, kind="stable")[:, :min(k, 10_000)]
    for r in range(b.shape[0]):
        assert set(j[r].tolist()) == set(wb[r].tolist()), r


@pytest.mark.parametrize("measure", ["dtw", "edr", "lcss", "erp", "dfrechet", "hausdorff"])
def test_matrix_gather_equals_matrix_entries(measure):
    """tsm_matrix_gather (per-query candidate rows) is bit-identical to the
    full matrix at the gathered entries, counts included; indices outside the
    database give NaN and count -1."""
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet, matrix, matrix_gather_raw, measure_id
    dev = torch.device("cuda", 0)
    Q = TrajSet.from_packed(*D.trajectory_set(37, seed=5), device=dev)
    Dset = TrajSet.from_packed(*D.trajectory_set(500, 1, 230, seed=6), device=dev)
    kw = dict(eps=D.EPS_DEG, gpoint=D.BOX_CENTRE, exact=True)
    full, fcnt = matrix(measure, Q, Dset, with_counts=True, **kw)
    rng = np.random.default_rng(7)
    cand = rng.integers(0, 500, (37, 301)).astype(np.int32)
    cand[3, 5] = -1
    cand[4, 7] = 500
    c = torch.from_numpy(cand).to(dev)
    out = torch.full((37, 320), -5.0, device=dev)
    cnt = torch.full((37, 320), -5, dtype=torch.int32, device=dev)
    matrix_gather_raw(measure, Q, Dset, c, out=out, counts=cnt, **kw)
    o, k = out.cpu().numpy(), cnt.cpu().numpy()
    f, fc = full.cpu().numpy(), fcnt.cpu().numpy()
    ok = (cand >= 0) & (cand < 500)
    qi = np.broadcast_to(np.arange(37)[:, None], cand.shape)
    np.testing.assert_array_equal(o[:, :301][ok], f[qi[ok], cand[ok]])
    assert np.isnan(o[3, 5]) and np.isnan(o[4, 7])
    assert (o[:, 301:] == -5.0).all()  # nothing past ncand is written
    if measure_id(measure) in (1, 2):
        np.testing.assert_array_equal(k[:, :301][ok], fc[qi[ok], cand[ok]])
        assert k[3, 5] == -1 and k[4, 7] == -1
    # a processing order of the queries (longest first) changes nothing in the result
    qo = torch.argsort(Q.lens, descending=True, stable=True).to(torch.int32)
    out2 = torch.full((37, 320), -5.0, device=dev)
    cnt2 = torch.full((37, 320), -5, dtype=torch.int32, device=dev)
    matrix_gather_raw(measure, Q, Dset, c, out=out2, counts=cnt2, q_order=qo, **kw)
    np.testing.assert_array_equal(out2.cpu().numpy(), o)
    np.testing.assert_array_equal(cnt2.cpu().numpy(), k)


def _scan_case(n=20000, nq=300, seed=21):
    """Embeddings like the filter's: 160 values, centred; queries are noisy
    copies of database rows, so the nearest distances are tiny next to |e|^2."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    E = (torch.randn(n, 160, generator=g) * 0.3).cuda()
    E -= E.double().mean(0).float()
    rows = torch.randint(0, n, (nq,), generator=g).cuda()
    Qe = E[rows] + (torch.randn(nq, 160, generator=g) * 1e-3).cuda()
    return E, Qe


def _scan_images(E, Qe, scale):
    from trajsimimeasures_b200 import _lib
    from trajsimimeasures_b200.engine import _ptr
    lib = _lib.load()

    def img(X, db):
        b = torch.empty(lib.tsm_scan_image_bytes(X.shape[0], int(db)), dtype=torch.uint8, device="cuda")
        nrm = torch.empty(X.shape[0], device="cuda") if db else None
        assert lib.tsm_scan_prepare(_ptr(X), X.shape[0], X.stride(0), scale, int(db), _ptr(b), _ptr(nrm), None) == 0
        return b, nrm
    (dimg, norms), (qimg, _) = img(E, True), img(Qe, False)
    return lib, dimg, norms, qimg


def test_scan_dense_matches_fp64_and_lists_match_dense():
    """tsm_scan (tcgen05, FP16 hi/lo split products, FP32 accumulation):
    dense d = |e_j|^2 - 2 e_q.e_j within 1e-5 of |e_q||e_j| of the FP64 value
    (a TF32 product is off by ~1e-3 of it) and the same top-50 up to near
    ties; in list mode exactly the pairs whose dense value is <= the
    threshold, with the dense values, over 3 query tiles (the last one
    partial) and a partial last database tile."""
    from trajsimimeasures_b200.engine import _ptr
    E, Qe = _scan_case()
    n, nq = E.shape[0], Qe.shape[0]
    scale = float(2.0 ** np.floor(np.log2(1024.0 / float(torch.cat([E, Qe]).abs().max()))))
    lib, dimg, norms, qimg = _scan_images(E, Qe, scale)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    dense = torch.full((nq, n + 3), -7.0, device="cuda")
    assert lib.tsm_scan(_ptr(qimg), nq, _ptr(dimg), n, scale, None, 0, None, None, None, _ptr(dense), n + 3,
                        _ptr(st), None) == 0
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    d = dense[:, :n].double()
    assert bool((dense[:, n:] == -7.0).all())  # nothing written past nd
    # a row stride that is a multiple of 4 floats takes the 16-byte stores: the same values
    dense4 = torch.full((nq, n + 4), -7.0, device="cuda")
    assert lib.tsm_scan(_ptr(qimg), nq, _ptr(dimg), n, scale, None, 0, None, None, None, _ptr(dense4), n + 4,
                        _ptr(st), None) == 0
    torch.cuda.synchronize()
    assert torch.equal(dense4[:, :n], dense[:, :n]) and bool((dense4[:, n:] == -7.0).all())
    E64, Q64 = E.double(), Qe.double()
    assert ((norms.double() - (E64 * E64).sum(1)).abs() <= 1e-5 * (E64 * E64).sum(1)).all()
    ref = (E64 * E64).sum(1)[None, :] - 2.0 * Q64 @ E64.T
    bound = Q64.norm(dim=1)[:, None] * E64.norm(dim=1)[None, :]
    err = ((d - ref).abs() / bound).max().item()
    assert err <= 1e-5, err
    top_k = torch.topk(d, 50, dim=1, largest=False).indices.cpu().numpy()
    top_r = torch.topk(ref, 50, dim=1, largest=False).indices.cpu().numpy()
    overlap = np.mean([len(np.intersect1d(a, b)) / 50 for a, b in zip(top_k, top_r)])
    assert overlap >= 0.98, overlap
    # list mode: threshold at each query's 100th smallest dense value
    thr = torch.kthvalue(dense[:, :n], 100, dim=1).values.contiguous()
    cap = 160
    idx = torch.full((nq, cap), -1, dtype=torch.int32, device="cuda")
    dd = torch.full((nq, cap), float("inf"), device="cuda")
    cnt = torch.zeros(nq, dtype=torch.int32, device="cuda")
    assert lib.tsm_scan(_ptr(qimg), nq, _ptr(dimg), n, scale, _ptr(thr), cap, _ptr(idx), _ptr(dd), _ptr(cnt), None,
                        0, _ptr(st), None) == 0
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    want = (dense[:, :n] <= thr[:, None])
    np.testing.assert_array_equal(cnt.cpu().numpy(), want.sum(1).cpu().numpy())
    dn = dense.cpu().numpy()
    for q in range(nq):
        c = int(cnt[q])
        got = np.sort(idx[q, :c].cpu().numpy())
        np.testing.assert_array_equal(got, np.nonzero(want[q].cpu().numpy())[0])
        np.testing.assert_array_equal(np.sort(dd[q, :c].cpu().numpy()), np.sort(dn[q, got]))


def test_scan_candidates_match_fp64_ranking():
    """SurrogateIndex-style candidates (sampled threshold, lists, exact
    selection) equal the FP64 top-c up to near ties, for several counts; a
    count that makes the list the whole database falls back to a dense scan."""
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet
    from trajsimimeasures_b200.knn import SurrogateIndex
    from trajsimimeasures_b200.surrogate import Encoder
    p, o, l = D.trajectory_set(30000, seed=31)
    Dset = TrajSet.from_packed(p, o, l)
    Q = TrajSet.from_packed(*D.trajectory_set(200, seed=32))
    idx = SurrogateIndex(Encoder.init(Dset, seed=3), Dset)
    eq = idx.enc.embed(Q)
    X = (idx.E * idx.wt).double()
    Y = ((eq - idx.mu) * idx.wt).double()
    ref = (X * X).sum(1)[None, :] - 2.0 * Y @ X.T
    for c in (50, 300, 5000):
        got = idx.candidates(Q, c).cpu().numpy()
        want = torch.topk(ref, c, dim=1, largest=False).indices.cpu().numpy()
        overlap = np.mean([len(np.intersect1d(a, b)) / c for a, b in zip(got, want)])
        assert overlap >= 0.995, (c, overlap)
        assert all(len(np.unique(r)) == c for r in got)
