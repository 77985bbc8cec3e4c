"""GPU tests of the learned filter's hand-written kernels: forward values and
gradients against an FP64 CPU autograd reference (oracle/encoder_ref.py), and
a short training run that must learn DTW order (Spearman rho)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _set(trajs):
    from trajsimimeasures_b200.engine import TrajSet
    return TrajSet.from_lists(trajs)


def test_encoder_gradients_match_fp64_autograd():
    from oracle import encoder_ref as R
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.surrogate import Encoder
    rng = np.random.default_rng(3)
    pts, off, lens = D._walks(rng, np.array([3, 30, 17, 1, 24, 9]), D.STEP_SIGMA)
    trajs = D.unpack(pts, off, lens)
    s = _set(trajs)
    enc = Encoder.init(s, seed=5)
    # larger weights than the init so that the gates leave their linear range
    enc.params.mul_(3.0)
    # distinct weights per resampled point of the skip (stored as logarithms)
    enc.params[-16:] = torch.log(torch.linspace(0.1, 0.4, 16, device=enc.params.device))
    ia, ib, y = np.array([0, 1, 2, 4, 5]), np.array([1, 2, 4, 5, 3]), np.array([0.1, 0.5, 0.2, 0.9, 0.3])
    w = np.array([1.0, 4.0, 25.0, 1.2, 11.1], dtype=np.float32)  # relative-error weights 1 / y^2
    loss, grad, pred = enc.loss_grad(s, np.arange(6), ia, ib, y, w)
    torch.cuda.synchronize()
    l_ref, g_ref, p_ref = R.loss_grad(enc.params.cpu().numpy(), trajs, enc.nrm, ia, ib, y, w)
    np.testing.assert_allclose(pred.cpu().numpy(), p_ref, rtol=2e-5, atol=1e-6)
    assert abs(loss.item() - l_ref) <= 1e-4 * abs(l_ref) + 1e-7
    g = grad.cpu().numpy().astype(np.float64)
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= 1e-4 * scale, np.abs(g - g_ref).max() / scale
    # every parameter block gets a gradient
    o = 0
    for name, shape in R.SIZES:
        n = int(np.prod(shape))
        assert np.abs(g_ref[o:o + n]).max() > 0, name
        o += n


def test_weight_gradients_long_batch_match_fp64_autograd():
    """The GRU weight gradients are reductions over every valid step of the
    batch, formed on the tensor cores from BF16 hi/lo operand parts (about
    2^-16 relative per product, FP32 accumulation).  24 trajectories of 20 to
    160 points: about 2,000 valid steps in a padded 24 x 160 block, so the K
    range spans several CTAs and stage boundaries fall inside trajectories."""
    from oracle import encoder_ref as R
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.surrogate import Encoder
    rng = np.random.default_rng(8)
    L = rng.integers(20, 161, 24)
    pts, off, lens = D._walks(rng, L, D.STEP_SIGMA)
    trajs = D.unpack(pts, off, lens)
    s = _set(trajs)
    enc = Encoder.init(s, seed=9)
    enc.params.mul_(2.0)
    ia, ib = np.arange(12), np.arange(12, 24)
    y = rng.uniform(0.05, 0.5, 12)
    loss, grad, _ = enc.loss_grad(s, np.arange(24), ia, ib, y)
    enc.check_training()
    _, g_ref, _ = R.loss_grad(enc.params.cpu().numpy(), trajs, enc.nrm, ia, ib, y)
    g = grad.cpu().numpy().astype(np.float64)
    o, blocks = 0, {}
    for name, shape in R.SIZES:
        n = int(np.prod(shape))
        blocks[name] = (o, o + n)
        o += n
    for name in ("w_ih", "w_hh"):  # the tensor-core reductions, each against its own largest gradient
        a, b = blocks[name]
        scale = np.abs(g_ref[a:b]).max()
        assert scale > 0
        assert np.abs(g[a:b] - g_ref[a:b]).max() <= 1e-4 * scale, (name, np.abs(g[a:b] - g_ref[a:b]).max() / scale)
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= 1e-4 * scale


def test_encoder_forward_long_batch():
    from oracle import encoder_ref as R
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.surrogate import Encoder
    rng = np.random.default_rng(4)
    L = rng.integers(20, 201, 40)
    pts, off, lens = D._walks(rng, L, D.STEP_SIGMA)
    trajs = D.unpack(pts, off, lens)
    s = _set(trajs)
    enc = Encoder.init(s, seed=6)
    e = enc.embed(s, batch=24, tensor_cores=False).cpu().numpy()  # two batches (16 trajectories per GRU CTA)
    W = R.unpack(enc.params.cpu().numpy())
    e_ref = R.embed(W, trajs[:6], enc.nrm).detach().numpy()
    np.testing.assert_allclose(e[:6], e_ref, rtol=1e-4, atol=1e-5)


def test_tensor_core_embedding_matches_bf16_operand_reference():
    """The tcgen05 inference kernel (tsm_enc_embed): against the FP64
    reference with a_t and h_t rounded to BF16 before the gate products, and
    against the FP32-activation training forward, over three 128-trajectory
    CTAs of lengths 1..230 (the last one partly filled)."""
    from oracle import encoder_ref as R
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.surrogate import Encoder
    rng = np.random.default_rng(11)
    L = np.concatenate([[1, 2, 230], rng.integers(1, 231, 297)])
    pts, off, lens = D._walks(rng, L, D.STEP_SIGMA)
    trajs = D.unpack(pts, off, lens)
    s = _set(trajs)
    enc = Encoder.init(s, seed=12)
    enc.params.mul_(2.0)  # gates away from their linear range
    e_tc = enc.embed(s, batch=300).cpu().numpy()
    e_fp = enc.embed(s, batch=300, tensor_cores=False).cpu().numpy()
    assert np.isfinite(e_tc).all()
    pick = [0, 1, 2, 3, 150, 299]
    W = R.unpack(enc.params.cpu().numpy())
    e_ref = R.embed(W, [trajs[i] for i in pick], enc.nrm, bf16_operands=True).detach().numpy()
    scale = np.abs(e_ref).max()
    err = np.abs(e_tc[pick] - e_ref).max() / scale
    assert err <= 2e-3, err
    # BF16 activations against FP32 ones: the same network to BF16 rounding
    assert np.abs(e_tc - e_fp).max() <= 3e-2 * np.abs(e_fp).max()


def test_training_learns_dtw_order():
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet
    from trajsimimeasures_b200.surrogate import Encoder, dtw_labels, spearman
    p, o, l = D.trajectory_set(4000, seed=8)
    s = TrajSet.from_packed(p, o, l)
    rng = np.random.default_rng(9)
    pa, pb = rng.integers(0, 4000, 30000), rng.integers(0, 4000, 30000)
    lab = dtw_labels(s, pa, pb)
    y = lab / lab.max()
    enc = Encoder.init(s, seed=1)
    hold = slice(27000, None)
    before = spearman(enc.predict_pairs(s, pa[hold], pb[hold]), y[hold])
    hist = enc.fit(s, pa[:27000], pb[:27000], y[:27000], epochs=6, batch_pairs=1024, lr=3e-3)
    after = spearman(enc.predict_pairs(s, pa[hold], pb[hold]), y[hold])
    assert hist[-1] < 0.5 * hist[0], hist
    assert after > 0.8 and after > before, (before, after)


def test_trained_filter_gains_over_untrained_and_exhaustive_and_falls_back():
    """What the learned part buys.  Over the same network untrained (same
    architecture, same initial weights, same candidate count): a higher
    recall@10 of the candidate sets.  Over the method without it
    (exhaustive exact DP): the trained encoder's candidates plus exact rerank
    reach recall@10 >= 0.99 while evaluating at most 2 % of the database per
    query (counted in DP evaluations, not timed).  A filter that cannot reach
    the target inside its budget hands the queries to the exhaustive search
    (exact results)."""
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet
    from trajsimimeasures_b200.knn import SurrogateIndex, knn_exhaustive, recall_at_k
    from trajsimimeasures_b200.surrogate import Encoder, dtw_labels, neighbour_pairs
    N = 20000
    p, o, l = D.trajectory_set(N, seed=12)
    Dset = TrajSet.from_packed(p, o, l)
    Q = TrajSet.from_packed(*D.trajectory_set(64, seed=13))
    _, exact = knn_exhaustive(Q, Dset, 10)
    rng = np.random.default_rng(14)
    pa, pb = rng.integers(0, N, 40000), rng.integers(0, N, 40000)
    na, nb = neighbour_pairs(Dset, 2000, k=10, seed=15)
    pa, pb = np.concatenate([pa, na]), np.concatenate([pb, nb])
    lab = dtw_labels(Dset, pa, pb)
    untrained = SurrogateIndex(Encoder.init(Dset, seed=2), Dset)
    enc = Encoder.init(Dset, seed=2)
    enc.fit(Dset, pa, pb, lab / lab.max(), epochs=6, batch_pairs=1024, lr=3e-3, relative=True)
    idx = SurrogateIndex(enc, Dset)
    # below saturation (a count where the untrained filter still misses
    # answers): trained strictly better at 20 candidates and on average
    rec = {c: (recall_at_k(idx.query(Q, 10, c=c)[1], exact), recall_at_k(untrained.query(Q, 10, c=c)[1], exact))
           for c in (10, 20, 40)}
    assert rec[20][0] > rec[20][1], rec
    assert sum(t - u for t, u in rec.values()) > 0.02, rec
    idx.LADDER = (40, 80, 160, 320, 400)
    cal = TrajSet.from_packed(*D.trajectory_set(64, seed=15))
    c, rec = idx.calibrate(cal, 10, target=0.99, max_fraction=0.02)
    assert c is not None and c <= 0.02 * N, rec
    _, got = idx.query(Q, 10)
    assert recall_at_k(got, exact) >= 0.99
    # budget too small to reach the target: no count is chosen, exhaustive answers
    idx.LADDER = (20,)
    c, rec = idx.calibrate(Q, 10, target=1.0, max_fraction=0.001)
    assert c is None, rec
    _, ans = idx.query(Q, 10)
    np.testing.assert_array_equal(ans.cpu().numpy(), exact.cpu().numpy())


def test_embed_wait_timeout_is_reported_and_context_survives():
    """The tensor-core GRU's waits are bounded.  The test hook announces one
    step's a_t copy on its mbarrier but never issues it, so every CTA's wait
    for it runs out (with a short limit) while no MMA is in flight.  The
    status word reports it (bit 1), tsm_enc_embed_status returns
    TSM_ETIMEOUT, Encoder.embed raises instead of returning NaN rows, and
    the context stays usable: a normal call afterwards gives the same
    embeddings as before."""
    import ctypes
    from trajsimimeasures_b200 import _lib, datagen as D
    from trajsimimeasures_b200.surrogate import Encoder
    rng = np.random.default_rng(8)
    pts, off, lens = D._walks(rng, rng.integers(20, 60, 300), D.STEP_SIGMA)
    s = _set(D.unpack(pts, off, lens))
    enc = Encoder.init(s, seed=9)
    before = enc.embed(s)
    torch.cuda.synchronize()
    assert torch.isfinite(before).all()
    lib = _lib.load()
    st = ctypes.c_int32(-1)
    assert lib.tsm_enc_embed_status(ctypes.c_void_p(enc._ews.data_ptr()), ctypes.byref(st), None) == 0
    assert st.value == 0
    enc._wait_override = (2_000_000, 3)  # ~1 ms of SM clocks; step 3's copy never issued
    with pytest.raises(_lib.TsmError, match="wait ran out"):
        enc.embed(s)
    rc = lib.tsm_enc_embed_status(ctypes.c_void_p(enc._ews.data_ptr()), ctypes.byref(st), None)
    assert rc == -4 and st.value & 1 and not st.value & 4, (rc, st.value)
    enc._wait_override = None
    after = enc.embed(s)
    torch.cuda.synchronize()
    assert torch.equal(before, after)
    assert lib.tsm_enc_embed_status(ctypes.c_void_p(enc._ews.data_ptr()), ctypes.byref(st), None) == 0
