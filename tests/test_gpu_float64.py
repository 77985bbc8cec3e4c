"""float64 inputs that float32 cannot hold, as the reference's drivers read
them: Porto near pairs in Mercator metres (x ~ -9.7e5, y ~ 5.0e6 m; eps 200 m,
gap point (0, 0): utilities/data_loader.py:78-79, config.py:52,
utilities/method_helper.py:25) and in lon/lat degrees.

Every entry point translates such inputs by an FP64 origin before rounding
them to float32 (core.pair_origins, core.set_origin).  These tests check the
GPU results against the FP64 restatement run on the ORIGINAL float64 inputs:
DTW/ERP/Frechet/Hausdorff within REL_TOL, EDR/LCSS counts equal; and, in
exact mode, bit-identity with the FP32 twin fed the same translated inputs.
"""
import numpy as np
import pytest
import torch

from conftest import REL_TOL, centred_pairs, rel_err

pytestmark = pytest.mark.gpu

MEAS = [0, 1, 2, 3, 4, 5]
NAMES = {0: "dtw", 1: "edr", 2: "lcss", 3: "erp", 4: "dfrechet", 5: "hausdorff"}


def _case(units, n=2000):
    from trajsimimeasures_b200 import datagen as D
    p, o, l, ia, ib = D.near_pairs_f64(n, units=units)
    eps, g = (D.MERC_EPS_M, (0.0, 0.0)) if units == "merc" else (D.EPS_DEG, D.BOX_CENTRE)
    return p, o, l, ia, ib, eps, g


@pytest.fixture(scope="module", params=["merc", "deg"])
def f64case(request):
    return _case(request.param)


@pytest.mark.parametrize("m", MEAS)
def test_pairs_float64_within_tolerance_of_fp64(oracle_mod, f64case, m):
    """core.pairs on padded float64 host arrays (the reference's input)."""
    from trajsimimeasures_b200 import core, datagen as D
    O = oracle_mod
    p, o, l, ia, ib, eps, g = f64case
    t1, t2 = D.pad(D.unpack(p, o, l, ia)), D.pad(D.unpack(p, o, l, ib))
    got, cnt = core.pairs(m, t1, l[ia], t2, l[ib], eps=eps, gpoint=g, counts=True)
    d64, c64 = O.pairs_idx(O.pairs_f64, m, p, o, l, ia, ib, eps=eps, gpoint=g)
    if m in (1, 2):
        np.testing.assert_array_equal(cnt, c64)
        np.testing.assert_array_equal(got, d64)
    else:
        assert rel_err(got, d64).max() <= REL_TOL, NAMES[m]


@pytest.mark.parametrize("m", MEAS)
def test_pairs_float64_exact_mode_bit_identical_to_twin(oracle_mod, f64case, m):
    """The kernels see exactly the translated inputs of centred_pairs."""
    from trajsimimeasures_b200 import core, datagen as D
    O = oracle_mod
    p, o, l, ia, ib, eps, g = f64case
    t1, t2 = D.pad(D.unpack(p, o, l, ia)), D.pad(D.unpack(p, o, l, ib))
    got, cnt = core.pairs(m, t1, l[ia], t2, l[ib], eps=eps, gpoint=g, exact=True, counts=True)
    p32, oa, la, ob, lb, gg = centred_pairs(m, p, o, l, ia, ib, g)
    want, wcnt = O.pairs_f32(m, p32, oa, la, ob, lb, eps=eps, gpoint=gg)
    if m in (1, 2):
        np.testing.assert_array_equal(cnt, wcnt)
    else:
        np.testing.assert_array_equal(got.astype(np.float32), want)


def test_list_and_device_float64_inputs_agree_with_padded(f64case):
    """Lists of float64 trajectories and float64 CUDA tensors take the same
    origins as padded host arrays, so all three give the same results."""
    from trajsimimeasures_b200 import core, datagen as D
    p, o, l, ia, ib, eps, g = f64case
    ia, ib = ia[:300], ib[:300]
    ta, tb = D.unpack(p, o, l, ia), D.unpack(p, o, l, ib)
    t1, t2 = D.pad(ta), D.pad(tb)
    for m in MEAS:
        kw = dict(eps=eps, gpoint=g)
        a = core.pairs(m, t1, l[ia], t2, l[ib], **kw)
        b = core.pairs(m, ta, None, tb, None, **kw)
        c = core.pairs(m, torch.from_numpy(t1).cuda(), l[ia], torch.from_numpy(t2).cuda(), l[ib], **kw)
        np.testing.assert_array_equal(a, b, err_msg=NAMES[m])
        np.testing.assert_array_equal(a, c.cpu().numpy(), err_msg=NAMES[m])


@pytest.mark.parametrize("units", ["merc", "deg"])
def test_matrix_and_allpairs_float64_within_bound(oracle_mod, units):
    """core.matrix / core.allpairs / core.matrix_many on float64 host sets:
    one FP64 origin G for the call, shared by Q and D.  A coordinate then
    carries at most 2^-24 |x - G| of rounding, so a distance at most
    2^-22.5 Rmax (Rmax = the call's largest |x - G|): the results are within
    REL_TOL relative plus K 2^-22.5 Rmax absolute, K = 1 for the max-type
    measures (Frechet, Hausdorff) and n1 + n2 cells for the sums (DTW, ERP).
    Pairs closer than ~1e5 2^-22.5 Rmax can therefore exceed REL_TOL here;
    core.pairs (one origin per pair) does not have this term."""
    from trajsimimeasures_b200 import core, datagen as D
    O = oracle_mod
    p, o, l, ia, ib, eps, g = _case(units, 150)
    idx = np.concatenate([ia, ib])
    trajs = D.unpack(p, o, l, idx)
    S = D.pad(trajs)
    ls = l[idx]
    q = S[:40]
    G = np.asarray(core.set_origin((S, ls)))
    rmax = max(float(np.abs(t - G).max()) for t in trajs)
    K = {0: ls[:40, None] + ls[None, :], 3: ls[:40, None] + ls[None, :], 4: 1, 5: 1}
    many = core.matrix_many(["dtw", "edr", "lcss", "erp", "dfrechet", "hausdorff"], q, ls[:40], S, ls, eps=eps,
                            gpoint=g)
    for m in MEAS:
        got, cnt = core.matrix(m, q, ls[:40], S, ls, eps=eps, gpoint=g, counts=True)
        pq = np.concatenate(trajs[:40])
        oq = np.concatenate([[0], np.cumsum(ls[:40])[:-1]])
        ps = np.concatenate(trajs)
        os_ = np.concatenate([[0], np.cumsum(ls)[:-1]])
        d64, c64 = O.matrix_idx(O.pairs_f64, m, pq, oq, ls[:40], ps, os_, ls, eps=eps, gpoint=g)
        if m in (1, 2):
            np.testing.assert_array_equal(cnt, c64)
        else:
            bound = REL_TOL * np.abs(d64) + K[m] * 2.0 ** -22.5 * rmax
            assert np.all(np.abs(got - d64) <= bound), (NAMES[m], rel_err(got, d64).max())
        np.testing.assert_array_equal(many[NAMES[m]], got, err_msg=NAMES[m])
        sym = core.allpairs(m, S, ls, eps=eps, gpoint=g)
        full = core.matrix(m, S, ls, S, ls, eps=eps, gpoint=g)
        np.testing.assert_array_equal(sym, full, err_msg=NAMES[m])
        np.testing.assert_array_equal(full[:40], got, err_msg=NAMES[m])
