"""CPU tests of trajsimimeasures_b200.data_loader against the reference's own
dataset classes: tests/golden/loader/pairs.npz holds an in-memory HDF5-layout
file and the items that utilities/data_loader.py (DatasetST_h5,
DatasetSynthetic) produced from it (tests/golden/make_loader_golden.py)."""
import os
import random

import numpy as np
import pytest

from conftest import GOLDEN_DIR

FIX = os.path.join(GOLDEN_DIR, "loader", "pairs.npz")


class _File(dict):
    """The mapping interface of an open h5py.File: datasets by path, attrs."""

    def __init__(self, items, attrs):
        super().__init__(items)
        self.attrs = attrs


def _file(z):
    lens, pts, ts = z["file_lens"], z["file_pts"], z["file_ts"]
    off = np.concatenate([[0], np.cumsum(lens)[:-1]])
    items = {"/trajs_len": lens.copy()}
    for i, (o, n) in enumerate(zip(off, lens)):
        items["/trajs_merc/%d" % i] = pts[o:o + n]
        items["/trajs_ts/%d" % i] = ts[o:o + n]
    return _File(items, {"merc_range": np.array([-9.7e5, -9.5e5, 5.0e6, 5.1e6]), "ts_range": np.array([0.0, 1e6])})


def _unpack(pts, lens):
    off = np.concatenate([[0], np.cumsum(lens)[:-1]])
    return [pts[o:o + n] for o, n in zip(off, lens)]


def _cases(z, prefix):
    return sorted({k.split("_")[0] for k in z.files if k.startswith(prefix)})


@pytest.fixture(scope="module")
def z():
    return np.load(FIX)


def test_st_h5_pairs_match_the_reference(z):
    from trajsimimeasures_b200.data_loader import DatasetST_h5
    cases = _cases(z, "st")
    assert len(cases) == 2
    for c in cases:
        temporal, num, lo, hi, seed = (int(v) for v in z[c + "_args"])
        ds = DatasetST_h5(_file(z), bool(temporal), num, lo, hi, seed)
        assert len(ds) == num
        ref = _unpack(z[c + "_pts"], z[c + "_lens"])
        got = [np.asarray(t, dtype=np.float64) for i in range(len(ds)) for t in ds[i]]
        assert len(got) == len(ref) == 2 * num
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(g.reshape(r.shape), r)
        np.testing.assert_array_equal(np.asarray(ds.merc_range), z[c + "_merc_range"])
        # every drawn trajectory is at least traj_len_min long, and one longer than
        # traj_len_max was read up to a length in [traj_len_min, traj_len_max]
        assert all(lo <= len(t) <= hi for i in range(len(ds)) for t in ds[i])


def test_synthetic_pairs_match_the_reference(z):
    from trajsimimeasures_b200.data_loader import DatasetSynthetic
    for c in _cases(z, "syn"):
        temporal, num, lo, hi, seed, np_seed = (int(v) for v in z[c + "_args"])
        ds = DatasetSynthetic(bool(temporal), num, lo, hi, seed)
        np.random.seed(np_seed)
        got = [np.asarray(t, dtype=np.float64) for i in range(len(ds)) for t in ds[i]]
        ref = _unpack(z[c + "_pts"], z[c + "_lens"])
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(g.reshape(r.shape), r)
        assert random.random() == float(z[c + "_random_state"][0])  # Python's generator: seeded, then untouched


def test_st_h5_feeds_the_heuristic_collate(z):
    """The dataset's items through the reference's collate (padded float64
    arrays and lengths, method_helper.heuristic_colllate_fn)."""
    from trajsimimeasures_b200.data_loader import DatasetST_h5
    from trajsimimeasures_b200.method_helper import heuristic_colllate_fn
    ds = DatasetST_h5(_file(z), False, 16, 20, 120, 5)
    t1, l1, t2, l2 = heuristic_colllate_fn([ds[i] for i in range(len(ds))], True)
    t1, t2 = np.asarray(t1), np.asarray(t2)
    assert t1.shape[0] == t2.shape[0] == 16 and t1.shape[-1] == 2
    for k in range(16):
        np.testing.assert_array_equal(t1[k, :l1[k]], np.asarray(ds[k][0]))
        np.testing.assert_array_equal(t2[k, :l2[k]], np.asarray(ds[k][1]))


def test_st_h5_rejects_a_file_with_too_few_trajectories(z):
    from trajsimimeasures_b200.data_loader import DatasetST_h5
    f = _file(z)
    with pytest.raises(ValueError):
        DatasetST_h5(f, False, 10 ** 6, 20, 120, 0)


def test_st_h5_path_needs_h5py():
    from trajsimimeasures_b200.data_loader import DatasetST_h5
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError, match="h5py"):
            DatasetST_h5("missing.h5", False, 4, 20, 200, 0)
    else:
        pytest.skip("h5py is installed here")
