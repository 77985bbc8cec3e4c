"""The reference's trajectory-pair datasets (utilities/data_loader.py), the
inputs of its timing drivers (test_trajsimi_time.py:58, test_knn_time.py:139,
test_clustering_time.py:64, test_trajsimi_time_DQ.py:58).

``DatasetST_h5`` reads the reference's HDF5 layout -- ``/trajs_len`` (one
length per trajectory), ``/trajs_merc/<i>`` (the i-th trajectory, [n, 2]
Mercator metres), ``/trajs_ts/<i>`` (its timestamps, for spatio-temporal
pairs) and the file attributes ``merc_range`` / ``ts_range`` -- from a path
(opened with h5py, which the caller provides: this package does not depend
on it) or from any object with the same mapping interface (an open
``h5py.File``, or a dict of arrays with an ``attrs`` dict, as the tests use).

The pairs are drawn as the reference draws them, so the same file and seed
give the same pairs: Python's ``random`` seeded once; trajectories shorter
than ``traj_len_min`` dropped; each one longer than ``traj_len_max`` given a
length uniform in [traj_len_min, traj_len_max] (one ``random.randint`` per
such trajectory, in index order) and read up to it; then two
``random.choices`` draws of ``num_trajs`` each, the first and second members
of the pairs.  Items are (traj1, traj2) pairs of float64 point lists, the
input of ``method_helper.heuristic_colllate_fn``.

``DatasetSynthetic`` (data_loader.py:114-144) draws each item's two
trajectories from NumPy's global generator at access time: uniform lengths
in [traj_len_min, traj_len_max] and points uniform in [0, 1)^2.
"""
from __future__ import annotations

import random

import numpy as np


def _open(source):
    if isinstance(source, (str, bytes)) or hasattr(source, "__fspath__"):
        try:
            import h5py
        except ImportError as e:
            raise ImportError("DatasetST_h5 reads a file path through h5py, which is not installed here; "
                              "pass an open h5py-like object instead") from e
        return h5py.File(source, "r"), True
    return source, False


def _attr(f, name):
    attrs = getattr(f, "attrs", {})
    if name not in attrs:
        return None
    v = attrs[name]
    return np.asarray(v).tolist() if isinstance(v, np.ndarray) else v


class DatasetST_h5:
    """Pairs of spatial (use_temporal False: [x, y]) or spatio-temporal
    ([x, y, t]) trajectories sampled with replacement from an HDF5 dataset
    (data_loader.py:52-111).  A torch ``Dataset`` by interface
    (``__getitem__`` / ``__len__``)."""

    def __init__(self, file_path, use_temporal: bool, num_trajs, traj_len_min, traj_len_max, seed):
        random.seed(seed)
        self.use_temporal = use_temporal
        self.traj_len_min = traj_len_min
        self.traj_len_max = traj_len_max
        self.data_length = num_trajs
        f, owned = _open(file_path)
        try:
            self.merc_range = _attr(f, "merc_range")
            self.ts_range = _attr(f, "ts_range")
            lens = np.asarray(f["/trajs_len"][:]).astype(np.int64).tolist()
            kept = [(i, n) for i, n in enumerate(lens) if n >= traj_len_min]
            # the length to read: trajectories over the maximum get a random one (randint per such trajectory)
            kept = [(i, random.randint(traj_len_min, traj_len_max) if n > traj_len_max else n) for i, n in kept]
            if len(kept) ** 2 < num_trajs:
                raise ValueError(f"{len(kept)} trajectories of at least {traj_len_min} points cannot give "
                                 f"{num_trajs} pairs")
            firsts = random.choices(kept, k=num_trajs)
            seconds = random.choices(kept, k=num_trajs)
            self.pairs = list(zip(firsts, seconds))  # ((index, length), (index, length))
            self.trajs = [(self._read(f, a), self._read(f, b)) for a, b in self.pairs]
        finally:
            if owned:
                f.close()

    def _read(self, f, iv):
        i, n = iv
        pts = np.asarray(f["/trajs_merc/%s" % i][:n], dtype=np.float64)
        if not self.use_temporal:
            return pts.tolist()
        ts = np.asarray(f["/trajs_ts/%s" % i][:n]).tolist()
        return [[p[0], p[1], t] for p, t in zip(pts.tolist(), ts)]

    def __getitem__(self, index):
        return self.trajs[index]

    def __len__(self):
        return self.data_length


class DatasetSynthetic:
    """Pairs of random trajectories in the unit square (data_loader.py:114-144):
    ``random.seed(seed)`` at construction, NumPy's global generator per item
    (lengths, then points, of each trajectory in turn; cumulative timestamps
    with steps uniform in [1, 59] for spatio-temporal pairs)."""

    def __init__(self, use_temporal: bool, num_trajs, traj_len_min, traj_len_max, seed):
        random.seed(seed)
        self.use_temporal = use_temporal
        self.traj_len_min = traj_len_min
        self.traj_len_max = traj_len_max
        self.num_trajs = num_trajs
        self.merc_range = [0.0, 1.0, 0.0, 1.0]

    def __getitem__(self, index):
        n1 = np.random.randint(self.traj_len_min, self.traj_len_max + 1)
        a = np.random.uniform(size=(n1, 2)).astype(np.float64).tolist()
        n2 = np.random.randint(self.traj_len_min, self.traj_len_max + 1)
        b = np.random.uniform(size=(n2, 2)).astype(np.float64).tolist()
        if not self.use_temporal:
            return (a, b)
        t1 = np.cumsum(np.random.randint(1, 60, size=n1), axis=0).tolist()
        t2 = np.cumsum(np.random.randint(1, 60, size=n2), axis=0).tolist()
        return ([[p[0], p[1], t] for p, t in zip(a, t1)], [[p[0], p[1], t] for p, t in zip(b, t2)])

    def __len__(self):
        return self.num_trajs
