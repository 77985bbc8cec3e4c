"""Generates tests/golden/loader/pairs.npz from the reference's own dataset
classes (utilities/data_loader.py: DatasetST_h5, DatasetSynthetic).

Run with a checkout of the reference at the path in the TSM_REFERENCE_ROOT
environment variable -- it is not needed afterwards:

    TSM_REFERENCE_ROOT=<reference checkout> python tests/golden/make_loader_golden.py

h5py is not installed here, so the reference module is imported with a
stand-in ``h5py`` module whose ``File`` returns an in-memory file: a dict of
NumPy arrays (``/trajs_len``, ``/trajs_merc/<i>``, ``/trajs_ts/<i>``) with an
``attrs`` dict (``merc_range``, ``ts_range``), seeded, with lengths on both
sides of the sampling bounds.  The fixture holds that file's contents, the
sampling arguments of each case and the reference's items (packed points and
lengths), so the test rebuilds the same file and compares item for item.
"""
from __future__ import annotations

import os
import random
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("TSM_REFERENCE_ROOT", "/root/reference")
OUT = os.path.join(HERE, "loader", "pairs.npz")

N_FILE = 60
ST_CASES = [  # (use_temporal, num_trajs, traj_len_min, traj_len_max, seed)
    (False, 40, 20, 120, 2000),  # trajectories over 120 points get a random length
    (True, 25, 30, 90, 7),
]
SYN_CASES = [(False, 10, 20, 120, 2000, 11), (True, 8, 5, 40, 3, 12)]  # + np.random seed before the items


class FakeFile(dict):
    def __init__(self, items, attrs):
        super().__init__(items)
        self.attrs = attrs

    def close(self):
        pass


def fake_contents(seed=3):
    rng = np.random.default_rng(seed)
    lens = rng.integers(5, 200, N_FILE)
    pts = rng.normal(0.0, 1000.0, (int(lens.sum()), 2)) + np.array([-9.6e5, 5.03e6])
    ts = np.concatenate([np.cumsum(rng.integers(1, 30, n)) for n in lens]).astype(np.int64)
    return lens.astype(np.int64), pts, ts


def fake_file(lens, pts, ts):
    off = np.concatenate([[0], np.cumsum(lens)[:-1]])
    items = {"/trajs_len": lens.copy()}
    for i, (o, n) in enumerate(zip(off, lens)):
        items["/trajs_merc/%d" % i] = pts[o:o + n]
        items["/trajs_ts/%d" % i] = ts[o:o + n]
    attrs = {"merc_range": np.array([-9.7e5, -9.5e5, 5.0e6, 5.1e6]), "ts_range": np.array([0.0, 1e6])}
    return FakeFile(items, attrs)


def pack(pairs):
    """[(traj1, traj2), ...] -> (points float64 [P, d], lengths int64 [2 * n])."""
    trajs = [t for ab in pairs for t in ab]
    lens = np.array([len(t) for t in trajs], dtype=np.int64)
    d = len(trajs[0][0]) if trajs and trajs[0] else 2
    pts = np.concatenate([np.asarray(t, dtype=np.float64).reshape(-1, d) for t in trajs])
    return pts, lens


def main():
    lens, pts, ts = fake_contents()
    stub = types.ModuleType("h5py")
    stub.File = lambda path, mode="r": fake_file(lens, pts, ts)
    sys.modules["h5py"] = stub
    sys.path.insert(0, REF)
    from utilities import data_loader as ref  # noqa: E402  the reference's module

    out = {"file_lens": lens, "file_pts": pts, "file_ts": ts}
    for k, (temporal, num, lo, hi, seed) in enumerate(ST_CASES):
        ds = ref.DatasetST_h5("unused.h5", temporal, num, lo, hi, seed)
        p, l = pack([ds[i] for i in range(len(ds))])
        out[f"st{k}_args"] = np.array([int(temporal), num, lo, hi, seed])
        out[f"st{k}_pts"], out[f"st{k}_lens"] = p, l
        out[f"st{k}_merc_range"] = np.asarray(ds.merc_range, dtype=np.float64)
    for k, (temporal, num, lo, hi, seed, np_seed) in enumerate(SYN_CASES):
        ds = ref.DatasetSynthetic(temporal, num, lo, hi, seed)
        np.random.seed(np_seed)
        p, l = pack([ds[i] for i in range(len(ds))])
        out[f"syn{k}_args"] = np.array([int(temporal), num, lo, hi, seed, np_seed])
        out[f"syn{k}_pts"], out[f"syn{k}_lens"] = p, l
        out[f"syn{k}_random_state"] = np.array([random.random()])  # Python's generator after construction + items
    np.savez_compressed(OUT, **out)
    print(OUT, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
