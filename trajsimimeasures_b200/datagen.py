"""Seeded synthetic trajectories standing in for the reference's datasets
(Porto, Geolife, ... are not available offline).

Random walks in a Porto-like box: start uniform in lon [-8.70, -8.55] x
lat [41.10, 41.20], i.i.d. N(0, sigma) steps per coordinate, cast to float32.
Seeds follow the reference's conventions: 2000 for databases and pairs
(config.py:8 `seed = 2000`), 2001 for queries (test_knn_time.py:181).

Workloads (sizes of the benchmark configurations):
  pairs_uniform   1,000 pairs, lengths U{20..200}, sigma 2e-4 deg
  set_uniform     2,000 trajectories (all-pairs 2000 x 2000), U{20..200}
  pairs_lognormal 500k pairs, lengths clip(round(lognormal(ln 60, 1.0)), 10, 2000),
                  per-trajectory sigma ~ U(5e-5, 5e-4) deg
  near_pairs      perturbed copies, so that EDR/LCSS threshold tests hit both sides
"""
from __future__ import annotations

import numpy as np

BOX = (-8.70, -8.55, 41.10, 41.20)  # lon_min, lon_max, lat_min, lat_max
BOX_CENTRE = (-8.625, 41.15)
EPS_DEG = 3e-4        # EDR/LCSS threshold for these inputs
STEP_SIGMA = 2e-4
SEED_DB = 2000
SEED_QUERY = 2001


def _walks(rng, lens, sigma, dtype=np.float32):
    """Packed random walks: pts [P, 2] (float32 unless dtype says otherwise),
    off int64 [N], lens int32 [N]."""
    lens = np.asarray(lens, dtype=np.int64)
    n = lens.shape[0]
    off = np.zeros(n, dtype=np.int64)
    if n > 1:
        np.cumsum(lens[:-1], out=off[1:])
    total = int(lens.sum())
    start = np.stack([rng.uniform(BOX[0], BOX[1], n), rng.uniform(BOX[2], BOX[3], n)], axis=1)
    sig = np.broadcast_to(np.asarray(sigma, dtype=np.float64), (n,))
    steps = rng.standard_normal((total, 2)) * np.repeat(sig, lens)[:, None]
    owner = np.repeat(np.arange(n), lens)
    first = np.zeros(total, dtype=bool)
    first[off[lens > 0]] = True
    steps[first] = 0.0
    # cumulative sum inside each trajectory: global cumsum minus the sum
    # before the trajectory's first point
    cs = np.cumsum(steps, axis=0)
    base = np.zeros((n, 2))
    nz = lens > 0
    base[nz] = cs[off[nz]] - steps[off[nz]]
    pts = start[owner] + cs - base[owner]
    return pts.astype(dtype), off, lens.astype(np.int32)


def uniform_lengths(rng, n, lo=20, hi=200):
    return rng.integers(lo, hi + 1, size=n)


def lognormal_lengths(rng, n, median=60.0, sigma=1.0, lo=10, hi=2000):
    return np.clip(np.round(rng.lognormal(np.log(median), sigma, size=n)), lo, hi).astype(np.int64)


def trajectory_set(n, lo=20, hi=200, seed=SEED_DB, sigma=STEP_SIGMA):
    """n random walks with lengths U{lo..hi}."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return _walks(rng, uniform_lengths(rng, n, lo, hi), sigma)


def pairs_uniform(n_pairs=1000, lo=20, hi=200, seed=SEED_DB, sigma=STEP_SIGMA):
    """Paired batch: 2*n_pairs walks; pair k = (k, n_pairs + k)."""
    pts, off, lens = trajectory_set(2 * n_pairs, lo, hi, seed, sigma)
    ia = np.arange(n_pairs, dtype=np.int64)
    return pts, off, lens, ia, ia + n_pairs


def pairs_lognormal(n_pairs=500_000, seed=SEED_DB, pool=None):
    """Uneven batch: lognormal lengths (median 60, sigma 1, clip [10, 2000]),
    per-trajectory step sigma U(5e-5, 5e-4).  With pool=None every pair has
    two fresh trajectories; else pairs are drawn from a pool of that size."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = 2 * n_pairs if pool is None else pool
    lens = lognormal_lengths(rng, n)
    sig = rng.uniform(5e-5, 5e-4, size=n)
    pts, off, lens = _walks(rng, lens, sig)
    if pool is None:
        ia = np.arange(n_pairs, dtype=np.int64)
        return pts, off, lens, ia, ia + n_pairs
    return pts, off, lens, rng.integers(0, n, n_pairs), rng.integers(0, n, n_pairs)


def near_pairs(n_pairs=200, lo=20, hi=200, seed=SEED_DB + 7, jitter=2e-4, sigma=STEP_SIGMA):
    """Pairs whose second trajectory is a jittered, resampled copy of the
    first, so a good share of the point pairs lie within EPS_DEG."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = uniform_lengths(rng, n_pairs, lo, hi)
    pts, off, lens = _walks(rng, lens, sigma)
    trajs = []
    for k in range(n_pairs):
        a = pts[off[k]:off[k] + lens[k]].astype(np.float64)
        keep = np.sort(rng.choice(lens[k], size=max(1, int(lens[k] * rng.uniform(0.6, 1.0))), replace=False))
        b = a[keep] + rng.normal(0.0, jitter, size=(keep.shape[0], 2))
        trajs.append(a.astype(np.float32))
        trajs.append(b.astype(np.float32))
    from .engine import pack_lists
    p, o, l = pack_lists(trajs)
    ia = np.arange(0, 2 * n_pairs, 2, dtype=np.int64)
    return p, o, l, ia, ia + 1


MERC_EPS_M = 200.0  # the reference's EDR/LCSS threshold on Mercator metres (config.py:52)


def lonlat_to_merc(lon, lat):
    """Spherical Web-Mercator metres of lon/lat degrees, the projection of the
    reference's trajs_merc datasets (utilities/tool_funcs.py:95-100): x = R
    lon, y = R/2 ln((1 + sin lat)/(1 - sin lat)), R = 6378137 m."""
    r = 6378137.0
    lon = np.asarray(lon, dtype=np.float64)
    t = np.sin(np.radians(np.asarray(lat, dtype=np.float64)))
    return r * np.radians(lon), 0.5 * r * np.log((1.0 + t) / (1.0 - t))


def near_pairs_f64(n_pairs=200, lo=20, hi=200, seed=SEED_DB + 8, units="merc"):
    """float64 near pairs as the reference's drivers read them: random walks
    in the Porto-like box, either in lon/lat degrees (step 2e-4 deg, jitter
    2e-4 deg, for eps = EPS_DEG) or projected to Mercator metres (step and
    jitter ~120 m, for eps = MERC_EPS_M = 200 m).  The second trajectory of a
    pair is a jittered, resampled copy of the first, so the EDR/LCSS threshold
    fires on both sides.  Coordinates are float64 values that float32 cannot
    hold.  -> (pts float64 [P, 2], off, lens, ia, ib)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = uniform_lengths(rng, n_pairs, lo, hi)
    sig, jit = (2e-4, 2e-4) if units == "deg" else (1e-3, 1e-3)
    pts, off, lens = _walks(rng, lens, sig, dtype=np.float64)
    trajs = []
    for k in range(n_pairs):
        a = pts[off[k]:off[k] + lens[k]]
        keep = np.sort(rng.choice(lens[k], size=max(1, int(lens[k] * rng.uniform(0.6, 1.0))), replace=False))
        b = a[keep] + rng.normal(0.0, jit, size=(keep.shape[0], 2))
        trajs += [a, b]
    if units == "merc":
        trajs = [np.stack(lonlat_to_merc(t[:, 0], t[:, 1]), axis=1) for t in trajs]
    elif units != "deg":
        raise ValueError(f"units must be 'deg' or 'merc', got {units!r}")
    lens = np.array([len(t) for t in trajs], dtype=np.int32)
    off = np.zeros(len(trajs), dtype=np.int64)
    np.cumsum(lens[:-1], out=off[1:])
    ia = np.arange(0, 2 * n_pairs, 2, dtype=np.int64)
    return np.concatenate(trajs).astype(np.float64), off, lens, ia, ia + 1


def unpack(pts, off, lens, idx=None):
    """Packed -> list of [n, 2] arrays (views, in the dtype of pts)."""
    idx = range(len(off)) if idx is None else idx
    return [pts[off[k]:off[k] + lens[k]] for k in idx]


def pad(trajs, width=None, dtype=np.float64):
    """List of [n, 2] -> zero-padded [N, width, 2] (the reference's
    pad_lists_to_array layout, utilities/tool_funcs.py:230-234)."""
    w = max((len(t) for t in trajs), default=0) if width is None else width
    arr = np.zeros((len(trajs), w, 2), dtype=dtype)
    for k, t in enumerate(trajs):
        arr[k, :len(t)] = t
    return arr
