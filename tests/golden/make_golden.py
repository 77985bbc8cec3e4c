"""Generates tests/golden/*.npz from the reference's own code.

Run with a checkout of the reference at the path in the TSM_REFERENCE_ROOT
environment variable -- it is not needed afterwards:

    NUMBA_ENABLE_CUDASIM=1 TSM_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py [--force]

For each case it runs
  * the reference GPU kernels of core/*.py (dtw, edr, lcss, erp, dfrechet
    through their public wrappers; Hausdorff through core.hausdorff's own
    kernel hausdorff_opt with a zero-initialised p2t buffer, because the
    wrapper allocates that buffer uninitialised and its host max then reads
    padded slots, core/hausdorff.py:114,121), executed by Numba's CUDA
    simulator on the CPU, and
  * the reference C++ measures (query/cpp/spatial/traj.cpp) through
    oracle/_ref/libtsm_ref.so,
on small seeded inputs.  Most cases use coordinates that are float32 values
(stored as float64 for the reference).  Two cases use float64 coordinates
that float32 cannot hold, as the reference's drivers read them: Porto near
pairs in Mercator metres with eps = 200 m and the default gap point (0, 0)
(utilities/data_loader.py:78-79, config.py:52), and in lon/lat degrees.  The
reference C++ measures take float32 points (query/cpp/spatial/point.h), so
those two cases carry no C++ outputs.  The fixtures hold the inputs (packed,
in their own dtype) and the outputs.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

os.environ.setdefault("NUMBA_ENABLE_CUDASIM", "1")
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("TSM_REFERENCE_ROOT", "/root/reference")
sys.path.insert(0, ROOT)
sys.path.insert(0, REF)

import core as refcore  # noqa: E402  the reference's core package
import importlib  # noqa: E402

ref_hausdorff_mod = importlib.import_module("core.hausdorff")
from numba import cuda  # noqa: E402

from trajsimimeasures_b200 import datagen as G  # noqa: E402
from trajsimimeasures_b200.engine import pack_lists  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle.build import build_ref  # noqa: E402

TPT = 4  # threads per pair in the simulator: exercises the strided column loop (pid += nthread)


def ref_hausdorff(t1, l1, t2, l2):
    trajs = np.stack([t1, t2], axis=1)
    lens = np.stack([l1, l2], axis=1)
    B = t1.shape[0]
    maxlen = int(lens.max())
    p2t = cuda.to_device(np.zeros((B, 2, maxlen)))
    ref_hausdorff_mod.hausdorff_opt[(B, 2, math.ceil(maxlen / TPT)), TPT](cuda.to_device(trajs), cuda.to_device(lens), p2t)
    return np.sqrt(p2t.copy_to_host().max(-1).max(-1))


def pack64(trajs):
    """pack_lists without the float32 rounding (float64 fixtures)."""
    lens = np.array([len(t) for t in trajs], dtype=np.int32)
    off = np.zeros(len(trajs), dtype=np.int64)
    np.cumsum(lens[:-1], out=off[1:])
    return np.concatenate([np.asarray(t, np.float64).reshape(-1, 2) for t in trajs]), off, lens


def run_case(name, trajs_a, trajs_b, eps, gpoint, f64=False):
    path = os.path.join(HERE, f"{name}.npz")
    if os.path.exists(path) and "--force" not in sys.argv:
        print(f"{path}: exists (--force regenerates)")
        return
    n = len(trajs_a)
    l1 = np.array([len(t) for t in trajs_a], dtype=np.int64)
    l2 = np.array([len(t) for t in trajs_b], dtype=np.int64)
    w = int(max(l1.max(), l2.max()))
    t1 = G.pad([np.asarray(t, np.float64) for t in trajs_a], w)
    t2 = G.pad([np.asarray(t, np.float64) for t in trajs_b], w)
    out = {}
    out["dtw"] = refcore.dtw(t1, l1, t2, l2, threads_per_traj=TPT)
    out["edr"] = refcore.edr(t1, l1, t2, l2, eps, threads_per_traj=TPT)
    out["lcss"] = refcore.lcss(t1, l1, t2, l2, eps, threads_per_traj=TPT)
    # core/erp.py sizes gpdists_g by max(len2) only (:106,:112) but writes
    # len1 entries into it (:32-34): a trailing dummy pair with len2 = width
    # keeps the reference in bounds; its output is dropped.
    t1e = np.concatenate([t1, np.zeros((1, w, 2))])
    t2e = np.concatenate([t2, np.zeros((1, w, 2))])
    out["erp"] = refcore.erp(t1e, np.append(l1, 1), t2e, np.append(l2, w), list(gpoint), threads_per_traj=TPT)[:n]
    out["dfrechet"] = refcore.dfrechet(t1, l1, t2, l2, threads_per_traj=TPT)
    out["hausdorff"] = ref_hausdorff(t1, l1, t2, l2)
    pts, off, lens = (pack64 if f64 else pack_lists)(list(trajs_a) + list(trajs_b))
    ia = np.arange(n)
    ib = ia + n
    cpp = {}
    if not f64:
        rs = O.RefSet(pts, off, lens)
        for m, key in ((O.DTW, "dtw"), (O.ERP, "erp"), (O.DFRECHET, "dfrechet"), (O.HAUSDORFF, "hausdorff")):
            cpp["cpp_" + key] = rs.pairs(m, ia, ib, gpoint=gpoint).astype(np.float64)
        rs.close()
    np.savez_compressed(path, pts=pts, off=off, lens=lens, ia=ia, ib=ib, eps=np.float64(eps),
                        gpoint=np.asarray(gpoint, np.float64), **out, **cpp)
    print(f"{path}: {n} pairs, lengths {lens.min()}..{lens.max()}")


def main():
    build_ref()
    rng = np.random.Generator(np.random.PCG64(12345))
    # 1. ragged random walks in the Porto-like box, lengths 1..40
    ls = [1, 2, 3, 4, 5, 7, 8, 13, 21, 31, 32, 33, 40]
    la = list(rng.choice(ls, 40)) + [1, 1, 2, 40]
    lb = list(rng.choice(ls, 40)) + [1, 2, 1, 40]
    pts, off, lens = G._walks(rng, np.array(la + lb), G.STEP_SIGMA)
    trajs = G.unpack(pts, off, lens)
    run_case("walks_ragged", trajs[:len(la)], trajs[len(la):], G.EPS_DEG, G.BOX_CENTRE)
    # 2. near pairs: EDR/LCSS threshold hits on both sides
    p, o, l, ia, ib = G.near_pairs(24, lo=5, hi=30, seed=777, jitter=2e-4)
    t = G.unpack(p, o, l)
    run_case("walks_near", [t[i] for i in ia], [t[i] for i in ib], G.EPS_DEG, G.BOX_CENTRE)
    # 3. identical and reversed trajectories
    base = G.unpack(*G.trajectory_set(8, 3, 25, seed=99))
    run_case("walks_self", base + base[:4], base[:4] + [b[::-1].copy() for b in base[4:]] + base[4:],
             G.EPS_DEG, G.BOX_CENTRE)
    # 4. the reference's own synthetic distribution (DatasetSynthetic: uniform
    #    [0,1]^2 points, utilities/data_loader.py:114-144), float32 values
    ua = [rng.uniform(size=(int(n), 2)).astype(np.float32) for n in rng.integers(1, 30, 16)]
    ub = [rng.uniform(size=(int(n), 2)).astype(np.float32) for n in rng.integers(1, 30, 16)]
    run_case("unit_square", ua, ub, 0.3, (0.0, 0.0))
    # 5, 6. float64 near pairs that float32 cannot hold: Porto in Mercator
    #    metres (eps 200 m, the drivers' default gap point (0, 0)) and in
    #    lon/lat degrees (eps 3e-4 deg, gap point at the box centre)
    for name, units, eps, g in (("merc_near_f64", "merc", G.MERC_EPS_M, (0.0, 0.0)),
                                ("lonlat_near_f64", "deg", G.EPS_DEG, G.BOX_CENTRE)):
        p, o, l, ia, ib = G.near_pairs_f64(24, lo=3, hi=30, seed=4242 if units == "merc" else 4343, units=units)
        t = G.unpack(p, o, l)
        run_case(name, [t[i] for i in ia], [t[i] for i in ib], eps, g, f64=True)


if __name__ == "__main__":
    main()
