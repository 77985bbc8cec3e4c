import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")

# Tolerances: DTW/ERP/Frechet/Hausdorff within 1e-5
# relative of the FP64 oracle; EDR/LCSS counts bit-exact.
REL_TOL = 1e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libtsm_b200.so")


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.lib()
    return O


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    both_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    both_nan = np.isnan(a) & np.isnan(b)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
    r[both_inf | both_nan] = 0.0
    return r


def centred_pairs(m, pts, off, lens, ia, ib, gpoint=(0.0, 0.0)):
    """A paired batch exactly as core.pairs hands it to the kernels: padded,
    translated by the FP64 origin(s) of core.pair_origins and rounded to
    float32.  -> (pts32, off_a, len_a, off_b, len_b, gpoint in the translated
    coordinates), for the FP32 twin."""
    from trajsimimeasures_b200 import core, datagen as D
    ia, ib = np.asarray(ia), np.asarray(ib)
    l1, l2 = np.asarray(lens)[ia], np.asarray(lens)[ib]
    w = max(1, int(max(l1.max(initial=0), l2.max(initial=0))))
    t1 = D.pad(D.unpack(pts, off, lens, ia), w)
    t2 = D.pad(D.unpack(pts, off, lens, ib), w)
    org = core.pair_origins(m, t1, l1, t2, l2)
    g = tuple(gpoint)
    if org is not None:
        o = org.reshape(-1, 1, 2)
        t1, t2 = t1 - o, t2 - o
        if org.ndim == 1:
            g = (g[0] - org[0], g[1] - org[1])
    n = len(ia)
    p32 = np.concatenate([t1.reshape(-1, 2), t2.reshape(-1, 2)]).astype(np.float32)
    k = np.arange(n, dtype=np.int64)
    return p32, k * w, l1, n * w + k * w, l2, g
