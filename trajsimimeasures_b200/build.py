"""Build step of the CUDA library: nvcc -> trajsimimeasures_b200/libtsm_b200.so.

The library is compiled for sm_100a only (B200).  It is a plain C-ABI shared
object (include/tsm.h) with the CUDA runtime linked statically, loaded by
trajsimimeasures_b200._lib through ctypes.  nvcc cross-compiles without a GPU.

    python -m trajsimimeasures_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libtsm_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + _headers()
    return any(os.path.getmtime(d) > t for d in deps)


OBJ_DIR = os.path.join(ROOT, "_build", "csrc")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles each .cu into an object (in parallel, one nvcc per source;
    only the stale ones) and links the shared library."""
    if not (force or _stale()):
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdrs = _headers()
    newest_hdr = max((os.path.getmtime(h) for h in hdrs), default=0.0)
    jobs = []
    for src in sources():
        obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), newest_hdr):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", "-I", INCLUDE, "-I", CSRC, "-o", obj + ".tmp", src]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append((cmd, obj))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        logs = list(ex.map(lambda j: _run(j[0]), jobs))
    for (_, obj) in jobs:
        os.replace(obj + ".tmp", obj)
    if verbose:
        sys.stderr.write("".join(logs))
    tmp = LIB + ".tmp"
    objs = [os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o") for src in sources()]
    _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
