"""Build recipe for the oracle (test infrastructure, not the product).

* ``build_oracle()`` compiles ``oracle/tsm_oracle.c`` (the FP64 restatement of
  the reference kernels and the FP32 same-arithmetic twin) into
  ``oracle/libtsm_oracle.so``.
* ``build_ref()`` compiles the reference's own C++ measures
  (``query/cpp/spatial/traj.cpp`` with ``point.cpp``, ``edge.cpp`` and
  ``utils/tool_funcs.cpp``), read in place from the reference checkout, plus
  ``oracle/ref_harness.cpp`` into ``oracle/_ref/libtsm_ref.so``.  traj.cpp
  includes ``Python.h``/numpy headers (lines 4-5) and defines
  ``Traj::TrajSimiGPU`` (lines 242-360), an embedded-CPython bridge; both are
  dropped on the way into the compiler (``sed`` into g++'s stdin), so no
  reference source is copied anywhere.  Outputs go to ``oracle/_ref/`` only.

Run as ``python -m oracle.build`` or through ``__graft_entry__.build()``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("TSM_REFERENCE_ROOT", "/root/reference")
REF_CPP = os.path.join(REF_ROOT, "query", "cpp")
ORACLE_SO = os.path.join(HERE, "libtsm_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libtsm_ref.so")


def _run(cmd, shell=False):
    r = subprocess.run(cmd, shell=shell, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {cmd}\n{r.stdout}\n{r.stderr}")
    return r


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "tsm_oracle.c")
    if force or _stale(ORACLE_SO, [src]):
        tmp = ORACLE_SO + ".tmp"
        _run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
              "-o", tmp, src, "-lm"])
        os.replace(tmp, ORACLE_SO)
    return ORACLE_SO


def _check_traj_cpp(path):
    with open(path) as f:
        lines = f.read().split("\n")
    ok = ("Python.h" in lines[3] and "numpy/arrayobject.h" in lines[4]
          and lines[241].startswith("int Traj::TrajSimiGPU") and lines[359].strip() == "}"
          and lines[362].startswith("std::istream& operator>>"))
    if not ok:
        raise RuntimeError(f"{path}: layout differs from the one this recipe strips (lines 4-5, 242-360)")


def build_ref(force: bool = False) -> str | None:
    """Returns the path of libtsm_ref.so, or None if the reference is absent."""
    traj = os.path.join(REF_CPP, "spatial", "traj.cpp")
    harness = os.path.join(HERE, "ref_harness.cpp")
    if not os.path.exists(traj):
        return REF_SO if os.path.exists(REF_SO) else None
    srcs = [traj, harness] + [os.path.join(REF_CPP, p) for p in
                              ("spatial/point.cpp", "spatial/edge.cpp", "utils/tool_funcs.cpp")]
    if not (force or _stale(REF_SO, srcs)):
        return REF_SO
    _check_traj_cpp(traj)
    os.makedirs(REF_DIR, exist_ok=True)
    inc = ["-I", os.path.join(REF_CPP, "spatial"), "-I", os.path.join(REF_CPP, "utils")]
    flags = ["g++", "-std=c++17", "-O3", "-DNDEBUG", "-fPIC", "-w"]
    objs = []
    for rel in ("spatial/point.cpp", "spatial/edge.cpp", "utils/tool_funcs.cpp"):
        o = os.path.join(REF_DIR, os.path.basename(rel).replace(".cpp", ".o"))
        _run(flags + inc + ["-c", os.path.join(REF_CPP, rel), "-o", o])
        objs.append(o)
    traj_o = os.path.join(REF_DIR, "traj.o")
    cmd = (f"sed -e '4,5d' -e '242,360d' '{traj}' | "
           f"{' '.join(flags)} {' '.join(inc)} -x c++ -c - -o '{traj_o}'")
    _run(cmd, shell=True)
    objs.append(traj_o)
    h_o = os.path.join(REF_DIR, "ref_harness.o")
    _run(flags + inc + ["-c", harness, "-o", h_o])
    objs.append(h_o)
    tmp = REF_SO + ".tmp"
    _run(["g++", "-shared", "-fPIC", "-o", tmp] + objs + ["-lpthread"])
    os.replace(tmp, REF_SO)
    return REF_SO


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
