"""Installs the reference's batched GPU measures into baseline/_ref/ (the
git-ignored install location of the reference) for bench.py's Numba arm.

The reference is not a pip-installable project (no setup.py or
pyproject.toml: `pip install --target baseline/_ref <reference>` stops with
"Neither 'setup.py' nor 'pyproject.toml' found").  Its GPU measures are the
plain-Python package core/ (Numba-CUDA kernels, core/dtw.py, edr.py, lcss.py,
erp.py, discret_frechet.py, hausdorff.py and their helpers), which needs no
build step, so installing it means copying that package, unmodified, to
baseline/_ref/core/.  Run it where a checkout of the reference exists:

    TSM_REFERENCE_ROOT=<reference checkout> python baseline/install_reference.py

baseline/_ref/ travels to the GPU box with the repository snapshot; it is not
part of the repository's history.
"""
from __future__ import annotations

import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEST = os.path.join(HERE, "_ref")


def install(ref_root: str) -> str:
    src = os.path.join(ref_root, "core")
    if not os.path.isfile(os.path.join(src, "__init__.py")):
        raise FileNotFoundError(f"no reference core package under {ref_root}")
    dst = os.path.join(DEST, "core")
    if os.path.isdir(dst):
        shutil.rmtree(dst)
    os.makedirs(DEST, exist_ok=True)
    shutil.copytree(src, dst, ignore=shutil.ignore_patterns("__pycache__", "*.pyc"))
    return dst


if __name__ == "__main__":
    root = os.environ.get("TSM_REFERENCE_ROOT")
    if not root:
        sys.exit("set TSM_REFERENCE_ROOT to the reference checkout")
    print(install(root))
