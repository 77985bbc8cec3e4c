"""CPU tests of the kernels' compiled resources (nvcc cross-compiles for
sm_100a without a GPU; ptxas reports each kernel's registers).

Occupancy is part of several kernels' design, and a register count is easy to
lose without a failing parity test: compiled into the scheduled kernel's ERP
tile tasks, the matrix kernels' four-block ERP pass once raised the whole
persistent kernel from 127 to 190 registers, cut its resident warps from 16 to
10 per SM and made the 500k-pair uneven batch 27 % slower with every result
unchanged."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

CSRC = os.path.join(ROOT, "trajsimimeasures_b200", "csrc")


def _nvcc():
    from trajsimimeasures_b200 import build as B
    return B.NVCC if os.path.exists(B.NVCC) else shutil.which("nvcc")


def _registers(source, tmp_path):
    """{mangled kernel name: registers per thread} of one translation unit,
    compiled with the library's own flags."""
    from trajsimimeasures_b200 import build as B
    nvcc = _nvcc()
    if not nvcc:
        pytest.skip("nvcc is not available")
    cmd = [nvcc] + B.ARCH + B.FLAGS + ["-Xptxas=-v", "-c", "-I", B.INCLUDE, "-I", B.CSRC, "-o",
                                       str(tmp_path / "k.o"), os.path.join(CSRC, source)]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-2000:]
    regs, cur = {}, None
    for line in (out.stdout + out.stderr).splitlines():
        m = re.search(r"Compiling entry function '(\S+)'", line)
        if m:
            cur = m.group(1)
        m = re.search(r"Used (\d+) registers", line)
        if m and cur:
            regs[cur] = int(m.group(1))
    return regs


def test_scheduled_kernel_keeps_sixteen_warps_per_sm(tmp_path):
    """The persistent scheduled kernel (128 threads per CTA, grid from the
    occupancy query) needs at most 128 registers per thread for 16 resident
    warps per SM (65,536 registers / (128 x 32))."""
    regs = _registers("tsm_k_sched_fast.cu", tmp_path)
    sched = {k: v for k, v in regs.items() if "dp_sched_kernel" in k}
    assert len(sched) == 2, sorted(regs)  # rows 4 and 8
    for name, r in sched.items():
        assert r <= 128, (name, r)


def test_paired_kernels_stay_below_the_four_block_pass(tmp_path):
    """The paired tile kernels run the two-block pass for every measure (the
    four-block ERP pass belongs to the matrix kernels): ERP's paired kernel
    stays near the other measures' register counts."""
    regs = _registers("tsm_k_pairs_fast.cu", tmp_path)
    pairs8 = {k: v for k, v in regs.items() if "dp_pairs_kernel" in k and "ELi8ELb0" in k}
    assert len(pairs8) == 5, sorted(regs)
    for name, r in pairs8.items():
        assert r <= 160, (name, r)
