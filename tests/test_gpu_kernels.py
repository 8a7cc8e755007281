"""Device building blocks checked on their own.

FixedDiv (csrc/common.cuh) replaces a division by the pass-constant theta in the subspace
pass; it must round exactly like CUDA's correctly rounded division.  The check program
(tests/kernels/fixed_div_check.cu) compares both bit for bit on 64 million random and
constructed pairs per precision (quotients near representable values and near midpoints,
divisors with all-ones mantissas, zeros, subnormals, infinities, NaNs).  The same program
checks the arg-min filter quotient_exceeds on 64 million random quotients per precision
with the running minimum at, just below, just above and far from the quotient: it must
never skip a quotient that could still be the minimum.

The pass epilogues run formk, formt, bmv and the K solves shared out over a warp
(csrc/warp_small.cuh); tests/kernels/warp_small_check.cu runs each warp routine and the
serial routine of csrc/small.cuh on the same inputs and requires bit-identical outputs and
info codes, on factorisations that succeed and on ones that fail.
"""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)

pytestmark = pytest.mark.gpu


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_fixed_divisor_quotient_rounds_like_division(tmp_path):
    _need_gpu()
    exe = tmp_path / "fixed_div_check"
    cmd = ["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
           "-fmad=false", os.path.join(HERE, "kernels", "fixed_div_check.cu"), "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(exe), "64"], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    assert run.stdout.count("0 mismatches") == 10, run.stdout
    assert run.stdout.count(": 0 violations") == 2, run.stdout


def test_warp_small_matrix_routines_match_serial(tmp_path):
    _need_gpu()
    exe = tmp_path / "warp_small_check"
    cmd = ["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
           "-fmad=false", os.path.join(HERE, "kernels", "warp_small_check.cu"), "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(exe), "20000"], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    assert run.stdout.count(": 0 mismatches") == 2, run.stdout
