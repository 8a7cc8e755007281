"""A program written against the reference's culbfgsb.h runs unchanged on this library."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def test_dropin_program_runs(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lbfgsb_b200
    lib_dir = os.path.dirname(lbfgsb_b200.LIB_PATH)
    exe = tmp_path / "dropin"
    cmd = ["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           f"-I{os.path.join(REPO, 'include')}", os.path.join(REPO, "tests", "dropin", "dropin_example.cu"),
           "-o", str(exe), f"-L{lib_dir}", "-llbfgsb_b200", f"-Xlinker=-rpath={lib_dir}"]
    subprocess.run(cmd, check=True, capture_output=True)
    res = subprocess.run([str(exe), "64"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "OK" in res.stdout


def test_reference_dsscfg_example_runs_unchanged():
    """The reference's own example program (examples/dsscfg/dsscfg_main.cpp with its
    dsscfg_cuda.cu and dsscfg_cpu.cpp), compiled unchanged against include/ (its
    #include "culbfgsb/culbfgsb.h" resolves to the drop-in adapter; it creates and destroys
    a cuBLAS handle itself) and linked against liblbfgsb_b200.so (oracle/Makefile target
    `dropin`, built where the reference tree is present).  Its CPU half asks for
    LCM_NO_ACCELERATION, which this GPU-only library answers with info = -1, so the program
    prints its CPU/CUDA comparison as failed; the CUDA results it prints must meet the
    reference's own checks (dsscfg_main.cpp:208, :224): the FP64 minimum within 1e-4 of the
    reference's FP64 result on this 256 x 256 problem, -1.01129586297, and the FP32 minimum
    within 1e-3 of the reference's FP32 result, -1.01110565662."""
    import re

    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import binding as OB
    if not os.path.exists(OB.DROPIN_EXE):
        pytest.skip("oracle/_ref/dsscfg_dropin was not built (needs the reference tree)")
    res = subprocess.run([OB.DROPIN_EXE], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    cuda = [float(v) for v in re.findall(r"CUDA result (\S+),", res.stdout)]
    assert len(cuda) == 2, res.stdout[-2000:]
    assert abs(cuda[0] - (-1.01129586297)) < 1e-4, cuda
    assert abs(cuda[1] - (-1.01110565662)) < 1e-3, cuda
    assert "CUDA iteration" in res.stdout
