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
