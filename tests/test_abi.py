"""CPU-side checks of the drop-in boundary (no GPU needed).

* liblbfgsb_b200.so loads and exports every function include/lbfgsb_b200.h declares;
* the ctypes mirrors have the C layouts;
* the defaults equal the reference's lbfgsbdefaultoption (culbfgsb/lbfgsb.cpp:43-66);
* a program written against the reference's culbfgsb.h API compiles unchanged against
  include/culbfgsb.h and links against the library.
"""
import os
import re
import subprocess
import ctypes as C

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "lbfgsb_b200.h")


@pytest.fixture(scope="module")
def LB():
    import lbfgsb_b200
    import build as B
    B.build()
    return lbfgsb_b200


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(lbfgsb_b200_[a-z0-9_]+)\s*\(", text))
    return sorted(n for n in names if not n.startswith("lbfgsb_b200_callback"))


def test_library_exports_every_declared_symbol(LB):
    lib = LB.load()
    names = declared_functions()
    assert len(names) >= 13
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(LB.EXPORTS) == names


def test_struct_layouts(LB):
    assert C.sizeof(LB.OptionF64) == 6 * 8 + 3 * 4 + 4
    assert C.sizeof(LB.OptionF32) == 6 * 4 + 3 * 4
    assert C.sizeof(LB.SummaryF64) == 3 * 8 + 2 * 4
    assert C.sizeof(LB.SummaryF32) == 3 * 4 + 2 * 4


def test_defaults_match_reference(LB):
    o = LB.default_option(np.float64)
    assert (o.eps_f, o.eps_g, o.eps_x) == (1e-15, 1e-15, 1e-15)
    assert o.hessian_approximate_dimension == 8 and o.max_iteration == 1000
    assert o.machine_epsilon == 1e-15 and o.step_scaling == 1.0
    assert o.machine_maximum == np.finfo(np.float64).max and o.mode == LB.MODE_CUDA
    o = LB.default_option(np.float32)
    assert o.machine_epsilon == np.float32(1e-8) and o.machine_maximum == np.finfo(np.float32).max


def test_dropin_header_compiles_and_links(LB, tmp_path):
    exe = tmp_path / "dropin"
    cmd = ["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           f"-I{os.path.join(REPO, 'include')}", os.path.join(REPO, "tests", "dropin", "dropin_example.cu"),
           "-o", str(exe), f"-L{os.path.dirname(LB.LIB_PATH)}", "-llbfgsb_b200",
           f"-Xlinker=-rpath={os.path.dirname(LB.LIB_PATH)}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    assert exe.exists()
