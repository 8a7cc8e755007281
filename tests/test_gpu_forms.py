"""The f32 entry point's precision forms against the FP64 oracle.

Forms: plain (vectors, history and scalars in float, like the reference's float path),
mixed (float vectors and history, double small matrices, Cauchy and line-search scalars)
and mixed with bf16 history storage.  The objective is evaluated in float in all three
(the oracle's float objective on the host), so the final f can only approach the FP64
optimum to within what a float objective resolves.  Measured final f against the FP64
oracle run of the same problem: plain 1.1e-7 .. 3.9e-6, mixed 4.1e-7 .. 3.2e-6,
bf16 history 1.4e-8 .. 2.8e-7 relative.  Bound: 1e-5 relative (the FP32 tolerance), the
run ends with a convergence code (1, 2 or 4), and x respects the declared bounds.
"""
import numpy as np
import pytest

from cases import apply_options, make_case

pytestmark = pytest.mark.gpu

CASES = ["synth_s32_f32", "synth_s32_f32_b002", "synth_s64_f32_b002", "quad_ties_f32",
         "quad_walk_many_f32"]


@pytest.fixture(scope="module")
def LB():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lbfgsb_b200
    lbfgsb_b200.load()
    return lbfgsb_b200


@pytest.fixture(scope="module")
def OB():
    from oracle import binding
    return binding


BOUND = {0: 1e-5, 1: 1e-6, 2: 1e-6}
# the mixed form's known miss of 1e-6 (float objective); still held to the FP32 tolerance
MIXED_MISS = {"synth_s64_f32_b002"}


def _final_rel(LB, OB, name, form):
    prob, dt, x0, over, stop = make_case(name)
    ref = OB.run_cpu("oracle", prob, np.float64, x0=x0,
                     option=apply_options(OB.default_option(np.float64), over))
    r = LB.solve(prob, np.float32, x0=x0, option=apply_options(LB.default_option(np.float32), over),
                 objective="host", form=form)
    fref = ref.evals[-1][0]
    return prob, r, abs(r.evals[-1][0] - fref) / max(1.0, abs(fref))


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("name", CASES)
def test_form_against_fp64_oracle(LB, OB, name, form):
    prob, r, rel = _final_rel(LB, OB, name, form)
    print(f"{name} form {form}: final f relative error {rel:.2e}")
    bound = 1e-5 if (form == 1 and name in MIXED_MISS) else BOUND[form]
    assert rel <= bound, rel
    assert r.info in (1, 2, 4)
    nbd = prob["nbd"]
    x = r.x.astype(np.float64)
    lo = prob["l"].astype(np.float32).astype(np.float64)
    hi = prob["u"].astype(np.float32).astype(np.float64)
    has_l = (nbd == 1) | (nbd == 2)
    has_u = (nbd == 2) | (nbd == 3)
    assert np.all(x[has_l] >= lo[has_l]) and np.all(x[has_u] <= hi[has_u])


@pytest.mark.xfail(reason="mixed form on s = 64, bounds +-0.02: the float objective's gradient "
                          "error moves the stopping point ~3e-6 from the FP64 optimum", strict=False)
@pytest.mark.parametrize("name", sorted(MIXED_MISS))
def test_mixed_form_one_in_a_million(LB, OB, name):
    _, _, rel = _final_rel(LB, OB, name, 1)
    assert rel <= 1e-6, rel
