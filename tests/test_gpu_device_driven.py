"""Device-driven solves (lbfgsb_b200_minimize_device_*) against host-driven solves.

Both run the same passes with the same device objective (csrc/objective.cu: the slot form
for the device-driven solve, the funcgrad form for the host-driven one, one kernel with the
same launch shape and reduction order), so every decision of the outer loop sees the same
state: the final x must be bit-identical, and the summary (info, iterations, residuals)
equal.  The host-driven solves are the ones the parity tests check against the oracle.
"""
import numpy as np
import pytest

from cases import apply_options, make_case

pytestmark = pytest.mark.gpu

CASES = ["synth_s16_f64", "synth_s32_f64", "synth_s32_f64_b005", "synth_s24_f64_b001_m5",
         "synth_s20_f64_unbounded", "synth_s20_f64_boxed", "synth_s20_f64_nbd13",
         "synth_s20_f64_fixedeq", "synth_s20_f64_x0out", "synth_s32_f64_maxit7",
         "synth_s64_f64_b001", "synth_s32_f32", "synth_s32_f32_b002", "synth_s64_f32_b002",
         "err_nbd4", "err_l_gt_u"]


@pytest.fixture(scope="module")
def LB():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lbfgsb_b200
    lbfgsb_b200.load()
    return lbfgsb_b200


def _pair(LB, prob, dt, x0, opt_over, **kw):
    a = LB.solve(prob, dt, x0=x0, option=apply_options(LB.default_option(dt), opt_over),
                 objective="device", record=False, **kw)
    b = LB.solve(prob, dt, x0=x0, option=apply_options(LB.default_option(dt), opt_over),
                 objective="device", record=False, driven="device", **kw)
    return a, b


def _same(a, b):
    assert (a.info, a.num_iteration) == (b.info, b.num_iteration)
    assert a.residual_g == b.residual_g and a.residual_x == b.residual_x
    assert a.residual_f == b.residual_f
    np.testing.assert_array_equal(a.x, b.x)


@pytest.mark.parametrize("name", CASES)
def test_device_driven_equals_host_driven(LB, name):
    prob, dt, x0, over, stop = make_case(name)
    a, b = _pair(LB, prob, dt, x0, over)
    _same(a, b)
    st = b.stats
    if a.info != -1:
        # one read of the state after k_init and one after projgr, then one per batch of
        # rounds: far fewer synchronisations than the host-driven solve's two per iteration
        assert st["rounds"] > 0 and st["host_syncs"] <= 2 + st["rounds"] // 4 + 1


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("name", ["synth_s32_f32_b002", "synth_s64_f32_b002"])
def test_device_driven_forms(LB, name, form):
    prob, dt, x0, over, stop = make_case(name)
    a, b = _pair(LB, prob, dt, x0, over, form=form)
    _same(a, b)


def test_device_driven_subspace_projection(LB):
    prob, dt, x0, over, stop = make_case("synth_s64_f64_b001")
    a, b = _pair(LB, prob, dt, x0, over, subsm_projection=True)
    _same(a, b)


def test_device_driven_full_size(LB):
    """n = 4096^2, FP64, 25 iterations (eps = 0): the benchmark's workload."""
    import synth
    prob = synth.synth_problem(4096, seed=0)
    over = {"eps_f": 0.0, "eps_g": 0.0, "eps_x": 0.0, "max_iteration": 24}
    a, b = _pair(LB, prob, np.float64, None, over)
    _same(a, b)
    assert b.num_iteration == 25
