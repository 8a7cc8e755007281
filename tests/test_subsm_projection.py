"""The L-BFGS-B 3.0 subspace step (lbfgsb_b200_ext.subsm_projection; off by default).

L-BFGS-B 3.0 (Morales and Nocedal, "Remark on Algorithm 778", ACM TOMS 38(1), 2011)
replaces the 2.1 truncation of the subspace step: the subspace minimizer is projected onto
the box, and the projected point is kept when it gives a descent direction from the
iterate; otherwise the 2.1 step truncated at the first bound is taken.  The reference
implements only 2.1, so the oracle restates the 3.0 step (oracle/lbfgsb_oracle_body.h,
subsm) and is checked here on the CPU:
  * a problem whose 2.1 steps are never truncated gives the 2.1 trace exactly;
  * problems with many truncated 2.1 steps converge to the same minimum (f within 1e-5
    relative) in fewer iterations.
On the GPU the 3.0 step must match the oracle's 3.0 step with the tolerances of the 2.1
parity tests (tests/test_gpu_parity.py): FP64 discrete traces equal until a
rounding-level near tie (at least 40 iterations here, all of them for the runs that never
diverge), f within 1e-10 per iteration on the agreed prefix, final f within 1e-5; FP32
the first 10 iterations' trace and final f within 1e-5.
"""
import numpy as np
import pytest

from cases import apply_options, make_case

TRACE_KEYS = ["nint", "nbreak", "nfree", "nenter", "nleave", "col", "head", "iword",
              "free_hash", "at_lower", "at_upper", "nfgv", "ifun"]
TRUNCATING_F64 = ["synth_s20_f64_boxed", "synth_s20_f64_nbd13", "synth_s24_f64_b001_m5",
                  "synth_s20_f64_x0out", "synth_s64_f64_b001"]


def _oracle(name, projection):
    from oracle import binding as OB
    prob, dt, x0, over, stop = make_case(name)
    return prob, dt, OB.run_cpu("oracle", prob, dt, x0=x0,
                                option=apply_options(OB.default_option(dt), over),
                                custom_stop_at=stop, trace=True, subsm_projection=projection)


def _relf(a, b):
    return abs(a - b) / max(1.0, abs(a))


def _first_divergence(ta, tb):
    for k, (a, b) in enumerate(zip(ta, tb)):
        if any(a[key] != b[key] for key in TRACE_KEYS):
            return k
    return min(len(ta), len(tb))


def test_oracle_projection_equals_21_without_truncation():
    _, _, a = _oracle("synth_s32_f64_b005", False)
    _, _, b = _oracle("synth_s32_f64_b005", True)
    assert not any(t["iword"] == 1 for t in a.trace)   # no 2.1 step is truncated
    assert [dict((k, t[k]) for k in TRACE_KEYS + ["f"]) for t in a.trace] == \
        [dict((k, t[k]) for k in TRACE_KEYS + ["f"]) for t in b.trace]
    assert np.array_equal(a.x, b.x)


@pytest.mark.parametrize("name", ["synth_s20_f64_boxed", "synth_s64_f64_b001",
                                  "synth_s32_f32_b002"])
def test_oracle_projection_converges_in_fewer_iterations(name):
    prob, _, a = _oracle(name, False)
    _, _, b = _oracle(name, True)
    assert sum(t["iword"] == 1 for t in a.trace) > 0     # 2.1 truncates here
    assert a.info == b.info == 1
    assert b.num_iteration < a.num_iteration
    assert _relf(a.trace[-1]["f"], b.trace[-1]["f"]) <= 1e-5
    nbd = prob["nbd"]
    has_l = (nbd == 1) | (nbd == 2)
    has_u = (nbd == 2) | (nbd == 3)
    assert np.all(b.x[has_l] >= prob["l"][has_l]) and np.all(b.x[has_u] <= prob["u"][has_u])


@pytest.fixture(scope="module")
def LB():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lbfgsb_b200
    lbfgsb_b200.load()
    return lbfgsb_b200


@pytest.mark.gpu
@pytest.mark.parametrize("name", TRUNCATING_F64)
def test_gpu_projection_matches_oracle_f64(LB, name):
    prob, dt, a = _oracle(name, True)
    _, _, x0, over, stop = make_case(name)
    b = LB.solve(prob, dt, x0=x0, option=apply_options(LB.default_option(dt), over),
                 objective="host", trace=True, custom_stop_at=stop, subsm_projection=True)
    assert sum(t["iword"] == 1 for t in a.trace) > 0
    k = _first_divergence(a.trace, b.trace)
    assert k >= min(40, len(a.trace)), f"trace diverges at iteration {k + 1}"
    for ra, rb in zip(a.trace[:k], b.trace[:k]):
        assert _relf(ra["f"], rb["f"]) <= 1e-10
    assert b.info == a.info
    assert _relf(a.trace[-1]["f"], b.trace[-1]["f"]) <= 1e-5
    if k == len(a.trace) == len(b.trace):
        assert b.num_iteration == a.num_iteration
        scale = max(1e-300, float(np.max(np.abs(a.x))))
        assert float(np.max(np.abs(a.x - b.x))) <= 1e-6 * scale
    nbd = prob["nbd"]
    has_l = (nbd == 1) | (nbd == 2)
    has_u = (nbd == 2) | (nbd == 3)
    assert np.all(b.x[has_l] >= prob["l"][has_l]) and np.all(b.x[has_u] <= prob["u"][has_u])


@pytest.mark.gpu
def test_gpu_projection_matches_oracle_f32(LB):
    prob, dt, a = _oracle("synth_s32_f32_b002", True)
    _, _, x0, over, stop = make_case("synth_s32_f32_b002")
    b = LB.solve(prob, dt, x0=x0, option=apply_options(LB.default_option(dt), over),
                 objective="host", trace=True, custom_stop_at=stop, subsm_projection=True)
    assert b.info == a.info
    assert _first_divergence(a.trace, b.trace) >= min(10, len(a.trace))
    assert _relf(a.trace[-1]["f"], b.trace[-1]["f"]) <= 1e-5


@pytest.mark.gpu
def test_gpu_projection_off_is_the_21_step(LB):
    """The switch left at 0 takes the 2.1 path: the same trace as a default solve."""
    name = "synth_s20_f64_nbd13"
    prob, dt, x0, over, stop = make_case(name)
    opt = apply_options(LB.default_option(dt), over)
    a = LB.solve(prob, dt, x0=x0, option=opt, objective="host", trace=True)
    b = LB.solve(prob, dt, x0=x0, option=opt, objective="host", trace=True,
                 subsm_projection=False)
    assert a.trace == b.trace
    assert np.array_equal(a.x, b.x)
