"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the reference goldens.

The funcgrad callback of these runs evaluates the objective on the host with the
oracle's own objective code, so for the same x the GPU path and the oracle see
bit-identical f and g: every difference comes from the solver.

Tolerances (stated per quantity; the GPU reductions sum in a different order than the
reference's sequential loops, so reals differ at rounding level and the discrete
decisions can only agree while the iterates agree):
  FP64  discrete per-iteration trace (breakpoints passed, free-set hash, entering /
        leaving counts, subspace truncation, evaluations) equal until the first
        rounding-level near tie; f per iteration within 1e-10 relative while the traces
        agree; for runs whose trace never diverges: same exit code and iteration count,
        final f within 1e-10 relative, final x within 1e-6 of max|x|; for a run that
        diverges after >= 100 identical iterations: f within 1e-10 for the first 50
        iterations and 1e-6 up to the divergence (the oracle's own sensitivity to a 1e-16
        perturbation of x0 reaches ~2e-7 there), final f within 1e-5 relative.
  FP32  (plain form, float scalars like the reference's float path) same exit code, the
        first 10 iterations' trace equal, final f within 1e-5 relative.
"""
import json
import os

import numpy as np
import pytest

from cases import CASES, apply_options, make_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TRACE_KEYS = ["nint", "nbreak", "nfree", "nenter", "nleave", "col", "head", "iword",
              "free_hash", "at_lower", "at_upper", "nfgv", "ifun"]


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


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "golden.json")) as fh:
        return json.load(fh)


def run_pair(LB, OB, name, **kw):
    prob, dt, x0, over, stop = make_case(name)
    a = OB.run_cpu("oracle", prob, dt, x0=x0, option=apply_options(OB.default_option(dt), over),
                   custom_stop_at=stop, trace=True)
    b = LB.solve(prob, dt, x0=x0, option=apply_options(LB.default_option(dt), over),
                 objective="host", trace=True, custom_stop_at=stop, **kw)
    return prob, dt, a, b


def first_divergence(ta, tb):
    for k, (a, b) in enumerate(zip(ta, tb)):
        if any(a[key] != b[key] for key in TRACE_KEYS):
            return k
    return min(len(ta), len(tb))


def relf(a, b):
    return abs(a - b) / max(1.0, abs(a))


F64_EXACT = [c for c in CASES if c.endswith("f64") or "_f64_" in c]
F64_EXACT = [c for c in F64_EXACT if c != "synth_s64_f64_b001"]
F32_CASES = [c for c in CASES if c.endswith("f32") or "_f32_" in c]


@pytest.mark.parametrize("name", F64_EXACT)
def test_f64_trace_matches_oracle(LB, OB, golden, name):
    prob, dt, a, b = run_pair(LB, OB, name)
    assert b.info == a.info == golden[name]["info"]
    k = first_divergence(a.trace, b.trace)
    assert k == len(a.trace) == len(b.trace), f"trace diverges at iteration {k + 1}"
    assert b.num_iteration == a.num_iteration
    for ra, rb in zip(a.trace, b.trace):
        assert relf(ra["f"], rb["f"]) <= 1e-10
    if a.trace:
        assert relf(a.trace[-1]["f"], b.trace[-1]["f"]) <= 1e-10
        # the reference's own last function value (golden fixture)
        assert relf(golden[name]["evals"][-1][0], b.evals[-1][0]) <= 1e-10
    scale = max(1e-300, float(np.max(np.abs(a.x))))
    assert float(np.max(np.abs(a.x - b.x))) <= 1e-6 * scale


def test_f64_long_tight_run(LB, OB, golden):
    """300 iterations against bounds of +-0.01.  This trajectory amplifies rounding: moving
    x0 by 1e-16 relative (or 1e-19 absolute) moves the oracle's own f by up to ~2e-7
    relative around iteration 100 while its discrete trace still agrees
    (tests/test_oracle_pin.py::test_long_tight_run_sensitivity).  So: the traces agree for
    at least the first 100 iterations, f within 1e-10 for the first 50 of them and within
    1e-6 up to the divergence; afterwards the runs take different but equally valid paths,
    and the final values agree to 1e-5 relative (the f-test stops at 1e-8 relative
    decrease per step)."""
    prob, dt, a, b = run_pair(LB, OB, "synth_s64_f64_b001")
    k = first_divergence(a.trace, b.trace)
    assert k >= 100
    for i, (ra, rb) in enumerate(zip(a.trace[:k], b.trace[:k])):
        assert relf(ra["f"], rb["f"]) <= (1e-10 if i < 50 else 1e-6)
    assert b.info == a.info
    assert relf(a.trace[-1]["f"], b.trace[-1]["f"]) <= 1e-5
    nbd = prob["nbd"]
    has_l = (nbd == 1) | (nbd == 2)
    has_u = (nbd == 2) | (nbd == 3)
    assert np.all(b.x[has_l] >= prob["l"][has_l]) and np.all(b.x[has_u] <= prob["u"][has_u])


@pytest.mark.parametrize("name", F32_CASES)
def test_f32_plain_matches_oracle(LB, OB, golden, name):
    prob, dt, a, b = run_pair(LB, OB, name)
    assert b.info == a.info == golden[name]["info"]
    assert first_divergence(a.trace, b.trace) >= min(10, len(a.trace))
    assert relf(a.trace[-1]["f"], b.trace[-1]["f"]) <= 1e-5
    assert relf(golden[name]["evals"][-1][0], b.trace[-1]["f"]) <= 1e-5


def test_many_breakpoints_walk(LB, OB):
    """The first Cauchy point passes 3278 breakpoints, more than three 1024-chunks of the
    device walk (radix-selected, sorted in shared memory, walked in key order)."""
    prob, dt, a, b = run_pair(LB, OB, "quad_walk_many_f64")
    assert a.trace[0]["nint"] > 3 * 1024
    assert b.trace[0]["nint"] == a.trace[0]["nint"]
    assert b.trace[0]["free_hash"] == a.trace[0]["free_hash"]
    assert relf(a.trace[0]["tsum"], b.trace[0]["tsum"]) <= 1e-12


def test_deterministic(LB):
    prob, dt, x0, over, stop = make_case("synth_s32_f64_b005")
    r1 = LB.solve(prob, dt, option=apply_options(LB.default_option(dt), over), objective="host")
    r2 = LB.solve(prob, dt, option=apply_options(LB.default_option(dt), over), objective="host")
    assert r1.evals == r2.evals
    np.testing.assert_array_equal(r1.x, r2.x)


def test_mode_no_acceleration_rejected(LB):
    prob, dt, x0, over, stop = make_case("synth_s16_f64")
    opt = apply_options(LB.default_option(dt), over)
    opt.mode = LB.MODE_NO_ACCELERATION
    with pytest.raises(RuntimeError):
        LB.solve(prob, dt, option=opt, objective="host")


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_device_objective_matches_host(LB, OB, dtype):
    """The synthetic objective kernel (csrc/objective.cu) against oracle/objective.c."""
    import ctypes as C
    import synth
    import torch
    prob = synth.synth_problem(48, seed=3)
    prob["kind"] = "synth"
    n = prob["nbd"].size
    rng = np.random.default_rng(0)
    x = (0.3 * rng.standard_normal(n)).astype(dtype)
    so = LB.SynthObjective(prob, single_precision_fields=dtype == np.float32)
    xd = torch.from_numpy(x).cuda()
    gd = torch.zeros_like(xd)
    real = C.c_double if dtype == np.float64 else C.c_float
    summ = LB.SummaryF64() if dtype == np.float64 else LB.SummaryF32()
    fbox = real()
    fn = (LB.CB64 if dtype == np.float64 else LB.CB32)(so.f64 if dtype == np.float64 else so.f32)
    fn(C.c_void_p(so.handle), C.cast(xd.data_ptr(), C.POINTER(real)), C.byref(fbox),
       C.cast(gd.data_ptr(), C.POINTER(real)), None, C.byref(summ))
    ev = OB.host_objective(prob, dtype)
    hg = np.zeros(n, dtype=dtype)
    hf = real()
    ev(x.ctypes.data_as(C.POINTER(real)), C.byref(hf), hg.ctypes.data_as(C.POINTER(real)))
    tol = 1e-12 if dtype == np.float64 else 2e-5
    assert abs(fbox.value - hf.value) <= tol * max(1.0, abs(hf.value))
    g = gd.cpu().numpy()
    assert float(np.max(np.abs(g - hg))) <= tol * max(1e-30, float(np.max(np.abs(hg)))) * 10
    so.close()


def test_config0_s256_full_solve(LB, OB):
    """The reference's config 0: s = 256 (n = 65,536), FP64, eps 1e-8, up to 1000
    iterations, host objective.  Measured: traces agree for 118 iterations (f within
    1.9e-10), then both runs stop on the f-test after 520-560 iterations with final f
    5e-6 apart.  The oracle itself, restarted from x0 moved by 1e-19, agrees for 123
    iterations and ends 1.0e-5 to 1.5e-5 away (test_config0_sensitivity), so the final
    f is compared within 5e-5."""
    import synth
    prob = synth.synth_problem(256, seed=0)
    prob["kind"] = "synth"
    over = {"eps_f": 1e-8, "eps_g": 1e-8, "eps_x": 1e-8, "max_iteration": 1000}
    a = OB.run_cpu("oracle", prob, np.float64, option=apply_options(OB.default_option(np.float64), over),
                   trace=True)
    b = LB.solve(prob, np.float64, option=apply_options(LB.default_option(np.float64), over),
                 objective="host", trace=True)
    k = first_divergence(a.trace, b.trace)
    assert k >= 100
    for i, (ra, rb) in enumerate(zip(a.trace[:k], b.trace[:k])):
        assert relf(ra["f"], rb["f"]) <= (1e-10 if i < 100 else 1e-9)
    assert b.info == a.info == 1
    assert relf(a.trace[-1]["f"], b.trace[-1]["f"]) <= 5e-5
    nbd = prob["nbd"]
    has_l = (nbd == 1) | (nbd == 2)
    has_u = (nbd == 2) | (nbd == 3)
    assert np.all(b.x[has_l] >= prob["l"][has_l]) and np.all(b.x[has_u] <= prob["u"][has_u])
    # final x and ||proj g||_inf, against the spread of the oracle's own ending: the oracle
    # restarted from x0 moved by 1e-19 gives the scale of the difference that the run's
    # conditioning allows (every rounding difference acts like such a move)
    xp = 1e-19 * np.random.default_rng(1).standard_normal(prob["nbd"].size)
    c = OB.run_cpu("oracle", prob, np.float64, x0=xp,
                   option=apply_options(OB.default_option(np.float64), over), record=False)
    dx_ref = float(np.max(np.abs(c.x - a.x)))
    dx = float(np.max(np.abs(b.x - a.x)))
    assert dx <= 4.0 * dx_ref + 1e-8, (dx, dx_ref)
    dg_ref = abs(c.residual_g - a.residual_g)
    dg = abs(b.residual_g - a.residual_g)
    assert dg <= 4.0 * max(dg_ref, 1e-3 * abs(a.residual_g)), (dg, dg_ref, a.residual_g)
