"""The oracle is pinned to the reference before anything is checked against it.

1. Against the golden fixtures recorded from the reference's own CPU L-BFGS-B
   (tests/golden/golden.json, made by tests/golden/make_golden.py from
   culbfgsb/lbfgsbcpu.cpp): every funcgrad point (f and the bytes of x), every
   after-iteration summary, the exit code and the final x must match bit for bit.
2. Against the live reference build (oracle/_ref/libref_lbfgsb.so) on further seeds and
   sizes, when that build is present.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import binding as B
from cases import CASES, apply_options, make_case

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "golden.json")
GOLDEN_X = os.path.join(HERE, "golden", "golden_x.npz")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as fh:
        return json.load(fh), np.load(GOLDEN_X)


def _run(which, name, trace=False):
    prob, dtype, x0, over, stop = make_case(name)
    opt = apply_options(B.default_option(dtype), over)
    return B.run_cpu(which, prob, dtype, x0=x0, option=opt, custom_stop_at=stop, trace=trace)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_golden(golden, name):
    gj, gx = golden
    g = gj[name]
    r = _run("oracle", name)
    assert r.info == g["info"]
    assert r.num_iteration == g["num_iteration"]
    assert [list(e) for e in r.evals] == [list(e) for e in g["evals"]]
    assert [list(e) for e in r.iters] == [list(e) for e in g["iters"]]
    assert hashlib.sha1(r.x.tobytes()).hexdigest()[:16] == g["x_sha1"]
    np.testing.assert_array_equal(r.x, gx[name])
    assert r.residual_g == g["residual_g"]


def test_golden_covers_the_walk_and_errors(golden):
    """The fixture set exercises breakpoint walks, truncated subspace steps, the
    entering/leaving corrections and every exit code the CPU path produces."""
    gj, _ = golden
    infos = {gj[c]["info"] for c in CASES}
    assert {-1, 0, 1, 4, 5} <= infos
    tr = _run("oracle", "synth_s64_f64_b001", trace=True).trace
    assert max(t["nint"] for t in tr) > 10
    assert sum(t["iword"] == 1 for t in tr) > 10
    assert sum(t["nenter"] for t in tr) > 0 and sum(t["nleave"] for t in tr) > 0


@pytest.mark.skipif(not B.ref_available(), reason="reference build not present")
@pytest.mark.parametrize("s,seed,bound,dtype", [
    (24, 21, 0.015, np.float64), (24, 22, 0.015, np.float32), (40, 23, 1.0, np.float64),
    (40, 24, 0.03, np.float64), (48, 25, 0.01, np.float32)])
def test_oracle_matches_live_reference(s, seed, bound, dtype):
    import synth
    prob = synth.synth_problem(s, seed=seed)
    prob["l"] = prob["l"] * bound
    prob["u"] = prob["u"] * bound
    opt = B.default_option(dtype)
    opt.eps_f = opt.eps_g = opt.eps_x = 1e-8
    a = B.run_cpu("ref", prob, dtype, option=opt)
    b = B.run_cpu("oracle", prob, dtype, option=opt)
    assert a.evals == b.evals
    assert a.iters == b.iters
    np.testing.assert_array_equal(a.x, b.x)
    assert a.info == b.info


TRACE_KEYS = ["nint", "nbreak", "nfree", "nenter", "nleave", "col", "head", "iword",
              "free_hash", "at_lower", "at_upper", "nfgv", "ifun"]


def test_long_tight_run_sensitivity():
    """The conditioning behind the GPU tolerance of synth_s64_f64_b001: moving the start
    point (x0 = 0) by 1e-19 leaves the oracle's discrete trace unchanged for at least 90
    iterations, yet moves its f by more than 1e-8 relative within that agreed prefix."""
    prob, dtype, x0, over, stop = make_case("synth_s64_f64_b001")
    opt = apply_options(B.default_option(dtype), over)
    a = B.run_cpu("oracle", prob, dtype, option=opt, trace=True)
    n = prob["nbd"].size
    xp = 1e-19 * np.random.default_rng(1).standard_normal(n)
    b = B.run_cpu("oracle", prob, dtype, x0=xp, option=opt, trace=True)
    k = 0
    worst = 0.0
    for ra, rb in zip(a.trace, b.trace):
        if any(ra[key] != rb[key] for key in TRACE_KEYS):
            break
        worst = max(worst, abs(ra["f"] - rb["f"]) / max(1.0, abs(ra["f"])))
        k += 1
    assert k >= 90
    assert worst > 1e-8


def _config0(opt_over=None):
    import synth
    prob = synth.synth_problem(256, seed=0)
    prob["kind"] = "synth"
    opt = B.default_option(np.float64)
    opt.eps_f = opt.eps_g = opt.eps_x = 1e-8
    opt.max_iteration = 1000
    return prob, opt


@pytest.mark.skipif(not B.ref_available(), reason="reference build not present")
def test_oracle_matches_live_reference_config0():
    """The full config-0 solve (s = 256, FP64, eps 1e-8), oracle against the reference
    build: every evaluation, every summary and the final x bit for bit."""
    prob, opt = _config0()
    a = B.run_cpu("ref", prob, np.float64, option=opt)
    b = B.run_cpu("oracle", prob, np.float64, option=opt)
    assert a.evals == b.evals
    assert a.iters == b.iters
    np.testing.assert_array_equal(a.x, b.x)
    assert a.info == b.info


def test_config0_sensitivity():
    """The conditioning behind the GPU tolerance of the config-0 solve: moving x0 = 0 by
    1e-19 keeps the oracle's discrete trace for at least 100 iterations, and the run then
    stops on the f-test at a final f more than 1e-6 (relative) away."""
    prob, opt = _config0()
    a = B.run_cpu("oracle", prob, np.float64, option=opt, trace=True)
    xp = 1e-19 * np.random.default_rng(1).standard_normal(prob["nbd"].size)
    b = B.run_cpu("oracle", prob, np.float64, x0=xp, option=opt, trace=True)
    k = 0
    for ra, rb in zip(a.trace, b.trace):
        if any(ra[key] != rb[key] for key in TRACE_KEYS):
            break
        k += 1
    assert k >= 100
    fa, fb = a.trace[-1]["f"], b.trace[-1]["f"]
    assert abs(fa - fb) / abs(fa) > 1e-6


# ---- dsscfg, the reference's own example objective ----------------------------------

def _dsscfg_eval(prob, dtype, source, x):
    import ctypes as C
    real = C.c_double if dtype == np.float64 else C.c_float
    f = real()
    g = np.zeros(x.size, dtype)
    xx = x.copy()
    B.host_objective(prob, dtype, source)(xx.ctypes.data_as(C.POINTER(real)), C.byref(f),
                                          g.ctypes.data_as(C.POINTER(real)))
    return f.value, g


@pytest.mark.skipif(not B.ref_available(), reason="reference build not present")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_dsscfg_objective_matches_reference(dtype):
    """oracle/objective.c's dsscfg against examples/dsscfg/dsscfg_cpu.cpp compiled from the
    reference: the start point, f and every gradient entry bit for bit, on 60 random
    points per grid (three grid shapes, values over four scales)."""
    for nx, ny in ((7, 5), (31, 47), (64, 64)):
        prob = B.dsscfg_problem(nx, ny, 1.0)
        np.testing.assert_array_equal(B.dsscfg_start(prob, dtype, "oracle"),
                                      B.dsscfg_start(prob, dtype, "ref"))
        for trial in range(20):
            rng = np.random.default_rng(100 + trial)
            x = (rng.random(nx * ny) * [0.01, 0.3, 1.0, 3.0][trial % 4]).astype(dtype)
            fa, ga = _dsscfg_eval(prob, dtype, "oracle", x)
            fb, gb = _dsscfg_eval(prob, dtype, "ref", x)
            assert fa == fb
            np.testing.assert_array_equal(ga, gb)


@pytest.mark.parametrize("nx,dtype,iters,evals,fmin", [
    (64, np.float64, 163, 169, -0.990070631538),
    (256, np.float64, 531, 550, -1.01129586297),
    (256, np.float32, 333, 354, -1.01110565662)])
def test_dsscfg_known_answers(nx, dtype, iters, evals, fmin):
    """The reference's own runs of its dsscfg example (lambda = 1, unbounded, standard
    start, eps 1e-8, 1000 iterations at most): iterations, evaluations and the smallest f
    seen (printed to 12 digits), reproduced by the oracle."""
    prob = B.dsscfg_problem(nx, nx, 1.0)
    opt = B.default_option(dtype)
    opt.eps_f = opt.eps_g = opt.eps_x = 1e-8
    opt.max_iteration = 1000
    r = B.run_cpu("oracle", prob, dtype, x0=B.dsscfg_start(prob, dtype), option=opt)
    assert r.info == 1 and r.num_iteration == iters and len(r.evals) == evals
    assert f"{min(e[0] for e in r.evals):.12g}" == f"{fmin:.12g}"


@pytest.mark.skipif(not B.ref_available(), reason="reference build not present")
@pytest.mark.parametrize("dtype,bounds", [(np.float64, None), (np.float32, None),
                                          (np.float64, (0.0, 0.25)), (np.float32, (0.0, 0.25))])
def test_dsscfg_solve_matches_reference(dtype, bounds):
    """64 x 64 dsscfg solves, unbounded and with 0 <= x <= 0.25: the reference build with
    its own objective against the oracle with objective.c, every evaluation bit for bit."""
    prob = B.dsscfg_problem(64, 64, 1.0, bounds)
    opt = B.default_option(dtype)
    opt.eps_f = opt.eps_g = opt.eps_x = 1e-8
    opt.max_iteration = 1000
    x0 = B.dsscfg_start(prob, dtype, "ref")
    a = B.run_cpu("ref", prob, dtype, x0=x0, option=opt, objective_source="ref")
    b = B.run_cpu("oracle", prob, dtype, x0=x0, option=opt)
    assert a.evals == b.evals and a.iters == b.iters and a.info == b.info
    np.testing.assert_array_equal(a.x, b.x)


def test_dsscfg_256_sensitivity():
    """The conditioning behind the GPU bound on the 256 x 256 dsscfg solve: starting from
    the standard x0 moved by 1e-15 relative, the oracle's smallest f differs from the
    unperturbed run's by more than 5e-8 relative."""
    prob = B.dsscfg_problem(256, 256)
    x0 = B.dsscfg_start(prob, np.float64)
    opt = B.default_option(np.float64)
    opt.eps_f = opt.eps_g = opt.eps_x = 1e-8
    opt.max_iteration = 1000
    a = B.run_cpu("oracle", prob, np.float64, x0=x0, option=opt)
    xp = x0 * (1 + 1e-15 * np.random.default_rng(1).standard_normal(x0.size))
    b = B.run_cpu("oracle", prob, np.float64, x0=xp, option=opt)
    fa = min(e[0] for e in a.evals)
    fb = min(e[0] for e in b.evals)
    assert abs(fa - fb) / abs(fa) > 5e-8
