"""Sharded solves (lbfgsb_b200_minimize_sharded_*): one problem split by index range over
several ranks, against the CPU oracle.

The ranks here are threads of one process on one GPU, each on its own stream, exchanging
their reduction rows through a host all-gather (lbfgsb_b200.ThreadAllGather): no kernel
waits on another rank's kernels, so the same kernels, exchanges and epilogues run as on
several GPUs, one rank per GPU.  The objective is the oracle's own host objective on the
whole x (rank 0 returns f, the others 0), so every difference from the oracle comes from
the solver.

Tolerances, as for single-GPU solves (the rank rows are folded in rank order, another
summation order than both the oracle's and the single-GPU solve's):
  FP64  the discrete per-iteration trace (breakpoints passed, free-set hash over global
        indices, entering / leaving counts, evaluations) equal to the oracle's for the
        whole run, f within 1e-10 relative at every iteration, the same exit code and
        iteration count, final x within 1e-6 of max|x|;
  FP32  the same exit code, the first 10 iterations' trace equal, final f within 1e-5.
"""
import numpy as np
import pytest

from cases import apply_options, make_case

pytestmark = pytest.mark.gpu

KEYS = ["nint", "nbreak", "nfree", "nenter", "nleave", "col", "head", "iword", "free_hash",
        "at_lower", "at_upper", "nfgv", "ifun"]


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


def run_pair(LB, OB, name, world, parts=None):
    prob, dt, x0, over, stop = make_case(name)
    assert x0 is None and stop is None
    a = OB.run_cpu("oracle", prob, dt, option=apply_options(OB.default_option(dt), over),
                   trace=True)
    b = LB.solve_sharded(prob, world, dt, option=apply_options(LB.default_option(dt), over),
                         trace=True, parts=parts)
    return a, b


def check_fp64(a, b):
    assert b.info == a.info and b.num_iteration == a.num_iteration
    assert len(a.trace) == len(b.trace)
    for ra, rb in zip(a.trace, b.trace):
        for k in KEYS:
            assert ra[k] == rb[k], (ra["iter"], k, ra[k], rb[k])
        rel = abs(ra["f"] - rb["f"]) / max(1.0, abs(ra["f"]))
        assert rel <= 1e-10, (ra["iter"], rel)
    scale = max(1.0, float(np.max(np.abs(a.x))))
    assert float(np.max(np.abs(a.x - b.x))) <= 1e-6 * scale
    # every rank ends with the same summary
    assert len(set(b.stats["ranks"])) == 1, b.stats["ranks"]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_bounded_walks(LB, OB, world):
    """A bounded problem with breakpoint walks and truncated subspace steps (s = 32, bounds
    +-0.05), 119 iterations; three ranks split 1024 variables 342 / 341 / 341, so no rank
    boundary falls on a tile boundary."""
    a, b = run_pair(LB, OB, "synth_s32_f64_b005", world)
    check_fp64(a, b)


def test_sharded_uneven_parts(LB, OB):
    """Ranks of very different sizes: one of 7 variables (fewer than m), one of 1000, one
    of 17."""
    a, b = run_pair(LB, OB, "synth_s32_f64_b005", 3, parts=[7, 1000, 17])
    check_fp64(a, b)


def test_sharded_long_walk(LB, OB):
    """A first Cauchy step that passes 3278 breakpoints: with two ranks every selection
    round takes at most 512 keys of each, so the walk runs several rounds and stops at a
    rank's frontier in between."""
    a, b = run_pair(LB, OB, "quad_walk_many_f64", 2)
    check_fp64(a, b)
    assert max(r["nint"] for r in b.trace) > 1024


@pytest.mark.parametrize("name", ["synth_s20_f64_boxed", "synth_s20_f64_nbd13",
                                  "synth_s20_f64_unbounded", "synth_s20_f64_fixedeq",
                                  "quad_ties_f64"])
def test_sharded_cases(LB, OB, name):
    a, b = run_pair(LB, OB, name, 2)
    check_fp64(a, b)


def test_sharded_fp32(LB, OB):
    a, b = run_pair(LB, OB, "synth_s32_f32_b002", 2)
    assert b.info == a.info
    for ra, rb in list(zip(a.trace, b.trace))[:10]:
        for k in KEYS:
            assert ra[k] == rb[k], (ra["iter"], k)
    fa, fb = a.trace[-1]["f"], b.trace[-1]["f"]
    assert abs(fa - fb) / max(1.0, abs(fa)) <= 1e-5


def test_sharded_input_errors(LB, OB):
    """errclb's checks run on every rank's variables and are combined: an nbd = 4 on one
    rank makes every rank return info = -1."""
    a, b = run_pair(LB, OB, "err_nbd4", 2)
    assert a.info == -1 and b.info == -1


def test_sharded_four_ranks(LB, OB):
    """s = 128 (n = 16,384, bounds +-0.05), four ranks of 4096 variables: several tiles and
    CTAs per rank; the first 40 iterations."""
    from cases import _synth
    prob = _synth(128, seed=12, bound=0.05)
    over = {"eps_f": 1e-8, "eps_g": 1e-8, "eps_x": 1e-8, "max_iteration": 40}
    a = OB.run_cpu("oracle", prob, np.float64, option=apply_options(OB.default_option(np.float64), over),
                   trace=True)
    b = LB.solve_sharded(prob, 4, np.float64,
                         option=apply_options(LB.default_option(np.float64), over), trace=True)
    check_fp64(a, b)


def test_sharded_mixed_form(LB, OB):
    """The mixed form (FP32 vectors and history, FP64 scalars) sharded over two ranks ends
    within 1e-5 of the same form on one GPU."""
    name = "synth_s32_f32_b002"
    prob, dt, x0, over, stop = make_case(name)
    opt = apply_options(LB.default_option(dt), over)
    one = LB.solve(prob, dt, option=opt, objective="host", form=LB.FORM_MIXED, trace=True)
    two = LB.solve_sharded(prob, 2, dt, option=apply_options(LB.default_option(dt), over),
                           form=LB.FORM_MIXED, trace=True)
    assert two.info == one.info
    fa, fb = one.trace[-1]["f"], two.trace[-1]["f"]
    assert abs(fa - fb) / max(1.0, abs(fa)) <= 1e-5


def test_one_rank_equals_plain_solve(LB):
    """A sharded solve of one rank splits every pass into the streaming launch and the
    one-CTA epilogue launch around an exchange of its own row: the iterates, the trace and
    the summary equal the plain solve's bit for bit."""
    prob, dt, x0, over, stop = make_case("synth_s32_f64_b005")
    a = LB.solve(prob, dt, option=apply_options(LB.default_option(dt), over), objective="host",
                 trace=True)
    b = LB.solve_sharded(prob, 1, dt, option=apply_options(LB.default_option(dt), over),
                         trace=True)
    assert (a.info, a.num_iteration) == (b.info, b.num_iteration)
    assert a.residual_g == b.residual_g and a.residual_f == b.residual_f
    assert np.array_equal(a.x, b.x)
    for ra, rb in zip(a.trace, b.trace):
        assert ra == rb, ra["iter"]
