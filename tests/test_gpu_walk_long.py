"""Long breakpoint walks: the first Cauchy steps of these tight-bound problems pass tens to
hundreds of thousands of breakpoints (the first iteration's nint: 54,757 and 217,112), many
chunks of the cooperative walk's grid-wide select.  FP64, the objective evaluated by the
oracle's code on the host: the trace of the first six iterations (breakpoints found and
passed, the free set, its hash, entering / leaving counts) must equal the oracle's and f
agree within 1e-10 relative; and the device-driven solve, whose rounds capture the
cooperative walk in a CUDA graph, must give the host-driven solve's result bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRACE_KEYS = ["nint", "nbreak", "nfree", "nenter", "nleave", "col", "head", "iword",
              "free_hash", "at_lower", "at_upper", "nfgv", "ifun"]
CASES = [(256, 1e-6, 54757), (512, 3e-7, 217112)]


@pytest.fixture(scope="module")
def LB():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lbfgsb_b200
    lbfgsb_b200.load()
    return lbfgsb_b200


def _prob(s, b):
    import synth
    p = dict(synth.synth_problem(s, seed=0), kind="synth")
    p["l"] = p["l"] * b
    p["u"] = p["u"] * b
    return p


def _opt(mod):
    o = mod.default_option(np.float64)
    o.eps_f = o.eps_g = o.eps_x = 0.0
    o.max_iteration = 5
    return o


@pytest.mark.parametrize("s,b,passed", CASES)
def test_long_walk_matches_oracle(LB, s, b, passed):
    from oracle import binding as OB
    prob = _prob(s, b)
    a = OB.run_cpu("oracle", prob, np.float64, option=_opt(OB), trace=True, record=False)
    r = LB.solve(prob, np.float64, option=_opt(LB), objective="host", trace=True, record=False)
    assert a.trace[0]["nint"] == passed  # the walk is as long as recorded above
    assert len(a.trace) == len(r.trace) == 6
    for ta, tb in zip(a.trace, r.trace):
        diff = {k: (ta[k], tb[k]) for k in TRACE_KEYS if ta[k] != tb[k]}
        assert not diff, (ta["iter"], diff)
        assert abs(ta["f"] - tb["f"]) <= 1e-10 * max(1.0, abs(ta["f"]))


@pytest.mark.parametrize("s,b,passed", CASES)
def test_long_walk_device_driven(LB, s, b, passed):
    prob = _prob(s, b)
    a = LB.solve(prob, np.float64, option=_opt(LB), objective="device", record=False)
    d = LB.solve(prob, np.float64, option=_opt(LB), objective="device", record=False, driven="device")
    assert (a.info, a.num_iteration) == (d.info, d.num_iteration)
    np.testing.assert_array_equal(a.x, d.x)
