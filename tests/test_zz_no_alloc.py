"""lbfgsb_b200_projgr_noalloc_f64: the projected-gradient norm with static scratch.

It must give what the existing entry point reports: inside the after-iteration callback of
lbfgsb_b200_minimize_f64 (a caller that must not allocate) it is called on every iterate,
and each value must equal, bit for bit, the summary.residual_g that the next callback sees
(the reference calls after_iteration before that iteration's projgr,
culbfgsb/lbfgsbcpu.cpp:388-395).  Called directly, two calls in a row on different sizes
must match a numpy restatement of projgr exactly, and at the largest size the scratch
holds (n = 2^25, 8192 CTAs) a batch of calls must leave the device's free memory and the
caching allocator's reserve unchanged.  Sizes beyond the static scratch are rejected before
any CUDA call.
"""
import ctypes as C

import numpy as np
import pytest

MAX_N = 1 << 25


@pytest.fixture(scope="module")
def LB():
    import lbfgsb_b200
    lbfgsb_b200.load()
    return lbfgsb_b200


def projgr_np(x, g, nbd, l, u):
    """culbfgsb/lbfgsbcpu.cpp:1390-1415 elementwise (exact in IEEE double)."""
    pg = g.copy()
    neg = g < 0
    hi = neg & (nbd != 0) & (nbd >= 2)
    lo = ~neg & (nbd != 0) & (nbd <= 2)
    du = x - u
    dl = x - l
    pg[hi] = np.where(du[hi] > g[hi], du[hi], g[hi])
    pg[lo] = np.where(dl[lo] < g[lo], dl[lo], g[lo])
    return float(np.max(np.abs(pg), initial=0.0))


def test_rejects_sizes_beyond_the_scratch(LB):
    lib = LB.load()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    for n in (MAX_N + 1, 1 << 30, -1):
        st = lib.lbfgsb_b200_projgr_noalloc_f64(n, dummy, dummy, dummy, dummy, dummy, dummy, None)
        assert st == 1  # LBFGSB_B200_ERR_ARGUMENT
        msg = lib.lbfgsb_b200_last_error().decode()
        assert "33554432" in msg and str(n) in msg
    st = lib.lbfgsb_b200_projgr_noalloc_f64(10, None, dummy, dummy, dummy, dummy, dummy, None)
    assert st == 1 and "null" in lib.lbfgsb_b200_last_error().decode()


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
def test_two_direct_calls_in_a_row(LB):
    torch = _cuda()
    lib = LB.load()
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(5)
    want = []
    keep = []
    for k, n in enumerate((3 * 4096 * 37 + 123, 5000)):
        x = rng.standard_normal(n)
        g = rng.standard_normal(n)
        l = x - np.abs(rng.standard_normal(n)) * (rng.random(n) < 0.7)  # some x on l
        u = x + np.abs(rng.standard_normal(n)) * (rng.random(n) < 0.7)
        nbd = rng.integers(0, 4, n).astype(np.int32)
        want.append(projgr_np(x, g, nbd, l, u))
        dev = [torch.from_numpy(a).cuda() for a in (x, g, nbd, l, u)]
        keep.append(dev)
        st = lib.lbfgsb_b200_projgr_noalloc_f64(n, *[t.data_ptr() for t in dev],
                                                out.data_ptr() + 8 * k, None)
        assert st == 0, lib.lbfgsb_b200_last_error()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert got[0] == want[0] and got[1] == want[1]


@pytest.mark.gpu
def test_matches_solver_residual_g_inside_callbacks(LB):
    """A solve on a 192 x 192 bounded grid (9 CTAs of the no-alloc kernel)."""
    torch = _cuda()
    import synth
    lib = LB.load()
    prob = synth.synth_problem(192, seed=4)
    prob["l"] = prob["l"] * 0.05
    prob["u"] = prob["u"] * 0.05
    n = prob["nbd"].size
    dev = torch.device("cuda", 0)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    l = torch.from_numpy(prob["l"]).to(dev)
    u = torch.from_numpy(prob["u"]).to(dev)
    nbd = torch.from_numpy(prob["nbd"]).to(dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)   # allocated before the solve
    host = np.zeros(1)
    so = LB.SynthObjective(prob)
    seen = []   # (value from the no-alloc call at iterate k, residual_g seen at callback k)
    errors = []

    def after(_user, xp, _fp, gp, stream, sp):
        st = lib.lbfgsb_b200_projgr_noalloc_f64(n, C.cast(xp, C.c_void_p), C.cast(gp, C.c_void_p),
                                                nbd.data_ptr(), l.data_ptr(), u.data_ptr(),
                                                out.data_ptr(), stream)
        if st != 0:
            errors.append(lib.lbfgsb_b200_last_error())
            return 0
        lib.lbfgsb_b200_copy(host.ctypes.data, out.data_ptr(), 8, 2)  # blocking, no allocation
        seen.append((float(host[0]), float(sp[0].residual_g)))
        return 0

    cb = LB.CB64(after)
    opt = LB.default_option(np.float64)
    opt.eps_f = opt.eps_g = opt.eps_x = 0.0
    opt.max_iteration = 25
    summ = LB.SummaryF64()
    st = lib.lbfgsb_b200_minimize_f64(n, x.data_ptr(), nbd.data_ptr(), l.data_ptr(), u.data_ptr(),
                                      C.byref(opt), so.f64, C.cast(cb, C.c_void_p).value, None,
                                      so.handle, None, C.byref(summ))
    torch.cuda.synchronize()
    so.close()
    assert st == 0 and not errors, errors
    assert len(seen) >= 20
    for k in range(len(seen) - 1):
        assert seen[k][0] == seen[k + 1][1], f"iterate {k + 1}"
    assert seen[-1][0] == summ.residual_g
    assert seen[0][0] > 0.0


@pytest.mark.gpu
def test_largest_size_allocates_nothing(LB):
    torch = _cuda()
    lib = LB.load()
    n = MAX_N
    rng = np.random.default_rng(9)
    x = rng.standard_normal(n)
    g = rng.standard_normal(n)
    l = x - np.abs(rng.standard_normal(n)) * (rng.random(n) < 0.5)
    u = x + np.abs(rng.standard_normal(n)) * (rng.random(n) < 0.5)
    nbd = rng.integers(0, 4, n).astype(np.int32)
    want = projgr_np(x, g, nbd, l, u)
    dev = [torch.from_numpy(a).cuda() for a in (x, g, nbd, l, u)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    ptrs = [t.data_ptr() for t in dev]
    assert lib.lbfgsb_b200_projgr_noalloc_f64(n, *ptrs, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(10):
        assert lib.lbfgsb_b200_projgr_noalloc_f64(n, *ptrs, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0 and torch.cuda.memory_reserved() == reserved0
    assert float(out.cpu()[0]) == want
