"""The serving front end (lbfgsb_b200_server_*): FP32 solves submitted one by one, admitted
in arrival order within an HBM budget and run on worker streams.

Every request must give exactly the x, exit code, iteration count and residuals of the
same solve run alone through lbfgsb_b200_minimize_ext_f32 with the server's precision
form; a budget that holds one solve's workspace at a time must admit one solve at a time
and still give the same results; a request whose workspace exceeds the whole budget is
refused at submit.  The workspace bound is host arithmetic and is checked without a GPU.
"""
import ctypes as C

import numpy as np
import pytest

SIDES = [16, 40, 64, 90, 128, 160]


def _lib():
    import lbfgsb_b200
    return lbfgsb_b200


def test_workspace_bound_covers_the_solve_arrays():
    LB = _lib()
    lib = LB.load()
    assert lib.lbfgsb_b200_workspace_bytes(0, 4, 1) == 0
    assert lib.lbfgsb_b200_workspace_bytes(100, 3, 1) == 0
    prev = 0
    for n in (1, 1000, 65536, 4194304):
        for real, form, hist in ((4, 1, 4), (4, 2, 2), (8, 0, 8)):
            b = lib.lbfgsb_b200_workspace_bytes(n, real, form)
            # six n-vectors of reals and the two history rings of 9 slots at least
            assert b >= n * 6 * real + 2 * 9 * n * hist
        b = lib.lbfgsb_b200_workspace_bytes(n, 4, 1)
        assert b > prev
        prev = b
    assert lib.lbfgsb_b200_workspace_bytes(4096, 4, 2) < lib.lbfgsb_b200_workspace_bytes(4096, 4, 1)


def test_server_calls_reject_bad_arguments():
    LB = _lib()
    lib = LB.load()
    opt = LB.default_option(np.float32)
    rid = C.c_longlong(-1)
    assert lib.lbfgsb_b200_server_submit_f32(None, 10, None, None, None, None, C.byref(opt),
                                             None, None, C.byref(rid)) == 1
    assert rid.value == -1
    summ = LB.SummaryF32()
    st = C.c_int(-5)
    lat = C.c_double()
    q = C.c_double()
    assert lib.lbfgsb_b200_server_wait(None, 0, C.byref(summ), C.byref(st), C.byref(lat),
                                       C.byref(q)) == 1
    assert lib.lbfgsb_b200_server_peak(None, None, None) == 1
    assert lib.lbfgsb_b200_server_destroy(None) == 1
    h = C.c_void_p()
    # a bad precision form or a null out-pointer is refused before any device call
    assert lib.lbfgsb_b200_server_create(2, 1 << 30, 7, C.byref(h)) == 1 and not h.value
    assert lib.lbfgsb_b200_server_create(2, 1 << 30, 1, None) == 1


def _setup(dtype=np.float32):
    import torch
    import synth
    LB = _lib()
    probs = [synth.synth_problem(s, seed=70 + i) for i, s in enumerate(SIDES)]
    for p in probs:
        p["l"] = p["l"] * 0.05
        p["u"] = p["u"] * 0.05
    objs = [LB.SynthObjective(p, single_precision_fields=True) for p in probs]
    dev = [dict(l=torch.from_numpy(p["l"].astype(dtype)).cuda(),
                u=torch.from_numpy(p["u"].astype(dtype)).cuda(),
                nbd=torch.from_numpy(p["nbd"]).cuda()) for p in probs]
    opt = LB.default_option(dtype)
    opt.eps_f = opt.eps_g = opt.eps_x = 1e-6
    opt.max_iteration = 150
    return probs, objs, dev, opt


def _solo(LB, lib, p, d, opt, obj, form):
    import torch
    x = torch.zeros(p["nbd"].size, dtype=torch.float32, device="cuda")
    s1 = LB.SummaryF32()
    ext = LB.Ext(form, 0, LB.TRACE_CB(), None)
    st = lib.lbfgsb_b200_minimize_ext_f32(p["nbd"].size, x.data_ptr(), d["nbd"].data_ptr(),
                                          d["l"].data_ptr(), d["u"].data_ptr(), C.byref(opt),
                                          obj.f32, None, None, obj.handle, None, C.byref(ext),
                                          C.byref(s1))
    torch.cuda.synchronize()
    assert st == 0
    return x, s1


@pytest.mark.gpu
@pytest.mark.parametrize("budget_kind", ["wide", "one_at_a_time"])
def test_server_results_equal_solo_solves(budget_kind):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    LB = _lib()
    lib = LB.load()
    probs, objs, dev, opt = _setup()
    form = LB.FORM_MIXED
    sizes = [lib.lbfgsb_b200_workspace_bytes(p["nbd"].size, 4, form) for p in probs]
    budget = 150 * 10**9 if budget_kind == "wide" else max(sizes) + min(sizes) // 2
    sv = LB.Server(workers=4, hbm_budget_bytes=budget, form=form)
    try:
        xs = [torch.zeros(p["nbd"].size, dtype=torch.float32, device="cuda") for p in probs]
        torch.cuda.synchronize()
        ids = []
        for k, p in enumerate(probs):
            rc, rid = sv.submit(p["nbd"].size, xs[k], dev[k]["nbd"], dev[k]["l"], dev[k]["u"],
                                opt, objs[k].f32, objs[k].handle)
            assert rc == 0
            ids.append(rid)
        results = [sv.wait(rid) for rid in ids]
        peak_bytes, peak_running = sv.peak()
    finally:
        sv.close()
    torch.cuda.synchronize()
    assert peak_bytes <= budget
    if budget_kind == "one_at_a_time":
        assert peak_running == 1
    else:
        assert peak_running >= 1
    for k, p in enumerate(probs):
        st, b, lat, q = results[k]
        assert st == 0, k
        assert lat >= q >= 0.0
        x1, s1 = _solo(LB, lib, p, dev[k], opt, objs[k], form)
        assert (b.info, b.num_iteration) == (s1.info, s1.num_iteration), k
        assert (b.residual_g, b.residual_f, b.residual_x) == (s1.residual_g, s1.residual_f,
                                                               s1.residual_x), k
        assert torch.equal(xs[k], x1), k
    for o in objs:
        o.close()


@pytest.mark.gpu
def test_server_refuses_a_request_beyond_its_budget():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    LB = _lib()
    lib = LB.load()
    probs, objs, dev, opt = _setup()
    small = lib.lbfgsb_b200_workspace_bytes(probs[0]["nbd"].size, 4, LB.FORM_MIXED)
    sv = LB.Server(workers=2, hbm_budget_bytes=small, form=LB.FORM_MIXED)
    try:
        big = len(probs) - 1
        x = torch.zeros(probs[big]["nbd"].size, dtype=torch.float32, device="cuda")
        rc, _ = sv.submit(probs[big]["nbd"].size, x, dev[big]["nbd"], dev[big]["l"],
                          dev[big]["u"], opt, objs[big].f32, objs[big].handle)
        assert rc == 1 and "budget" in lib.lbfgsb_b200_last_error().decode()
        x0 = torch.zeros(probs[0]["nbd"].size, dtype=torch.float32, device="cuda")
        rc, rid = sv.submit(probs[0]["nbd"].size, x0, dev[0]["nbd"], dev[0]["l"], dev[0]["u"],
                            opt, objs[0].f32, objs[0].handle)
        assert rc == 0
        st, _, _, _ = sv.wait(rid)
        assert st == 0
    finally:
        sv.close()
    for o in objs:
        o.close()
