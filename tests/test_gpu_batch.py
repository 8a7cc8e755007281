"""Batched independent solves (lbfgsb_b200_minimize_batch_*): ten synthetic bounded grid
problems of different sizes (n from 256 to 90,000) solved side by side on four worker
streams must give, instance by instance, exactly the x, exit code, iteration count and
residuals of the same problem solved alone."""
import ctypes as C

import numpy as np
import pytest

SIDES = [16, 33, 48, 64, 100, 127, 128, 200, 256, 300]


def _lib():
    import lbfgsb_b200
    return lbfgsb_b200


def test_batch_rejects_null_arguments():
    LB = _lib()
    lib = LB.load()
    opt = LB.default_option(np.float64)
    summ = (LB.SummaryF64 * 1)()
    stat = (C.c_int * 1)()
    rc = lib.lbfgsb_b200_minimize_batch_f64(1, None, None, None, None, None, C.byref(opt), None,
                                            None, 2, summ, stat, None)
    assert rc == 1 and "null" in lib.lbfgsb_b200_last_error().decode()
    assert lib.lbfgsb_b200_minimize_batch_f64(0, None, None, None, None, None, C.byref(opt),
                                              None, None, 2, summ, stat, None) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_batch_equals_solo_solves(dtype):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import synth
    LB = _lib()
    lib = LB.load()
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    probs = [synth.synth_problem(s, seed=40 + i) for i, s in enumerate(SIDES)]
    for p in probs:
        p["l"] = p["l"] * 0.05
        p["u"] = p["u"] * 0.05
    objs = [LB.SynthObjective(p, single_precision_fields=dtype == np.float32) for p in probs]
    dev = [dict(x=torch.zeros(p["nbd"].size, dtype=tdt, device="cuda"),
                l=torch.from_numpy(p["l"].astype(dtype)).cuda(),
                u=torch.from_numpy(p["u"].astype(dtype)).cuda(),
                nbd=torch.from_numpy(p["nbd"]).cuda()) for p in probs]
    opt = LB.default_option(dtype)
    opt.eps_f = opt.eps_g = opt.eps_x = 1e-8
    opt.max_iteration = 200
    fg = objs[0].f64 if dtype == np.float64 else objs[0].f32
    rc, stat, summ, secs = LB.solve_batch([p["nbd"].size for p in probs], [d["x"] for d in dev],
                                          [d["nbd"] for d in dev], [d["l"] for d in dev],
                                          [d["u"] for d in dev], opt, fg,
                                          [o.handle for o in objs], concurrency=4, dtype=dtype)
    torch.cuda.synchronize()
    assert rc == 0 and stat == [0] * len(probs)
    fn = lib.lbfgsb_b200_minimize_f64 if dtype == np.float64 else lib.lbfgsb_b200_minimize_f32
    for k, p in enumerate(probs):
        x = torch.zeros(p["nbd"].size, dtype=tdt, device="cuda")
        s1 = LB.SummaryF64() if dtype == np.float64 else LB.SummaryF32()
        st = fn(p["nbd"].size, x.data_ptr(), dev[k]["nbd"].data_ptr(), dev[k]["l"].data_ptr(),
                dev[k]["u"].data_ptr(), C.byref(opt), fg, None, None, objs[k].handle, None,
                C.byref(s1))
        torch.cuda.synchronize()
        assert st == 0
        b = summ[k]
        assert (b.info, b.num_iteration) == (s1.info, s1.num_iteration), k
        assert (b.residual_g, b.residual_f, b.residual_x) == (s1.residual_g, s1.residual_f,
                                                               s1.residual_x), k
        assert torch.equal(dev[k]["x"], x), k
        assert secs[k] > 0
    for o in objs:
        o.close()
