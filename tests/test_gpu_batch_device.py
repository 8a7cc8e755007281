"""Batched device-driven solves (lbfgsb_b200_minimize_batch_device_*): many instances of
different sizes advanced by one launch per pass.

* the device generator of the batch's problems gives synth.py's fields bit for bit;
* an instance's result is the same alone and in the mix (bit for bit: it runs the same
  launches on its own reduction rows, whatever else is in the batch);
* the batched solves reach the single-instance solves' minima and the oracle's (the
  reductions are grouped differently, so the iterates agree to rounding level only: final f
  within 1e-6 relative in FP64, 1e-5 in FP32).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def LB():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lbfgsb_b200
    lbfgsb_b200.load()
    return lbfgsb_b200


def _download(LB, ptr, count, dtype):
    out = np.empty(count, dtype=dtype)
    assert LB.load().lbfgsb_b200_copy(out.ctypes.data, C.c_void_p(ptr), out.nbytes, 2) == 0
    return out


def test_device_generator_matches_host(LB):
    import synth
    sides, seeds = [16, 33, 64], [3, 11, 12345]
    bt = LB.SynthBatch(sides, seeds, single_precision_fields=False, dtype=np.float64)
    for p, (s, seed) in enumerate(zip(sides, seeds)):
        ref = synth.synth_problem(s, seed=seed)
        l, u, nbd, fields = bt.problem(p)
        n = s * s
        for name, ptr in zip(("kappa", "w", "t", "b"), fields):
            np.testing.assert_array_equal(_download(LB, ptr, n, np.float64), ref[name])
        np.testing.assert_array_equal(_download(LB, nbd, n, np.int32), ref["nbd"])
        np.testing.assert_array_equal(_download(LB, l, n, np.float64), ref["l"])
        np.testing.assert_array_equal(_download(LB, u, n, np.float64), ref["u"])
    bt.close()


def _batch(LB, sides, seeds, dtype, form=0, ids=None, eps_g=1e-6, max_iteration=500):
    import torch
    bt = LB.SynthBatch(sides, seeds, single_precision_fields=(dtype == np.float32), dtype=dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    ids = list(range(len(sides))) if ids is None else ids
    xs = [torch.zeros(sides[p] * sides[p], dtype=tdt, device="cuda") for p in ids]
    opt = LB.default_option(dtype)
    opt.eps_g = eps_g
    opt.max_iteration = max_iteration
    rc, stat, summ, stats = LB.solve_batch_device(bt, xs, opt, form=form, ids=ids)
    torch.cuda.synchronize()
    assert rc == 0, LB.load().lbfgsb_b200_last_error()
    assert all(s == 0 for s in stat)
    out = [(x.cpu().numpy(), sm.info, sm.num_iteration, float(sm.residual_g)) for x, sm in zip(xs, summ)]
    bt.close()
    return out, stats


SIDES = [16, 23, 32, 40, 47, 64, 17, 30, 55, 64]
SEEDS = [101 + k for k in range(len(SIDES))]


@pytest.mark.parametrize("dtype,form", [(np.float32, 0), (np.float32, 1), (np.float64, 0)])
def test_same_alone_and_in_the_mix(LB, dtype, form):
    mix, stats = _batch(LB, SIDES, SEEDS, dtype, form=form)
    assert stats["rounds"] > 0 and stats["total_launches"] > 0
    for p in (0, 4, 8):
        alone, _ = _batch(LB, SIDES, SEEDS, dtype, form=form, ids=[p])
        xa, info_a, it_a, g_a = alone[0]
        xm, info_m, it_m, g_m = mix[p]
        assert (info_a, it_a, g_a) == (info_m, it_m, g_m)
        np.testing.assert_array_equal(xa, xm)


def test_batch_reaches_single_solve_and_oracle_minima(LB):
    import synth
    from oracle import binding as OB
    sides, seeds = [16, 24, 32], [7, 8, 9]
    res, _ = _batch(LB, sides, seeds, np.float64, eps_g=1e-8)
    for (x, info, it, _), s, seed in zip(res, sides, seeds):
        prob = synth.synth_problem(s, seed=seed)
        o = LB.default_option(np.float64)
        o.eps_f = o.eps_g = o.eps_x = 1e-8
        single = LB.solve(prob, np.float64, option=o, objective="device", record=False)
        oo = OB.default_option(np.float64)
        oo.eps_f = oo.eps_g = oo.eps_x = 1e-8
        orc = OB.run_cpu("oracle", dict(prob, kind="synth"), np.float64, option=oo, record=False)
        fb = LB.synth_value(prob, x)
        fs = LB.synth_value(prob, single.x)
        fo = LB.synth_value(prob, orc.x)
        assert info in (1, 2, 4), info
        assert abs(fb - fs) <= 1e-6 * max(1.0, abs(fs)), (fb, fs)
        assert abs(fb - fo) <= 1e-6 * max(1.0, abs(fo)), (fb, fo)


def test_batch_f32_reaches_fp64_minima(LB):
    import synth
    sides, seeds = [20, 36], [31, 32]
    res32, _ = _batch(LB, sides, seeds, np.float32)
    res64, _ = _batch(LB, sides, seeds, np.float64, eps_g=1e-8)
    for (x32, *_), (x64, *_), s, seed in zip(res32, res64, sides, seeds):
        prob = synth.synth_problem(s, seed=seed)
        f32 = LB.synth_value(prob, x32.astype(np.float64))
        f64 = LB.synth_value(prob, x64)
        assert abs(f32 - f64) <= 1e-5 * max(1.0, abs(f64)), (f32, f64)
