"""Named parity cases shared by the golden-fixture generator and the tests.

Each case is a bounded (or unbounded) problem from lbfgsb-gpu_b200/synth.py or a separable
quadratic, with the option overrides and the start point that exercise one behaviour of
the reference's CPU path (culbfgsb/lbfgsbcpu.cpp): breakpoint walks, ties, zero gradients,
nbd = 1/3 variables, l == u variables, projection of an infeasible start, ring sizes
m < 8, the iteration limit, the user stopping callback and the input-validation errors.
"""
from __future__ import annotations

import os
import sys

import numpy as np

_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
_PKG = os.path.join(_REPO, "lbfgsb-gpu_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)
import synth  # noqa: E402


def _synth(s, seed=1, bound=1.0, nbd_mix=True):
    p = synth.synth_problem(s, seed=seed, nbd_mix=nbd_mix)
    p["l"] = p["l"] * bound
    p["u"] = p["u"] * bound
    p["kind"] = "synth"
    return p


def _quad(n, a, c, l, u, nbd):
    return {"kind": "quad", "s": 0, "a": np.asarray(a, float), "c": np.asarray(c, float),
            "l": np.asarray(l, float), "u": np.asarray(u, float),
            "nbd": np.asarray(nbd, np.int32)}


def make_case(name: str):
    """Return (problem, dtype, x0 or None, option overrides dict, custom_stop_at)."""
    f64, f32 = np.float64, np.float32
    tight = {"eps_f": 1e-8, "eps_g": 1e-8, "eps_x": 1e-8}
    if name == "synth_s16_f64":
        return _synth(16), f64, None, tight, None
    if name == "synth_s32_f64":
        return _synth(32), f64, None, tight, None
    if name == "synth_s32_f32":
        return _synth(32), f32, None, tight, None
    if name == "synth_s32_f64_b005":
        return _synth(32, seed=2, bound=0.05), f64, None, tight, None
    if name == "synth_s32_f32_b002":
        return _synth(32, seed=3, bound=0.02), f32, None, tight, None
    if name == "synth_s24_f64_b001_m5":
        return _synth(24, seed=4, bound=0.01), f64, None, dict(tight, hessian_approximate_dimension=5), None
    if name == "synth_s20_f64_unbounded":
        p = _synth(20, seed=5)
        p["nbd"][:] = 0
        return p, f64, None, tight, None
    if name == "synth_s20_f64_boxed":
        return _synth(20, seed=6, bound=0.02, nbd_mix=False), f64, None, tight, None
    if name == "synth_s20_f64_nbd13":
        p = _synth(20, seed=7, bound=0.02)
        r = np.arange(p["nbd"].size)
        p["nbd"][r % 5 == 1] = 3
        p["nbd"][r % 7 == 2] = 1
        return p, f64, None, tight, None
    if name == "synth_s20_f64_fixedeq":
        p = _synth(20, seed=8, bound=0.02)
        r = np.arange(p["nbd"].size)
        sel = r % 9 == 4
        p["nbd"][sel] = 2
        p["l"][sel] = 0.003
        p["u"][sel] = 0.003
        return p, f64, None, tight, None
    if name == "synth_s20_f64_x0out":
        p = _synth(20, seed=9, bound=0.02)
        x0 = 0.05 * np.sin(np.arange(p["nbd"].size) * 0.7)
        return p, f64, x0, tight, None
    if name == "synth_s32_f64_maxit7":
        return _synth(32, seed=10, bound=0.02), f64, None, dict(tight, max_iteration=7), None
    if name == "synth_s16_f64_custom3":
        return _synth(16, seed=11), f64, None, tight, 3
    if name == "synth_s64_f64_b001":
        return _synth(64, seed=1, bound=0.01), f64, None, tight, None
    if name == "synth_s64_f32_b002":
        return _synth(64, seed=1, bound=0.02), f32, None, tight, None
    if name in ("quad_ties_f64", "quad_ties_f32"):
        n = 64
        k = np.arange(n)
        a = np.where(k % 2 == 0, 1.0, 3.0)
        c = np.where(k % 3 == 0, 2.0, -1.5)
        l = np.full(n, -0.5)
        u = np.full(n, 0.5)
        nbd = np.full(n, 2, np.int32)
        nbd[k % 8 == 5] = 0
        return _quad(n, a, c, l, u, nbd), (f64 if name.endswith("64") else f32), None, tight, None
    if name == "quad_zero_grad_f64":
        n = 48
        k = np.arange(n)
        x0 = 0.1 * np.cos(k)
        a = 1.0 + 0.1 * (k % 5)
        c = np.where(k % 4 == 0, x0, 0.8 * np.sin(3.0 * k))
        return _quad(n, a, c, np.full(n, -0.3), np.full(n, 0.3), np.full(n, 2, np.int32)), f64, x0, tight, None
    if name in ("quad_walk_many_f64", "quad_walk_many_f32"):
        # ~3000 breakpoints are passed by the first Cauchy step (more than one 1024-chunk of
        # the device walk), then the walk stops inside the remaining segment
        n = 4096
        k = np.arange(n)
        far = k % 4 != 3
        sign = np.where(k % 2 == 0, 1.0, -1.0)
        c = np.where(far, 3.0 * sign * (1.0 + k / n), 0.5 * sign)
        a = 1.0 + 0.25 * ((k * 7) % 5)
        return (_quad(n, a, c, np.full(n, -1.0), np.full(n, 1.0), np.full(n, 2, np.int32)),
                (f64 if name.endswith("64") else f32), None, tight, None)
    if name == "err_nbd4":
        p = _synth(4)
        p["nbd"][3] = 4
        return p, f64, None, tight, None
    if name == "err_l_gt_u":
        p = _synth(4)
        p["nbd"][5] = 2
        p["l"][5] = 0.5
        p["u"][5] = -0.5
        return p, f64, None, tight, None
    if name == "err_n_lt_m":
        p = _quad(4, np.ones(4), np.zeros(4), -np.ones(4), np.ones(4), np.full(4, 2, np.int32))
        return p, f64, None, tight, None
    raise KeyError(name)


CASES = [
    "synth_s16_f64", "synth_s32_f64", "synth_s32_f32", "synth_s32_f64_b005",
    "synth_s32_f32_b002", "synth_s24_f64_b001_m5", "synth_s20_f64_unbounded",
    "synth_s20_f64_boxed", "synth_s20_f64_nbd13", "synth_s20_f64_fixedeq",
    "synth_s20_f64_x0out", "synth_s32_f64_maxit7", "synth_s16_f64_custom3",
    "synth_s64_f64_b001", "synth_s64_f32_b002", "quad_ties_f64", "quad_ties_f32",
    "quad_zero_grad_f64", "quad_walk_many_f64", "quad_walk_many_f32", "err_nbd4",
    "err_l_gt_u", "err_n_lt_m",
]


def apply_options(opt, overrides: dict):
    for k, v in overrides.items():
        setattr(opt, k, v)
    return opt
