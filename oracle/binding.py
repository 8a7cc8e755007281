"""ctypes binding of the CPU checkers (TEST INFRASTRUCTURE).

Used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm:
  * liboracle.so          -- the plain-C restatement of the reference CPU L-BFGS-B
                             (lbfgsb_oracle.c) with a per-iteration trace;
  * _ref/libref_lbfgsb.so -- the reference's own culbfgsb/lbfgsbcpu.cpp built from the
                             reference sources (Makefile here), the pin for the restatement.
Both run the synthetic objective of objective.c on host arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_lbfgsb.so")
DROPIN_EXE = os.path.join(HERE, "_ref", "dsscfg_dropin")


class SummaryF64(C.Structure):
    _fields_ = [("residual_g", C.c_double), ("residual_f", C.c_double),
                ("residual_x", C.c_double), ("num_iteration", C.c_int), ("info", C.c_int)]


class SummaryF32(C.Structure):
    _fields_ = [("residual_g", C.c_float), ("residual_f", C.c_float),
                ("residual_x", C.c_float), ("num_iteration", C.c_int), ("info", C.c_int)]


class OptionF64(C.Structure):
    _fields_ = [("machine_epsilon", C.c_double), ("machine_maximum", C.c_double),
                ("step_scaling", C.c_double), ("eps_g", C.c_double), ("eps_f", C.c_double),
                ("eps_x", C.c_double), ("hessian_approximate_dimension", C.c_int),
                ("max_iteration", C.c_int)]


class OptionF32(C.Structure):
    _fields_ = [("machine_epsilon", C.c_float), ("machine_maximum", C.c_float),
                ("step_scaling", C.c_float), ("eps_g", C.c_float), ("eps_f", C.c_float),
                ("eps_x", C.c_float), ("hessian_approximate_dimension", C.c_int),
                ("max_iteration", C.c_int)]


class TraceRec(C.Structure):
    _fields_ = [("iter", C.c_int), ("nint", C.c_int), ("nbreak", C.c_int), ("nfree", C.c_int),
                ("nenter", C.c_int), ("nleave", C.c_int), ("col", C.c_int), ("head", C.c_int),
                ("nfgv", C.c_int), ("ifun", C.c_int), ("iword", C.c_int), ("reset", C.c_int),
                ("free_hash", C.c_ulonglong), ("at_lower", C.c_ulonglong),
                ("at_upper", C.c_ulonglong), ("f", C.c_double), ("theta", C.c_double),
                ("stp", C.c_double), ("dtm", C.c_double), ("tsum", C.c_double),
                ("gd", C.c_double), ("gdold", C.c_double), ("dtd", C.c_double),
                ("stpmx", C.c_double), ("f1_0", C.c_double), ("f2_0", C.c_double),
                ("dbg", C.c_double * 8)]


CB64 = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                   C.POINTER(C.c_double), C.POINTER(SummaryF64))
CB32 = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                   C.POINTER(C.c_float), C.POINTER(SummaryF32))
TRACE_CB = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(TraceRec))

_TRACE_KEYS = [f for f, _ in TraceRec._fields_]


def build(reference_dir: str | None = None, quiet: bool = True) -> None:
    """Build liboracle.so, and the reference build when `reference_dir` (or the
    environment variable LBFGSB_REFERENCE_DIR) names a reference tree."""
    cmd = ["make", "-C", HERE, os.path.join(HERE, "liboracle.so")]
    subprocess.run(cmd, check=True, capture_output=quiet)
    ref_dir = reference_dir or os.environ.get("LBFGSB_REFERENCE_DIR")
    if ref_dir and os.path.isfile(os.path.join(ref_dir, "culbfgsb", "lbfgsbcpu.cpp")):
        subprocess.run(["make", "-C", HERE, "ref", f"REFERENCE_DIR={ref_dir}"], check=True,
                       capture_output=quiet)
        # the reference's dsscfg example program on this library's drop-in header (needs
        # the built library)
        lib = os.path.join(os.path.dirname(HERE), "lbfgsb-gpu_b200", "liblbfgsb_b200.so")
        if os.path.exists(lib):
            subprocess.run(["make", "-C", HERE, "dropin", f"REFERENCE_DIR={ref_dir}"],
                           check=True, capture_output=quiet)


_libs: dict[str, C.CDLL] = {}


def _load(path: str) -> C.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        _libs[path] = lib
    return _libs[path]


def oracle_lib() -> C.CDLL:
    lib = _load(ORACLE_SO)
    for sfx, opt, summ, cb in (("f64", OptionF64, SummaryF64, CB64),
                               ("f32", OptionF32, SummaryF32, CB32)):
        fn = getattr(lib, f"orc_lbfgsb_minimize_{sfx}")
        fn.restype = None
        real = C.c_double if sfx == "f64" else C.c_float
        fn.argtypes = [C.c_int, C.POINTER(real), C.POINTER(C.c_int), C.POINTER(real),
                       C.POINTER(real), C.POINTER(opt), cb, cb, cb, C.c_void_p, TRACE_CB,
                       C.c_void_p, C.POINTER(summ)]
    return lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib() -> C.CDLL:
    lib = _load(REF_SO)
    for sfx, opt, summ, cb in (("f64", OptionF64, SummaryF64, CB64),
                               ("f32", OptionF32, SummaryF32, CB32)):
        fn = getattr(lib, f"ref_lbfgsb_minimize_{sfx}")
        fn.restype = None
        real = C.c_double if sfx == "f64" else C.c_float
        fn.argtypes = [C.c_int, C.POINTER(real), C.POINTER(C.c_int), C.POINTER(real),
                       C.POINTER(real), C.POINTER(opt), cb, cb, cb, C.c_void_p,
                       C.POINTER(summ)]
    return lib


def default_option(dtype) -> C.Structure:
    """lbfgsbdefaultoption (culbfgsb/lbfgsb.cpp:43-66)."""
    if np.dtype(dtype) == np.float64:
        o = OptionF64(1e-15, np.finfo(np.float64).max, 1.0, 1e-15, 1e-15, 1e-15, 8, 1000)
    else:
        o = OptionF32(1e-8, np.finfo(np.float32).max, 1.0, 1e-15, 1e-15, 1e-15, 8, 1000)
    return o


@dataclass
class RunResult:
    x: np.ndarray
    info: int
    num_iteration: int
    residual_g: float
    residual_f: float
    residual_x: float
    evals: list = field(default_factory=list)    # (f, x-digest) at every funcgrad call
    iters: list = field(default_factory=list)    # summary at every after-iteration call
    trace: list = field(default_factory=list)    # oracle trace records (dicts)


def _digest(a: np.ndarray) -> str:
    import hashlib
    return hashlib.sha1(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def host_objective(prob: dict, dtype, source: str = "oracle"):
    """Host objective callback body for a problem dict: (xp, fp, gp) pointers -> fills f, g.

    prob["kind"] == "synth" (default): the grid objective of objective.c with fields
    kappa, w, t, b, minus the constant prob["f_offset"] when that is given; "quad": the
    separable quadratic with vectors a, c; "dsscfg": the
    steady-state combustion objective on an nx x ny grid with parameter lam, from
    objective.c (source "oracle") or from the reference's own example code (source
    "ref", the reference build)."""
    is64 = np.dtype(dtype) == np.float64
    real = C.c_double if is64 else C.c_float
    sfx = "f64" if is64 else "f32"
    kind = prob.get("kind", "synth")
    if kind == "dsscfg":
        lib = _load(ORACLE_SO if source == "oracle" else REF_SO)
        fn = getattr(lib, f"{'orc' if source == 'oracle' else 'ref'}_dsscfg_eval_{sfx}")
        fn.restype = None
        fn.argtypes = [C.c_int, C.c_int, real] + [C.POINTER(real)] * 3
        nx, ny, lam = int(prob["nx"]), int(prob["ny"]), float(prob["lam"])

        def evaluate_dsscfg(xp, fp, gp):
            fn(nx, ny, lam, xp, fp, gp)

        return evaluate_dsscfg
    lib = _load(ORACLE_SO)
    names = ("kappa", "w", "t", "b") if kind == "synth" else ("a", "c")
    arrs = [np.ascontiguousarray(prob[k], dtype=np.float64) for k in names]
    ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
    lead = int(prob["s"]) if kind == "synth" else int(prob["nbd"].size)
    f0 = float(prob.get("f_offset", 0.0))
    if kind == "synth" and f0 != 0.0:
        # f minus the constant f0, subtracted before f is rounded (objective.c)
        fn = getattr(lib, f"orc_synth_eval_off_{sfx}")
        fn.restype = None
        fn.argtypes = [C.c_int] + [C.POINTER(C.c_double)] * 4 + [C.c_double] + \
            [C.POINTER(real)] * 3

        def evaluate_off(xp, fp, gp):
            fn(lead, *ptrs, f0, xp, fp, gp)

        evaluate_off.keepalive = arrs  # type: ignore[attr-defined]
        return evaluate_off
    fn = getattr(lib, f"orc_{kind}_eval_{sfx}")
    fn.restype = None
    fn.argtypes = [C.c_int] + [C.POINTER(C.c_double)] * len(arrs) + [C.POINTER(real)] * 3

    def evaluate_ptr(xp, fp, gp):
        fn(lead, *ptrs, xp, fp, gp)

    evaluate_ptr.keepalive = arrs  # type: ignore[attr-defined]
    return evaluate_ptr


def dsscfg_problem(nx: int, ny: int, lam: float = 1.0, bounds=None) -> dict:
    """The reference example's problem: unbounded (nbd = 0, as dsscfg_main.cpp:66-80) or,
    with bounds=(lo, hi), nbd = 2 everywhere."""
    n = nx * ny
    p = {"kind": "dsscfg", "nx": nx, "ny": ny, "lam": lam, "s": 0}
    if bounds is None:
        p.update(l=np.zeros(n), u=np.zeros(n), nbd=np.zeros(n, np.int32))
    else:
        p.update(l=np.full(n, float(bounds[0])), u=np.full(n, float(bounds[1])),
                 nbd=np.full(n, 2, np.int32))
    return p


def dsscfg_start(prob: dict, dtype, source: str = "oracle") -> np.ndarray:
    """The standard start point ('XS') of the dsscfg problem."""
    is64 = np.dtype(dtype) == np.float64
    real = C.c_double if is64 else C.c_float
    lib = _load(ORACLE_SO if source == "oracle" else REF_SO)
    fn = getattr(lib, f"{'orc' if source == 'oracle' else 'ref'}_dsscfg_start_{'f64' if is64 else 'f32'}")
    fn.restype = None
    fn.argtypes = [C.c_int, C.c_int, real, C.POINTER(real)]
    x = np.zeros(int(prob["nx"]) * int(prob["ny"]), dtype=dtype)
    fn(int(prob["nx"]), int(prob["ny"]), float(prob["lam"]), x.ctypes.data_as(C.POINTER(real)))
    return x


def run_cpu(which: str, prob: dict, dtype=np.float64, x0=None, option=None, record=True,
            trace=False, custom_stop_at: int | None = None,
            objective_source: str = "oracle", subsm_projection: bool = False) -> RunResult:
    """Run the oracle ('oracle') or the reference build ('ref') on a synthetic problem.
    subsm_projection: the oracle's L-BFGS-B 3.0 subspace step (the reference has only 2.1)."""
    dtype = np.dtype(dtype)
    is64 = dtype == np.float64
    real = C.c_double if is64 else C.c_float
    cbt = CB64 if is64 else CB32
    summ = SummaryF64() if is64 else SummaryF32()
    n = prob["nbd"].size
    x = np.zeros(n, dtype=dtype) if x0 is None else np.array(x0, dtype=dtype)
    l = np.ascontiguousarray(prob["l"], dtype=dtype)
    u = np.ascontiguousarray(prob["u"], dtype=dtype)
    nbd = np.ascontiguousarray(prob["nbd"], dtype=np.int32)
    opt = option if option is not None else default_option(dtype)
    ev = host_objective(prob, dtype, objective_source)
    res = RunResult(x=x, info=0, num_iteration=0, residual_g=0, residual_f=0, residual_x=0)

    def fg(user, xp, fp, gp, sp):
        ev(xp, fp, gp)
        if record:
            xa = np.ctypeslib.as_array(xp, shape=(n,))
            res.evals.append((float(fp[0]), _digest(xa)))
        return 0

    def after(user, xp, fp, gp, sp):
        if record:
            s = sp[0]
            res.iters.append((s.num_iteration, float(s.residual_g), float(s.residual_f),
                              float(s.residual_x), float(fp[0])))
        return 0

    def stop(user, xp, fp, gp, sp):
        return 1 if (custom_stop_at is not None and sp[0].num_iteration >= custom_stop_at) else 0

    cb_fg, cb_after = cbt(fg), cbt(after)
    cb_stop = cbt(stop) if custom_stop_at is not None else cbt()

    def tr(user, recp):
        r = recp[0]
        res.trace.append({k: (list(getattr(r, k)) if k == 'dbg' else getattr(r, k)) for k in _TRACE_KEYS})

    sfx = "f64" if is64 else "f32"
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    if subsm_projection and which != "oracle":
        raise ValueError("the reference build has only the 2.1 subspace step")
    if which == "oracle":
        lib = oracle_lib()
        fn = getattr(lib, f"orc_lbfgsb_minimize_{sfx}")
        cb_tr = TRACE_CB(tr) if trace else TRACE_CB()
        lib.orc_set_subsm_projection(1 if subsm_projection else 0)
        try:
            fn(n, P(x, real), P(nbd, C.c_int), P(l, real), P(u, real), C.byref(opt), cb_fg,
               cb_after, cb_stop, None, cb_tr, None, C.byref(summ))
        finally:
            lib.orc_set_subsm_projection(0)
    elif which == "ref":
        fn = getattr(ref_lib(), f"ref_lbfgsb_minimize_{sfx}")
        fn(n, P(x, real), P(nbd, C.c_int), P(l, real), P(u, real), C.byref(opt), cb_fg,
           cb_after, cb_stop, None, C.byref(summ))
    else:
        raise ValueError(which)
    res.x = x
    res.info = summ.info
    res.num_iteration = summ.num_iteration
    res.residual_g = float(summ.residual_g)
    res.residual_f = float(summ.residual_f)
    res.residual_x = float(summ.residual_x)
    return res
