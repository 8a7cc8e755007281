"""ctypes binding of liblbfgsb_b200.so for tests, smoke and bench.

The library itself is C++/CUDA behind the C ABI of include/lbfgsb_b200.h; this module only
loads it (and fails loudly if it has not been built: there is no fallback), mirrors the
structs, and offers a small driver that runs one solve on device buffers allocated with
torch.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbfgsb_b200.so")

MODE_NO_ACCELERATION, MODE_CUDA = 0, 1
FORM_PLAIN, FORM_MIXED, FORM_MIXED_BF16 = 0, 1, 2
MAX_KERNELS = 16


class OptionF64(C.Structure):
    _fields_ = [("machine_epsilon", C.c_double), ("machine_maximum", C.c_double),
                ("step_scaling", C.c_double), ("eps_g", C.c_double), ("eps_f", C.c_double),
                ("eps_x", C.c_double), ("hessian_approximate_dimension", C.c_int),
                ("max_iteration", C.c_int), ("mode", C.c_int)]


class OptionF32(C.Structure):
    _fields_ = [("machine_epsilon", C.c_float), ("machine_maximum", C.c_float),
                ("step_scaling", C.c_float), ("eps_g", C.c_float), ("eps_f", C.c_float),
                ("eps_x", C.c_float), ("hessian_approximate_dimension", C.c_int),
                ("max_iteration", C.c_int), ("mode", C.c_int)]


class SummaryF64(C.Structure):
    _fields_ = [("residual_g", C.c_double), ("residual_f", C.c_double),
                ("residual_x", C.c_double), ("num_iteration", C.c_int), ("info", C.c_int)]


class SummaryF32(C.Structure):
    _fields_ = [("residual_g", C.c_float), ("residual_f", C.c_float),
                ("residual_x", C.c_float), ("num_iteration", C.c_int), ("info", C.c_int)]


class TraceRecord(C.Structure):
    _fields_ = [("iter", C.c_int), ("nint", C.c_int), ("nbreak", C.c_int), ("nfree", C.c_int),
                ("nenter", C.c_int), ("nleave", C.c_int), ("col", C.c_int), ("head", C.c_int),
                ("nfgv", C.c_int), ("ifun", C.c_int), ("iword", C.c_int), ("reset", C.c_int),
                ("free_hash", C.c_ulonglong), ("at_lower", C.c_ulonglong),
                ("at_upper", C.c_ulonglong), ("f", C.c_double), ("theta", C.c_double),
                ("stp", C.c_double), ("dtm", C.c_double), ("tsum", C.c_double),
                ("gd", C.c_double), ("gdold", C.c_double), ("dtd", C.c_double),
                ("stpmx", C.c_double), ("f1_0", C.c_double), ("f2_0", C.c_double),
                ("dbg", C.c_double * 8)]


TRACE_CB = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(TraceRecord))


class Ext(C.Structure):
    _fields_ = [("form", C.c_int), ("profile", C.c_int), ("trace", TRACE_CB),
                ("trace_user", C.c_void_p), ("subsm_projection", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("kernels", C.c_int), ("name", (C.c_char * 32) * MAX_KERNELS),
                ("launches", C.c_longlong * MAX_KERNELS), ("ms", C.c_double * MAX_KERNELS),
                ("bytes", C.c_double * MAX_KERNELS), ("total_launches", C.c_longlong),
                ("host_syncs", C.c_longlong), ("evaluations", C.c_longlong),
                ("bytes_per_iteration_model", C.c_double), ("rounds", C.c_longlong)]


# allgather(user, send, recv, count, stream) of a sharded solve (device pointers)
ALLGATHER_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p)


class Shard(C.Structure):
    _fields_ = [("rank", C.c_int), ("world", C.c_int), ("n_global", C.c_int),
                ("offset", C.c_int), ("allgather", C.c_void_p), ("allgather_user", C.c_void_p)]


CB64 = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                   C.POINTER(C.c_double), C.c_void_p, C.POINTER(SummaryF64))
CB32 = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                   C.POINTER(C.c_float), C.c_void_p, C.POINTER(SummaryF32))

# every symbol include/lbfgsb_b200.h declares
EXPORTS = [
    "lbfgsb_b200_default_option_f64", "lbfgsb_b200_default_option_f32",
    "lbfgsb_b200_minimize_f64", "lbfgsb_b200_minimize_f32",
    "lbfgsb_b200_minimize_ext_f64", "lbfgsb_b200_minimize_ext_f32",
    "lbfgsb_b200_last_stats", "lbfgsb_b200_last_error", "lbfgsb_b200_synth_create",
    "lbfgsb_b200_synth_destroy", "lbfgsb_b200_synth_set_offset", "lbfgsb_b200_synth_funcgrad_f64",
    "lbfgsb_b200_synth_funcgrad_f32", "lbfgsb_b200_copy", "lbfgsb_b200_projgr_noalloc_f64",
    "lbfgsb_b200_trim_memory", "lbfgsb_b200_dsscfg_create", "lbfgsb_b200_dsscfg_destroy",
    "lbfgsb_b200_dsscfg_funcgrad_f64", "lbfgsb_b200_dsscfg_funcgrad_f32",
    "lbfgsb_b200_dsscfg_start_f64", "lbfgsb_b200_dsscfg_start_f32",
    "lbfgsb_b200_minimize_batch_f64", "lbfgsb_b200_minimize_batch_f32",
    "lbfgsb_b200_workspace_bytes", "lbfgsb_b200_server_create", "lbfgsb_b200_server_submit_f32",
    "lbfgsb_b200_server_wait", "lbfgsb_b200_server_peak", "lbfgsb_b200_server_destroy",
    "lbfgsb_b200_minimize_device_f64", "lbfgsb_b200_minimize_device_f32",
    "lbfgsb_b200_synth_device_f64", "lbfgsb_b200_synth_device_f32",
    "lbfgsb_b200_minimize_batch_device_f64", "lbfgsb_b200_minimize_batch_device_f32",
    "lbfgsb_b200_batch_tiles_per_cta", "lbfgsb_b200_synth_batch_create",
    "lbfgsb_b200_synth_batch_destroy", "lbfgsb_b200_synth_batch_problem",
    "lbfgsb_b200_synth_batch_f64", "lbfgsb_b200_synth_batch_f32",
    "lbfgsb_b200_batch_server_create_f32", "lbfgsb_b200_batch_server_submit_f32",
    "lbfgsb_b200_batch_server_wait", "lbfgsb_b200_batch_server_peak",
    "lbfgsb_b200_batch_server_destroy", "lbfgsb_b200_batch_request_bytes",
    "lbfgsb_b200_minimize_sharded_f64", "lbfgsb_b200_minimize_sharded_f32",
]

_lib = None


def load() -> C.CDLL:
    """Load the built library; raises if it is missing (build with build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with lbfgsb-gpu_b200/build.py "
                           "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for sfx, real, opt, summ, cb in (("f64", C.c_double, OptionF64, SummaryF64, CB64),
                                     ("f32", C.c_float, OptionF32, SummaryF32, CB32)):
        fn = getattr(lib, f"lbfgsb_b200_minimize_ext_{sfx}")
        fn.restype = C.c_int
        fn.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.POINTER(opt), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.c_void_p, C.POINTER(Ext), C.POINTER(summ)]
        fn = getattr(lib, f"lbfgsb_b200_minimize_{sfx}")
        fn.restype = C.c_int
        fn.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.POINTER(opt), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.c_void_p, C.POINTER(summ)]
        fn = getattr(lib, f"lbfgsb_b200_default_option_{sfx}")
        fn.restype = None
        fn.argtypes = [C.POINTER(opt)]
        fn = getattr(lib, f"lbfgsb_b200_minimize_device_{sfx}")
        fn.restype = C.c_int
        fn.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.POINTER(opt), C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Ext),
                       C.POINTER(summ)]
        fn = getattr(lib, f"lbfgsb_b200_minimize_sharded_{sfx}")
        fn.restype = C.c_int
        fn.argtypes = [C.POINTER(Shard), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.c_void_p, C.POINTER(opt), C.c_void_p, C.c_void_p, C.c_void_p,
                       C.c_void_p, C.c_void_p, C.POINTER(Ext), C.POINTER(summ)]
    lib.lbfgsb_b200_last_stats.restype = C.c_int
    lib.lbfgsb_b200_last_stats.argtypes = [C.POINTER(Stats)]
    lib.lbfgsb_b200_last_error.restype = C.c_char_p
    lib.lbfgsb_b200_synth_create.restype = C.c_void_p
    lib.lbfgsb_b200_synth_create.argtypes = [C.c_int] + [C.c_void_p] * 4 + [C.c_int]
    lib.lbfgsb_b200_synth_destroy.restype = None
    lib.lbfgsb_b200_synth_destroy.argtypes = [C.c_void_p]
    lib.lbfgsb_b200_synth_set_offset.restype = None
    lib.lbfgsb_b200_synth_set_offset.argtypes = [C.c_void_p, C.c_double]
    lib.lbfgsb_b200_copy.restype = C.c_int
    lib.lbfgsb_b200_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    for sfx, opt, summ in (("f64", OptionF64, SummaryF64), ("f32", OptionF32, SummaryF32)):
        fn = getattr(lib, f"lbfgsb_b200_minimize_batch_{sfx}")
        fn.restype = C.c_int
        fn.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.POINTER(opt), C.c_void_p, C.c_void_p, C.c_int, C.POINTER(summ),
                       C.c_void_p, C.c_void_p]
    for sfx, opt, summ in (("f64", OptionF64, SummaryF64), ("f32", OptionF32, SummaryF32)):
        fn = getattr(lib, f"lbfgsb_b200_minimize_batch_device_{sfx}")
        fn.restype = C.c_int
        fn.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.c_void_p, C.POINTER(opt), C.c_void_p, C.c_void_p, C.c_void_p,
                       C.POINTER(Ext), C.POINTER(summ), C.c_void_p]
    lib.lbfgsb_b200_batch_tiles_per_cta.restype = C.c_int
    lib.lbfgsb_b200_batch_tiles_per_cta.argtypes = [C.c_int, C.c_int]
    lib.lbfgsb_b200_synth_batch_create.restype = C.c_void_p
    lib.lbfgsb_b200_synth_batch_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    lib.lbfgsb_b200_synth_batch_destroy.restype = None
    lib.lbfgsb_b200_synth_batch_destroy.argtypes = [C.c_void_p]
    lib.lbfgsb_b200_synth_batch_problem.restype = C.c_int
    lib.lbfgsb_b200_synth_batch_problem.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                                                    C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                                    C.c_void_p]
    lib.lbfgsb_b200_batch_server_create_f32.restype = C.c_int
    lib.lbfgsb_b200_batch_server_create_f32.argtypes = [C.c_ulonglong, C.c_int, C.POINTER(OptionF32),
                                                        C.c_void_p, C.c_void_p, C.c_int,
                                                        C.POINTER(C.c_void_p)]
    lib.lbfgsb_b200_batch_server_submit_f32.restype = C.c_int
    lib.lbfgsb_b200_batch_server_submit_f32.argtypes = [C.c_void_p, C.c_int, C.c_int] + \
        [C.c_void_p] * 4 + [C.POINTER(C.c_longlong)]
    lib.lbfgsb_b200_batch_server_wait.restype = C.c_int
    lib.lbfgsb_b200_batch_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(SummaryF32),
                                                  C.POINTER(C.c_int), C.POINTER(C.c_double),
                                                  C.POINTER(C.c_double)]
    lib.lbfgsb_b200_batch_server_peak.restype = C.c_int
    lib.lbfgsb_b200_batch_server_peak.argtypes = [C.c_void_p, C.POINTER(C.c_ulonglong), C.POINTER(C.c_int)]
    lib.lbfgsb_b200_batch_request_bytes.restype = C.c_ulonglong
    lib.lbfgsb_b200_batch_request_bytes.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.lbfgsb_b200_batch_server_destroy.restype = C.c_int
    lib.lbfgsb_b200_batch_server_destroy.argtypes = [C.c_void_p]
    lib.lbfgsb_b200_dsscfg_create.restype = C.c_void_p
    lib.lbfgsb_b200_dsscfg_create.argtypes = [C.c_int, C.c_int, C.c_double]
    lib.lbfgsb_b200_dsscfg_destroy.restype = None
    lib.lbfgsb_b200_dsscfg_destroy.argtypes = [C.c_void_p]
    for sfx in ("f64", "f32"):
        fn = getattr(lib, f"lbfgsb_b200_dsscfg_start_{sfx}")
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.lbfgsb_b200_projgr_noalloc_f64.restype = C.c_int
    lib.lbfgsb_b200_projgr_noalloc_f64.argtypes = [C.c_int] + [C.c_void_p] * 7
    lib.lbfgsb_b200_workspace_bytes.restype = C.c_ulonglong
    lib.lbfgsb_b200_workspace_bytes.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.lbfgsb_b200_server_create.restype = C.c_int
    lib.lbfgsb_b200_server_create.argtypes = [C.c_int, C.c_ulonglong, C.c_int, C.POINTER(C.c_void_p)]
    lib.lbfgsb_b200_server_submit_f32.restype = C.c_int
    lib.lbfgsb_b200_server_submit_f32.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 4 + \
        [C.POINTER(OptionF32), C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong)]
    lib.lbfgsb_b200_server_wait.restype = C.c_int
    lib.lbfgsb_b200_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(SummaryF32),
                                            C.POINTER(C.c_int), C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]
    lib.lbfgsb_b200_server_peak.restype = C.c_int
    lib.lbfgsb_b200_server_peak.argtypes = [C.c_void_p, C.POINTER(C.c_ulonglong), C.POINTER(C.c_int)]
    lib.lbfgsb_b200_server_destroy.restype = C.c_int
    lib.lbfgsb_b200_server_destroy.argtypes = [C.c_void_p]
    _lib = lib
    return lib


def default_option(dtype):
    lib = load()
    if np.dtype(dtype) == np.float64:
        o = OptionF64()
        lib.lbfgsb_b200_default_option_f64(C.byref(o))
    else:
        o = OptionF32()
        lib.lbfgsb_b200_default_option_f32(C.byref(o))
    return o


def last_stats() -> dict:
    st = Stats()
    load().lbfgsb_b200_last_stats(C.byref(st))
    out = {"kernels": {}, "total_launches": st.total_launches, "host_syncs": st.host_syncs,
           "evaluations": st.evaluations, "rounds": st.rounds,
           "bytes_per_iteration_model": st.bytes_per_iteration_model}
    for k in range(st.kernels):
        name = bytes(st.name[k]).split(b"\0", 1)[0].decode()
        out["kernels"][name] = {"launches": st.launches[k], "ms": st.ms[k],
                                "bytes": st.bytes[k]}
    return out


def solve_batch(ns, xs, nbds, ls, us, option, funcgrad, users, concurrency=16, dtype=np.float64):
    """lbfgsb_b200_minimize_batch over device tensors (lists of torch tensors); returns
    (status, per-instance statuses, summaries, seconds)."""
    lib = load()
    k = len(ns)
    is64 = np.dtype(dtype) == np.float64
    ptrs = lambda ts: (C.c_void_p * k)(*[t.data_ptr() for t in ts])  # noqa: E731
    n_arr = (C.c_int * k)(*ns)
    summ = ((SummaryF64 if is64 else SummaryF32) * k)()
    stat = (C.c_int * k)()
    secs = (C.c_double * k)()
    us_arr = (C.c_void_p * k)(*users)
    fn = lib.lbfgsb_b200_minimize_batch_f64 if is64 else lib.lbfgsb_b200_minimize_batch_f32
    rc = fn(k, n_arr, ptrs(xs), ptrs(nbds), ptrs(ls), ptrs(us), C.byref(option), funcgrad,
            us_arr, concurrency, summ, stat, secs)
    return rc, list(stat), list(summ), list(secs)


class Server:
    """The serving front end (lbfgsb_b200_server_*): FP32 solves queued one by one,
    admitted in arrival order within an HBM budget, run on `workers` streams."""

    def __init__(self, workers=16, hbm_budget_bytes=150 * 10**9, form=FORM_MIXED):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.lbfgsb_b200_server_create(workers, hbm_budget_bytes, form, C.byref(h))
        if rc != 0:
            raise RuntimeError(self.lib.lbfgsb_b200_last_error().decode())
        self.handle = h

    def submit(self, n, x, nbd, l, u, option, funcgrad, user):
        """Queue one solve on device tensors; returns (status, request id)."""
        rid = C.c_longlong(-1)
        rc = self.lib.lbfgsb_b200_server_submit_f32(self.handle, n, x.data_ptr(), nbd.data_ptr(),
                                                    l.data_ptr(), u.data_ptr(), C.byref(option),
                                                    funcgrad, user, C.byref(rid))
        return rc, rid.value

    def wait(self, rid):
        """(status, summary, seconds from submit to result, seconds waiting for admission)."""
        summ = SummaryF32()
        st = C.c_int(-1)
        lat = C.c_double()
        q = C.c_double()
        rc = self.lib.lbfgsb_b200_server_wait(self.handle, rid, C.byref(summ), C.byref(st),
                                              C.byref(lat), C.byref(q))
        if rc != 0:
            raise RuntimeError(self.lib.lbfgsb_b200_last_error().decode())
        return st.value, summ, lat.value, q.value

    def peak(self):
        b = C.c_ulonglong()
        r = C.c_int()
        self.lib.lbfgsb_b200_server_peak(self.handle, C.byref(b), C.byref(r))
        return b.value, r.value

    def close(self):
        if self.handle:
            self.lib.lbfgsb_b200_server_destroy(self.handle)
            self.handle = None


class DsscfgObjective:
    """The device dsscfg objective of csrc/dsscfg.cu (the reference example's problem)."""

    def __init__(self, nx: int, ny: int, lam: float = 1.0):
        lib = load()
        self.nx, self.ny = nx, ny
        self.handle = lib.lbfgsb_b200_dsscfg_create(nx, ny, lam)
        if not self.handle:
            raise RuntimeError("lbfgsb_b200_dsscfg_create failed")
        self.f64 = C.cast(lib.lbfgsb_b200_dsscfg_funcgrad_f64, C.c_void_p).value
        self.f32 = C.cast(lib.lbfgsb_b200_dsscfg_funcgrad_f32, C.c_void_p).value

    def start(self, x_dev_ptr: int, dtype=np.float64, stream=None) -> None:
        lib = load()
        fn = lib.lbfgsb_b200_dsscfg_start_f64 if np.dtype(dtype) == np.float64 else \
            lib.lbfgsb_b200_dsscfg_start_f32
        if fn(self.handle, x_dev_ptr, stream) != 0:
            raise RuntimeError("lbfgsb_b200_dsscfg_start failed")

    def close(self) -> None:
        if self.handle:
            load().lbfgsb_b200_dsscfg_destroy(self.handle)
            self.handle = None


class SynthObjective:
    """The device objective of csrc/objective.cu for a synth.py problem."""

    def __init__(self, prob: dict, single_precision_fields: bool = False):
        lib = load()
        self._fields = [np.ascontiguousarray(prob[k], dtype=np.float64)
                        for k in ("kappa", "w", "t", "b")]
        self.handle = lib.lbfgsb_b200_synth_create(
            int(prob["s"]), *[a.ctypes.data for a in self._fields],
            1 if single_precision_fields else 0)
        if not self.handle:
            raise RuntimeError("lbfgsb_b200_synth_create failed")
        if prob.get("f_offset", 0.0):
            lib.lbfgsb_b200_synth_set_offset(self.handle, float(prob["f_offset"]))
        self.f64 = C.cast(lib.lbfgsb_b200_synth_funcgrad_f64, C.c_void_p).value
        self.f32 = C.cast(lib.lbfgsb_b200_synth_funcgrad_f32, C.c_void_p).value
        # the device-driven forms (lbfgsb_b200_device_objective_*)
        self.d64 = C.cast(lib.lbfgsb_b200_synth_device_f64, C.c_void_p).value
        self.d32 = C.cast(lib.lbfgsb_b200_synth_device_f32, C.c_void_p).value

    def close(self):
        if self.handle:
            load().lbfgsb_b200_synth_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def synth_value(prob: dict, x0=None) -> float:
    """f of a synth.py problem at x0 (default 0; a host array), evaluated in FP64 by the
    device objective; at 0 it is the f_offset that lets a float f resolve the decrease of
    the first iterations."""
    import torch
    lib = load()
    n = int(prob["nbd"].size)
    so = SynthObjective({k: v for k, v in prob.items() if k != "f_offset"})
    if x0 is None:
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
    else:
        x = torch.from_numpy(np.ascontiguousarray(x0, dtype=np.float64)).to("cuda")
    g = torch.empty_like(x)
    f = C.c_double(0.0)
    fn = lib.lbfgsb_b200_synth_funcgrad_f64
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p, C.c_void_p, C.c_void_p]
    fn(so.handle, x.data_ptr(), C.byref(f), g.data_ptr(), None, None)
    torch.cuda.synchronize()
    so.close()
    return float(f.value)


class SynthBatch:
    """A batch of synth.py problems generated on the device (lbfgsb_b200_synth_batch_*):
    problem p has grid side sides[p] and seed seeds[p]; its l, u (in the solver precision)
    and nbd stay on the device."""

    def __init__(self, sides, seeds, single_precision_fields=True, dtype=np.float32):
        lib = load()
        self.count = len(sides)
        self.sides = [int(v) for v in sides]
        self.n = [v * v for v in self.sides]
        self.dtype = np.dtype(dtype)
        sd = (C.c_int * self.count)(*self.sides)
        se = (C.c_ulonglong * self.count)(*[int(v) for v in seeds])
        self.handle = lib.lbfgsb_b200_synth_batch_create(self.count, sd, se,
                                                         1 if single_precision_fields else 0,
                                                         self.dtype.itemsize)
        if not self.handle:
            raise RuntimeError("lbfgsb_b200_synth_batch_create failed")
        self.objective = C.cast(lib.lbfgsb_b200_synth_batch_f64 if self.dtype == np.float64
                                else lib.lbfgsb_b200_synth_batch_f32, C.c_void_p).value

    def problem(self, p):
        """(l, u, nbd, [kappa, w, t, b]) device pointers of problem p."""
        lib = load()
        l, u, nbd = C.c_void_p(), C.c_void_p(), C.c_void_p()
        fields = (C.c_void_p * 4)()
        if lib.lbfgsb_b200_synth_batch_problem(self.handle, p, C.byref(l), C.byref(u),
                                               C.byref(nbd), fields) != 0:
            raise IndexError(p)
        return l.value, u.value, nbd.value, [fields[k] for k in range(4)]

    def close(self):
        if self.handle:
            load().lbfgsb_b200_synth_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_batch_device(batch: "SynthBatch", xs, option, form: int = FORM_PLAIN,
                       subsm_projection: bool = False, ids=None):
    """lbfgsb_b200_minimize_batch_device over the problems `ids` (default all) of a
    SynthBatch (the objective's ids are the batch's problem indices); xs: device tensors
    (start points in, solutions out).  Returns (status, per-instance statuses, summaries,
    stats)."""
    lib = load()
    ids = list(range(batch.count)) if ids is None else list(ids)
    k = len(ids)
    is64 = batch.dtype == np.float64
    probs = [batch.problem(p) for p in ids]
    n_arr = (C.c_int * k)(*[batch.n[p] for p in ids])
    id_arr = (C.c_int * k)(*ids)
    ptr = lambda v: (C.c_void_p * k)(*v)  # noqa: E731
    summ = ((SummaryF64 if is64 else SummaryF32) * k)()
    stat = (C.c_int * k)()
    ext = Ext(form, 0, TRACE_CB(), None, 1 if subsm_projection else 0)
    fn = lib.lbfgsb_b200_minimize_batch_device_f64 if is64 else lib.lbfgsb_b200_minimize_batch_device_f32
    rc = fn(k, id_arr, n_arr, ptr([t.data_ptr() for t in xs]), ptr([p[2] for p in probs]),
            ptr([p[0] for p in probs]), ptr([p[1] for p in probs]), C.byref(option),
            batch.objective, batch.handle, None, C.byref(ext), summ, stat)
    return rc, list(stat), list(summ), last_stats()


class BatchServer:
    """The continuous-batching server (lbfgsb_b200_batch_server_*) over a SynthBatch's
    batched objective: FP32 solves admitted in arrival order within an HBM budget and
    advanced together on the device."""

    def __init__(self, batch: "SynthBatch", option, hbm_budget_bytes=150 * 10**9,
                 form=FORM_MIXED, rounds_per_loop=4):
        self.lib = load()
        self.batch = batch
        h = C.c_void_p()
        rc = self.lib.lbfgsb_b200_batch_server_create_f32(hbm_budget_bytes, form, C.byref(option),
                                                          batch.objective, batch.handle,
                                                          rounds_per_loop, C.byref(h))
        if rc != 0:
            raise RuntimeError(self.lib.lbfgsb_b200_last_error().decode())
        self.handle = h

    def submit(self, p, x):
        """Queue problem p of the batch with start point / result tensor x; returns
        (status, ticket)."""
        l, u, nbd, _ = self.batch.problem(p)
        t = C.c_longlong(-1)
        rc = self.lib.lbfgsb_b200_batch_server_submit_f32(self.handle, p, self.batch.n[p],
                                                          x.data_ptr(), nbd, l, u, C.byref(t))
        return rc, t.value

    def wait(self, ticket):
        """(status, summary, seconds from submit to result, seconds to admission)."""
        summ = SummaryF32()
        st = C.c_int(-1)
        lat = C.c_double()
        q = C.c_double()
        rc = self.lib.lbfgsb_b200_batch_server_wait(self.handle, ticket, C.byref(summ),
                                                    C.byref(st), C.byref(lat), C.byref(q))
        if rc != 0:
            raise RuntimeError(self.lib.lbfgsb_b200_last_error().decode())
        return st.value, summ, lat.value, q.value

    def peak(self):
        b = C.c_ulonglong()
        r = C.c_int()
        self.lib.lbfgsb_b200_batch_server_peak(self.handle, C.byref(b), C.byref(r))
        return b.value, r.value

    def close(self):
        if self.handle:
            self.lib.lbfgsb_b200_batch_server_destroy(self.handle)
            self.handle = None


def _digest(a: np.ndarray) -> str:
    return hashlib.sha1(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


@dataclass
class GpuResult:
    x: np.ndarray
    info: int
    num_iteration: int
    residual_g: float
    residual_f: float
    residual_x: float
    status: int
    evals: list = field(default_factory=list)
    iters: list = field(default_factory=list)
    trace: list = field(default_factory=list)
    stats: dict = field(default_factory=dict)


_TRACE_KEYS = [f for f, _ in TraceRecord._fields_]


def solve(prob: dict, dtype=np.float64, x0=None, option=None, objective: str = "host",
          form: int = FORM_PLAIN, trace: bool = False, record: bool = True,
          custom_stop_at: int | None = None, profile: bool = False, stream=None,
          subsm_projection: bool = False, driven: str = "host") -> GpuResult:
    """One solve on the GPU through the C ABI.

    subsm_projection: the L-BFGS-B 3.0 subspace step (lbfgsb_b200_ext.subsm_projection)
    instead of the reference's 2.1 step.
    driven="device": lbfgsb_b200_minimize_device with the device synthetic objective (the
    outer loop on the device; objective must be "device", no trace or callbacks).

    objective="host": funcgrad copies x to the host and evaluates the CPU objective of
    oracle/objective.c (so f and g are bit-identical to what the oracle sees);
    objective="device": the device objective of csrc/objective.cu (synthetic problems).
    """
    import torch

    lib = load()
    dtype = np.dtype(dtype)
    is64 = dtype == np.float64
    tdt = torch.float64 if is64 else torch.float32
    n = int(prob["nbd"].size)
    dev = torch.device("cuda:0")
    x_np = np.zeros(n, dtype=dtype) if x0 is None else np.asarray(x0, dtype=dtype)
    x = torch.from_numpy(np.ascontiguousarray(x_np)).to(dev)
    l = torch.from_numpy(np.ascontiguousarray(prob["l"], dtype=dtype)).to(dev)
    u = torch.from_numpy(np.ascontiguousarray(prob["u"], dtype=dtype)).to(dev)
    nbd = torch.from_numpy(np.ascontiguousarray(prob["nbd"], dtype=np.int32)).to(dev)
    opt = option if option is not None else default_option(dtype)
    summ = SummaryF64() if is64 else SummaryF32()
    cbt = CB64 if is64 else CB32
    res = GpuResult(x=x_np, info=0, num_iteration=0, residual_g=0, residual_f=0,
                    residual_x=0, status=0)
    keep = []
    user = None
    if objective == "host":
        import sys
        repo = os.path.dirname(HERE)
        if repo not in sys.path:
            sys.path.insert(0, repo)
        from oracle import binding as OB  # test glue: the CPU objective of the oracle
        ev = OB.host_objective(prob, dtype)
        hx = np.zeros(n, dtype=dtype)
        hg = np.zeros(n, dtype=dtype)
        real = C.c_double if is64 else C.c_float
        fbox = (real * 1)()

        def fg(_user, xp, fp, gp, _stream, _sp):
            torch.cuda.current_stream().synchronize()
            lib.lbfgsb_b200_copy(hx.ctypes.data, C.cast(xp, C.c_void_p), hx.nbytes, 2)
            ev(hx.ctypes.data_as(C.POINTER(real)), fbox, hg.ctypes.data_as(C.POINTER(real)))
            lib.lbfgsb_b200_copy(C.cast(gp, C.c_void_p), hg.ctypes.data, hg.nbytes, 1)
            fp[0] = fbox[0]
            if record:
                res.evals.append((float(fbox[0]), _digest(hx)))
            return 0

        cb = cbt(fg)
        keep.append(cb)
        fg_ptr = C.cast(cb, C.c_void_p).value
    elif objective == "device":
        so = SynthObjective(prob, single_precision_fields=not is64)
        keep.append(so)
        user = so.handle
        fg_ptr = so.f64 if is64 else so.f32
    else:
        raise ValueError(objective)

    def after(_user, xp, fp, gp, _stream, sp):
        if record:
            s = sp[0]
            res.iters.append((s.num_iteration, float(s.residual_g), float(s.residual_f),
                              float(s.residual_x), float(fp[0])))
        return 0

    def stop(_user, xp, fp, gp, _stream, sp):
        return 1 if (custom_stop_at is not None and sp[0].num_iteration >= custom_stop_at) else 0

    cb_after = cbt(after)
    keep.append(cb_after)
    after_ptr = C.cast(cb_after, C.c_void_p).value if record else None
    stop_ptr = None
    if custom_stop_at is not None:
        cb_stop = cbt(stop)
        keep.append(cb_stop)
        stop_ptr = C.cast(cb_stop, C.c_void_p).value

    def tr(_user, rp):
        r = rp[0]
        res.trace.append({k: (list(getattr(r, k)) if k == 'dbg' else getattr(r, k)) for k in _TRACE_KEYS})

    cb_tr = TRACE_CB(tr) if trace else TRACE_CB()
    keep.append(cb_tr)
    ext = Ext(form, 1 if profile else 0, cb_tr, None, 1 if subsm_projection else 0)
    sfx = "f64" if is64 else "f32"
    torch.cuda.synchronize()
    if driven == "device":
        if objective != "device" or trace or custom_stop_at is not None:
            raise ValueError("a device-driven solve takes the device objective and no callbacks")
        so = keep[0]
        fn = getattr(lib, f"lbfgsb_b200_minimize_device_{sfx}")
        status = fn(n, x.data_ptr(), nbd.data_ptr(), l.data_ptr(), u.data_ptr(), C.byref(opt),
                    so.d64 if is64 else so.d32, so.handle, stream, C.byref(ext), C.byref(summ))
    else:
        fn = getattr(lib, f"lbfgsb_b200_minimize_ext_{sfx}")
        status = fn(n, x.data_ptr(), nbd.data_ptr(), l.data_ptr(), u.data_ptr(), C.byref(opt),
                    fg_ptr, after_ptr, stop_ptr, user, stream, C.byref(ext), C.byref(summ))
    torch.cuda.synchronize()
    if status != 0:
        raise RuntimeError(f"lbfgsb_b200 status {status}: {lib.lbfgsb_b200_last_error()}")
    res.status = status
    res.x = x.cpu().numpy()
    res.info = summ.info
    res.num_iteration = summ.num_iteration
    res.residual_g = float(summ.residual_g)
    res.residual_f = float(summ.residual_f)
    res.residual_x = float(summ.residual_x)
    res.stats = last_stats()
    return res


class ThreadAllGather:
    """All-gather among `world` threads of one process, for sharded solves whose ranks share
    one GPU (each rank a thread with its own stream).  Every call waits for the rank's
    stream, stages its `count` doubles on the host, meets the other ranks at a barrier and
    copies everyone's values to recv; no kernel waits on another rank's kernels.  A rank that
    does not arrive within `timeout` seconds breaks the barrier, and the call returns 1."""

    def __init__(self, world: int, timeout: float = 120.0):
        import threading
        self.world = world
        self.barrier = threading.Barrier(world, timeout=timeout)
        self.slots = [None] * world

    def callback(self, rank: int):
        import torch
        lib = load()

        def gather(_user, send, recv, count, stream):
            try:
                torch.cuda.ExternalStream(stream).synchronize() if stream else torch.cuda.synchronize()
                mine = np.empty(count, dtype=np.float64)
                lib.lbfgsb_b200_copy(mine.ctypes.data, send, mine.nbytes, 2)
                self.slots[rank] = mine
                self.barrier.wait()
                allv = np.concatenate(self.slots)
                lib.lbfgsb_b200_copy(recv, allv.ctypes.data, allv.nbytes, 1)
                self.barrier.wait()
                return 0
            except Exception:  # a broken barrier: another rank left
                self.barrier.abort()
                return 1

        return ALLGATHER_CB(gather)


def solve_sharded(prob: dict, world: int, dtype=np.float64, option=None, form: int = FORM_PLAIN,
                  trace: bool = False, parts=None, timeout: float = 120.0) -> GpuResult:
    """One problem split by index range over `world` ranks that share cuda:0: each rank is a
    thread calling lbfgsb_b200_minimize_sharded_* on its own stream, with a ThreadAllGather.
    The objective is evaluated on the host by the oracle's objective (oracle/objective.c) on
    the whole x, gathered from the ranks; rank 0 returns f and the others 0.  parts: the
    ranks' sizes (default: np.array_split's).  Returns rank 0's result with the whole x."""
    import sys
    import threading

    import torch

    lib = load()
    repo = os.path.dirname(HERE)
    if repo not in sys.path:
        sys.path.insert(0, repo)
    from oracle import binding as OB  # test glue: the CPU objective of the oracle

    dtype = np.dtype(dtype)
    is64 = dtype == np.float64
    n = int(prob["nbd"].size)
    sizes = list(parts) if parts is not None else [len(a) for a in np.array_split(np.arange(n), world)]
    assert len(sizes) == world and sum(sizes) == n
    offs = [int(v) for v in np.concatenate([[0], np.cumsum(sizes)[:-1]])]
    real = C.c_double if is64 else C.c_float
    cbt = CB64 if is64 else CB32
    sfx = "f64" if is64 else "f32"
    ev = OB.host_objective(prob, dtype)
    hx = np.zeros(n, dtype=dtype)
    hg = np.zeros(n, dtype=dtype)
    fbox = (real * 1)()
    bar = threading.Barrier(world, timeout=timeout)
    ag = ThreadAllGather(world, timeout)
    results = [None] * world
    keep = []

    def rank_main(r):
        torch.cuda.set_device(0)
        dev = torch.device("cuda:0")
        stream = torch.cuda.Stream(device=dev)
        lo, nr = offs[r], sizes[r]
        with torch.cuda.stream(stream):
            x = torch.zeros(nr, dtype=torch.float64 if is64 else torch.float32, device=dev)
            l = torch.from_numpy(np.ascontiguousarray(prob["l"][lo:lo + nr], dtype=dtype)).to(dev)
            u = torch.from_numpy(np.ascontiguousarray(prob["u"][lo:lo + nr], dtype=dtype)).to(dev)
            nbd = torch.from_numpy(np.ascontiguousarray(prob["nbd"][lo:lo + nr], dtype=np.int32)).to(dev)
        stream.synchronize()
        res = GpuResult(x=None, info=0, num_iteration=0, residual_g=0, residual_f=0,
                        residual_x=0, status=0)

        def fg(_user, xp, fp, gp, sp, _summ):
            try:
                torch.cuda.ExternalStream(sp).synchronize()
                part = np.empty(nr, dtype=dtype)
                lib.lbfgsb_b200_copy(part.ctypes.data, C.cast(xp, C.c_void_p), part.nbytes, 2)
                hx[lo:lo + nr] = part
                bar.wait()
                if r == 0:
                    ev(hx.ctypes.data_as(C.POINTER(real)), fbox, hg.ctypes.data_as(C.POINTER(real)))
                bar.wait()
                gpart = np.ascontiguousarray(hg[lo:lo + nr])
                lib.lbfgsb_b200_copy(C.cast(gp, C.c_void_p), gpart.ctypes.data, gpart.nbytes, 1)
                fp[0] = fbox[0] if r == 0 else 0.0
                if r == 0:
                    res.evals.append(float(fbox[0]))
                bar.wait()
                return 0
            except Exception:
                bar.abort()
                return 1

        def tr(_user, rp):
            rec = rp[0]
            res.trace.append({k: (list(getattr(rec, k)) if k == 'dbg' else getattr(rec, k))
                              for k in _TRACE_KEYS})

        cb = cbt(fg)
        cb_tr = TRACE_CB(tr) if trace else TRACE_CB()
        gcb = ag.callback(r)
        keep.extend([cb, cb_tr, gcb])
        sh = Shard(r, world, n, lo, C.cast(gcb, C.c_void_p).value, None)
        ext = Ext(form, 0, cb_tr, None, 0)
        summ = SummaryF64() if is64 else SummaryF32()
        opt = option if option is not None else default_option(dtype)
        fn = getattr(lib, f"lbfgsb_b200_minimize_sharded_{sfx}")
        status = fn(C.byref(sh), nr, x.data_ptr(), nbd.data_ptr(), l.data_ptr(), u.data_ptr(),
                    C.byref(opt), C.cast(cb, C.c_void_p).value, None, None, None,
                    C.c_void_p(stream.cuda_stream), C.byref(ext), C.byref(summ))
        stream.synchronize()
        res.status = status
        res.x = x.cpu().numpy()
        res.info = summ.info
        res.num_iteration = summ.num_iteration
        res.residual_g = float(summ.residual_g)
        res.residual_f = float(summ.residual_f)
        res.residual_x = float(summ.residual_x)
        if status != 0:
            res.stats = {"error": lib.lbfgsb_b200_last_error().decode()}
            bar.abort()
        results[r] = res

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for r, res in enumerate(results):
        if res is None or res.status != 0:
            raise RuntimeError(f"sharded rank {r} failed: {None if res is None else res.stats}")
    out = results[0]
    out.x = np.concatenate([res.x for res in results])
    out.stats = {"ranks": [(res.info, res.num_iteration, res.residual_g, res.residual_f)
                           for res in results]}
    return out


class _DeviceArray:
    """A raw device pointer seen as a 1-D float64 CUDA array (__cuda_array_interface__), so
    that torch can wrap it without a copy."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def shard_ranges(n: int, world: int) -> list:
    """The index ranges (offset, size) of `world` ranks over n variables, as contiguous
    blocks in rank order (sizes differ by at most one)."""
    base, extra = divmod(n, world)
    out, off = [], 0
    for r in range(world):
        size = base + (1 if r < extra else 0)
        out.append((off, size))
        off += size
    return out


class DistAllGather:
    """The all-gather of a sharded solve over a torch.distributed process group, one process
    per GPU: with the nccl backend, send and recv are device pointers and the NCCL all-gather
    is enqueued on the solver's stream (no host synchronisation); with gloo (CPU), send and
    recv are host pointers and the exchange completes before the call returns."""

    def __init__(self, group=None, device: bool = True):
        self.group = group
        self.device = device

    def exchange(self, send: int, recv: int, count: int, stream=None) -> int:
        import torch
        import torch.distributed as dist
        world = dist.get_world_size(self.group)
        if self.device:
            s_t = torch.as_tensor(_DeviceArray(send, count), device="cuda")
            r_t = torch.as_tensor(_DeviceArray(recv, world * count), device="cuda")
            st = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
            with torch.cuda.stream(st):
                dist.all_gather_into_tensor(r_t, s_t, group=self.group)
        else:
            s_np = np.ctypeslib.as_array(C.cast(send, C.POINTER(C.c_double)), shape=(count,))
            r_np = np.ctypeslib.as_array(C.cast(recv, C.POINTER(C.c_double)), shape=(world * count,))
            out = torch.from_numpy(r_np)
            dist.all_gather_into_tensor(out, torch.from_numpy(s_np).clone(), group=self.group)
        return 0

    def callback(self):
        def gather(_user, send, recv, count, stream):
            try:
                return self.exchange(send, recv, count, stream)
            except Exception:
                return 1
        self._cb = ALLGATHER_CB(gather)
        return self._cb
