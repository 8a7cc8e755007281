"""Benchmark of the L-BFGS-B iteration at n = 4096^2 (the headline config).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--side S] [--dtype f64|f32]

A step is one L-BFGS-B iteration (Cauchy point, subspace step, line search with its
function evaluations, memory update) of the plain solve of the synthetic bounded problem
of lbfgsb-gpu_b200/synth.py on an S x S grid (default 4096: n = 16,777,216), FP64.  The
tolerances eps_f = eps_g = eps_x are 0 so every run performs exactly W + K iterations
(the stopping tests still run every iteration).  The FP64 form is the headline: in FP32
f ~ 0.45 cannot resolve this problem's per-iteration decrease (~1e-8 relative) at this
size and the reference's f-test ends the solve after one iteration, in the reference as
here.

ours:      W untimed iterations, then exactly K iterations timed with CUDA events on the
           solver's stream between two after-iteration callbacks (barrier + synchronize on
           both sides), inputs resident in HBM (vectors far larger than the 126 MB L2).
           e2e: one solve of K iterations through the C ABI from pinned host buffers:
           the host-to-device copies of x0, l, u, nbd, the whole call (workspace, start
           point, K iterations) and the device-to-host copy of x inside the timed region,
           after one untimed call of the same (allocator and memory-pool warm-up).
           The objective's fields are the user's problem data and are uploaded before.
batched:   the batched workload (4,096 FP32 solves of n from 1,024 to 262,144) in one
           batched device-driven solve, against a 32-problem sample of plain solves one
           after another and the reference's CPU path on the host cores.
serving:   a 400-request sample of the Poisson request stream through the continuous-
           batching server, with p50 / p99 latency, beside the same requests one at a time.
forms:     the precision forms at 4096^2 and 2048^2 with each pass's HBM fraction.
walk:      a first Cauchy step that passes ~9e5 breakpoints (n = 1024^2).
dsscfg:    the reference's only published workload (its dsscfg example): our GPU path with
           the device dsscfg objective against the reference's CPU path with its own
           objective, at 256^2 FP64 and 2048^2 FP32, beside the published speedups.
reference: the reference's own CPU L-BFGS-B (culbfgsb/lbfgsbcpu.cpp built into
           oracle/_ref/) on the same problem on the host, single thread (the reference has
           no threading), a bounded number of iterations.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "lbfgsb-gpu_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

UNIT = "iters/s"


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s earlier pool measurement; MEASURED_PEAKS.json absent)"


def ncu_traffic():
    """Per-element DRAM bytes per launch, from a committed ncu capture summary."""
    try:
        with open(os.path.join(REPO, "profiles", "ncu_traffic.json")) as fh:
            return json.load(fh)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"bench_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
            # the timed work starts once the sampler has produced its first sample
            t0 = time.time()
            while time.time() - t0 < 5.0:
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[0]) for r in rows]
        mx = float(rows[0][1])
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows)}


def make_problem(side: int, seed: int = 0):
    import synth
    return synth.synth_problem(side, seed=seed)


class Runner:
    """Solves of one synthetic problem through the C ABI on device-resident inputs:
    eps_f = eps_g = eps_x = 0, so a solve of `iters` iterations runs exactly that many.
    FP32 solves subtract f0 = f(x0) (FP64) from the objective, so that a float f resolves
    the ~1e-8 decrease of an iteration (the minimiser and g are unchanged)."""

    def __init__(self, LB, lib, prob, dtype: str, form: int, dev):
        import torch
        self.LB, self.lib, self.dev = LB, lib, dev
        self.is64 = dtype == "f64"
        self.dt = np.float64 if self.is64 else np.float32
        tdt = torch.float64 if self.is64 else torch.float32
        self.form = form
        if not self.is64:
            prob = dict(prob, f_offset=LB.synth_value(prob))
        self.prob = prob
        self.n = prob["nbd"].size
        self.so = LB.SynthObjective(prob, single_precision_fields=not self.is64)
        self.fg = self.so.f64 if self.is64 else self.so.f32
        self.x = torch.zeros(self.n, dtype=tdt, device=dev)
        self.l = torch.from_numpy(prob["l"].astype(self.dt)).to(dev)
        self.u = torch.from_numpy(prob["u"].astype(self.dt)).to(dev)
        self.nbd = torch.from_numpy(prob["nbd"]).to(dev)
        self.cbt = LB.CB64 if self.is64 else LB.CB32
        self.summ_t = LB.SummaryF64 if self.is64 else LB.SummaryF32
        self.minimize = lib.lbfgsb_b200_minimize_ext_f64 if self.is64 else lib.lbfgsb_b200_minimize_ext_f32

    def option(self, iters):
        o = self.LB.default_option(self.dt)
        o.eps_f = o.eps_g = o.eps_x = 0.0
        o.max_iteration = iters - 1  # the solve stops after iteration `iters`
        return o

    def solve(self, iters, after=None, profile=False):
        import torch
        self.x.zero_()
        summ = self.summ_t()
        ext = self.LB.Ext(self.form, 1 if profile else 0, self.LB.TRACE_CB(), None)
        st = self.minimize(self.n, self.x.data_ptr(), self.nbd.data_ptr(), self.l.data_ptr(),
                           self.u.data_ptr(), C.byref(self.option(iters)), self.fg, after, None,
                           self.so.handle, None, C.byref(ext), C.byref(summ))
        torch.cuda.synchronize()
        if st != 0:
            raise RuntimeError(f"status {st}: {self.lib.lbfgsb_b200_last_error()}")
        return summ, self.LB.last_stats()

    def steady_kernels(self, W, K):
        """Per-kernel launches, summed CUDA-event ms and algorithmic bytes per launch over
        iterations W+1 .. W+K (two profiled solves, W and W+K iterations, subtracted)."""
        _, st_w = self.solve(W, profile=True)
        _, st_wk = self.solve(W + K, profile=True)
        kern = {}
        for name, v in st_wk["kernels"].items():
            launches = v["launches"] - st_w["kernels"][name]["launches"]
            kms = v["ms"] - st_w["kernels"][name]["ms"]
            if launches > 0:
                kern[name] = {"launches": launches, "ms": kms, "bytes": v["bytes"]}
        evals_k = st_wk["evaluations"] - st_w["evaluations"]
        launches_k = st_wk["total_launches"] - st_w["total_launches"] + evals_k  # + objective
        return kern, evals_k, launches_k, st_wk["bytes_per_iteration_model"]

    def timed(self, W, K, dist=None, sampler=None):
        """ms of iterations W+1 .. W+K, CUDA events recorded in the after-iteration callback
        on the solver's stream."""
        import torch
        ev = {"start": torch.cuda.Event(enable_timing=True), "end": torch.cuda.Event(enable_timing=True)}

        def after_cb(_user, _x, _f, _g, _stream, sp):
            it = sp[0].num_iteration
            if it == W:
                torch.cuda.synchronize()
                if dist is not None:
                    dist.barrier()
                ev["start"].record()
            elif it == W + K:
                ev["end"].record()
                ev["end"].synchronize()
            return 0

        cb = self.cbt(after_cb)
        if sampler is not None:
            with sampler:
                summ, _ = self.solve(W + K, after=C.cast(cb, C.c_void_p).value)
        else:
            summ, _ = self.solve(W + K, after=C.cast(cb, C.c_void_p).value)
        torch.cuda.synchronize()
        if summ.num_iteration != W + K:
            raise RuntimeError(f"solve stopped early: {summ.num_iteration} iterations, info {summ.info}")
        return ev["start"].elapsed_time(ev["end"])

    def solve_device(self, iters):
        """The same solve through lbfgsb_b200_minimize_device (the outer loop on the device,
        the objective's f left in device memory)."""
        import torch
        self.x.zero_()
        summ = self.summ_t()
        ext = self.LB.Ext(self.form, 0, self.LB.TRACE_CB(), None)
        fn = self.lib.lbfgsb_b200_minimize_device_f64 if self.is64 else self.lib.lbfgsb_b200_minimize_device_f32
        st = fn(self.n, self.x.data_ptr(), self.nbd.data_ptr(), self.l.data_ptr(), self.u.data_ptr(),
                C.byref(self.option(iters)), self.so.d64 if self.is64 else self.so.d32, self.so.handle,
                None, C.byref(ext), C.byref(summ))
        torch.cuda.synchronize()
        if st != 0:
            raise RuntimeError(f"status {st}: {self.lib.lbfgsb_b200_last_error()}")
        return summ, self.LB.last_stats()

    def timed_device(self, W, K):
        """ms of K device-driven iterations: a solve of W + K iterations less one of W, each
        timed with CUDA events around the call (the set-up of the two solves cancels)."""
        import torch
        out = []
        for iters in (W, W + K):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            summ, st = self.solve_device(iters)
            e1.record()
            e1.synchronize()
            if summ.num_iteration != iters:
                raise RuntimeError(f"device-driven solve stopped early: {summ.num_iteration}")
            out.append((e0.elapsed_time(e1), st))
        st = dict(out[1][1])
        st["timed_launches"] = out[1][1]["total_launches"] - out[0][1]["total_launches"]
        return out[1][0] - out[0][0], st

    def close(self):
        self.so.close()


def roofline_of(kern, n, hbm, hbm_kind, traffic_table=None):
    """The dominant kernel (most summed time) with its achieved algorithmic GB/s and the
    fraction of the HBM peak, and every kernel's share, average time and GB/s."""
    if not kern:
        return None, {}
    name, v = max(kern.items(), key=lambda kv: kv[1]["ms"])
    avg_s = v["ms"] / v["launches"] / 1000.0
    achieved = v["bytes"] / avg_s / 1e9
    traffic = None
    if traffic_table and name in traffic_table.get("bytes_per_element", {}):
        traffic = traffic_table["bytes_per_element"][name] * n
    roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm,
            "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
            "peak_source": hbm_kind,
            "algorithmic_bytes_per_launch": v["bytes"], "avg_launch_ms": avg_s * 1000.0}
    total = sum(x["ms"] for x in kern.values())
    per_kernel = {}
    for k, v in kern.items():
        gbps = (v["bytes"] / (v["ms"] / v["launches"] / 1000.0) / 1e9) if v["bytes"] else None
        per_kernel[k] = {"launches": v["launches"], "avg_ms": v["ms"] / v["launches"],
                         "share": v["ms"] / total, "GBps": gbps,
                         "frac": (gbps / hbm) if gbps else None}
    return roof, per_kernel


def run_ours(args, rank: int, world: int, dist):
    import torch
    import lbfgsb_b200 as LB

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    lib = LB.load()
    is64 = args.dtype == "f64"
    dt = np.float64 if is64 else np.float32
    tdt = torch.float64 if is64 else torch.float32
    prob = make_problem(args.side, seed=rank)
    n = prob["nbd"].size
    W, K = args.warmup, args.steps
    run = Runner(LB, lib, prob, args.dtype, args.form if not is64 else 0, dev)
    prob = run.prob
    option = run.option

    # warm the whole path once (allocator pool, module load)
    run.solve(2)

    # ---- headline: K iterations after W, timed between after-iteration callbacks ----
    sampler = ClockSampler(dev.index)
    ms = run.timed(W, K, dist=dist, sampler=sampler)
    if dist is not None:
        dist.barrier()

    # ---- per-kernel device times of the K steady-state iterations (profiled runs) ----
    kern, evals_k, launches_k, model_bytes = run.steady_kernels(W, K)

    # ---- the same iterations device-driven (lbfgsb_b200_minimize_device) ----
    run.solve_device(2)
    ms_dev, st_dev = run.timed_device(W, K)

    # ---- e2e through the C ABI from pinned host buffers ----
    hx = torch.zeros(n, dtype=tdt).pin_memory()
    hl = torch.from_numpy(prob["l"].astype(dt)).pin_memory()
    hu = torch.from_numpy(prob["u"].astype(dt)).pin_memory()
    hn = torch.from_numpy(prob["nbd"]).pin_memory()
    hout = torch.empty(n, dtype=tdt).pin_memory()
    # the objective's fields are the user's problem data, set up before the solve call
    so2 = LB.SynthObjective(prob, single_precision_fields=not is64)
    ext2 = LB.Ext(run.form, 0, LB.TRACE_CB(), None)
    def e2e_once():
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        dx = hx.to(dev, non_blocking=True)
        dl = hl.to(dev, non_blocking=True)
        du = hu.to(dev, non_blocking=True)
        dn = hn.to(dev, non_blocking=True)
        summ2 = run.summ_t()
        st = run.minimize(n, dx.data_ptr(), dn.data_ptr(), dl.data_ptr(), du.data_ptr(),
                          C.byref(option(K)), so2.f64 if is64 else so2.f32, None, None,
                          so2.handle, None, C.byref(ext2), C.byref(summ2))
        hout.copy_(dx, non_blocking=True)
        e1.record()
        e1.synchronize()
        if st != 0:
            raise RuntimeError(f"status {st}")
        return e0.elapsed_time(e1), summ2

    # one untimed call first: the device buffers of the copies come from torch's caching
    # allocator and the solver's workspace from its pool, whose first growth maps memory
    e2e_once()
    e2e_ms, summ2 = e2e_once()
    so2.close()
    h2d = hx.nbytes + hl.nbytes + hu.nbytes + hn.nbytes
    d2h = hout.nbytes + 8 * summ2.num_iteration  # x and the per-evaluation f
    run.close()

    # ---- gather over ranks (max time) ----
    ms, e2e_ms, ms_dev = max_over_ranks([ms, e2e_ms, ms_dev], dist, dev)
    return {"ms_dev": ms_dev, "dev_rounds": st_dev["rounds"], "dev_syncs": st_dev["host_syncs"],
            "dev_launches": st_dev["total_launches"], "dev_timed_launches": st_dev["timed_launches"],
            "ms": ms, "kern": kern, "launches_k": launches_k, "evals_k": evals_k,
            "clocks": sampler.summary(), "e2e_ms": e2e_ms, "e2e_iters": summ2.num_iteration,
            "h2d": h2d, "d2h": d2h, "n": n, "model_bytes_iter": model_bytes}


def forms_compare(hbm, hbm_kind, sides=(4096, 2048), W=5, K=20, err_iters=300):
    """The precision forms at n = 4096^2 and 2048^2 (the same synthetic problem, seed 0):
    FP64 plain, FP32 plain, FP32 mixed (FP64 small-matrix, Cauchy and line-search scalars)
    and FP32 mixed with BF16 history storage.  Per form: ms per iteration of K iterations
    after W (CUDA events), every solver kernel's algorithmic GB/s and fraction of the HBM
    peak over those iterations, and, after err_iters iterations of each form from the same
    start, the FP32 forms' f, x and ||proj g||_inf against the FP64 run's."""
    import torch
    import lbfgsb_b200 as LB
    lib = LB.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    out = {}
    for side in sides:
        prob = make_problem(side, seed=0)
        rows = {}
        ref = None
        for key, dtype, form in (("f64_plain", "f64", 0), ("f32_plain", "f32", 0),
                                 ("f32_mixed", "f32", 1), ("f32_mixed_bf16", "f32", 2)):
            run = Runner(LB, lib, prob, dtype, form, dev)
            run.solve(2)
            ms = run.timed(W, K)
            kern, evals_k, launches_k, _ = run.steady_kernels(W, K)
            roof, per_kernel = roofline_of(kern, run.n, hbm, hbm_kind)
            pg = []

            def after(_u, _x, _f, _g, _s, sp):
                pg.append(float(sp[0].residual_g))
                return 0

            cb = run.cbt(after)
            summ, _ = run.solve(err_iters, after=C.cast(cb, C.c_void_p).value)
            x = run.x.double().cpu().numpy()
            row = {"ms_per_iteration": ms / K, "iters_per_s": 1000.0 * K / ms,
                   "evaluations_per_iteration": evals_k / K,
                   "solver_kernels_ms_per_iteration": sum(v["ms"] for v in kern.values()) / K,
                   "kernels": per_kernel, "dominant": roof,
                   "min_kernel_frac": min((v["frac"] for v in per_kernel.values()
                                           if v["frac"] is not None and v["share"] > 0.05),
                                          default=None),
                   "after_iterations": summ.num_iteration, "info": summ.info,
                   "proj_g_inf": pg[-1] if pg else None}
            # f at the final x, in FP64 (the FP32 forms report f - f0)
            fx = LB.synth_value(prob, x)
            row["f"] = fx
            if dtype == "f64":
                ref = (fx, x, row["proj_g_inf"])
            else:
                row["vs_f64"] = {"f_rel": abs(fx - ref[0]) / max(1.0, abs(ref[0])),
                                 "x_max_abs": float(np.max(np.abs(x - ref[1]))),
                                 "proj_g_inf_rel": abs(row["proj_g_inf"] - ref[2]) / max(ref[2], 1e-300)}
            rows[key] = row
            run.close()
        out[f"n{side}sq"] = rows
    out["note"] = ("FP32 forms subtract f0 = f(0) (FP64) in the objective so that f resolves the "
                   "per-iteration decrease; errors compare the iterates after the same number "
                   "of iterations from the same start (not converged solves)")
    return out


def walk_timing(side: int = 1024, bound: float = 7.5e-8):
    """The breakpoint walk at scale: the synthetic problem on a side x side grid with bounds
    +-bound, so tight that the first Cauchy steps pass most breakpoints; FP64, the device
    objective, the first three iterations profiled.  Reports the cooperative walk's launches
    and time, and the breakpoints listed and passed by the first iteration's walk."""
    import lbfgsb_b200 as LB
    prob = make_problem(side)
    prob["l"] = prob["l"] * bound
    prob["u"] = prob["u"] * bound
    o = LB.default_option(np.float64)
    o.eps_f = o.eps_g = o.eps_x = 0.0
    o.max_iteration = 2
    LB.solve(prob, np.float64, option=o, objective="device", record=False)
    r = LB.solve(prob, np.float64, option=o, objective="device", record=False, profile=True,
                 trace=True)
    k = r.stats["kernels"].get("k_walk_coop", {"launches": 0, "ms": 0.0})
    t0 = r.trace[0]
    return {"n": side * side, "bound": bound, "walk_launches": k["launches"],
            "walk_ms_total": k["ms"], "walk_ms_per_launch": k["ms"] / max(1, k["launches"]),
            "breakpoints_listed_iter1": t0["nbreak"], "segments_walked_iter1": t0["nint"],
            "ns_per_segment": 1e6 * k["ms"] / max(1, sum(t["nint"] for t in r.trace)),
            "iterations": r.num_iteration}


def dsscfg_compare():
    """The reference's own published workload (its dsscfg example, README.md:23: GPU/CPU
    speedup 10.15x at 256^2 FP64 and 36.86x at 2048^2 FP32, RTX 2080 Ti vs i9-9900K): our
    GPU path with the device dsscfg objective (csrc/dsscfg.cu), whole solves from the
    standard start (lambda = 1, unbounded, eps 1e-8, at most 1000 iterations), timed with
    CUDA events around the call; against the reference's CPU path with its own dsscfg
    objective (oracle/_ref), a bounded sample of iterations on one host core."""
    import torch
    import lbfgsb_b200 as LB
    from oracle import binding as OB
    lib = LB.load()
    out = {"published_gpu_cpu_speedup": {"fp64_256": 10.15, "fp32_2048": 36.86,
                                         "hardware": "RTX 2080 Ti vs i9-9900K",
                                         "source": "README.md:23"}}
    for key, nx, dt, cpu_iters in (("fp64_256", 256, np.float64, 60), ("fp32_2048", 2048, np.float32, 3)):
        n = nx * nx
        tdt = torch.float64 if dt == np.float64 else torch.float32
        d = LB.DsscfgObjective(nx, nx)
        x = torch.zeros(n, dtype=tdt, device="cuda")
        zeros = torch.zeros(n, dtype=tdt, device="cuda")
        nbd = torch.zeros(n, dtype=torch.int32, device="cuda")
        fn = lib.lbfgsb_b200_minimize_f64 if dt == np.float64 else lib.lbfgsb_b200_minimize_f32
        summ = LB.SummaryF64() if dt == np.float64 else LB.SummaryF32()

        def solve(iters):
            d.start(x.data_ptr(), dt)
            o = LB.default_option(dt)
            o.eps_f = o.eps_g = o.eps_x = 1e-8
            o.max_iteration = iters
            st = fn(n, x.data_ptr(), nbd.data_ptr(), zeros.data_ptr(), zeros.data_ptr(), C.byref(o),
                    d.f64 if dt == np.float64 else d.f32, None, None, d.handle, None, C.byref(summ))
            if st != 0:
                raise RuntimeError(lib.lbfgsb_b200_last_error())

        solve(5)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        solve(1000)
        e1.record()
        e1.synchronize()
        gpu_s = e0.elapsed_time(e1) / 1000.0
        gpu = {"iterations": summ.num_iteration, "info": summ.info,
               "iters_per_s": summ.num_iteration / gpu_s, "seconds": gpu_s}
        d.close()
        cpu = None
        if OB.ref_available():
            prob = OB.dsscfg_problem(nx, nx)
            x0 = OB.dsscfg_start(prob, dt, "ref")
            o = OB.default_option(dt)
            o.eps_f = o.eps_g = o.eps_x = 1e-8
            o.max_iteration = cpu_iters
            t0 = time.perf_counter()
            r = OB.run_cpu("ref", prob, dt, x0=x0, option=o, objective_source="ref", record=False)
            secs = time.perf_counter() - t0
            cpu = {"iterations": r.num_iteration, "iters_per_s": r.num_iteration / secs,
                   "sample": f"first {r.num_iteration} iterations of the same solve, 1 thread"}
        out[key] = {"gpu": gpu, "cpu_reference": cpu,
                    "speedup": (gpu["iters_per_s"] / cpu["iters_per_s"]) if cpu else None}
    return out


def _cpu_batch_worker(args):
    """One reference CPU solve (oracle/_ref, lbfgsbcpu.cpp) of a batched-workload instance;
    returns its wall seconds.  Runs in a spawned process."""
    side, seed, eps_g, max_it = args
    import sys as _sys
    for _p in (REPO, os.path.join(REPO, "lbfgsb-gpu_b200")):
        if _p not in _sys.path:
            _sys.path.insert(0, _p)
    import synth
    from oracle import binding as OB
    prob = dict(synth.synth_problem(int(side), seed=int(seed)), kind="synth")
    o = OB.default_option(np.float32)
    o.eps_g = eps_g
    o.max_iteration = max_it
    t0 = time.perf_counter()
    OB.run_cpu("ref", prob, np.float32, option=o, record=False)
    return time.perf_counter() - t0


def batched_compare(count: int = 4096, seq_sample: int = 32, cpu_budget_s: float = 25.0):
    """The batched workload: `count` independent FP32 solves of the synthetic bounded grid
    problem, problem k with seed 100 + k and grid side log-uniform in [32, 512] (n 1,024 ..
    262,144), m = 8, eps_g = 1e-6, at most 500 iterations.  Fields are generated on the
    device (bit-identical to synth.py).  All of them are solved together by
    lbfgsb_b200_minimize_batch_device_f32 (one launch per pass for every live instance);
    the sequential baseline is the plain GPU form (lbfgsb_b200_minimize_f32, host-driven, the
    reference's API) solving a sample of the same problems one after another (every
    count/seq_sample-th problem), its rate taken as the sequential rate; the CPU baseline is
    the reference's CPU path, one solve per host core, on the first problems for a bounded
    time."""
    import torch
    import lbfgsb_b200 as LB
    import synth
    lib = LB.load()
    rng = np.random.default_rng(3)
    sides = np.rint(np.exp(rng.uniform(np.log(32), np.log(512), count))).astype(int)
    seeds = [100 + k for k in range(count)]
    bt = LB.SynthBatch(sides, seeds, single_precision_fields=True, dtype=np.float32)
    opt = LB.default_option(np.float32)
    opt.eps_g = 1e-6
    opt.max_iteration = 500
    xs = [torch.zeros(int(n), dtype=torch.float32, device="cuda") for n in bt.n]
    # warm the pool and the module on a few instances
    LB.solve_batch_device(bt, xs[:8], opt, ids=list(range(8)))
    for x in xs[:8]:
        x.zero_()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rc, stat, summ, st = LB.solve_batch_device(bt, xs, opt)
    e1.record()
    e1.synchronize()
    if rc != 0:
        raise RuntimeError(lib.lbfgsb_b200_last_error())
    batched_s = e0.elapsed_time(e1) / 1000.0
    its = np.array([sm.num_iteration for sm in summ])
    infos = np.array([sm.info for sm in summ])
    # sequential plain GPU solves of a sample of the same problems
    sample = list(range(0, count, max(1, count // seq_sample)))[:seq_sample]
    seq_s = 0.0
    seq_its = []
    for p in sample:
        prob = synth.synth_problem(int(sides[p]), seed=seeds[p])
        so = LB.SynthObjective(prob, single_precision_fields=True)
        x = torch.zeros(int(bt.n[p]), dtype=torch.float32, device="cuda")
        l = torch.from_numpy(prob["l"].astype(np.float32)).cuda()
        u = torch.from_numpy(prob["u"].astype(np.float32)).cuda()
        nbd = torch.from_numpy(prob["nbd"]).cuda()
        sm = LB.SummaryF32()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = lib.lbfgsb_b200_minimize_f32(int(bt.n[p]), x.data_ptr(), nbd.data_ptr(), l.data_ptr(),
                                         u.data_ptr(), C.byref(opt), so.f32, None, None, so.handle,
                                         None, C.byref(sm))
        torch.cuda.synchronize()
        seq_s += time.perf_counter() - t0
        seq_its.append(sm.num_iteration)
        so.close()
        if r != 0:
            raise RuntimeError(lib.lbfgsb_b200_last_error())
    seq_rate = len(sample) / seq_s
    # reference CPU path, one solve per host core, on the first problems, bounded time
    cpu = None
    try:
        from oracle import binding as OB
        if OB.ref_available():
            import multiprocessing as mp
            cores = os.cpu_count() or 1
            ctx = mp.get_context("spawn")
            jobs = [(int(sides[p]), seeds[p], 1e-6, 500) for p in range(count)]
            done = 0
            t0 = time.perf_counter()
            with ctx.Pool(cores) as pool:
                for secs in pool.imap(_cpu_batch_worker, jobs[:cores * 4]):
                    done += 1
                    if time.perf_counter() - t0 > cpu_budget_s and done >= cores:
                        break
                pool.terminate()
            wall = time.perf_counter() - t0
            cpu = {"value": done / wall, "unit": "solves/s", "cores": cores, "kind": "reference",
                   "sample": f"{done} of the same problems (the first ones), one reference "
                             f"lbfgsbcpu.cpp solve per host core, {wall:.1f} s"}
    except Exception as exc:  # noqa: BLE001 - the CPU baseline is reported, never required
        cpu = {"unavailable": str(exc)[:200]}
    bt.close()
    return {"instances": count, "n_total": int(sum(bt.n)),
            "n_range": [int(min(bt.n)), int(max(bt.n))],
            "batched_solves_per_s": count / batched_s, "batched_seconds": batched_s,
            "rounds": st["rounds"], "launches": st["total_launches"],
            "host_syncs": st["host_syncs"],
            "iterations_mean": float(its.mean()), "iterations_max": int(its.max()),
            "converged": int(np.sum(np.isin(infos, [1, 2, 4]))), "hit_max_iteration": int(np.sum(infos == 5)),
            "sequential_plain_solves_per_s": seq_rate,
            "sequential_sample": f"{len(sample)} of the problems (every {max(1, count // seq_sample)}th), "
                                 "lbfgsb_b200_minimize_f32 one after another",
            "sequential_iterations_mean": float(np.mean(seq_its)),
            "speedup_vs_sequential": (count / batched_s) / seq_rate,
            "cpu_baseline": cpu}


def serving_compare(count: int = 400, rate: float = 2000.0, seq_sample: int = 16):
    """A bounded sample of the serving workload: `count` solve requests with Poisson arrivals
    at `rate` per second, request k a synthetic bounded grid problem with seed 500 + k and
    grid side log-uniform in [64, 2048] (n 4,096 .. 4,194,304), FP32 vectors with FP64
    small-matrix steps, eps_g = 1e-6, at most 500 iterations, admitted against a 150 GB HBM
    budget by the continuous-batching server (lbfgsb_b200_batch_server_*); latency is submit
    to result.  One-at-a-time baseline: the same solves one after another through the same
    engine alone (a sample of every count/seq_sample-th request), replayed through a first
    come, first served single server with the same arrivals."""
    import torch
    import lbfgsb_b200 as LB
    lib = LB.load()
    rng = np.random.default_rng(4)
    sides = np.rint(np.exp(rng.uniform(np.log(64), np.log(2048), count))).astype(int)
    gaps = rng.exponential(1.0 / rate, count)
    arrivals = np.cumsum(gaps) - gaps[0]
    bt = LB.SynthBatch(sides, [500 + k for k in range(count)], single_precision_fields=True,
                       dtype=np.float32)
    opt = LB.default_option(np.float32)
    opt.eps_g = 1e-6
    opt.max_iteration = 500
    form = LB.FORM_MIXED
    xs = [torch.zeros(int(n), dtype=torch.float32, device="cuda") for n in bt.n]
    # one-at-a-time solves of a sample (also warms the pool for the largest sizes)
    sample = list(range(0, count, max(1, count // seq_sample)))[:seq_sample]
    solo = {}
    for p in sample:
        x = torch.zeros(int(bt.n[p]), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc, stat, summ, _ = LB.solve_batch_device(bt, [x], opt, form=form, ids=[p])
        torch.cuda.synchronize()
        solo[p] = (time.perf_counter() - t0, x, summ[0])
    mean_solo = float(np.mean([v[0] for v in solo.values()]))
    sv = LB.BatchServer(bt, opt, hbm_budget_bytes=150 * 10**9, form=form, rounds_per_loop=4)
    torch.cuda.synchronize()
    tickets = []
    t0 = time.perf_counter()
    for k in range(count):
        delay = t0 + arrivals[k] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        rc, t = sv.submit(k, xs[k])
        if rc != 0:
            raise RuntimeError(lib.lbfgsb_b200_last_error().decode())
        tickets.append(t)
    outs = [sv.wait(t) for t in tickets]
    span = time.perf_counter() - t0
    peak_bytes, peak_live = sv.peak()
    sv.close()
    torch.cuda.synchronize()
    same = all(outs[p][0] == 0 and torch.equal(xs[p], solo[p][1]) and
               (outs[p][1].info, outs[p][1].num_iteration) == (solo[p][2].info, solo[p][2].num_iteration)
               for p in sample)
    lat = np.array([o[2] for o in outs])
    its = np.array([o[1].num_iteration for o in outs])
    # FCFS single server with the mean measured solo time per request
    finish, lat1 = 0.0, []
    for a in arrivals:
        finish = max(a, finish) + mean_solo
        lat1.append(finish - a)
    bt.close()
    return {"requests": count, "offered_per_s": rate, "arrival_span_s": float(arrivals[-1]),
            "hbm_budget_gb": 150, "n_range": [int(min(bt.n)), int(max(bt.n))],
            "n_total": int(sum(bt.n)), "solves_per_s": count / span,
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)),
            "peak_admitted": peak_live, "peak_workspace_gb": peak_bytes / 1e9,
            "iterations_mean": float(its.mean()),
            "one_at_a_time_solves_per_s": 1.0 / mean_solo,
            "one_at_a_time_p50_latency_s": float(np.percentile(lat1, 50)),
            "one_at_a_time_p99_latency_s": float(np.percentile(lat1, 99)),
            "one_at_a_time_sample": f"{len(sample)} requests solved alone (every "
                                    f"{max(1, count // seq_sample)}th), mean {mean_solo:.3f} s",
            "same_alone_and_in_mix": bool(same),
            "note": f"{count} requests of the 60 s stream at the same arrival rate; the offered "
                    "load exceeds the GPU's capacity, so the queue builds up"}


def max_over_ranks(values, dist, device):
    """Each value's maximum over the ranks (the job's time is its slowest rank's)."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def job_throughput(world: int, steps: int, ms: float) -> float:
    """Whole-job iterations/s: every rank runs `steps` iterations of its own replica."""
    return world * steps / (ms / 1000.0)


def cpu_reference(side: int, dtype: str, warm: int, timed: int, budget_s: float = 60.0):
    """The reference's CPU path (oracle/_ref, built from culbfgsb/lbfgsbcpu.cpp) on the same
    problem; iterations timed between after-iteration callbacks, single thread."""
    from oracle import binding as OB
    if not OB.ref_available():
        return None
    dt = np.float64 if dtype == "f64" else np.float32
    prob = make_problem(side)
    prob["kind"] = "synth"
    opt = OB.default_option(dt)
    opt.eps_f = opt.eps_g = opt.eps_x = 0.0
    lib = OB.ref_lib()
    ev = OB.host_objective(prob, dt)
    n = prob["nbd"].size
    x = np.zeros(n, dtype=dt)
    l = prob["l"].astype(dt)
    u = prob["u"].astype(dt)
    nbd = prob["nbd"].astype(np.int32)
    marks = {}
    real = C.c_double if dt == np.float64 else C.c_float
    cbt = OB.CB64 if dt == np.float64 else OB.CB32
    summ = OB.SummaryF64() if dt == np.float64 else OB.SummaryF32()
    t_start = [time.perf_counter()]

    def fg(_u, xp, fp, gp, _s):
        ev(xp, fp, gp)
        return 0

    def after(_u, xp, fp, gp, sp):
        marks[sp[0].num_iteration] = time.perf_counter()
        return 0

    def stop(_u, xp, fp, gp, sp):
        it = sp[0].num_iteration
        done = it >= warm + timed or (it > warm and time.perf_counter() - marks[warm] > budget_s)
        return 1 if done else 0

    cbs = [cbt(fg), cbt(after), cbt(stop)]
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    opt.max_iteration = warm + timed + 1
    fn = getattr(lib, "ref_lbfgsb_minimize_" + dtype)
    fn(n, P(x, real), P(nbd, C.c_int), P(l, real), P(u, real), C.byref(opt), cbs[0], cbs[1],
       cbs[2], None, C.byref(summ))
    last = max(marks)
    iters = last - warm
    secs = marks[last] - marks[warm]
    return {"value": iters / secs, "iters": iters, "secs": secs, "n": n}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--side", type=int, default=4096)
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--form", type=int, default=0, choices=[0, 1, 2],
                    help="f32 precision form: 0 plain, 1 mixed, 2 mixed with bf16 history")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    global METRIC
    METRIC = f"L-BFGS-B iterations/s at n={args.side}^2"
    config = {"workload": f"plain L-BFGS-B solve, synthetic bounded grid problem {args.side}x{args.side} "
                          f"(n={args.side * args.side}), m=8, 80% boxed / 10% lower / 10% free",
              "side": args.side, "n": args.side * args.side, "m": 8, "instances_per_gpu": 1,
              "l2": "inputs larger than L2 (every n-vector > 126 MB)"}

    if args.impl == "reference":
        if rank != 0:
            return
        warm = 1
        timed = max(1, min(args.steps, 3))
        r = cpu_reference(args.side, args.dtype, warm, timed)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable":
                              "reference CPU build oracle/_ref/libref_lbfgsb.so is missing"}))
            return
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "impl": "reference",
                "n_gpus": args.gpus, "steps": r["iters"], "warmup": warm,
                "ms_per_step": 1000.0 / r["value"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
                "config": config,
                "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                                 "sample": f"{r['iters']} iterations after {warm} of the full "
                                           f"n={r['n']} problem, reference lbfgsbcpu.cpp, 1 thread"},
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td
    try:
        r = run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    if rank != 0:
        return
    K = args.steps
    # the headline is the faster of the two drivers of the same iterations (same kernels):
    # host-driven through the reference's callback API, or device-driven
    v_host = job_throughput(world, K, r["ms"])
    v_dev = job_throughput(world, K, r["ms_dev"])
    # the device-driven figure is a difference of two solves; when both launched the same
    # rounds (the host polls in groups of rounds) the difference counts no launches and the
    # host-driven figure is used
    use_dev = v_dev > v_host and r["dev_timed_launches"] > 0
    value = v_dev if use_dev else v_host
    ms_step = (r["ms_dev"] if use_dev else r["ms"]) / K
    config["driver"] = ("device-driven: lbfgsb_b200_minimize_device, rounds captured in a CUDA graph"
                        if use_dev else
                        "host-driven: lbfgsb_b200_minimize_ext, the reference's callback API")
    hbm, hbm_kind = peaks()
    kern = r["kern"]
    roof, per_kernel = roofline_of(kern, r["n"], hbm, hbm_kind, ncu_traffic())
    solver_ms = sum(v["ms"] for v in kern.values())
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        c = cpu_reference(args.side, args.dtype, 1, 2)
        if c:
            cpu = {"value": c["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"{c['iters']} iterations (after 1) of the same n={c['n']} problem, "
                             "reference lbfgsbcpu.cpp built from source, 1 thread"}
    dss = None
    batched = None
    serving = None
    forms = None
    walk = None
    if not args.no_cpu_baseline and world == 1:
        forms = forms_compare(hbm, hbm_kind)
        walk = walk_timing()
        dss = dsscfg_compare()
        batched = batched_compare()
        serving = serving_compare()
    e2e_iters = max(1, r["e2e_iters"])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
        "config": config,
        "e2e": {"value": job_throughput(world, e2e_iters, r["e2e_ms"]), "unit": UNIT,
                "h2d_bytes_per_step": r["h2d"] / e2e_iters,
                "d2h_bytes_per_step": r["d2h"] / e2e_iters},
        "gpu_launches": (r["dev_timed_launches"] if use_dev else r["launches_k"]),
        "host_driven": {"value": v_host, "ms_per_step": r["ms"] / K, "launches": r["launches_k"]},
        "device_driven": {"value": v_dev, "ms_per_step": r["ms_dev"] / K,
                          "rounds_whole_solve": r["dev_rounds"], "host_syncs_whole_solve": r["dev_syncs"],
                          "launches_whole_solve": r["dev_launches"],
                          "timing": "a solve of W+K iterations less one of W, CUDA events around each call"},
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": r["clocks"],
        "solver_kernels_ms_per_step": solver_ms / K,
        "evaluations_per_step": r["evals_k"] / K,
        "hbm_GBps_model": r["model_bytes_iter"] / (solver_ms / K / 1000.0) / 1e9 if solver_ms else None,
        "kernels": per_kernel,
        "forms": forms,
        "walk": walk,
        "dsscfg": dss,
        "serving": serving,
        "batched": batched,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
