"""Autotuner of the batched passes: tiles per CTA for each instance-size bucket.

    python lbfgsb-gpu_b200/autotune.py [--write] [--out LOG]

For each bucket of csrc/batch_tune.h (n <= 4096, <= 16384, <= 65536, <= 262144, larger) a
batch of synthetic FP32 problems with grid sides inside the bucket is solved by
lbfgsb_b200_minimize_batch_device_f32 for a fixed number of iterations (eps = 0), once per
candidate tiles-per-CTA value (set with lbfgsb_b200_batch_tiles_per_cta), and timed with
CUDA events; the fastest candidate of each bucket wins.  --write rewrites csrc/batch_tune.h
with the winners (rebuild the library afterwards); the timings go to stdout (JSON) and to
--out.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

# grid sides per bucket (n = side^2 inside the bucket) and how many problems of each
BUCKETS = [
    {"name": "n<=4096", "sides": (32, 64), "count": 1024},
    {"name": "n<=16384", "sides": (65, 128), "count": 512},
    {"name": "n<=65536", "sides": (129, 256), "count": 256},
    {"name": "n<=262144", "sides": (257, 512), "count": 96},
    {"name": "n>262144", "sides": (513, 1024), "count": 24},
]
CANDIDATES = [4, 8, 16, 32, 64, 128, 1024]
ITERATIONS = 30


def time_bucket(LB, lib, bucket_index, spec, tiles, seed=7):
    import torch
    rng = np.random.default_rng(seed + bucket_index)
    lo, hi = spec["sides"]
    sides = rng.integers(lo, hi + 1, spec["count"])
    bt = LB.SynthBatch(sides, [1000 * bucket_index + k for k in range(len(sides))],
                       single_precision_fields=True, dtype=np.float32)
    opt = LB.default_option(np.float32)
    opt.eps_f = opt.eps_g = opt.eps_x = 0.0
    opt.max_iteration = ITERATIONS - 1
    out = {}
    for t in tiles:
        lib.lbfgsb_b200_batch_tiles_per_cta(bucket_index, t)
        xs = [torch.zeros(int(n), dtype=torch.float32, device="cuda") for n in bt.n]
        LB.solve_batch_device(bt, xs[:4], opt, ids=[0, 1, 2, 3])  # warm the sizes
        for x in xs:
            x.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        rc, stat, summ, _ = LB.solve_batch_device(bt, xs, opt)
        e1.record()
        e1.synchronize()
        if rc != 0:
            raise RuntimeError(lib.lbfgsb_b200_last_error())
        out[t] = e0.elapsed_time(e1)
    lib.lbfgsb_b200_batch_tiles_per_cta(bucket_index, 0)
    bt.close()
    return out


def write_header(winners):
    path = os.path.join(HERE, "csrc", "batch_tune.h")
    body = ", ".join(str(w) for w in winners)
    text = f"""// batch_tune.h -- tiles per CTA of the batched passes by instance size, the table that
// lbfgsb-gpu_b200/autotune.py writes after timing batched solves on the GPU.
// Buckets: n <= 4096, <= 16384, <= 65536, <= 262144, larger.
#pragma once

namespace lbfgsb_b200 {{
constexpr int kTuneBuckets = 5;
constexpr int kTunedTilesPerCta[kTuneBuckets] = {{{body}}};
}}  // namespace lbfgsb_b200
"""
    with open(path, "w") as fh:
        fh.write(text)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--write", action="store_true")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    import torch
    import lbfgsb_b200 as LB
    if not torch.cuda.is_available():
        raise SystemExit("the autotuner needs a CUDA device")
    lib = LB.load()
    result = {"iterations": ITERATIONS, "buckets": []}
    winners = []
    for b, spec in enumerate(BUCKETS):
        ms = time_bucket(LB, lib, b, spec, CANDIDATES)
        best = min(ms, key=ms.get)
        winners.append(best)
        result["buckets"].append({"bucket": spec["name"], "sides": spec["sides"],
                                  "problems": spec["count"], "ms": ms, "tiles_per_cta": best})
    result["winners"] = winners
    text = json.dumps(result, indent=1)
    print(text)
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(text)
    if args.write:
        write_header(winners)


if __name__ == "__main__":
    main()
