"""Record golden fixtures from the reference's own CPU L-BFGS-B.

Runs every case of cases.py through oracle/_ref/libref_lbfgsb.so (culbfgsb/lbfgsbcpu.cpp
compiled from the reference sources by oracle/Makefile) and writes
  golden.json   -- per case: info, num_iteration, residuals, every funcgrad point as
                   (f, sha1 of x bytes), every after-iteration summary, sha1 of the final x;
  golden_x.npz  -- the final x of every case.
Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from oracle import binding as B  # noqa: E402
from cases import CASES, apply_options, make_case  # noqa: E402


def record(which: str, name: str):
    prob, dtype, x0, over, stop = make_case(name)
    opt = apply_options(B.default_option(dtype), over)
    r = B.run_cpu(which, prob, dtype, x0=x0, option=opt, custom_stop_at=stop)
    return r, {
        "dtype": np.dtype(dtype).name,
        "info": r.info,
        "num_iteration": r.num_iteration,
        "residual_g": r.residual_g,
        "residual_f": r.residual_f,
        "residual_x": r.residual_x,
        "evals": r.evals,
        "iters": r.iters,
        "x_sha1": hashlib.sha1(r.x.tobytes()).hexdigest()[:16],
    }


def main():
    B.build()
    if not B.ref_available():
        raise SystemExit("reference build missing: oracle/_ref/libref_lbfgsb.so")
    out, xs = {}, {}
    for name in CASES:
        r, rec = record("ref", name)
        out[name] = rec
        xs[name] = r.x
        print(f"{name:28s} info={rec['info']:2d} iters={rec['num_iteration']:4d} "
              f"evals={len(rec['evals'])}")
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(out, fh, indent=0)
    np.savez_compressed(os.path.join(HERE, "golden_x.npz"), **xs)


if __name__ == "__main__":
    main()
