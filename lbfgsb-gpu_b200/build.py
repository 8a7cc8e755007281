"""Build recipe of liblbfgsb_b200.so (sm_100a only).

    python lbfgsb-gpu_b200/build.py        # or __graft_entry__.build()

nvcc compiles each csrc/*.cu translation unit (in parallel, objects in _build/) for
compute_100a/sm_100a with -fmad=false (elementwise steps must round like the reference's
scalar code; reductions use explicit fma()) and links lbfgsb-gpu_b200/liblbfgsb_b200.so, in
the source tree, so the built library travels with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liblbfgsb_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in
           ("driver.cu", "batch.cu", "objective.cu", "dsscfg.cu", "noalloc.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in
           ("common.cuh", "small.cuh", "state.cuh", "reduce.cuh", "tiles.cuh", "warp_small.cuh",
            "passes.cuh", "walk.cuh", "rounds.cuh", "host.cuh", "batch_tune.h", "shard.cuh")]
HEADERS.append(os.path.join(REPO, "include", "lbfgsb_b200.h"))

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-fmad=false", "-Xcompiler", "-fPIC", f"-I{os.path.join(REPO, 'include')}",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA 12.9 toolkit is required to build")
    return cand


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compile each translation unit to an object in parallel, then link the library."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.basename(src) + ".o") for src in SOURCES]
    cmds = [[nvcc(), *NVCC_FLAGS, *(extra or []), "-c", "-o", obj, src]
            for src, obj in zip(SOURCES, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), flush=True)
    with ThreadPoolExecutor(max_workers=len(cmds)) as pool:
        results = list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for res in results:
        if res.returncode != 0 or (extra and res.stderr):
            sys.stderr.write(res.stdout + res.stderr)
    if any(res.returncode != 0 for res in results):
        raise RuntimeError("nvcc failed building liblbfgsb_b200.so")
    link = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB + ".tmp", *objs]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed linking liblbfgsb_b200.so")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None
    print(build(force=force or bool(extra), verbose=True, extra=extra))
