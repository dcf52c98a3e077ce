"""Builds libmontmul_b200.so in-tree for sm_100a (the reference's build.rs step, montmul/build.rs).

The kernels of each transform length are compiled as their own object (mm_inst.cu with
-DMM_M=m), in parallel, then linked with the host backend into one shared library next to this
file. Run `python -m montmul_b200.build` (add --force to rebuild everything).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmontmul_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
LOG_NS = range(2, 14)   # shared-memory lengths: n = 4 .. 8192 (L = 8 .. 16384)


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".hpp"))] + \
           [os.path.join(HERE, "..", "include", "montmul_b200.h")]


def _stale(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _compile(args):
    cmd, obj, log = args
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {obj}:\n{r.stderr[-4000:]}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    heads = _headers()
    nv = nvcc()
    jobs_list, objs = [], []
    for m in LOG_NS:
        obj = os.path.join(BUILD, f"mm_inst_{m}.o")
        src = os.path.join(CSRC, "mm_inst.cu")
        objs.append(obj)
        if force or _stale(obj, [src] + heads):
            jobs_list.append(([nv, *ARCH, *FLAGS, f"-DMM_M={m}", "-c", src, "-o", obj], obj, obj + ".log"))
    for name in ("mm_backend", "mm_global", "mm_cluster", "mm_cluster_half", "mm_mixed", "mm_transform", "mm_peak",
                 "mm_noalloc"):
        obj = os.path.join(BUILD, f"{name}.o")
        src = os.path.join(CSRC, f"{name}.cu")
        objs.append(obj)
        if force or _stale(obj, [src] + heads):
            jobs_list.append(([nv, *ARCH, *FLAGS, "-c", src, "-o", obj], obj, obj + ".log"))
    if jobs_list:
        n = jobs or max(1, min(len(jobs_list), os.cpu_count() or 1))
        with ThreadPoolExecutor(n) as ex:
            for obj in ex.map(_compile, jobs_list):
                if verbose:
                    print("built", os.path.relpath(obj, HERE))
    if force or _stale(LIB, objs):
        subprocess.run([nv, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], check=True)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs, verbose=True))


if __name__ == "__main__":
    sys.exit(main())
