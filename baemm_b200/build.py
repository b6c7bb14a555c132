"""Build libbaemm_cuda.so in-tree for sm_100a (B200).

    python -m baemm_b200.build          # incremental
    python -m baemm_b200.build --clean  # rebuild everything

Every translation unit in baemm_b200/csrc/*.cu is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo`` (plus the per-file flags
in FILE_FLAGS) into baemm_b200/_build/, then linked (static CUDA runtime) into
baemm_b200/libbaemm_cuda.so.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libbaemm_cuda.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]
# Per-file flags.  The tensor-core form flushes FP32 denormals (|x| < 1.2e-38)
# to zero: its rsqrt and sincos then skip the denormal handling.  On the
# 153600-triangle torus with 64 right-hand sides this is 142.0 vs 144.8 ms,
# with the same error.  The entries, right-hand sides and sums there are many
# orders of magnitude above the denormal range.
FILE_FLAGS = {"tc.cu": ["-ftz=true"]}


def _newer(src: str, dst: str, deps: list[str]) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return os.path.getmtime(src) > t or any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, extra: list[str]) -> str:
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    return (r.stdout + r.stderr).strip()


def build(clean: bool = False, verbose: bool = False, ptxas_verbose: bool = False, jobs: int = 0) -> str:
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h")))
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    todo = []
    objs = []
    for s in sources:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if clean or ptxas_verbose or _newer(s, o, headers):
            todo.append((s, o))
    if todo:
        n = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=n) as ex:
            futs = {ex.submit(_compile, s, o, extra + FILE_FLAGS.get(os.path.basename(s), [])): s
                    for s, o in todo}
            for f in cf.as_completed(futs):
                msg = f.result()
                if (verbose or ptxas_verbose) and msg:
                    print(f"--- {os.path.basename(futs[f])}\n{msg}")
    if todo or not os.path.exists(OUT):
        tmp = OUT + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-cudart", "static", *objs, "-o", tmp]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, OUT)
    return OUT


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=0)
    a = ap.parse_args(argv)
    out = build(a.clean, a.verbose, a.ptxas_verbose, a.jobs)
    print(out)


if __name__ == "__main__":
    sys.exit(main())
