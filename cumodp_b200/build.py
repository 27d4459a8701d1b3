"""Build libcumodp.so (the C-ABI library) in-tree for sm_100a.

    python -m cumodp_b200.build [--force] [-j N] [--ptxas-v]

Each csrc/*.cu is compiled to an object under cumodp_b200/_build/ with
``nvcc -gencode arch=compute_100a,code=sm_100a``; the objects are linked into
cumodp_b200/libcumodp.so against the CUDA runtime.  Rebuilds only what
changed (sources or any header in csrc/ or include/).  bench/percall.c (the
benchmark's one-call-per-product loop in C) becomes libcumodp_percall.so.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcumodp.so")
PERCALL = os.path.join(HERE, "libcumodp_percall.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I" + os.path.join(ROOT, "include")]


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(SRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, force: bool, ptxas_v: bool) -> str:
    obj = os.path.join(OUT, os.path.basename(src) + ".o")
    newest = max(os.path.getmtime(src), _headers_mtime(), os.path.getmtime(__file__))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    if ptxas_v:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if ptxas_v:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, jobs: int = 8, ptxas_v: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(SRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, ptxas_v), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    _build_percall(force)
    return LIB


def _build_percall(force: bool) -> None:
    """bench/percall.c -> libcumodp_percall.so: a C loop of one product call each (benchmark driver)."""
    src = os.path.join(HERE, "bench", "percall.c")
    if not os.path.exists(src):
        return
    if not force and os.path.exists(PERCALL) and os.path.getmtime(PERCALL) >= max(os.path.getmtime(src),
                                                                                  os.path.getmtime(LIB)):
        return
    cmd = [os.environ.get("CC", "gcc"), "-O2", "-shared", "-fPIC", "-I" + os.path.join(ROOT, "include"), src,
           "-o", PERCALL, "-L" + HERE, "-lcumodp", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"percall driver build failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.ptxas_v))
