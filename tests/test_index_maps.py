"""Bounds and collision check of every kernel index map, on the CPU.

Compiles tests/index_maps_check.cu (the kernels' own __host__ __device__ index
functions, compiled for the host) with nvcc and runs it: every level of every
row and column plan touches each shared-memory word exactly once, the fast
address paths equal the plain swizzle, twiddle reads stay in their tables,
16-column tiles keep their half-warps on opposite bank halves, and the
digit-reversal maps are permutations.  No GPU is involved.
"""
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_index_maps_in_bounds_and_bijective():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc absent")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "index_maps_check")
        r = subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                            "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "include"),
                            os.path.join(ROOT, "tests", "index_maps_check.cu"), "-o", exe],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]
        out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stdout[-2000:]
        assert out.stdout.strip().endswith("OK: 0 failures")
