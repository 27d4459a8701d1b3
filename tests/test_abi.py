"""The C-ABI library loads and exports every function include/*.h declares (CPU only)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src):
            name = m.group(1)
            prefix = src[max(0, m.start() - 80):m.start()]
            # a declaration: the name follows a type at the start of a statement
            stmt = re.split(r"[;{}]", prefix)[-1]
            # inline C++ forwarders (list_stockham_b200.h) are not exports
            if re.search(r"(^|[;}\n])\s*(const\s+)?[A-Za-z_][A-Za-z0-9_ ]*[\s\*]+$", prefix) and \
                    name not in ("if", "defined", "sizeof") and not re.search(r"\binline\b", stmt):
                names.add(name)
    return sorted(names)


def test_header_declares_reference_entry_points():
    names = set(declared_functions())
    for ref in ("is_cuda_enabled", "num_of_cuda_devices", "is_double_float_enabled",
                "global_memory_in_bytes", "global_memory_in_megabytes", "can_call_fftmul_uni",
                "cumodp_fft_uni", "cumodp_invfft_uni", "cumodp_fft_bivariate",
                "cumodp_invfft_bivariate", "cumodp_fftmul_uni", "init_cuda_scube"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    from cumodp_b200 import LIB_PATH
    lib = ctypes.CDLL(LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_queries_without_gpu_do_not_crash():
    import cumodp_b200 as cm
    # on a machine without a GPU these report "no device"; with one, a device
    n = cm.num_of_cuda_devices()
    assert n >= 0
    assert cm.is_cuda_enabled() == (n > 0)


def test_modpn_links_against_this_library():
    """modpn with its GPU dispatch links unchanged against libcumodp.so (no GPU call)."""
    import oracle
    if not oracle.modpn_gpu_available():
        pytest.skip("modpn GPU-dispatch build absent (needs the reference sources)")
    import subprocess
    out = subprocess.run(["ldd", oracle.MODPN_GPU_SO], capture_output=True, text=True).stdout
    assert "libcumodp.so" in out
    lib = ctypes.CDLL(oracle.MODPN_GPU_SO)  # resolves cumodp_fftmul_uni / can_call_fftmul_uni
    assert hasattr(lib, "modpn_gpu_fftmul")


def test_cpp_forwarding_header_compiles():
    """include/list_stockham_b200.h and stockham_b200.h give the reference's C++ overloads."""
    import shutil
    import subprocess
    import tempfile
    gxx = shutil.which("g++")
    cuda_inc = "/usr/local/cuda/include"
    if not gxx or not os.path.isdir(cuda_inc):
        pytest.skip("g++ or CUDA headers absent")
    src = (
        '#include "list_stockham_b200.h"\n'
        '#include "stockham_b200.h"\n'
        "void use(sfixn* X, const sfixn* W) {\n"
        "  cumodp_err a = list_stockham_dev(X, 4, 10, 3, 469762049);\n"
        "  cumodp_err b = list_stockham_dev(X, 4, 10, W, 469762049);\n"
        "  cumodp_err c = bi_stockham_poly_mul_dev(64, 6, 512, 9, X, X + 32768, 469762049);\n"
        "  stockham_dev(X, 1024, 10, 3, 469762049);\n"
        "  stockham_dev(X, 1024, 10, W, 469762049);\n"
        "  inverse_stockham_dev(X, 1024, 10, 3, 469762049);\n"
        "  inverse_stockham_dev(X, 1024, 10, W, 469762049);\n"
        "  stockham_host(X, 1024, 10, 3, 469762049);\n"
        "  inverse_stockham_host(X, 1024, 10, 3, 469762049);\n"
        "  stockham_poly_mul_dev(1024, 10, X, X + 1024, 469762049);\n"
        "  stockham_poly_mul_host(10, X, 5, W, 5, W, 469762049);\n"
        "  (void)a; (void)b; (void)c;\n}\n")
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "use.cpp")
        open(f, "w").write(src)
        r = subprocess.run([gxx, "-fsyntax-only", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc, f],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
