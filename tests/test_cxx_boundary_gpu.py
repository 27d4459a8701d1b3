"""The reference's C++ boundary, called from compiled C++.

include/stockham_b200.h gives the overloads of the reference's
include/stockham.h:39-94 (stockham_dev x2, inverse_stockham_dev x2,
stockham_host, inverse_stockham_host, stockham_poly_mul_dev,
stockham_poly_mul_host) and include/list_stockham_b200.h those of
list_stockham_dev and bi_stockham_poly_mul_dev.  tests/cxx_boundary.cpp calls
each of them from C++ the way the reference's internal callers do; its
results must equal the oracle's (bit-exact: integer results).
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P = 469762049
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


@pytest.fixture(scope="module")
def drv(cm, tmp_path_factory):
    gxx = shutil.which("g++")
    cuda = "/usr/local/cuda"
    if not gxx or not os.path.isdir(os.path.join(cuda, "include")):
        pytest.skip("g++ or the CUDA headers are absent")
    cm.lib()  # the library instance the driver links against is the one already loaded
    libdir = os.path.join(ROOT, "cumodp_b200")
    out = str(tmp_path_factory.mktemp("cxx") / "libcxx_boundary.so")
    cmd = [gxx, "-O1", "-shared", "-fPIC", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(cuda, "include"), os.path.join(ROOT, "tests", "cxx_boundary.cpp"), "-o", out,
           "-L", libdir, "-lcumodp", "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath," + libdir,
           "-Wl,-rpath," + os.path.join(cuda, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    L = C.CDLL(out)
    L.cxx_transform.argtypes = [_i32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int]
    L.cxx_poly_mul_dev.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, C.c_int32]
    L.cxx_poly_mul_host.argtypes = [C.c_int32, _i32p, C.c_int32, _i32p, C.c_int32, _i32p, C.c_int32]
    L.cxx_list.argtypes = [_i32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int]
    L.cxx_bi_mul.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, C.c_int32]
    return L


def _cyclic(a, b, n, oracle_mod):
    h = oracle_mod.polymul(a, b, P).astype(np.uint64)
    out = h[:n].copy()
    out[:len(h) - n] += h[n:]
    return (out % P).astype(np.uint32)


@pytest.mark.parametrize("k", [0, 1, 3, 6, 12, 15, 20])
def test_transform_overloads(drv, oracle_mod, k):
    n = 1 << k
    x = SplitMix64(900 + k).residues(n, P)
    w = oracle_mod.primitive_root(k, P)
    want = oracle_mod.ntt(x, w, P)
    for mode in (0, 1, 4):  # stockham_dev(w), stockham_dev(W), stockham_host
        y = x.view(np.int32).copy()
        assert drv.cxx_transform(y, n, k, w, P, mode) == 0
        assert np.array_equal(y.view(np.uint32), want), mode
    for mode in (2, 3, 5):  # inverse_stockham_dev(w), inverse_stockham_dev(W of w^-1), inverse_stockham_host
        y = want.view(np.int32).copy()
        assert drv.cxx_transform(y, n, k, w, P, mode) == 0
        assert np.array_equal(y.view(np.uint32), x), mode


def test_transform_overload_rejects_wrong_length(drv):
    y = np.zeros(64, np.int32)
    assert drv.cxx_transform(y, 63, 6, 1, P, 0) != 0


@pytest.mark.parametrize("e", [0, 2, 4, 5, 8, 12, 13, 14, 16, 21])
def test_poly_mul_dev_is_the_cyclic_convolution(drv, oracle_mod, e):
    """stockham_poly_mul_dev(n, e, F, G, p): F <- DFT^-1(DFT F * DFT G), full-length operands (wrap-around)."""
    n = 1 << e
    r = SplitMix64(1000 + e)
    f, g = r.residues(n, P), r.residues(n, P)
    F, G = f.view(np.int32).copy(), g.view(np.int32).copy()
    assert drv.cxx_poly_mul_dev(n, e, F, G, P) == 0
    assert np.array_equal(F.view(np.uint32), _cyclic(f, g, n, oracle_mod))
    assert np.array_equal(G.view(np.uint32), g)  # G is left unchanged


def test_poly_mul_dev_padded_is_the_product(drv, oracle_mod):
    """With deg F + deg G < n the cyclic convolution is the polynomial product (the reference's use)."""
    e, n = 17, 1 << 17
    r = SplitMix64(1100)
    f = np.zeros(n, np.uint32)
    g = np.zeros(n, np.uint32)
    f[:50000] = r.residues(50000, P)
    g[:60000] = r.residues(60000, P)
    F, G = f.view(np.int32).copy(), g.view(np.int32).copy()
    assert drv.cxx_poly_mul_dev(n, e, F, G, P) == 0
    want = oracle_mod.polymul(f[:50000], g[:60000], P)
    assert np.array_equal(F.view(np.uint32)[:len(want)], want)
    assert not F[len(want):].any()


def test_poly_mul_dev_past_the_product_kernels(drv):
    """e = 26 (composed from natural-order transforms): times c x^s is a rotation of F by s, times c."""
    e, n = 26, 1 << 26
    r = SplitMix64(1200)
    f = r.residues(n, P)
    s, c = 12345677, 987654
    g = np.zeros(n, np.uint32)
    g[s] = c
    F, G = f.view(np.int32).copy(), g.view(np.int32).copy()
    assert drv.cxx_poly_mul_dev(n, e, F, G, P) == 0
    want = (np.roll(f, s).astype(np.uint64) * c % P).astype(np.uint32)
    assert np.array_equal(F.view(np.uint32), want)


@pytest.mark.parametrize("df,dg,dh", [(100, 200, 300), (4095, 4095, 8190), (30000, 20000, 60000), (500, 40, 100)])
def test_poly_mul_host(drv, oracle_mod, df, dg, dh):
    r = SplitMix64(1300 + df)
    f, g = r.residues(df + 1, P), r.residues(dg + 1, P)
    H = np.full(dh + 1, -1, np.int32)
    assert drv.cxx_poly_mul_host(dh, H, df, f.view(np.int32), dg, g.view(np.int32), P) == 0
    want = np.zeros(dh + 1, np.uint32)
    prod = oracle_mod.polymul(f, g, P)
    want[:min(dh + 1, len(prod))] = prod[:dh + 1]
    assert np.array_equal(H.view(np.uint32), want)


@pytest.mark.parametrize("use_table", [0, 1])
@pytest.mark.parametrize("k", [1, 10])
def test_list_overloads(drv, oracle_mod, use_table, k):
    m = 5
    x = SplitMix64(1400 + use_table).residues(m << k, P)
    w = oracle_mod.primitive_root(k, P)
    X = x.view(np.int32).copy()
    assert drv.cxx_list(X, m, k, w, P, use_table) == 0
    for i in range(m):
        assert np.array_equal(X.view(np.uint32)[i << k:(i + 1) << k], oracle_mod.ntt(x[i << k:(i + 1) << k], w, P))


def test_bivariate_mul_overload(drv, oracle_mod):
    em, en = 6, 9
    r = SplitMix64(1500)
    F = np.zeros((1 << em, 1 << en), np.uint32)
    G = np.zeros((1 << em, 1 << en), np.uint32)
    F[:20, :200] = r.residues(20 * 200, P).reshape(20, 200)
    G[:30, :150] = r.residues(30 * 150, P).reshape(30, 150)
    want = oracle_mod.bivariate_mul(F[:20, :200], G[:30, :150], P)
    Fd = F.reshape(-1).view(np.int32).copy()
    assert drv.cxx_bi_mul(em, en, Fd, G.reshape(-1).view(np.int32).copy(), P) == 0
    got = Fd.view(np.uint32).reshape(1 << em, 1 << en)
    assert np.array_equal(got[:want.shape[0], :want.shape[1]], want)
    assert not got[want.shape[0]:].any() and not got[:, want.shape[1]:].any()
