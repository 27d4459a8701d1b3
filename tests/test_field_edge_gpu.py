"""The field primitives and register DFTs at the edges of their stated ranges.

csrc/field.cuh states: mul_shoup(a, w) in [0, 2p) for any 32-bit a (w < p);
mul_mont(a, b) = a b 2^-32 mod p in [0, 2p) whenever a b < 2^32 p;
red2: [0, 4p) -> [0, 2p); red1: [0, 2p) -> [0, p).  csrc/ntt_engine.cuh
states the register DFTs' input and output ranges (DIF: [0, 2p) -> [0, 2p),
or outputs j >= 1 in [0, 4p) with TW; DIT: [0, 4p) -> [0, 4p)).  Random
residues rarely reach those edges, so tests/field_edge.cu runs the device
code on the edge operands themselves (2^32 - 1, 4p - 1, 2p - 1, p - 1, the
Montgomery bound) for the five test primes, and every result is checked
against exact integer arithmetic here: the value mod p and the range.
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
PRIMES = [469762049, 754974721, 962592769, 950009857, 940572673]
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


@pytest.fixture(scope="module")
def fe(cm, tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc absent")
    out = str(tmp_path_factory.mktemp("fe") / "libfield_edge.so")
    r = subprocess.run([nvcc, "-O3", "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                        "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
                        os.path.join(ROOT, "tests", "field_edge.cu"), "-o", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    L = C.CDLL(out)
    L.field_edge.argtypes = [_u32p, _u32p, C.c_int, C.c_uint32, C.c_uint32, _u32p]
    L.dft32.argtypes = [_u32p, C.c_int, C.c_uint32, _u32p, C.c_int, _u32p]
    return L


def _pinv_neg(p):
    return (-pow(p, -1, 1 << 32)) % (1 << 32)


def _edges(p):
    return [0, 1, 2, p - 2, p - 1, p, p + 1, 2 * p - 1, 2 * p, 2 * p + 1, 3 * p, 4 * p - 2, 4 * p - 1,
            1 << 30, (1 << 31) - 1, 1 << 31, (1 << 32) - 2, (1 << 32) - 1]


@pytest.mark.parametrize("p", PRIMES)
def test_mul_shoup_mul_mont_red_at_the_edges(fe, p):
    rnd = SplitMix64(p)
    xs = _edges(p) + [int(v) for v in rnd.residues(16, 1 << 32)]
    ws = [0, 1, 2, (p - 1) // 2, (p + 1) // 2, p - 2, p - 1] + [int(v) for v in rnd.residues(9, p)]
    pairs = [(x, w) for x in xs for w in ws]
    # Montgomery at its bound: the largest b with a b < 2^32 p, for edge a
    for a in [x for x in xs if x > 0]:
        b = min((1 << 32) - 1, ((1 << 32) * p - 1) // a)
        pairs += [(a, b), (a, max(0, b - 1))]
    a = np.array([x for x, _ in pairs], np.uint32)
    b = np.array([y for _, y in pairs], np.uint32)
    out = np.empty(4 * len(pairs), np.uint32)
    assert fe.field_edge(a, b, len(pairs), p, _pinv_neg(p), out) == 0
    out = out.reshape(-1, 4).astype(object)
    rinv = pow(1 << 32, -1, p)
    for (x, y), (shoup, mont, r2, r1) in zip(pairs, out):
        if y < p:
            assert shoup < 2 * p and shoup % p == x * y % p, (p, x, y, shoup)
        if x * y < (1 << 32) * p:
            assert mont < 2 * p and mont % p == x * y * rinv % p, (p, x, y, mont)
        if x < 4 * p:
            assert r2 < 2 * p and r2 % (2 * p) == x % (2 * p), (p, x, r2)
        if x < 2 * p:
            assert r1 < p and r1 == x % p, (p, x, r1)


def _bitrev5(j):
    return int(f"{j:05b}"[::-1], 2)


@pytest.mark.parametrize("p", PRIMES)
def test_register_dft32_ranges_at_the_edges(fe, oracle_mod, p):
    w = oracle_mod.primitive_root(5, p)
    wi = pow(w, p - 2, p)
    fwd = np.array([pow(w, j, p) for j in range(16)], np.uint32)
    inv = np.array([pow(wi, j, p) for j in range(16)], np.uint32)
    rnd = SplitMix64(3 * p)

    def vectors(top):
        v = [[top - 1] * 32, [0] * 32, [(top - 1) if j % 2 else 0 for j in range(32)],
             [(top - 1) if j < 16 else 0 for j in range(32)], [p] * 32, [p - 1] * 32]
        v += [[int(t) for t in rnd.residues(32, top)] for _ in range(26)]
        return np.array(v, np.uint32)

    # forward DIF: inputs in [0, 2p); x[j] ends holding X[bitrev(j)]
    for dirn in (0, 2):
        x = vectors(2 * p)
        y = np.empty_like(x)
        assert fe.dft32(x.reshape(-1), len(x), p, fwd, dirn, y.reshape(-1)) == 0
        for xv, yv in zip(x.tolist(), y.tolist()):
            for j in range(32):
                k = _bitrev5(j)
                want = sum(xv[i] * pow(w, i * k, p) for i in range(32)) % p
                bound = 4 * p if (dirn == 2 and j >= 1) else 2 * p
                assert yv[j] < bound and yv[j] % p == want, (p, dirn, j)
    # inverse DIT: inputs in [0, 4p) (PRE: inputs j >= 1 in [0, 2p)); x[j] holds Y[bitrev(j)],
    # output j is 32 y[j] = sum_k Y[k] w^-jk, in [0, 4p)
    for dirn in (1, 3):
        x = vectors(4 * p)
        if dirn == 3:
            x[:, 1:] %= 2 * p
        y = np.empty_like(x)
        assert fe.dft32(x.reshape(-1), len(x), p, inv, dirn, y.reshape(-1)) == 0
        for xv, yv in zip(x.tolist(), y.tolist()):
            Y = [0] * 32
            for j in range(32):
                Y[_bitrev5(j)] = xv[j]
            for j in range(32):
                want = sum(Y[k] * pow(wi, j * k, p) for k in range(32)) % p
                assert yv[j] < 4 * p and yv[j] % p == want, (p, dirn, j)
