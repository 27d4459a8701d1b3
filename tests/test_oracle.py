"""Pins the CPU oracle before it is trusted as the checker (CPU only).

* exact integer products against the reference's golden files
  (benchmark/*.test, committed gzipped under tests/golden/);
* the two-convolution helpers against the reference's unit-test KATs
  (unit_tests/test_two_convolution_poly_mul.cpp, parsed into unit_kats.json);
* the mod-p product against modpn's own FFT multiply (EX_Mont_FFTMul,
  modpn/src/FMUL.c:2015-2030) compiled from the reference sources, when
  that build is present;
* the transform against the DFT definition.
"""
import gzip
import json
import os

import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
P0 = 469762049


def read_golden(name):
    with gzip.open(os.path.join(GOLDEN, name), "rt") as fh:
        lines = [ln.split() for ln in fh.read().strip().split("\n")]
    return [[int(v) for v in ln] for ln in lines[:3]]


FIXED_WIDTH = sorted(f for f in os.listdir(GOLDEN) if f.startswith("bench_n") and "_p" in f)
BIG = sorted(f for f in os.listdir(GOLDEN) if f.startswith("bench_n") and "_p" not in f)
KATS = json.load(open(os.path.join(GOLDEN, "unit_kats.json")))


def test_golden_inventory():
    # every size of the reference's fixed-width golden set is present
    sizes = {int(f.split("_")[1][1:]) for f in FIXED_WIDTH}
    assert {32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384} <= sizes
    assert len(KATS["products"]) >= 8 and len(KATS["limb_split"]) >= 4


@pytest.mark.parametrize("name", FIXED_WIDTH)
def test_i128_oracle_matches_golden_files(oracle_mod, name):
    a, b, c = read_golden(name)
    got = oracle_mod.polymul_i128(np.array(a, np.int64), np.array(b, np.int64))
    assert got == c


@pytest.mark.parametrize("name", BIG)
def test_big_golden_files_are_products(oracle_mod, name):
    """The big-coefficient files are self-consistent exact products (python ints).

    Up to 256 terms by the schoolbook; the longer files by the evaluation
    identity c(t) = a(t) b(t) mod q at seeded points t and the prime
    q = 2^127 - 1 (a wrong coefficient survives one point with probability
    at most deg / q)."""
    a, b, c = read_golden(name)
    assert len(c) == len(a) + len(b) - 1
    if len(a) <= 256:
        assert oracle_mod.bigint_polymul(a, b) == c
        return
    q = (1 << 127) - 1

    def ev(poly, t):
        acc = 0
        for v in reversed(poly):
            acc = (acc * t + v) % q
        return acc
    for t in (3, 0x1234567890ABCDEF1234567, q - 2):
        assert ev(c, t) == ev(a, t) * ev(b, t) % q


def test_unit_kat_products(oracle_mod):
    for case in KATS["products"]:
        got = oracle_mod.polymul_i128(np.array(case["a"], np.int64), np.array(case["b"], np.int64))
        assert got == case["c"]


def test_unit_kat_bit_width(oracle_mod):
    for case in KATS["bit_width"]:
        if max(abs(v) for v in case["a"] + case["b"]) >= 1 << 63:
            continue  # beyond int64 (the 160-bit case)
        got = oracle_mod.bit_width(np.array(case["a"], np.int64), np.array(case["b"], np.int64))
        assert got == case["expected"]


def test_unit_kat_limb_split(oracle_mod):
    for case in KATS["limb_split"]:
        got = oracle_mod.limb_split(np.array(case["a"], np.int64), case["K"], case["M"], case["prime"])
        assert got.tolist() == case["expected"]


def test_unit_kat_scale_x(oracle_mod):
    for case in KATS["scale_x"]:
        got = oracle_mod.scale_x(np.array(case["A"], np.uint32), case["K"], case["theta"], case["prime"])
        assert got.tolist() == case["expected"]


def test_dft_definition(oracle_mod):
    for p in (P0, 257, 962592769):
        for k in (1, 3, 8):
            if k > oracle_mod.fourier_degree(p):
                continue
            r = SplitMix64(p + k)
            x = r.residues(1 << k, p)
            w = oracle_mod.primitive_root(k, p)
            assert oracle_mod.pow_mod(w, 1 << k, p) == 1 and (k == 0 or oracle_mod.pow_mod(w, 1 << (k - 1), p) != 1)
            want = [sum(int(x[i]) * pow(w, i * j, p) for i in range(len(x))) % p for j in range(len(x))]
            assert oracle_mod.dft_naive(x, w, p).tolist() == want
            assert oracle_mod.ntt(x, w, p).tolist() == want
            assert np.array_equal(oracle_mod.intt(oracle_mod.ntt(x, w, p), w, p), x)


@pytest.mark.parametrize("da,db", [(0, 0), (7, 3), (137, 138), (300, 299), (4095, 4095), (1, 20000), (65535, 65535)])
def test_polymul_oracle_vs_schoolbook_and_modpn(oracle_mod, da, db):
    r = SplitMix64(da * 1000 + db)
    a, b = r.residues(da + 1, P0), r.residues(db + 1, P0)
    fast = oracle_mod.polymul(a, b, P0)
    if da * db <= 20_000_000:
        assert np.array_equal(fast, oracle_mod.polymul_school(a, b, P0))
    if oracle_mod.ref_available():
        assert np.array_equal(fast, oracle_mod.ref_polymul(a, b, P0))


def test_modpn_batch_threads(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference build absent")
    r = SplitMix64(5)
    pairs = [(r.residues(n, P0), r.residues(m, P0)) for n, m in [(10, 20), (500, 700), (3000, 3000), (1, 1)]]
    outs = oracle_mod.ref_polymul_batch(pairs, P0, threads=3)
    for (a, b), h in zip(pairs, outs):
        assert np.array_equal(h, oracle_mod.polymul_school(a, b, P0))


def test_crt_signed(oracle_mod):
    ps = [962592769, 950009857, 940572673]
    P = ps[0] * ps[1] * ps[2]
    for v in [0, 1, -1, 10**20, -(10**20), P // 2, -(P // 2) + 1, 2**80 + 12345]:
        assert oracle_mod.crt_signed([v % q for q in ps], ps) == v
    assert oracle_mod.crt_signed([7 % 962592769, 7 % 950009857], ps[:2]) == 7


def test_oracle_bivariate_mul_matches_direct_sum(oracle_mod):
    """The Kronecker-substitution bivariate product equals the direct double sum."""
    p = 469762049
    r = np.random.default_rng(5)
    for (a, b), (c, d) in [((3, 3), (3, 3)), ((4, 7), (6, 2)), ((1, 9), (5, 1)), ((13, 11), (8, 17))]:
        F = r.integers(0, p, (a, b)).astype(np.uint32)
        G = r.integers(0, p, (c, d)).astype(np.uint32)
        H = np.zeros((a + c - 1, b + d - 1), dtype=object)
        for y in range(a):
            for x in range(b):
                H[y:y + c, x:x + d] += int(F[y, x]) * G.astype(object)
        assert np.array_equal(oracle_mod.bivariate_mul(F, G, p), (H % p).astype(np.uint32))


def test_oracle_subproduct_level_is_monic_product(oracle_mod):
    p = 469762049
    r = np.random.default_rng(9)
    for l in (1, 2, 5, 16):
        M = r.integers(0, p, 4 * l).astype(np.uint32)
        out = oracle_mod.subproduct_level(M, l, p)
        for j in range(2):
            a = [int(v) for v in M[2 * j * l:(2 * j + 1) * l]] + [1]
            b = [int(v) for v in M[(2 * j + 1) * l:(2 * j + 2) * l]] + [1]
            h = [0] * (2 * l + 1)
            for i, x in enumerate(a):
                for k, y in enumerate(b):
                    h[i + k] = (h[i + k] + x * y) % p
            assert [int(v) for v in out[2 * j * l:(2 * j + 2) * l]] == h[:2 * l]
