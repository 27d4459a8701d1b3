"""Exact integer products (two-convolution path) vs golden files, KATs and the __int128 oracle."""
import gzip
import json
import os

import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64, seed_for

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu


def read_golden(name):
    with gzip.open(os.path.join(GOLDEN, name), "rt") as fh:
        return [[int(v) for v in ln.split()] for ln in fh.read().strip().split("\n")[:3]]


FIXED = sorted(f for f in os.listdir(GOLDEN) if f.startswith("bench_n") and "_p" in f)


@pytest.mark.parametrize("name", FIXED)
@pytest.mark.parametrize("method", [0, 1])
def test_reference_golden_files(cm, name, method):
    a, b, c = read_golden(name)
    assert cm.twoconv_mul(np.array(a, np.int64), np.array(b, np.int64), method=method) == c


def test_unit_kat_products(cm):
    kats = json.load(open(os.path.join(GOLDEN, "unit_kats.json")))
    for case in kats["products"]:
        for method in (0, 1):
            assert cm.twoconv_mul(np.array(case["a"], np.int64), np.array(case["b"], np.int64), method) == case["c"]


def test_unit_kat_bit_width(cm):
    kats = json.load(open(os.path.join(GOLDEN, "unit_kats.json")))
    for case in kats["bit_width"]:
        if max(abs(v) for v in case["a"] + case["b"]) >= 1 << 63:
            continue
        assert cm.twoconv_bit_width(np.array(case["a"], np.int64), np.array(case["b"], np.int64)) == case["expected"]


@pytest.mark.parametrize("d", [8191, 16383])
@pytest.mark.parametrize("method", [0, 1])
def test_c3_signed_vs_i128_schoolbook(cm, oracle_mod, d, method):
    r = SplitMix64(seed_for(2) + d)
    a = r.int64_in(d + 1, 10**10)
    b = r.int64_in(d + 1, 10**10)
    assert cm.twoconv_mul(a, b, method) == oracle_mod.polymul_i128(a, b)


@pytest.mark.parametrize("bits,n,m", [(1, 50, 70), (20, 3000, 1), (40, 1000, 1000), (52, 4096, 300),
                                      (60, 40, 200), (62, 2, 2), (61, 8, 4)])
def test_widths_and_shapes(cm, oracle_mod, bits, n, m):
    r = SplitMix64(bits * 7 + n)
    bound = (1 << bits) - 1
    a = r.int64_in(n, bound)
    b = r.int64_in(m, bound)
    a[0] = bound  # make the width exact
    assert cm.twoconv_mul(a, b) == oracle_mod.polymul_i128(a, b)


def test_plan_choices(cm):
    # C3 shape: 34-bit coefficients, 16384 terms: one convolution over three primes
    assert cm.twoconv_plan(34, 34, 16384, 16384) == (1, 34, 3)
    # the two-prime limb split of the same shape: K=2 limbs of 17 bits
    assert cm.twoconv_plan(34, 34, 16384, 16384, method=1) == (2, 17, 2)


def test_overflow_rejected(cm):
    a = np.full(1000, (1 << 62), np.int64)
    with pytest.raises(cm.CumodpError) as e:
        cm.twoconv_mul(a, a)
    assert e.value.code == cm.ASSUMPTION_ERROR


def test_zero_and_extremes(cm, oracle_mod):
    a = np.zeros(10, np.int64)
    b = np.array([-(2**40), 2**40, 0, 1], np.int64)
    assert cm.twoconv_mul(a, b) == [0] * 13
    assert cm.twoconv_mul(b, b) == oracle_mod.polymul_i128(b, b)


def _words_mod(c_words: np.ndarray, q: int) -> np.ndarray:
    """Signed 128-bit (lo, hi) words -> residues mod q (Python ints, vectorised on object arrays)."""
    lo = c_words[0::2].view(np.uint64).astype(object)
    hi = c_words[1::2].astype(object)  # signed high word
    return (hi * (1 << 64) + lo) % q


def _eval_mod(coeffs, t: int, q: int) -> int:
    acc = 0
    for v in reversed(list(coeffs)):
        acc = (acc * t + int(v)) % q
    return acc


def test_long_product_past_the_reference_primes(cm, oracle_mod):
    """2^21 + 10 coefficients times 100 (transform 2^22, past 962592769's order): exact vs the __int128 oracle."""
    r = SplitMix64(seed_for(2) + 77)
    a, b = r.int64_in((1 << 21) + 10, 10**10), r.int64_in(100, 10**10)
    got = cm.twoconv_mul(a, b)
    want = oracle_mod.polymul_i128(a, b)
    bad = [i for i, (x, y) in enumerate(zip(got, want)) if x != y]
    assert len(got) == len(want) and not bad, (len(bad), bad[:5])
    with pytest.raises(cm.CumodpError) as e:  # the reference's forced two-prime scheme has no such plan
        cm.twoconv_mul(a, b, method=1)
    assert e.value.code == cm.FFT_SIZE_TOO_LARGE


def test_serving_sized_int64_product(cm):
    """Degrees 2^20 x 2^20, |c| <= 10^10 (the largest int64 request of the serving workload): the product's
    values mod q = 2^61 - 1 at two points equal a(t) b(t) mod q (size-independent identity), host and device entries."""
    import ctypes as C

    import torch
    r = SplitMix64(seed_for(4) + 5)
    n = (1 << 20) + 1
    a, b = r.int64_in(n, 10**10), r.int64_in(n, 10**10)
    c = cm.twoconv_mul(a, b, raw=True)
    q = (1 << 61) - 1
    cm_mod = _words_mod(c, q)
    for t in (3, 1234567891011):
        assert _eval_mod(cm_mod, t, q) == _eval_mod(a, t, q) * _eval_mod(b, t, q) % q
    bw = cm.twoconv_bit_width(a, b)
    dA, dB = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    dC = torch.empty(2 * (2 * n - 1), dtype=torch.int64, device="cuda")
    rc = cm.lib().cumodp_twoconv_mul_i64_dev(n, dA.data_ptr(), n, dB.data_ptr(), dC.data_ptr(), bw, 0, C.c_void_p(0))
    assert rc == 0
    assert np.array_equal(dC.cpu().numpy(), c)
