"""Big-coefficient exact products through the C ABI (bit-exact).

cumodp_twoconv_mul_big is the general two_convolution_poly_mul of the
reference (src/two_convolution_poly_mul.cu:532-569, mpz coefficients).  The
checkers: the reference's own golden files benchmark/n{32..512}.test
(32..512-bit coefficients, committed under tests/golden/) and the oracle's
schoolbook over Python ints for seeded signed cases.
"""
import gzip
import os

import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BIG = sorted(f for f in os.listdir(GOLDEN) if f.startswith("bench_n") and "_p" not in f)


def read_golden(name):
    with gzip.open(os.path.join(GOLDEN, name), "rt") as fh:
        lines = [ln.split() for ln in fh.read().strip().split("\n")]
    return [[int(v) for v in ln] for ln in lines[:3]]


def big_ints(r, n, bits, signed=True):
    words = (bits + 63) // 64
    raw = r.next_u64(n * words).reshape(n, words)
    out = []
    for row in raw:
        v = 0
        for w in row[::-1]:
            v = (v << 64) | int(w)
        v &= (1 << bits) - 1
        out.append(-v if signed and (int(row[0]) & 1) else v)
    return out


@pytest.mark.parametrize("name", BIG)
def test_reference_golden_files(cm, name):
    a, b, c = read_golden(name)
    assert cm.twoconv_mul_big(a, b) == c


@pytest.mark.parametrize("bits,na,nb", [(1, 5, 7), (63, 40, 33), (64, 40, 33), (65, 17, 100), (200, 64, 64),
                                        (1024, 96, 80), (2048, 20, 30), (4095, 8, 9), (300, 1, 500),
                                        (100, 2000, 3)])
def test_signed_products_match_oracle(cm, oracle_mod, bits, na, nb):
    r = SplitMix64(bits * 1000 + na * 7 + nb)
    a, b = big_ints(r, na, bits), big_ints(r, nb, bits)
    assert cm.twoconv_mul_big(a, b) == oracle_mod.bigint_polymul(a, b)


def test_edge_values(cm, oracle_mod):
    """Zeros, powers of two (negation carries through zero low words), extreme widths."""
    a = [0, -(1 << 128), (1 << 128), -(1 << 4095) + 1, (1 << 4095) - 1, -1, 1, 0]
    b = [-(1 << 64), 0, 3, -(1 << 4000), 7]
    assert cm.twoconv_mul_big(a, b) == oracle_mod.bigint_polymul(a, b)
    assert cm.twoconv_mul_big([0, 0], [0]) == [0, 0]


def test_wider_input_words_and_truncated_output(cm, oracle_mod):
    r = SplitMix64(0xC0DA0401)
    a, b = big_ints(r, 50, 150), big_ints(r, 60, 150)
    want = oracle_mod.bigint_polymul(a, b)
    assert cm.twoconv_mul_big(a, b, in_words=8) == want
    # out_words narrower than the product: the low words, two's complement
    got = cm.twoconv_mul_big(a, b, out_words=2)
    assert got == [((v + (1 << 127)) % (1 << 128)) - (1 << 127) for v in want]


def test_large_1024_bit_product_properties(cm, oracle_mod):
    """4096 x 4096 coefficients of 1024 bits: checked at sampled coefficients and by
    evaluation at x = 1 and x = -1 (sums of coefficients), size-independent identities."""
    r = SplitMix64(0xC0DA0402)
    n = 4096
    a, b = big_ints(r, n, 1024), big_ints(r, n, 1024)
    got = cm.twoconv_mul_big(a, b)
    assert len(got) == 2 * n - 1
    assert sum(got) == sum(a) * sum(b)
    alt = lambda v: sum(x if i % 2 == 0 else -x for i, x in enumerate(v))
    assert alt(got) == alt(a) * alt(b)
    for k in (0, 1, 17, n - 1, n, 2 * n - 2):
        want = sum(a[i] * b[k - i] for i in range(max(0, k - n + 1), min(k, n - 1) + 1))
        assert got[k] == want


def test_plan_bound(cm):
    for bw, n in [(32, 32), (1024, 1024), (4096, 4096), (64, 1 << 20)]:
        K, M, npr, lg = cm.twoconv_big_plan(bw, n, n)
        assert K * M >= bw and npr in (3, 4) and lg <= 24
