"""Parity of the CUDA product path with the CPU oracle (bit-exact).

Every case goes through the C ABI (libcumodp.so via ctypes).  The checker is
the oracle's schoolbook product (small cases), its radix-2 transform product
(large cases), and modpn's own FFT multiply when the compiled reference is
present.
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

P0 = 469762049
PRIMES = [469762049, 754974721, 962592769, 950009857, 940572673]

pytestmark = pytest.mark.gpu


def _rand(r, n, p):
    return r.residues(n, p)


@pytest.mark.parametrize("p", PRIMES)
@pytest.mark.parametrize("da,db", [(0, 0), (1, 0), (5, 9), (31, 0), (16, 15), (100, 27), (255, 256),
                                   (1000, 3), (2047, 2048), (4095, 4095), (3000, 5000), (8191, 8191)])
def test_single_cta_products(cm, oracle_mod, p, da, db):
    r = SplitMix64(hash((p, da, db)) & 0xFFFFFFFF)
    a, b = _rand(r, da + 1, p), _rand(r, db + 1, p)
    want = oracle_mod.polymul_school(a, b, p) if da * db < 4_000_000 else oracle_mod.polymul(a, b, p)
    got = cm.fftmul_uni(a, b, p)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("p", [469762049, 962592769])
@pytest.mark.parametrize("da,db", [(8192, 8191), (16383, 16383), (12345, 40000), (65535, 65535),
                                   (100000, 1), (2**17 - 1, 2**17), (2**19 - 1, 2**19 - 1)])
def test_three_pass_products(cm, oracle_mod, p, da, db):
    r = SplitMix64(hash((p, da, db, 3)) & 0xFFFFFFFF)
    a, b = _rand(r, da + 1, p), _rand(r, db + 1, p)
    want = oracle_mod.polymul(a, b, p)
    got = cm.fftmul_uni(a, b, p)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("da,db", [(600000, 100), (100, 600000), (5000000, 10), (3000000, 3000000)])
def test_column_pass_long_operands(cm, oracle_mod, da, db):
    """Transforms of 2^20 and 2^23 words (1024- and 512-row columns) where an
    operand is longer than half the transform, so its columns have no zero
    half, and a balanced 2^23 case."""
    r = SplitMix64(hash((da, db, 5)) & 0xFFFFFFFF)
    a, b = _rand(r, da + 1, P0), _rand(r, db + 1, P0)
    assert np.array_equal(cm.fftmul_uni(a, b, P0), oracle_mod.polymul(a, b, P0))


@pytest.mark.parametrize("da,db,off", [(2**19 - 1, 2**19 - 1, 1), (2**19 - 1, 2**19 - 1, 3), (700000, 2**19 - 10, 2),
                                       (2**22 - 1, 2**22 - 1, 1)])
def test_column_pass_unaligned_device_operands(cm, oracle_mod, da, db, off):
    """Device operands that start off a 16-byte boundary (offsets of 4-12
    bytes), through cumodp_fftmul_uni_dev."""
    import torch
    r = SplitMix64(hash((da, db, off)) & 0xFFFFFFFF)
    a, b = _rand(r, da + 1, P0), _rand(r, db + 1, P0)
    ta = torch.zeros(da + 1 + off, dtype=torch.int32, device="cuda")
    tb = torch.zeros(db + 1 + off, dtype=torch.int32, device="cuda")
    ta[off:] = torch.from_numpy(a.view(np.int32)).cuda()
    tb[off:] = torch.from_numpy(b.view(np.int32)).cuda()
    lh = da + db + 1
    th = torch.zeros(lh + off, dtype=torch.int32, device="cuda")
    cm.fftmul_uni_dev(th.data_ptr() + 4 * off, lh, ta.data_ptr() + 4 * off, da, tb.data_ptr() + 4 * off, db, P0)
    torch.cuda.synchronize()
    got = th[off:].cpu().numpy().view(np.uint32)
    assert np.array_equal(got, oracle_mod.polymul(a, b, P0))


@pytest.mark.parametrize("da,db,dh", [(2**19 - 1, 2**19 - 1, 100000), (2**20 - 1, 2**20 - 1, 2**20 + 12345),
                                      (2**19 - 1, 2**19 - 1, 2**20 + 40)])
def test_output_length_contract_large(cm, oracle_mod, da, db, dh):
    """Truncated and zero-extended outputs of 2^20 and 2^21 transforms (the
    pipelined inverse column pass stops at lh)."""
    r = SplitMix64(da + 3 * dh)
    a, b = _rand(r, da + 1, P0), _rand(r, db + 1, P0)
    full = oracle_mod.polymul(a, b, P0)
    got = cm.fftmul_uni(a, b, P0, dh=dh)
    want = np.zeros(dh + 1, dtype=np.uint32)
    k = min(dh + 1, len(full))
    want[:k] = full[:k]
    assert np.array_equal(got, want)


def test_c1_config_vs_modpn(cm, oracle_mod):
    """4095 x 4095 mod 469762049 (transform 8192) against modpn's own product."""
    r = SplitMix64(0xC0DA0000)
    a, b = _rand(r, 4096, P0), _rand(r, 4096, P0)
    got = cm.fftmul_uni(a, b, P0)
    assert np.array_equal(got, oracle_mod.polymul_school(a, b, P0))
    if oracle_mod.ref_available():
        assert np.array_equal(got, oracle_mod.ref_polymul(a, b, P0))


def test_c2_product_2_24(cm, oracle_mod):
    """Product of two degree 2^23-1 polynomials (transform 2^24) vs the oracle."""
    r = SplitMix64(0xC0DA0001)
    n = 1 << 23
    a, b = _rand(r, n, P0), _rand(r, n, P0)
    got = cm.fftmul_uni(a, b, P0)
    want = oracle_mod.polymul(a, b, P0)
    assert np.array_equal(got, want)


def test_product_2_25(cm, oracle_mod):
    """Transform 2^25, the longest of the three-pass kernels (2^11-row columns x 2^14-word rows);
    the same product through the batch entry, beside a small one."""
    r = SplitMix64(0xC0DA0025)
    a, b = _rand(r, (1 << 24) + 5, P0), _rand(r, (1 << 24) - 77, P0)
    want = oracle_mod.polymul(a, b, P0)
    assert np.array_equal(cm.fftmul_uni(a, b, P0), want)
    c, d = _rand(r, 300, P0), _rand(r, 1000, P0)
    got = cm.fftmul_batch([(a, b), (c, d)], P0)
    assert np.array_equal(got[0], want)
    assert np.array_equal(got[1], oracle_mod.polymul_school(c, d, P0))


@pytest.mark.parametrize("p,order", [(962592769, 21), (950009857, 21), (940572673, 20), (754974721, 24)])
def test_products_at_the_primes_2_adic_order(cm, oracle_mod, p, order):
    """The longest product each prime allows (transform 2^order, 2^order - 1 coefficients) is
    computed; a product of 2^order + 1 coefficients is refused with CUMODP_FFT_SIZE_TOO_LARGE."""
    r = SplitMix64(p ^ 0x5A5A)
    half = 1 << (order - 1)
    a, b = _rand(r, half, p), _rand(r, half, p)
    assert np.array_equal(cm.fftmul_uni(a, b, p), oracle_mod.polymul(a, b, p))
    with pytest.raises(cm.CumodpError) as e:
        cm.fftmul_uni(np.append(a, [1, 1]).astype(np.uint32), b, p)
    assert e.value.code == cm.FFT_SIZE_TOO_LARGE


def test_split_product_2_26(cm, oracle_mod):
    """Transform 2^26 (the 2-adic order of 469762049): beyond the three-pass kernels' 2^25 the
    operands are cut into 2^24-coefficient pieces whose pairwise products are added at their
    offsets.  Full length, truncated inside a piece, zero fill past the product, and H over F
    through the device entry."""
    import torch

    r = SplitMix64(0xC0DA0026)
    la, lb = (1 << 25) - 3, (1 << 25) - 1000
    a, b = _rand(r, la, P0), _rand(r, lb, P0)
    want = oracle_mod.polymul(a, b, P0)
    assert len(want) > 1 << 25
    assert np.array_equal(cm.fftmul_uni(a, b, P0), want)
    dh = (1 << 24) + 12345
    assert np.array_equal(cm.fftmul_uni(a, b, P0, dh=dh), want[:dh + 1])
    got = cm.fftmul_uni(a, b, P0, dh=len(want) + 98)
    assert np.array_equal(got[:len(want)], want) and not got[len(want):].any()
    lh = (1 << 25) + 4321
    buf = torch.zeros(max(la, lh), dtype=torch.int32, device="cuda")
    buf[:la] = torch.from_numpy(a.view(np.int32)).cuda()
    g = torch.from_numpy(b.view(np.int32)).cuda()
    cm.fftmul_uni_dev(buf.data_ptr(), lh, buf.data_ptr(), la - 1, g.data_ptr(), lb - 1, P0)
    torch.cuda.synchronize()
    assert np.array_equal(buf[:lh].cpu().numpy().view(np.uint32), want[:lh])


def test_split_product_unbalanced(cm):
    """A long operand times a short one past 2^25 (three pieces of the long operand against one of
    the short): equal to the sum of two three-pass products, a_lo * b + x^m (a_hi * b)."""
    r = SplitMix64(0xC0DA0027)
    m = (1 << 25) - 1000  # a[:m] * b and a[m:] * b stay within 2^25
    a, b = _rand(r, (1 << 25) + 9, P0), _rand(r, 700, P0)
    assert len(a) + len(b) - 1 > 1 << 25
    lo, hi = cm.fftmul_uni(a[:m], b, P0), cm.fftmul_uni(a[m:], b, P0)
    want = np.zeros(len(a) + len(b) - 1, dtype=np.uint64)
    want[:len(lo)] += lo
    want[m:m + len(hi)] += hi
    assert np.array_equal(cm.fftmul_uni(a, b, P0), (want % P0).astype(np.uint32))


@pytest.mark.parametrize("da,db,dh", [(100, 50, 20), (100, 50, 150), (100, 50, 400), (4095, 4095, 9000),
                                      (20000, 20000, 100), (20000, 20000, 70000)])
def test_output_length_contract(cm, oracle_mod, da, db, dh):
    """dh < da+db truncates; dh > da+db zero-fills exactly dh+1 words."""
    r = SplitMix64(da * 7 + dh)
    a, b = _rand(r, da + 1, P0), _rand(r, db + 1, P0)
    full = oracle_mod.polymul(a, b, P0)
    got = cm.fftmul_uni(a, b, P0, dh=dh)
    want = np.zeros(dh + 1, dtype=np.uint32)
    k = min(dh + 1, len(full))
    want[:k] = full[:k]
    assert np.array_equal(got, want)


def test_small_fourier_primes(cm, oracle_mod):
    for p, d in [(257, 100), (7681, 200), (12289, 1000), (40961, 4000)]:
        r = SplitMix64(p)
        a, b = _rand(r, d + 1, p), _rand(r, d + 1, p)
        assert np.array_equal(cm.fftmul_uni(a, b, p), oracle_mod.polymul_school(a, b, p))


def test_errors(cm):
    with pytest.raises(cm.CumodpError) as e:
        cm.fftmul_uni(np.ones(4, np.uint32), np.ones(4, np.uint32), 1000)  # not prime
    assert e.value.code == cm.ASSUMPTION_ERROR
    with pytest.raises(cm.CumodpError) as e:  # 257: 2-adic order 8 -> at most 256 points
        cm.fftmul_uni(np.ones(200, np.uint32), np.ones(200, np.uint32), 257)
    assert e.value.code == cm.FFT_SIZE_TOO_LARGE
    # the library keeps working after an error
    a = np.arange(10, dtype=np.uint32)
    assert cm.fftmul_uni(a, a, P0)[0] == 0


def test_inputs_above_p_are_reduced(cm, oracle_mod):
    """Inputs are taken as unsigned 32-bit words and reduced mod p on load."""
    r = SplitMix64(77)
    a = r.next_u64(300).astype(np.uint32)
    b = r.next_u64(200).astype(np.uint32)
    want = oracle_mod.polymul_school(a % P0, b % P0, P0)
    assert np.array_equal(cm.fftmul_uni(a, b, P0), want)


def test_comparison_switches_give_the_same_products(cm):
    """CUMODP_COL_PIPE=0 (one-tile-per-CTA column passes) and CUMODP_ROWTAB=0
    (factor tables built inside every row CTA) select other kernels for the
    same products: a 2^21 and a 2^23 product must come out identical."""
    import os
    import subprocess
    import sys
    code = (
        "import numpy as np, cumodp_b200 as cm\n"
        "from cumodp_b200.workloads import SplitMix64\n"
        "r = SplitMix64(99); p = 469762049\n"
        "out = []\n"
        "for d in (2**20 - 1, 2**22 - 1):\n"
        "    a, b = r.residues(d + 1, p), r.residues(d + 1, p)\n"
        "    h = cm.fftmul_uni(a, b, p)\n"
        "    out.append(int((h.astype(np.uint64) * np.arange(1, len(h) + 1, dtype=np.uint64)).sum() % (2**61 - 1)))\n"
        "print(out)\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = []
    for extra in ({}, {"CUMODP_COL_PIPE": "0", "CUMODP_ROWTAB": "0"}):
        env = dict(os.environ, PYTHONPATH=root, **extra)
        out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr[-2000:]
        res.append(out.stdout.strip().splitlines()[-1])
    assert res[0] == res[1]


_FIRST_USE = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import cumodp_b200 as cm
from cumodp_b200.workloads import SplitMix64
# the first products of this process, each on a prime and size nothing here has used yet: the
# library builds and uploads its tables inside the call, then launches on a non-blocking stream
st = torch.cuda.Stream()
r = SplitMix64(424242)
bad = 0
cases = [(645922817, 300000, 250000), (595591169, 70000, 90000), (377487361, 20000, 30000),
         (167772161, 500000, 600000), (998244353, 5000, 3000), (897581057, 130000, 1)]
outs = []
with torch.cuda.stream(st):
    for p, na, nb in cases:
        a, b = r.residues(na, p), r.residues(nb, p)
        F = torch.from_numpy(a.view(np.int32)).cuda(non_blocking=True)
        G = torch.from_numpy(b.view(np.int32)).cuda(non_blocking=True)
        H = torch.empty(na + nb - 1, dtype=torch.int32, device="cuda")
        cm.fftmul_uni_dev(H.data_ptr(), na + nb - 1, F.data_ptr(), na - 1, G.data_ptr(), nb - 1, p, st.cuda_stream)
        outs.append((p, a, b, H))
st.synchronize()
for p, a, b, H in outs:
    bad += not np.array_equal(H.cpu().numpy().view(np.uint32), cm.fftmul_uni(a, b, p))
print("BAD", bad)
"""


def test_first_use_tables_on_a_non_blocking_stream(cm, tmp_path):
    """A fresh process's first products (new primes and sizes: tables built and uploaded inside the call)
    launched on a non-blocking stream equal the host entry's products: the upload has landed before the
    kernels that read it run."""
    import os
    import subprocess
    import sys
    script = tmp_path / "first_use.py"
    script.write_text(_FIRST_USE)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, str(script), root], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "BAD 0" in out.stdout, out.stdout[-2000:]
