"""Bit-exact against the reference's own GPU path on the same inputs.

The reference's stockham_poly_mul_host (src/stockham.cu:562-611, the body of
cumodp_fftmul_uni) and its transforms stockham_host / inverse_stockham_host
(src/stockham.cu:479-503, the bodies of cumodp_fft_uni / cumodp_invfft_uni)
are compiled from the reference sources for sm_100a by `make -C oracle
ref_gpu` and run as shipped; this library's entry points must return the
same words.
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64, seed_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("da,db", [(200, 100), (4095, 4095), (20000, 12345), (65535, 65535)])
def test_same_words_as_reference_gpu(cm, oracle_mod, da, db):
    if not oracle_mod.ref_gpu_available():
        pytest.skip("reference GPU build absent (make -C oracle ref_gpu)")
    p = 469762049
    r = SplitMix64(seed_for(0) + da)
    a, b = r.residues(da + 1, p), r.residues(db + 1, p)
    assert np.array_equal(cm.fftmul_uni(a, b, p), oracle_mod.ref_gpu_polymul(a, b, p))


def test_same_words_as_reference_gpu_2_24(cm, oracle_mod):
    """The benchmark's size: degree 2^23 - 1 squared-size product (transform 2^24)."""
    if not oracle_mod.ref_gpu_available():
        pytest.skip("reference GPU build absent (make -C oracle ref_gpu)")
    import time
    p = 469762049
    r = SplitMix64(seed_for(1))
    a, b = r.residues(1 << 23, p), r.residues(1 << 23, p)
    ours = cm.fftmul_uni(a, b, p)
    ref = oracle_mod.ref_gpu_polymul(a, b, p)
    assert np.array_equal(ours, ref)
    # informational: both through their host entry points (copies included)
    t0 = time.perf_counter()
    cm.fftmul_uni(a, b, p)
    t1 = time.perf_counter()
    oracle_mod.ref_gpu_polymul(a, b, p)
    t2 = time.perf_counter()
    print(f"\n2^24 product, host entry points: this library {1e3 * (t1 - t0):.2f} ms, "
          f"reference GPU path {1e3 * (t2 - t1):.2f} ms")


@pytest.mark.parametrize("k", list(range(8, 25)))
def test_transforms_same_words_as_reference_gpu(cm, oracle_mod, k):
    """cumodp_fft_uni / cumodp_invfft_uni against the reference's own GPU transforms
    (stockham_host / inverse_stockham_host, src/stockham.cu:479-503, run as shipped)
    with the reference's own root, k = 8 ... 24."""
    if not oracle_mod.ref_gpu_available():
        pytest.skip("reference GPU build absent (make -C oracle ref_gpu)")
    for p in (469762049, 754974721) if k in (8, 13, 20) else (469762049,):
        x = SplitMix64(seed_for(2) + k).residues(1 << k, p)
        w = oracle_mod.primitive_root(k, p)
        y = cm.fft_uni(x, w, p)
        assert np.array_equal(y, oracle_mod.ref_gpu_fft(x, w, p))
        assert np.array_equal(cm.invfft_uni(y, w, p), oracle_mod.ref_gpu_fft(y, w, p, inverse=True))
