"""Natural-order transforms through the C ABI vs the oracle (bit-exact).

cumodp_fft_uni / cumodp_invfft_uni (reference src/modpn.cu:181-210) and the
bivariate pair (src/modpn.cu:215-244): the checker is the DFT definition
(oracle or_dft_naive for small sizes, or_ntt for large ones) with the
caller's root, including the reference's own deterministic root
(primitive_root, include/inlines.h:460-485).
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

P0 = 469762049
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [0, 1, 3, 5, 6, 8, 10, 13, 14, 15, 16, 18, 20, 21])
@pytest.mark.parametrize("p", [469762049, 962592769])
def test_fft_uni_matches_dft(cm, oracle_mod, k, p):
    r = SplitMix64(k * 31 + p)
    x = r.residues(1 << k, p)
    w = oracle_mod.primitive_root(k, p) if k > 0 else 1
    want = oracle_mod.dft_naive(x, w, p) if k <= 10 else oracle_mod.ntt(x, w, p)
    got = cm.fft_uni(x, w, p)
    assert np.array_equal(got, want)
    back = cm.invfft_uni(got, w, p)
    assert np.array_equal(back, x)


def test_fft_uni_2_24_round_trip(cm, oracle_mod):
    """The headline-size transform: 2^24 points, forward vs oracle, then inverse round trip."""
    k = 24
    r = SplitMix64(0xC0DA0001)
    x = r.residues(1 << k, P0)
    w = oracle_mod.primitive_root(k, P0)
    got = cm.fft_uni(x, w, P0)
    assert np.array_equal(got, oracle_mod.ntt(x, w, P0))
    assert np.array_equal(cm.invfft_uni(got, w, P0), x)


@pytest.mark.parametrize("k", [25, 26])
def test_fft_uni_beyond_2_24(cm, oracle_mod, k):
    """2^25: the four-step kernels with 2^11-row columns; 2^26 (the 2-adic order of 469762049): one
    radix-2 step over HBM, two 2^25 transforms and an interleave.  Forward vs oracle, inverse
    round trip (the inverse's 2^-26 is applied in the split step)."""
    r = SplitMix64(0xC0DA0000 + k)
    x = r.residues(1 << k, P0)
    w = oracle_mod.primitive_root(k, P0)
    got = cm.fft_uni(x, w, P0)
    assert np.array_equal(got, oracle_mod.ntt(x, w, P0))
    assert np.array_equal(cm.invfft_uni(got, w, P0), x)


def test_uni_fft_tst_identity(cm, oracle_mod):
    """The reference's self-test uni_fft_tst (src/modpn.cu:416-449): X[i] = i, FFT then inverse = identity."""
    for k in (8, 12, 16):
        x = np.arange(1 << k, dtype=np.uint32)
        w = oracle_mod.primitive_root(k, P0)
        assert np.array_equal(cm.invfft_uni(cm.fft_uni(x, w, P0), w, P0), x)


def test_fft_uni_rejects_bad_root(cm):
    x = np.arange(256, dtype=np.uint32)
    with pytest.raises(cm.CumodpError) as e:
        cm.fft_uni(x, 2, P0)  # 2 is not a primitive 256th root
    assert e.value.code == cm.ASSUMPTION_ERROR


@pytest.mark.parametrize("em,en", [(0, 6), (1, 6), (3, 8), (8, 8), (5, 10), (10, 12), (6, 14),
                                   (12, 6), (13, 7), (16, 6), (6, 15), (3, 17)])
def test_bivariate_matches_row_column_dft(cm, oracle_mod, em, en):
    """Columns up to 2^11 and rows up to 2^14 run fused (column pass + row pass); longer ones as
    list transforms of the rows and of the transposed columns."""
    p = P0
    r = SplitMix64(em * 100 + en)
    X = r.residues(1 << (em + en), p).reshape(1 << em, 1 << en)
    wm = oracle_mod.primitive_root(em, p) if em else 1
    wn = oracle_mod.primitive_root(en, p)
    # (DFT_m (x) I_n)(I_m (x) DFT_n): rows then columns
    rows = np.stack([oracle_mod.ntt(X[i], wn, p) for i in range(X.shape[0])])
    want = np.stack([oracle_mod.ntt(rows[:, j], wm, p) if em else rows[:, j] for j in range(X.shape[1])], axis=1)
    got = cm.fft_bivariate(X, em, wm, en, wn, p).reshape(X.shape)
    assert np.array_equal(got, want)
    back = cm.fft_bivariate(got, em, wm, en, wn, p, inverse=True).reshape(X.shape)
    assert np.array_equal(back, X)


@pytest.mark.parametrize("em,en", [(4, 8), (11, 14), (12, 6)])
def test_fft_bivariate_dev_equals_host_entry(cm, em, en):
    """The device-pointer 2-D transform gives the host entry's result, forward and inverse."""
    import torch

    r = SplitMix64(em * 1000 + en)
    x = r.residues(1 << (em + en), P0)
    wm, wn = pow(3, (P0 - 1) >> em, P0), pow(3, (P0 - 1) >> en, P0)
    want = cm.fft_bivariate(x, em, wm, en, wn, P0)
    d = torch.from_numpy(x.view(np.int32)).cuda()
    cm.fft_bivariate_dev(d.data_ptr(), em, wm, en, wn, P0)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), want.reshape(-1))
    cm.fft_bivariate_dev(d.data_ptr(), em, wm, en, wn, P0, inverse=True)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), x)
