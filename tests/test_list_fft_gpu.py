"""List transform I_m (x) DFT_n through the C ABI vs the oracle (bit-exact).

cumodp_list_fft_dev replaces the reference's list_stockham_dev
(src/list_stockham.cu:595-665): m independent natural-order transforms of
length 2^k, in place on a device array.  The checker applies the DFT
definition (oracle dft_naive / ntt) row by row.
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu
P0 = 469762049


def _run(cm, x, m, k, w, p, inverse=False):
    import torch
    d = torch.from_numpy(x.view(np.int32).copy()).cuda()
    cm.list_fft_dev(d.data_ptr(), m, k, w, p, inverse)
    torch.cuda.synchronize()
    return d.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("m,k", [(1, 0), (7, 1), (5, 3), (300, 5), (3, 6), (17, 10), (100, 12),
                                 (9, 14), (3, 16), (2, 18), (5, 15), (70, 16), (3, 20)])
@pytest.mark.parametrize("p", [469762049, 962592769])
def test_list_fft_matches_rowwise_dft(cm, oracle_mod, m, k, p):
    r = SplitMix64(m * 1000 + k * 7 + p)
    x = r.residues(m << k, p)
    w = oracle_mod.primitive_root(k, p) if k > 0 else 1
    got = _run(cm, x, m, k, w, p)
    rows = x.reshape(m, 1 << k)
    for i in sorted({0, m // 2, m - 1}):
        want = oracle_mod.dft_naive(rows[i], w, p) if k <= 10 else oracle_mod.ntt(rows[i], w, p)
        assert np.array_equal(got.reshape(m, 1 << k)[i], want), i
    back = _run(cm, got, m, k, w, p, inverse=True)
    assert np.array_equal(back, x)


@pytest.mark.parametrize("m,k", [(2, 22), (5, 24)])
def test_list_fft_long_rows(cm, oracle_mod, m, k):
    """Rows of 2^22 and 2^24 words mod 469762049 (2-adic order 26); five 2^24-word rows take two
    launches of the batched four-step passes (at most 2^26 words in flight)."""
    r = SplitMix64(m * 1000 + k * 7)
    x = r.residues(m << k, P0)
    w = oracle_mod.primitive_root(k, P0)
    got = _run(cm, x, m, k, w, P0)
    rows = x.reshape(m, 1 << k)
    for i in sorted({0, m // 2, m - 1}):
        assert np.array_equal(got.reshape(m, 1 << k)[i], oracle_mod.ntt(rows[i], w, P0)), i
    assert np.array_equal(_run(cm, got, m, k, w, P0, inverse=True), x)


def test_list_fft_every_row_small(cm, oracle_mod):
    """Every row checked: 64 rows of 2^8 (the reference's taylor_shift / evaluation sizes)."""
    m, k, p = 64, 8, P0
    x = SplitMix64(0xC0DA0101).residues(m << k, p)
    w = oracle_mod.primitive_root(k, p)
    got = _run(cm, x, m, k, w, p).reshape(m, 1 << k)
    for i, row in enumerate(x.reshape(m, 1 << k)):
        assert np.array_equal(got[i], oracle_mod.dft_naive(row, w, p)), i


def test_list_fft_empty_and_bad_root(cm, oracle_mod):
    import torch
    d = torch.zeros(1 << 10, dtype=torch.int32, device="cuda")
    cm.list_fft_dev(d.data_ptr(), 0, 10, oracle_mod.primitive_root(10, P0), P0)
    with pytest.raises(cm.CumodpError) as e:
        cm.list_fft_dev(d.data_ptr(), 1, 10, 2, P0)
    assert e.value.code == cm.ASSUMPTION_ERROR
