"""Bivariate product through the C ABI vs the oracle (bit-exact).

cumodp_bivariate_mul replaces bi_stockham_poly_mul_host
(reference src/list_stockham.cu:1352-1390) and cumodp_bivariate_mul_dev
replaces bi_stockham_poly_mul_dev (src/list_stockham.cu:1317-1348).
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu
P0 = 469762049


def _rand(r, ny, nx, p):
    return r.residues(ny * nx, p).reshape(ny, nx)


def test_reference_doc_example(cm, oracle_mod):
    """f = (1 + 2x) + (3 + 4x + 5x^2)y + (6 + 7x^2)y^2 (fft_aux.cu:614-628), squared."""
    f = np.array([[1, 2, 0], [3, 4, 5], [6, 0, 7]], np.uint32)
    got = cm.bivariate_mul(f, f, P0)
    assert np.array_equal(got, oracle_mod.bivariate_mul(f, f, P0))
    assert got[0, 0] == 1 and got[0, 1] == 4 and got[4, 4] == 49


@pytest.mark.parametrize("sf,sg", [((1, 1), (1, 1)), ((1, 100), (1, 50)), ((100, 1), (50, 1)),
                                   ((20, 30), (25, 17)), ((64, 64), (64, 64)), ((7, 300), (5, 200)),
                                   ((300, 7), (200, 5)), ((150, 120), (90, 140))])
@pytest.mark.parametrize("p", [469762049, 962592769])
def test_bivariate_mul_matches_oracle(cm, oracle_mod, sf, sg, p):
    r = SplitMix64(sf[0] * 7919 + sf[1] * 31 + sg[0] * 3 + sg[1] + p)
    F, G = _rand(r, *sf, p), _rand(r, *sg, p)
    assert np.array_equal(cm.bivariate_mul(F, G, p), oracle_mod.bivariate_mul(F, G, p))


def test_bivariate_mul_dev_cyclic_grid(cm, oracle_mod):
    """The device entry on a padded 2^em x 2^en grid; a cyclic wrap case checked too."""
    import torch
    p, em, en = P0, 6, 9
    r = SplitMix64(0xC0DA0201)
    F = np.zeros((1 << em, 1 << en), np.uint32)
    G = np.zeros_like(F)
    F[:30, :200] = _rand(r, 30, 200, p)
    G[:34, :300] = _rand(r, 34, 300, p)
    dF = torch.from_numpy(F.view(np.int32).copy()).cuda()
    dG = torch.from_numpy(G.view(np.int32).copy()).cuda()
    cm.bivariate_mul_dev(em, en, dF.data_ptr(), dG.data_ptr(), p)
    torch.cuda.synchronize()
    got = dF.cpu().numpy().view(np.uint32)
    want = oracle_mod.bivariate_mul(F[:30, :200], G[:34, :300], p)
    assert np.array_equal(got[:63, :499], want)
    assert not got[63:].any() and not got[:, 499:].any()
    # wrap: operands filling the grid give the 2-D cyclic convolution
    A = _rand(r, 1 << 3, 1 << 6, p)
    B = _rand(r, 1 << 3, 1 << 6, p)
    lin = oracle_mod.bivariate_mul(A, B, p).astype(np.uint64)
    cyc = np.zeros((8, 64), np.uint64)
    for y in range(lin.shape[0]):
        for x in range(lin.shape[1]):
            cyc[y % 8, x % 64] = (cyc[y % 8, x % 64] + lin[y, x]) % p
    dA = torch.from_numpy(A.view(np.int32).copy()).cuda()
    dB = torch.from_numpy(B.view(np.int32).copy()).cuda()
    cm.bivariate_mul_dev(3, 6, dA.data_ptr(), dB.data_ptr(), p)
    torch.cuda.synchronize()
    assert np.array_equal(dA.cpu().numpy().view(np.uint32), cyc.astype(np.uint32))
