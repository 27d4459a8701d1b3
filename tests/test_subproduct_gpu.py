"""One subproduct-tree level through the C ABI vs the oracle (bit-exact).

cumodp_subproduct_level_dev replaces the FFT level step of the reference's
subProductTree (src/fastPolyEvaluation.cu:604-650).
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu


def _level(cm, M, l, npairs, p):
    import torch
    dM = torch.from_numpy(M.view(np.int32).copy()).cuda()
    dO = torch.full((2 * l * npairs,), -1, dtype=torch.int32, device="cuda")
    cm.subproduct_level_dev(l, npairs, dM.data_ptr(), dO.data_ptr(), p)
    torch.cuda.synchronize()
    return dO.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("l,npairs", [(1, 1), (1, 64), (2, 33), (128, 512), (256, 100), (1000, 7),
                                      (4096, 16), (8192, 4), (1 << 15, 2), (1 << 17, 1)])
@pytest.mark.parametrize("p", [469762049, 962592769])
def test_level_matches_oracle(cm, oracle_mod, l, npairs, p):
    r = SplitMix64(l * 131 + npairs + p)
    M = r.residues(2 * npairs * l, p)
    got = _level(cm, M, l, npairs, p)
    idx = sorted({0, npairs // 2, npairs - 1})
    want = oracle_mod.subproduct_level(np.concatenate([M[2 * j * l:(2 * j + 2) * l] for j in idx]), l, p)
    got_sel = np.concatenate([got[2 * j * l:(2 * j + 2) * l] for j in idx])
    assert np.array_equal(got_sel, want)


def test_tree_from_roots_gives_prod_x_minus_u(cm, oracle_mod):
    """Build a whole subproduct tree from 2^10 linear factors x - u_i, level by level,
    and check the root polynomial vanishes at every u_i (a size-independent property)."""
    import torch
    p, k = 469762049, 10
    u = SplitMix64(0xC0DA0301).residues(1 << k, p)
    M = ((p - u.astype(np.int64)) % p).astype(np.uint32)  # x - u: constant term -u
    dM = torch.from_numpy(M.view(np.int32).copy()).cuda()
    l = 1
    for _ in range(k):
        npairs = len(M) // (2 * l)
        dO = torch.empty(len(M), dtype=torch.int32, device="cuda")
        cm.subproduct_level_dev(l, npairs, dM.data_ptr(), dO.data_ptr(), p)
        dM, l = dO, 2 * l
    torch.cuda.synchronize()
    root = np.append(dM.cpu().numpy().view(np.uint32), 1).astype(object)  # monic degree 2^k
    for x in u[:16]:
        acc = 0
        for c in root[::-1]:
            acc = (acc * int(x) + int(c)) % p
        assert acc == 0


def test_level_rejects_overlap(cm):
    import torch
    d = torch.zeros(64, dtype=torch.int32, device="cuda")
    with pytest.raises(cm.CumodpError) as e:
        cm.subproduct_level_dev(8, 4, d.data_ptr(), d.data_ptr(), 469762049)
    assert e.value.code == cm.ASSUMPTION_ERROR
