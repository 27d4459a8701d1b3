"""The no-allocation product entry point against the allocating one.

Some users of this library cannot let it call cudaMalloc: a service whose
device memory is handed out by its own pool allocator, a plugin loaded after
the host has partitioned all device memory, or latency-critical code that
cannot afford cudaMalloc's implicit synchronisation.
cumodp_fftmul_uni_dev_noalloc serves them: its scratch is a fixed array in
the library's device data segment, and every call rewrites the twiddle tables
of its own prime and size there.  Its products must equal those of
cumodp_fftmul_uni_dev word for word (integer results: tolerance 0).

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu


def _dev(x, torch):
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda()


def _both(cm, torch, r, da, db, p):
    a = _dev(r.residues(da + 1, p), torch)
    b = _dev(r.residues(db + 1, p), torch)
    lh = da + db + 1
    want = torch.empty(lh, dtype=torch.int32, device="cuda")
    got = torch.full((lh,), -1, dtype=torch.int32, device="cuda")
    cm.fftmul_uni_dev(want.data_ptr(), lh, a.data_ptr(), da, b.data_ptr(), db, p)
    cm.fftmul_uni_dev_noalloc(got.data_ptr(), lh, a.data_ptr(), da, b.data_ptr(), db, p)
    torch.cuda.synchronize()
    return got, want


def test_noalloc_matches_allocating_entry_point_twice(cm):
    import torch
    r = SplitMix64(2024)
    # two calls in a row, both on the three-pass path that uses the scratch
    # array, the second with another prime and size
    for da, db, p in [(100000, 80000, 469762049), (300000, 250000, 962592769)]:
        got, want = _both(cm, torch, r, da, db, p)
        assert torch.equal(got, want)  # exact: integer results, tolerance 0


def test_noalloc_alternating_primes_and_sizes(cm):
    """A, B, A: each call writes its own tables, so returning to A after B is exact."""
    import torch
    r = SplitMix64(2026)
    for da, db, p in [(70000, 60000, 469762049), (8000, 7000, 754974721), (70000, 60000, 469762049),
                      (200000, 150000, 754974721), (8000, 7000, 469762049)]:
        got, want = _both(cm, torch, r, da, db, p)
        assert torch.equal(got, want), (da, db, p)


def test_noalloc_single_cta_sizes_and_limit(cm):
    import torch
    r = SplitMix64(2025)
    p = 469762049
    # transforms 2^13, 2^12 and 2^14 (one CTA; the largest row-table layout of that path)
    for da, db in [(4095, 4095), (10, 3000), (8000, 7999)]:
        got, want = _both(cm, torch, r, da, db, p)
        assert torch.equal(got, want)
    # beyond the stated maximum (transform 2^21): rejected before any work
    big = torch.zeros(1 << 20, dtype=torch.int32, device="cuda")
    out = torch.zeros(2 << 20, dtype=torch.int32, device="cuda")
    with pytest.raises(cm.CumodpError) as e:
        cm.fftmul_uni_dev_noalloc(out.data_ptr(), (2 << 20) - 1, big.data_ptr(), (1 << 20) - 1,
                                  big.data_ptr(), (1 << 20) - 1, p)
    assert e.value.code == cm.FFT_SIZE_TOO_LARGE


def test_noalloc_largest_row_tables_and_limit_size(cm):
    """Transform 2^19 (2^14-word rows: the full row-table region) and 2^20 (the stated maximum)."""
    import torch
    r = SplitMix64(2027)
    for da, db, p in [(200000, 199999, 962592769), ((1 << 19) - 1, (1 << 19) - 1, 469762049)]:
        got, want = _both(cm, torch, r, da, db, p)
        assert torch.equal(got, want)


def test_noalloc_makes_no_device_allocation(cm, oracle_mod):
    """With every library allocation forced to fail, a prime and size never used before still work."""
    import torch
    p = 998244353  # 119 * 2^23 + 1: used by no other test of this file
    r = SplitMix64(2028)
    fa, fb = r.residues(40001, p), r.residues(30001, p)
    a, b = _dev(fa, torch), _dev(fb, torch)
    out = torch.full((70001,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    cm.inject_alloc_failures(1 << 30)
    try:
        cm.fftmul_uni_dev_noalloc(out.data_ptr(), 70001, a.data_ptr(), 40000, b.data_ptr(), 30000, p)
        torch.cuda.synchronize()
    finally:
        cm.inject_alloc_failures(0)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), oracle_mod.polymul(fa, fb, p))
