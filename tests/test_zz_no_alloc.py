"""The no-allocation product entry point against the allocating one.

cumodp_fftmul_uni_dev_noalloc exists for callers that cannot allocate device
memory (work captured into another component's CUDA graph, device memory
owned by a pool allocator, plugins loaded after the host partitioned device
memory): it takes its scratch from a fixed array in the library's device data
segment.  This file is collected last so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh
process.
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu


def _dev(x, torch):
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda()


def test_noalloc_matches_allocating_entry_point_twice(cm):
    import torch
    r = SplitMix64(2024)
    # two calls in a row, both on the three-pass path that uses the scratch
    # array, the second with another prime and size so the tables reload
    for da, db, p in [(100000, 80000, 469762049), (300000, 250000, 962592769)]:
        a = _dev(r.residues(da + 1, p), torch)
        b = _dev(r.residues(db + 1, p), torch)
        lh = da + db + 1
        want = torch.empty(lh, dtype=torch.int32, device="cuda")
        got = torch.full((lh,), -1, dtype=torch.int32, device="cuda")
        cm.fftmul_uni_dev(want.data_ptr(), lh, a.data_ptr(), da, b.data_ptr(), db, p)
        cm.fftmul_uni_dev_noalloc(got.data_ptr(), lh, a.data_ptr(), da, b.data_ptr(), db, p)
        torch.cuda.synchronize()
        assert torch.equal(got, want)  # exact: integer results, tolerance 0


def test_noalloc_single_cta_sizes_and_limit(cm):
    import torch
    r = SplitMix64(2025)
    p = 469762049
    for da, db in [(4095, 4095), (10, 3000)]:
        a = _dev(r.residues(da + 1, p), torch)
        b = _dev(r.residues(db + 1, p), torch)
        lh = da + db + 1
        want = torch.empty(lh, dtype=torch.int32, device="cuda")
        got = torch.empty(lh, dtype=torch.int32, device="cuda")
        cm.fftmul_uni_dev(want.data_ptr(), lh, a.data_ptr(), da, b.data_ptr(), db, p)
        cm.fftmul_uni_dev_noalloc(got.data_ptr(), lh, a.data_ptr(), da, b.data_ptr(), db, p)
        torch.cuda.synchronize()
        assert torch.equal(got, want)
    # beyond the stated maximum (transform 2^21): rejected before any work
    big = torch.zeros(1 << 20, dtype=torch.int32, device="cuda")
    out = torch.zeros(2 << 20, dtype=torch.int32, device="cuda")
    with pytest.raises(cm.CumodpError) as e:
        cm.fftmul_uni_dev_noalloc(out.data_ptr(), (2 << 20) - 1, big.data_ptr(), (1 << 20) - 1,
                                  big.data_ptr(), (1 << 20) - 1, p)
    assert e.value.code == cm.FFT_SIZE_TOO_LARGE
