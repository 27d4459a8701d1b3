"""Host-side fault injection: forced device-allocation failures.

An allocation the library needs fails (cumodp_inject_alloc_failures, no GPU
fault involved): the call reports CUMODP_OUT_OF_MEMORY, nothing half-built is
cached, and the same call succeeds bit-exact afterwards.  The reference has no
such path (cudaMalloc failures go unchecked, src/stockham.cu:579-610).
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _no_leftover_injection(cm):
    yield
    cm.inject_alloc_failures(0)


def test_product_table_allocation_failure_then_recovery(cm, oracle_mod):
    p = 595591169  # a prime no other test uses: its tables are built here
    r = SplitMix64(0xC0DA0601)
    a, b = r.residues(300001, p), r.residues(200000, p)
    cm.inject_alloc_failures(1)
    with pytest.raises(cm.CumodpError) as e:
        cm.fftmul_uni(a, b, p)
    assert e.value.code == cm.OUT_OF_MEMORY
    assert np.array_equal(cm.fftmul_uni(a, b, p), oracle_mod.polymul(a, b, p))


@pytest.mark.parametrize("failures", [1, 2, 3])
def test_batch_plan_allocation_failure_then_recovery(cm, oracle_mod, failures):
    p = 377487361  # unused elsewhere; a batch shape of its own
    r = SplitMix64(0xC0DA0602 + failures)
    # classes of 2^8-2^12 only (the work-queue kernel): the autotuner times the 2^13 and 2^14 classes
    # (scratch allocations of its own, whose failure only falls back to the default choice), these not
    pairs = [(r.residues(int(d), p), r.residues(int(d) + 7, p)) for d in (100 + failures, 1000, 2000)] * 20
    cm.inject_alloc_failures(failures)
    with pytest.raises(cm.CumodpError) as e:
        cm.fftmul_batch(pairs, p)
    assert e.value.code == cm.OUT_OF_MEMORY
    cm.inject_alloc_failures(0)
    outs = cm.fftmul_batch(pairs, p)
    for (a, b), h in zip(pairs, outs):
        assert np.array_equal(h, oracle_mod.polymul(a, b, p))


def test_server_lane_allocation_failure_is_contained(cm, oracle_mod):
    """A lane's buffers are sized at creation (here for a 3 MB device budget, about 1 MB each); a request
    larger than that grows them, and that growth is made to fail."""
    p = 469762049
    r = SplitMix64(0xC0DA0603)
    a, b = r.residues(300000, p), r.residues(300000, p)
    with cm.Server(lanes=1, memory_budget=3 << 20) as srv:
        cm.inject_alloc_failures(1)  # the lane's growth for this request
        rid, _ = srv.submit_mod(a, b, p)
        assert srv.wait(rid) == cm.OUT_OF_MEMORY
        rid, out = srv.submit_mod(a, b, p)
        assert srv.wait(rid) == 0
        assert np.array_equal(out, oracle_mod.polymul(a, b, p))
