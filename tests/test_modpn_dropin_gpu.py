"""modpn, unmodified, calling this library as its GPU backend.

modpn's FMUL.c compiled with its GPU dispatch (-D_cuda_modp_) and linked
against libcumodp.so (oracle/Makefile target modpn_gpu): for transform sizes
>= 2^16 modpn itself calls can_call_fftmul_uni and then
cumodp_fftmul_uni(n1 - 1, A, degA, A, degB, B, p) with the result in place
(modpn/src/FMUL.c:1943-1957).  The product must equal the oracle's.

modpn falls back to its own CPU product, silently, whenever the library
returns an error (FMUL.c:1945-1956), so an equal product alone does not show
that the library ran: the library's pass tracer counts the kernels launched
during modpn's call.  Sizes at or above modpn's GPU threshold (transform
2^16) must launch them; a smaller product must launch none (modpn keeps it on
the CPU).
"""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("da,db", [(40000, 30000), (65535, 65535), (100000, 3), (300, 200)])
def test_modpn_through_libcumodp(oracle_mod, cm, da, db):
    if not oracle_mod.modpn_gpu_available():
        pytest.skip("modpn GPU-dispatch build absent (make -C oracle modpn_gpu)")
    p = 469762049
    r = SplitMix64(da + 7 * db)
    a, b = r.residues(da + 1, p), r.residues(db + 1, p)
    cm.trace_passes(True)
    cm.trace_report(reset=True)
    try:
        got = oracle_mod.modpn_gpu_polymul(a, b, p)
        launches = sum(cnt for cnt, _ in cm.trace_report(reset=True).values())
    finally:
        cm.trace_passes(False)
    assert np.array_equal(got, oracle_mod.polymul(a, b, p))
    gpu_sized = (da + db + 1) > (1 << 15)  # modpn's transform of at least 2^16 points
    if gpu_sized:
        assert launches > 0, "modpn computed the product without the library (CPU fallback)"
    else:
        assert launches == 0
