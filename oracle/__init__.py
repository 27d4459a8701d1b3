"""CPU oracle for the polynomial product path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm import this package, and only as the checker or the timed CPU
reference.  The shipped library (``cumodp_b200``) never imports it.

Two shared libraries are wrapped here:

* ``liboracle.so`` -- our plain-C restatement of the reference arithmetic
  (``oracle.c``; each function cites the reference file:line it follows);
* ``_ref/libmodpn_ref.so`` -- the reference's own CPU FFT multiply, modpn's
  ``EX_Mont_FFTMul`` (modpn/src/FMUL.c:2015-2030), compiled from the
  reference sources by ``oracle/Makefile`` (``make ref``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmodpn_ref.so")
MODPN_GPU_SO = os.path.join(HERE, "_ref", "libmodpn_gpu.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libcumodp_refgpu.so")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def reference_present() -> bool:
    """Whether the reference sources the ``ref`` targets compile are present
    (``make has-ref``: the Makefile's REF, or the CUMODP_REFERENCE variable)."""
    return subprocess.run(["make", "-s", "-C", HERE, "has-ref"], capture_output=True).returncode == 0


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and, when ``ref``, the modpn reference builds)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"])
        subprocess.check_call(["make", "-s", "-C", HERE, "modpn_gpu"])
        subprocess.check_call(["make", "-s", "-C", HERE, "ref_gpu"])


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.or_pow.restype = C.c_uint32
        L.or_pow.argtypes = [C.c_uint32, C.c_uint64, C.c_uint32]
        L.or_inv.restype = C.c_uint32
        L.or_inv.argtypes = [C.c_uint32, C.c_uint32]
        L.or_fourier_degree.restype = C.c_int
        L.or_fourier_degree.argtypes = [C.c_uint32]
        L.or_primitive_root.restype = C.c_uint32
        L.or_primitive_root.argtypes = [C.c_int, C.c_uint32]
        L.or_dft_naive.argtypes = [C.c_int, _u32p, C.c_uint32, C.c_uint32, _u32p]
        L.or_ntt.argtypes = [_u32p, C.c_int, C.c_uint32, C.c_uint32]
        L.or_intt.argtypes = [_u32p, C.c_int, C.c_uint32, C.c_uint32]
        L.or_polymul_school.argtypes = [C.c_int, _u32p, C.c_int, _u32p, _u32p, C.c_uint32]
        L.or_polymul_ntt.restype = C.c_int
        L.or_polymul_ntt.argtypes = [C.c_int, _u32p, C.c_int, _u32p, _u32p, C.c_uint32]
        L.or_polymul_i128.argtypes = [C.c_int, _i64p, C.c_int, _i64p, _u64p]
        L.or_bit_width.restype = C.c_int
        L.or_bit_width.argtypes = [C.c_int, _i64p, C.c_int, _i64p]
        L.or_limb_split.argtypes = [C.c_int, _i64p, C.c_int, C.c_int, C.c_uint32, _u32p]
        L.or_scale_x.argtypes = [C.c_int, _u32p, C.c_int, C.c_uint32, C.c_uint32]
        L.or_crt_signed.argtypes = [C.c_int, _u32p, _u32p, C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The compiled reference (modpn) CPU product; raises if it was not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref)")
        L = C.CDLL(REF_SO)
        L.ref_init_prime.restype = C.c_int
        L.ref_init_prime.argtypes = [C.c_int32]
        L.ref_fftmul.restype = C.c_int
        L.ref_fftmul.argtypes = [C.c_int32, _i32p, C.c_int32, _i32p, _i32p, C.c_int32]
        _l = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
        L.ref_fftmul_batch.restype = C.c_int
        L.ref_fftmul_batch.argtypes = [C.c_int, _i32p, _l, _i32p, _i32p, _l, _i32p, _l,
                                       _i32p, C.c_int32, C.c_int]
        _ref = L
    return _ref


# ------------------------------------------------------------ python API --

def pow_mod(a: int, e: int, p: int) -> int:
    return int(lib().or_pow(a, e, p))


def inv_mod(a: int, p: int) -> int:
    return int(lib().or_inv(a, p))


def fourier_degree(p: int) -> int:
    return int(lib().or_fourier_degree(p))


def primitive_root(e: int, p: int) -> int:
    """The reference's deterministic 2^e-th root (include/inlines.h:460-485).

    Defined for e >= 1 (the reference's search shifts by e - 1; for e = 0 it
    never ends): the primitive 1st root is 1, returned without the search."""
    if e == 0:
        return 1
    if e < 0:
        raise ValueError("e >= 0")
    return int(lib().or_primitive_root(e, p))


def dft_naive(x: np.ndarray, w: int, p: int) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.uint32)
    out = np.empty_like(x)
    lib().or_dft_naive(len(x), x, w, p, out)
    return out


def ntt(x: np.ndarray, w: int, p: int) -> np.ndarray:
    x = np.array(x, dtype=np.uint32, copy=True)
    k = int(len(x)).bit_length() - 1
    assert len(x) == 1 << k
    lib().or_ntt(x, k, w, p)
    return x


def intt(x: np.ndarray, w: int, p: int) -> np.ndarray:
    x = np.array(x, dtype=np.uint32, copy=True)
    k = int(len(x)).bit_length() - 1
    assert len(x) == 1 << k
    lib().or_intt(x, k, w, p)
    return x


def polymul_school(a: np.ndarray, b: np.ndarray, p: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    h = np.empty(len(a) + len(b) - 1, dtype=np.uint32)
    lib().or_polymul_school(len(a) - 1, a, len(b) - 1, b, h, p)
    return h


def polymul(a: np.ndarray, b: np.ndarray, p: int) -> np.ndarray:
    """Product mod p through the oracle's own radix-2 transforms."""
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    h = np.empty(len(a) + len(b) - 1, dtype=np.uint32)
    if lib().or_polymul_ntt(len(a) - 1, a, len(b) - 1, b, h, p) != 0:
        raise ValueError("transform size exceeds the prime's 2-adic order")
    return h


def bivariate_mul(F: np.ndarray, G: np.ndarray, p: int) -> np.ndarray:
    """Bivariate product mod p of 2-D arrays indexed [y, x].

    Follows bi_stockham_poly_mul_host (reference src/list_stockham.cu:1352-1390):
    the product of the (nx, ny)-dense operands, here computed by Kronecker
    substitution x^i y^j -> z^(j X + i) with X = nxf + nxg - 1 (no carry
    between y-rows) and the oracle's univariate product.
    """
    F = np.asarray(F, dtype=np.uint32)
    G = np.asarray(G, dtype=np.uint32)
    (nyf, nxf), (nyg, nxg) = F.shape, G.shape
    X, Y = nxf + nxg - 1, nyf + nyg - 1
    f = np.zeros(nyf * X, np.uint32)
    g = np.zeros(nyg * X, np.uint32)
    f.reshape(nyf, X)[:, :nxf] = F % p
    g.reshape(nyg, X)[:, :nxg] = G % p
    h = polymul_school(f, g, p) if len(f) * len(g) <= 1 << 22 else polymul(f, g, p)
    assert not h[Y * X:].any()  # the product's degree is below Y X
    out = np.zeros(Y * X, np.uint32)
    out[:min(len(h), Y * X)] = h[:Y * X]
    return out.reshape(Y, X)


def subproduct_level(M: np.ndarray, l: int, p: int) -> np.ndarray:
    """One subproduct-tree level of monic polynomials stored without leading coefficient.

    Follows subProductTree's FFT level step (reference
    src/fastPolyEvaluation.cu:604-650 with pointAdd2 :83-92 and pointAdd
    :153-158): out[j] = (x^l + M[2j]) (x^l + M[2j+1]) - x^(2l), 2l words.
    Computed here with explicit leading ones and the oracle's product.
    """
    M = np.asarray(M, dtype=np.uint32).reshape(-1, l)
    out = np.empty((M.shape[0] // 2, 2 * l), np.uint32)
    for j in range(M.shape[0] // 2):
        a = np.append(M[2 * j] % p, 1).astype(np.uint32)
        b = np.append(M[2 * j + 1] % p, 1).astype(np.uint32)
        h = polymul_school(a, b, p) if l <= 512 else polymul(a, b, p)
        assert h[2 * l] == 1
        out[j] = h[:2 * l]
    return out.reshape(-1)


def bigint_polymul(a, b) -> list:
    """Exact product of big-integer polynomials (Python ints, schoolbook).

    The reference's general two_convolution_poly_mul
    (src/two_convolution_poly_mul.cu:532-569) and its benchmark's Kronecker
    baseline (benchmark/bench_two_convolution_poly_mul.cpp:11-100) both
    compute this exact product; schoolbook over Python ints is its
    definition (small cases only).
    """
    a = [int(v) for v in a]
    b = [int(v) for v in b]
    out = [0] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        if x:
            for j, y in enumerate(b):
                out[i + j] += x * y
    return out


def polymul_i128(a: np.ndarray, b: np.ndarray) -> list[int]:
    """Exact integer product (Python ints) by __int128 schoolbook."""
    a = np.ascontiguousarray(a, dtype=np.int64)
    b = np.ascontiguousarray(b, dtype=np.int64)
    n = len(a) + len(b) - 1
    h = np.empty(2 * n, dtype=np.uint64)
    lib().or_polymul_i128(len(a) - 1, a, len(b) - 1, b, h)
    return i128_pairs_to_int(h)


def i128_pairs_to_int(h: np.ndarray) -> list[int]:
    lo = h[0::2].astype(object)
    hi = h[1::2].astype(object)
    out = []
    for l, hh in zip(lo, hi):
        v = int(l) | (int(hh) << 64)
        if v >= 1 << 127:
            v -= 1 << 128
        out.append(v)
    return out


def bit_width(a: np.ndarray, b: np.ndarray) -> int:
    a = np.ascontiguousarray(a, dtype=np.int64)
    b = np.ascontiguousarray(b, dtype=np.int64)
    return int(lib().or_bit_width(len(a), a, len(b), b))


def limb_split(a: np.ndarray, K: int, M: int, p: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int64)
    out = np.empty(len(a) * K, dtype=np.uint32)
    lib().or_limb_split(len(a), a, K, M, p, out)
    return out


def scale_x(A: np.ndarray, K: int, theta: int, p: int) -> np.ndarray:
    A = np.array(A, dtype=np.uint32, copy=True)
    lib().or_scale_x(len(A), A, K, theta, p)
    return A


def crt_signed(residues, primes) -> int:
    r = np.ascontiguousarray(residues, dtype=np.uint32)
    p = np.ascontiguousarray(primes, dtype=np.uint32)
    lo, hi = C.c_uint64(), C.c_uint64()
    lib().or_crt_signed(len(r), r, p, C.byref(lo), C.byref(hi))
    v = lo.value | (hi.value << 64)
    return v - (1 << 128) if v >= 1 << 127 else v


def ref_polymul(a: np.ndarray, b: np.ndarray, p: int) -> np.ndarray:
    """The reference's own CPU product: modpn EX_Mont_FFTMul."""
    L = ref()
    if L.ref_init_prime(p) != 0:
        raise RuntimeError("prime table full")
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    h = np.empty(len(a) + len(b) - 1, dtype=np.int32)
    if L.ref_fftmul(len(a) - 1, a, len(b) - 1, b, h, p) != 0:
        raise RuntimeError("modpn product failed")
    return h.view(np.uint32)


def modpn_gpu_available() -> bool:
    return os.path.exists(MODPN_GPU_SO)


_mg = None


def modpn_gpu_polymul(a: np.ndarray, b: np.ndarray, p: int) -> np.ndarray:
    """modpn's in-place product with its GPU dispatch compiled in, linked to libcumodp.so.

    For transform sizes >= 2^16 modpn itself calls can_call_fftmul_uni and
    cumodp_fftmul_uni (modpn/src/FMUL.c:1943-1957); below that it multiplies
    on the CPU.  Used to show the library is a drop-in for modpn.
    """
    global _mg
    if _mg is None:
        _mg = C.CDLL(MODPN_GPU_SO)
        _mg.modpn_gpu_fftmul.restype = C.c_int
        _mg.modpn_gpu_fftmul.argtypes = [C.c_int32, _i32p, C.c_int32, _i32p, _i32p, C.c_int32]
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint32).view(np.int32))
    b = np.ascontiguousarray(np.asarray(b, dtype=np.uint32).view(np.int32))
    h = np.empty(len(a) + len(b) - 1, dtype=np.int32)
    if _mg.modpn_gpu_fftmul(len(a) - 1, a, len(b) - 1, b, h, p) != 0:
        raise RuntimeError("modpn prime error")
    return h.view(np.uint32)


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


_rg = None


def ref_gpu_polymul(a: np.ndarray, b: np.ndarray, p: int) -> np.ndarray:
    """The reference's own GPU product (stockham_poly_mul_host, src/stockham.cu:562-611).

    Runs the reference as shipped (radix-2 Stockham, synchronised launches,
    per-call allocation).  Transform sizes below 256 are refused by the
    reference itself (it returns with H untouched), so callers keep to
    len(a) + len(b) - 1 > 128.
    """
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint32).view(np.int32))
    b = np.ascontiguousarray(np.asarray(b, dtype=np.uint32).view(np.int32))
    dh = len(a) + len(b) - 2
    h = np.zeros(dh + 1, dtype=np.int32)
    rc = _ref_gpu_lib().ref_gpu_fftmul(dh, h, len(a) - 1, a, len(b) - 1, b, p)
    if rc != 0:
        raise RuntimeError(f"reference GPU product failed: CUDA error {rc}")
    return h.view(np.uint32)


def _ref_gpu_lib():
    global _rg
    if _rg is None:
        _rg = C.CDLL(REF_GPU_SO)
        _rg.ref_gpu_fftmul.restype = C.c_int
        _rg.ref_gpu_fftmul.argtypes = [C.c_int, _i32p, C.c_int, _i32p, C.c_int, _i32p, C.c_int]
        _rg.ref_gpu_fft_host.restype = C.c_int
        _rg.ref_gpu_fft_host.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        _rg.ref_gpu_time_fft_dev.restype = C.c_int
        _rg.ref_gpu_time_fft_dev.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.POINTER(C.c_float)]
        _rg.ref_gpu_time_polymul_dev.restype = C.c_int
        _rg.ref_gpu_time_polymul_dev.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                 C.POINTER(C.c_float)]
    return _rg


def ref_gpu_fft(x: np.ndarray, w: int, p: int, inverse: bool = False) -> np.ndarray:
    """The reference's own GPU transform, host to host: stockham_host, or
    inverse_stockham_host with the forward root w (src/stockham.cu:479-503)."""
    x = np.array(np.asarray(x, dtype=np.uint32).view(np.int32), copy=True)
    k = int(len(x)).bit_length() - 1
    assert len(x) == 1 << k
    rc = _ref_gpu_lib().ref_gpu_fft_host(x, len(x), k, w, p, int(inverse))
    if rc != 0:
        raise RuntimeError(f"reference GPU transform failed: CUDA error {rc}")
    return x.view(np.uint32)


def ref_gpu_time_fft_dev(x_ptr: int, k: int, w: int, p: int, reps: int) -> float:
    """Mean ms of the reference's stockham_dev on a device array (CUDA events)."""
    ms = C.c_float(0)
    rc = _ref_gpu_lib().ref_gpu_time_fft_dev(x_ptr, 1 << k, k, w, p, reps, C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU transform failed: CUDA error {rc}")
    return float(ms.value)


def ref_gpu_time_polymul_dev(f_ptr: int, g_ptr: int, e: int, p: int, reps: int) -> float:
    """Mean ms of the reference's stockham_poly_mul_dev on device arrays of 2^e words (CUDA events)."""
    ms = C.c_float(0)
    rc = _ref_gpu_lib().ref_gpu_time_polymul_dev(f_ptr, g_ptr, 1 << e, e, p, reps, C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU product failed: CUDA error {rc}")
    return float(ms.value)


class quiet_stdout:
    """Sends file descriptor 1 to /dev/null while the reference's GPU product
    runs: stockham_poly_mul_host prints its timing to stdout on every call
    (src/stockham.cu:600), which would mix with a caller's own output."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        C.CDLL(None).fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False


def ref_polymul_batch(pairs, p: int, threads: int):
    """Many independent modpn products over ``threads`` host threads.

    ``pairs`` is a list of (a, b) uint32 arrays; returns the list of products.
    """
    L = ref()
    L.ref_init_prime(p)
    da = np.array([len(a) - 1 for a, _ in pairs], dtype=np.int32)
    db = np.array([len(b) - 1 for _, b in pairs], dtype=np.int32)
    a_off = np.zeros(len(pairs), dtype=np.int64)
    b_off = np.zeros(len(pairs), dtype=np.int64)
    h_off = np.zeros(len(pairs), dtype=np.int64)
    a_off[1:] = np.cumsum(da + 1)[:-1]
    b_off[1:] = np.cumsum(db + 1)[:-1]
    h_off[1:] = np.cumsum(da + db + 1)[:-1]
    A = np.concatenate([np.asarray(a, dtype=np.uint32) for a, _ in pairs]).view(np.int32)
    B = np.concatenate([np.asarray(b, dtype=np.uint32) for _, b in pairs]).view(np.int32)
    H = np.empty(int((da + db + 1).sum()), dtype=np.int32)
    fails = L.ref_fftmul_batch(len(pairs), da, a_off, A, db, b_off, B, h_off, H, p, threads)
    if fails:
        raise RuntimeError(f"{fails} modpn products failed")
    return [H[h_off[i]:h_off[i] + da[i] + db[i] + 1].view(np.uint32) for i in range(len(pairs))]
