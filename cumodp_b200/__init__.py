"""cumodp_b200 -- B200-native FFT-based polynomial products over Fourier primes.

The product is the C-ABI library ``libcumodp.so`` (declared in
``include/cumodp.h``); this module is a thin ctypes binding over it whose
functions mirror the reference's entry points (src/modpn.cu:181-261) and
their error behaviour: a non-zero ``cumodp_err`` raises ``CumodpError``
carrying the reference's numeric code.

There is no CPU fallback: every call goes to the CUDA library, and importing
the binding fails loudly if ``libcumodp.so`` has not been built
(``python -m cumodp_b200.build``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcumodp.so")

# cumodp_err codes (include/types.h:123-146 of the reference)
SUCCESS = 0x000
FAILURE = 0x001
ASSUMPTION_ERROR = 0x002
NO_CUDA_DEVICE = 0x100
FFT_ERROR = 0x200
FOURIER_DEGREE_TOO_SMALL = 0x201
FFT_SIZE_TOO_LARGE = 0x202
FFT_SIZE_TOO_SMALL = 0x203
OUT_OF_MEMORY = 0x401

# Fourier primes used by the reference (its benchmark configurations, two-convolution).
P_469762049 = 469762049   # 7 * 2^26 + 1
P_754974721 = 754974721   # 45 * 2^24 + 1
TWOCONV_PRIMES = (962592769, 950009857, 940572673)


class CumodpError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = _lib().cumodp_error_string(code).decode() if _LIB is not None else ""
        super().__init__(f"{what}: cumodp_err 0x{code:03x} ({msg})")


_LIB = None


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("memory_budget", C.c_size_t), ("max_batch", C.c_int),
                ("batch_window_us", C.c_int), ("lanes", C.c_int), ("inject_fault_batch", C.c_int),
                ("host_budget", C.c_size_t)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_longlong), ("failed", C.c_longlong), ("batches", C.c_longlong),
                ("pending", C.c_longlong), ("inflight_bytes", C.c_size_t), ("p50_us", C.c_double),
                ("p99_us", C.c_double), ("max_us", C.c_double), ("products_per_s", C.c_double)]


_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cumodp_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.cumodp_error_string.restype = C.c_char_p
        L.cumodp_error_string.argtypes = [C.c_int]
        for name in ("is_cuda_enabled", "num_of_cuda_devices", "is_double_float_enabled"):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = []
        L.global_memory_in_bytes.restype = C.c_uint
        L.global_memory_in_bytes.argtypes = []
        L.global_memory_in_megabytes.restype = C.c_float
        L.global_memory_in_megabytes.argtypes = []
        L.can_call_fftmul_uni.restype = C.c_int
        L.can_call_fftmul_uni.argtypes = [C.c_int32, C.c_int32]
        L.cumodp_fftmul_uni.restype = C.c_int
        L.cumodp_fftmul_uni.argtypes = [C.c_int32, _i32p, C.c_int32, _i32p, C.c_int32, _i32p, C.c_int32]
        L.cumodp_fftmul_uni_dev.restype = C.c_int
        L.cumodp_fftmul_uni_dev.argtypes = [C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                            C.c_void_p, C.c_int32, C.c_void_p]
        for name in ("cumodp_fft_uni", "cumodp_invfft_uni"):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = [_i32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        for name in ("cumodp_fft_bivariate", "cumodp_invfft_bivariate"):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = [_i32p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        L.cumodp_fftmul_batch.restype = C.c_int
        L.cumodp_fftmul_batch.argtypes = [C.c_int, _i32p, _i64p, _i32p, _i32p, _i64p, _i32p, _i64p,
                                          _i32p, C.c_int32]
        L.cumodp_fftmul_batch_dev.restype = C.c_int
        L.cumodp_fftmul_batch_dev.argtypes = [C.c_int, _i32p, _i64p, C.c_void_p, _i32p, _i64p, C.c_void_p,
                                              _i64p, C.c_void_p, C.c_int32, C.c_void_p]
        L.cumodp_fftmul_uni_dev_noalloc.restype = C.c_int
        L.cumodp_fftmul_uni_dev_noalloc.argtypes = [C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                                    C.c_void_p, C.c_int32, C.c_void_p]
        L.cumodp_fft_uni_dev.restype = C.c_int
        L.cumodp_fft_uni_dev.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                                         C.c_void_p]
        L.cumodp_fft_bivariate_dev.restype = C.c_int
        L.cumodp_fft_bivariate_dev.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                               C.c_int, C.c_void_p]
        L.cumodp_list_fft_dev.restype = C.c_int
        L.cumodp_list_fft_dev.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                                          C.c_void_p]
        L.cumodp_bivariate_mul_dev.restype = C.c_int
        L.cumodp_bivariate_mul_dev.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
        L.cumodp_bivariate_mul.restype = C.c_int
        L.cumodp_bivariate_mul.argtypes = [C.c_int32, C.c_int32, _i32p, C.c_int32, C.c_int32, _i32p, _i32p,
                                           C.c_int32]
        L.cumodp_subproduct_level_dev.restype = C.c_int
        L.cumodp_subproduct_level_dev.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                                  C.c_void_p]
        L.cumodp_twoconv_mul_big.restype = C.c_int
        L.cumodp_twoconv_mul_big.argtypes = [C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, C.c_int,
                                             C.c_void_p, C.c_int]
        L.cumodp_twoconv_mul_big_dev.restype = C.c_int
        L.cumodp_twoconv_mul_big_dev.argtypes = [C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, C.c_int,
                                                 C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.cumodp_twoconv_big_bit_width.restype = C.c_int
        L.cumodp_twoconv_big_bit_width.argtypes = [C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p, C.c_int]
        L.cumodp_twoconv_big_out_words.restype = C.c_int
        L.cumodp_twoconv_big_out_words.argtypes = [C.c_longlong, C.c_longlong, C.c_int]
        L.cumodp_twoconv_big_plan.restype = C.c_int
        L.cumodp_twoconv_big_plan.argtypes = [C.c_int, C.c_longlong, C.c_longlong, C.POINTER(C.c_int),
                                              C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.cumodp_inject_alloc_failures.restype = None
        L.cumodp_inject_alloc_failures.argtypes = [C.c_int]
        L.cumodp_select_device.restype = C.c_int
        L.cumodp_select_device.argtypes = [C.c_int]
        L.cumodp_trace_passes.restype = None
        L.cumodp_trace_passes.argtypes = [C.c_int]
        L.cumodp_trace_report.restype = C.c_size_t
        L.cumodp_trace_report.argtypes = [C.c_char_p, C.c_size_t, C.c_int]
        L.cumodp_twoconv_mul_i64.restype = C.c_int
        L.cumodp_twoconv_mul_i64.argtypes = [C.c_longlong, _i64p, C.c_longlong, _i64p, _i64p, C.c_int]
        L.cumodp_twoconv_mul_i64_dev.restype = C.c_int
        L.cumodp_twoconv_mul_i64_dev.argtypes = [C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p,
                                                 C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.cumodp_twoconv_bit_width.restype = C.c_int
        L.cumodp_twoconv_bit_width.argtypes = [C.c_longlong, _i64p, C.c_longlong, _i64p]
        L.cumodp_twoconv_plan.restype = C.c_int
        L.cumodp_twoconv_plan.argtypes = [C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.c_int,
                                          C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.cumodp_server_default_config.restype = None
        L.cumodp_server_default_config.argtypes = [C.POINTER(ServerConfig)]
        L.cumodp_server_create.restype = C.c_void_p
        L.cumodp_server_create.argtypes = [C.POINTER(ServerConfig)]
        L.cumodp_server_submit_mod.restype = C.c_longlong
        L.cumodp_server_submit_mod.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                               C.c_void_p]
        L.cumodp_server_submit_i64.restype = C.c_longlong
        L.cumodp_server_submit_i64.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p,
                                               C.c_void_p]
        L.cumodp_server_poll.restype = C.c_int
        L.cumodp_server_poll.argtypes = [C.c_void_p, C.c_longlong]
        L.cumodp_server_wait.restype = C.c_int
        L.cumodp_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong]
        L.cumodp_server_replay.restype = C.c_int
        L.cumodp_server_replay.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                           C.c_void_p, C.POINTER(C.c_double)]
        L.cumodp_server_register.restype = C.c_int
        L.cumodp_server_register.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.cumodp_server_unregister.restype = C.c_int
        L.cumodp_server_unregister.argtypes = [C.c_void_p, C.c_void_p]
        L.cumodp_server_get_stats.restype = None
        L.cumodp_server_get_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.cumodp_server_reset_stats.restype = None
        L.cumodp_server_reset_stats.argtypes = [C.c_void_p]
        L.cumodp_server_destroy.restype = None
        L.cumodp_server_destroy.argtypes = [C.c_void_p]
        L.cumodp_device_bytes_in_use.restype = C.c_size_t
        L.cumodp_device_bytes_in_use.argtypes = []
        _LIB = L
    return _LIB


def lib():
    """The loaded libcumodp.so (ctypes CDLL)."""
    return _lib()


def _check(code: int, what: str) -> None:
    if code != SUCCESS:
        raise CumodpError(code, what)


def _as_i32(x) -> np.ndarray:
    """32-bit words of x as an int32 view (no copy for contiguous int32/uint32 input)."""
    a = np.asarray(x)
    if a.dtype == np.int32:
        return np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        return np.ascontiguousarray(a).view(np.int32)
    return np.ascontiguousarray(a.astype(np.uint32).view(np.int32))


# ------------------------------------------------------------- queries ----

def is_cuda_enabled() -> bool:
    return bool(_lib().is_cuda_enabled())


def num_of_cuda_devices() -> int:
    return int(_lib().num_of_cuda_devices())


def can_call_fftmul_uni(df: int, dg: int) -> bool:
    return bool(_lib().can_call_fftmul_uni(df, dg))


# ------------------------------------------------------------ products ----

def fftmul_uni(F, G, p: int, dh: int | None = None) -> np.ndarray:
    """H = F * G mod p through ``cumodp_fftmul_uni`` (host arrays).

    Returns dh+1 coefficients (default dh = deg F + deg G) as uint32.
    """
    f = _as_i32(F)
    g = _as_i32(G)
    if dh is None:
        dh = len(f) + len(g) - 2
    h = np.empty(dh + 1, dtype=np.int32)
    _check(_lib().cumodp_fftmul_uni(dh, h, len(f) - 1, f, len(g) - 1, g, p), "cumodp_fftmul_uni")
    return h.view(np.uint32)


def fftmul_uni_dev(h_ptr: int, lh: int, f_ptr: int, df: int, g_ptr: int, dg: int, p: int,
                   stream: int = 0) -> None:
    """Device-pointer product: lh words of H = F * G mod p (``cumodp_fftmul_uni_dev``)."""
    _check(_lib().cumodp_fftmul_uni_dev(lh, h_ptr, df, f_ptr, dg, g_ptr, p, stream or None),
           "cumodp_fftmul_uni_dev")


def fftmul_uni_dev_noalloc(h_ptr: int, lh: int, f_ptr: int, df: int, g_ptr: int, dg: int, p: int,
                           stream: int = 0) -> None:
    """Device-pointer product that allocates no device memory (``cumodp_fftmul_uni_dev_noalloc``).

    For callers that may not allocate device memory (pool-owned device
    memory, plugins in a host that partitioned device memory, latency-critical
    code that cannot take cudaMalloc's implicit synchronisation).  Scratch is
    a fixed ~8.4 MiB array in the library's device data segment, whose tables
    every call rewrites; products up to df + dg + 1 <= 2^20; calls that
    overlap on the GPU race on that array.
    """
    _check(_lib().cumodp_fftmul_uni_dev_noalloc(lh, h_ptr, df, f_ptr, dg, g_ptr, p, stream or None),
           "cumodp_fftmul_uni_dev_noalloc")


# ----------------------------------------------------------- transforms ----

def fft_uni(X, w: int, p: int) -> np.ndarray:
    """Natural-order DFT with root w (``cumodp_fft_uni``); returns a new array."""
    x = _as_i32(X).copy()
    n = len(x)
    k = n.bit_length() - 1
    _check(_lib().cumodp_fft_uni(x, n, k, w, p), "cumodp_fft_uni")
    return x.view(np.uint32)


def invfft_uni(X, w: int, p: int) -> np.ndarray:
    """Inverse of fft_uni: DFT with w^-1 scaled by n^-1 (``cumodp_invfft_uni``)."""
    x = _as_i32(X).copy()
    n = len(x)
    k = n.bit_length() - 1
    _check(_lib().cumodp_invfft_uni(x, n, k, w, p), "cumodp_invfft_uni")
    return x.view(np.uint32)


def fft_bivariate(X, em: int, wm: int, en: int, wn: int, p: int, inverse: bool = False) -> np.ndarray:
    """2-D DFT of a row-major 2^em x 2^en array (``cumodp_fft_bivariate``)."""
    x = _as_i32(X).reshape(-1).copy()
    assert len(x) == 1 << (em + en)
    f = _lib().cumodp_invfft_bivariate if inverse else _lib().cumodp_fft_bivariate
    _check(f(x, em, wm, en, wn, p), "cumodp_fft_bivariate")
    return x.view(np.uint32)


# ------------------------------------------------------------- batches ----

def _batch_layout(pairs):
    df = np.array([len(a) - 1 for a, _ in pairs], dtype=np.int32)
    dg = np.array([len(b) - 1 for _, b in pairs], dtype=np.int32)
    f_off = np.zeros(len(pairs), dtype=np.int64)
    g_off = np.zeros(len(pairs), dtype=np.int64)
    h_off = np.zeros(len(pairs), dtype=np.int64)
    if len(pairs):
        f_off[1:] = np.cumsum(df.astype(np.int64) + 1)[:-1]
        g_off[1:] = np.cumsum(dg.astype(np.int64) + 1)[:-1]
        h_off[1:] = np.cumsum(df.astype(np.int64) + dg + 1)[:-1]
    return df, dg, f_off, g_off, h_off


def fftmul_batch(pairs, p: int):
    """Products of many (F, G) pairs mod p in one batched call (``cumodp_fftmul_batch``)."""
    df, dg, f_off, g_off, h_off = _batch_layout(pairs)
    F = np.concatenate([_as_i32(a) for a, _ in pairs]) if pairs else np.zeros(1, np.int32)
    G = np.concatenate([_as_i32(b) for _, b in pairs]) if pairs else np.zeros(1, np.int32)
    H = np.empty(max(1, int((df.astype(np.int64) + dg + 1).sum())), dtype=np.int32)
    _check(_lib().cumodp_fftmul_batch(len(pairs), df, f_off, F, dg, g_off, G, h_off, H, p),
           "cumodp_fftmul_batch")
    Hu = H.view(np.uint32)
    return [Hu[h_off[i]:h_off[i] + df[i] + dg[i] + 1] for i in range(len(pairs))]


def fftmul_batch_dev(df, f_off, f_ptr: int, dg, g_off, g_ptr: int, h_off, h_ptr: int, p: int,
                     stream: int = 0) -> None:
    """Device-resident batch (``cumodp_fftmul_batch_dev``); offsets/degrees are host arrays."""
    df = np.ascontiguousarray(df, dtype=np.int32)
    dg = np.ascontiguousarray(dg, dtype=np.int32)
    f_off = np.ascontiguousarray(f_off, dtype=np.int64)
    g_off = np.ascontiguousarray(g_off, dtype=np.int64)
    h_off = np.ascontiguousarray(h_off, dtype=np.int64)
    _check(_lib().cumodp_fftmul_batch_dev(len(df), df, f_off, f_ptr, dg, g_off, g_ptr, h_off, h_ptr, p,
                                          stream or None), "cumodp_fftmul_batch_dev")


def fft_uni_dev(x_ptr: int, k: int, w: int, p: int, inverse: bool = False, stream: int = 0) -> None:
    """In-place natural-order transform of 2^k device words (``cumodp_fft_uni_dev``)."""
    _check(_lib().cumodp_fft_uni_dev(x_ptr, 1 << k, k, w, p, int(inverse), stream or None),
           "cumodp_fft_uni_dev")


def fft_bivariate_dev(x_ptr: int, em: int, wm: int, en: int, wn: int, p: int, inverse: bool = False,
                      stream: int = 0) -> None:
    """In-place 2-D transform of a 2^em x 2^en device array (``cumodp_fft_bivariate_dev``)."""
    _check(_lib().cumodp_fft_bivariate_dev(x_ptr, em, wm, en, wn, p, int(inverse), stream or None),
           "cumodp_fft_bivariate_dev")


def list_fft_dev(x_ptr: int, m: int, k: int, w: int, p: int, inverse: bool = False, stream: int = 0) -> None:
    """m natural-order transforms of 2^k device words each, in place (``cumodp_list_fft_dev``)."""
    _check(_lib().cumodp_list_fft_dev(x_ptr, m, k, w, p, int(inverse), stream or None), "cumodp_list_fft_dev")


def bivariate_mul(F, G, p: int) -> np.ndarray:
    """Bivariate product mod p (``cumodp_bivariate_mul``).

    F, G: 2-D arrays indexed [y, x] (row j holds the coefficients of y^j).
    Returns the product as a uint32 array of shape (nyf + nyg - 1, nxf + nxg - 1).
    """
    F = np.asarray(F)
    G = np.asarray(G)
    (nyf, nxf), (nyg, nxg) = F.shape, G.shape
    f = _as_i32(np.ascontiguousarray(F).reshape(-1))
    g = _as_i32(np.ascontiguousarray(G).reshape(-1))
    h = np.empty((nyf + nyg - 1) * (nxf + nxg - 1), dtype=np.int32)
    _check(_lib().cumodp_bivariate_mul(nxf, nyf, f, nxg, nyg, g, h, p), "cumodp_bivariate_mul")
    return h.view(np.uint32).reshape(nyf + nyg - 1, nxf + nxg - 1)


def bivariate_mul_dev(em: int, en: int, f_ptr: int, g_ptr: int, p: int, stream: int = 0) -> None:
    """In-place 2-D cyclic convolution on a 2^em x 2^en device grid (``cumodp_bivariate_mul_dev``)."""
    _check(_lib().cumodp_bivariate_mul_dev(em, en, f_ptr, g_ptr, p, stream or None), "cumodp_bivariate_mul_dev")


def subproduct_level_dev(l: int, npairs: int, in_ptr: int, out_ptr: int, p: int, stream: int = 0) -> None:
    """One subproduct-tree level on device arrays (``cumodp_subproduct_level_dev``)."""
    _check(_lib().cumodp_subproduct_level_dev(l, npairs, in_ptr, out_ptr, p, stream or None),
           "cumodp_subproduct_level_dev")


def inject_alloc_failures(count: int) -> None:
    """Host-side fault injection: the next `count` device allocations fail (0 cancels)."""
    _lib().cumodp_inject_alloc_failures(count)


def select_device(dev: int) -> None:
    _check(_lib().cumodp_select_device(dev), "cumodp_select_device")


def trace_passes(enable: bool) -> None:
    """Bracket every (non-captured) kernel launch with CUDA events."""
    _lib().cumodp_trace_passes(int(enable))


def trace_report(reset: bool = True) -> dict:
    """{kernel: (launches, total_ms)} accumulated since the last reset."""
    n = _lib().cumodp_trace_report(None, 0, 0)
    buf = C.create_string_buffer(n + 1)
    _lib().cumodp_trace_report(buf, n + 1, int(reset))
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out


# ------------------------------------------------------ exact products ----

def int128_words_to_ints(w: np.ndarray) -> list:
    """(lo, hi) int64 word pairs -> Python ints."""
    lo = w[0::2].astype(np.uint64).astype(object)
    hi = w[1::2].astype(np.int64).astype(object)
    return [int(h) * (1 << 64) + int(l) for l, h in zip(lo, hi)]


def twoconv_mul(a, b, method: int = 0, raw: bool = False):
    """Exact product of int64 polynomials (``cumodp_twoconv_mul_i64``).

    Returns the na+nb-1 coefficients as Python ints (or the raw (lo, hi)
    int64 words when ``raw``).  method 1 forces the two-prime limb split.
    """
    a = np.ascontiguousarray(a, dtype=np.int64)
    b = np.ascontiguousarray(b, dtype=np.int64)
    c = np.empty(2 * (len(a) + len(b) - 1), dtype=np.int64)
    _check(_lib().cumodp_twoconv_mul_i64(len(a), a, len(b), b, c, method), "cumodp_twoconv_mul_i64")
    return c if raw else int128_words_to_ints(c)


def twoconv_bit_width(a, b) -> int:
    a = np.ascontiguousarray(a, dtype=np.int64)
    b = np.ascontiguousarray(b, dtype=np.int64)
    return int(_lib().cumodp_twoconv_bit_width(len(a), a, len(b), b))


def twoconv_plan(bit_width_a: int, bit_width_b: int, na: int, nb: int, method: int = 0):
    """(K, M, number of primes) the exact product would use."""
    K, M, npr = C.c_int(), C.c_int(), C.c_int()
    _check(_lib().cumodp_twoconv_plan(bit_width_a, bit_width_b, na, nb, method, C.byref(K), C.byref(M),
                                      C.byref(npr)), "cumodp_twoconv_plan")
    return K.value, M.value, npr.value


def ints_to_words(values, words: int) -> np.ndarray:
    """Python ints -> `words` little-endian 64-bit two's-complement words each."""
    out = np.empty(len(values) * words, dtype=np.uint64)
    mask = (1 << (64 * words)) - 1
    for i, v in enumerate(values):
        u = int(v) & mask
        out[i * words:(i + 1) * words] = [(u >> (64 * k)) & 0xFFFFFFFFFFFFFFFF for k in range(words)]
    return out


def words_to_ints(w: np.ndarray, words: int) -> list:
    """`words` little-endian 64-bit two's-complement words each -> Python ints."""
    w = np.asarray(w, dtype=np.uint64).reshape(-1, words)
    top = 1 << (64 * words)
    res = []
    for row in w:
        u = 0
        for k in range(words - 1, -1, -1):
            u = (u << 64) | int(row[k])
        res.append(u - top if u >> (64 * words - 1) else u)
    return res


def twoconv_big_words(values) -> int:
    """64-bit words a signed coefficient list needs (two's complement)."""
    bits = max((abs(int(v)).bit_length() for v in values), default=0) + 1
    return max(1, (bits + 63) // 64)


def twoconv_mul_big(a, b, in_words: int | None = None, out_words: int | None = None):
    """Exact product of big-integer polynomials (``cumodp_twoconv_mul_big``); Python ints in and out."""
    if in_words is None:
        in_words = max(twoconv_big_words(a), twoconv_big_words(b))
    wa, wb = ints_to_words(a, in_words), ints_to_words(b, in_words)
    if out_words is None:
        bw = int(_lib().cumodp_twoconv_big_bit_width(len(a), wa.ctypes.data, len(b), wb.ctypes.data, in_words))
        out_words = int(_lib().cumodp_twoconv_big_out_words(len(a), len(b), bw))
    c = np.empty((len(a) + len(b) - 1) * out_words, dtype=np.uint64)
    _check(_lib().cumodp_twoconv_mul_big(len(a), wa.ctypes.data, len(b), wb.ctypes.data, in_words, c.ctypes.data,
                                         out_words), "cumodp_twoconv_mul_big")
    return words_to_ints(c, out_words)


def twoconv_big_plan(bit_width: int, na: int, nb: int):
    """(K, M, number of primes, log2 transform length) of the big-coefficient product."""
    K, M, npr, lg = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    _check(_lib().cumodp_twoconv_big_plan(bit_width, na, nb, C.byref(K), C.byref(M), C.byref(npr), C.byref(lg)),
           "cumodp_twoconv_big_plan")
    return K.value, M.value, npr.value, lg.value


# ------------------------------------------------------------- serving ----

class Server:
    """Continuous-batching request loop (``cumodp_server_*``).

    submit_mod / submit_i64 copy the inputs and return (request id, output
    array); the output array is filled when wait(id) returns 0.
    """

    def __init__(self, device: int = 0, memory_budget: int = 0, max_batch: int = 512,
                 batch_window_us: int = 50, lanes: int = 4, inject_fault_batch: int = 0, host_budget: int = 0):
        cfg = ServerConfig()
        _lib().cumodp_server_default_config(C.byref(cfg))
        cfg.device, cfg.memory_budget, cfg.max_batch = device, memory_budget, max_batch
        cfg.batch_window_us, cfg.lanes, cfg.inject_fault_batch = batch_window_us, lanes, inject_fault_batch
        cfg.host_budget = host_budget
        self._h = _lib().cumodp_server_create(C.byref(cfg))
        if not self._h:
            raise CumodpError(NO_CUDA_DEVICE, "cumodp_server_create")
        self._outs = {}
        self._regs = []

    def submit_mod(self, F, G, p: int):
        f = _as_i32(F)
        g = _as_i32(G)
        out = np.empty(len(f) + len(g) - 1, dtype=np.int32)
        rid = _lib().cumodp_server_submit_mod(self._h, p, len(f) - 1, f.ctypes.data, len(g) - 1, g.ctypes.data,
                                              out.ctypes.data)
        if rid < 0:
            raise CumodpError(ASSUMPTION_ERROR, "cumodp_server_submit_mod")
        self._outs[rid] = out
        return rid, out.view(np.uint32)

    def submit_i64(self, a, b):
        a = np.ascontiguousarray(a, dtype=np.int64)
        b = np.ascontiguousarray(b, dtype=np.int64)
        out = np.empty(2 * (len(a) + len(b) - 1), dtype=np.int64)
        rid = _lib().cumodp_server_submit_i64(self._h, len(a), a.ctypes.data, len(b), b.ctypes.data,
                                              out.ctypes.data)
        if rid < 0:
            raise CumodpError(ASSUMPTION_ERROR, "cumodp_server_submit_i64")
        self._outs[rid] = out
        return rid, out

    def replay(self, arrival_us, requests, threads: int = 4, outputs=None):
        """Open-loop replay of a timed trace by native threads (``cumodp_server_replay``).

        requests[i] = (a, b, p): p = None for an exact int64 product, else the
        prime of a product mod p (a, b residue arrays).  outputs[i] (optional)
        receives the result; without it results are dropped.  Returns
        (status array, latency array in microseconds from the scheduled
        arrival to the result, span in microseconds).
        """
        n = len(requests)
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        assert len(arr) == n
        kind = np.empty(n, np.int32)
        pr = np.zeros(n, np.int32)
        la = np.empty(n, np.int64)
        lb = np.empty(n, np.int64)
        keep = []
        pa = (C.c_void_p * max(n, 1))()
        pb = (C.c_void_p * max(n, 1))()
        for i, (a, b, p) in enumerate(requests):
            if p is None:
                a = np.ascontiguousarray(a, dtype=np.int64)
                b = np.ascontiguousarray(b, dtype=np.int64)
                kind[i] = 1
            else:
                a, b = _as_i32(a), _as_i32(b)
                kind[i], pr[i] = 0, p
            keep += [a, b]
            la[i], lb[i] = len(a), len(b)
            pa[i], pb[i] = a.ctypes.data, b.ctypes.data
        ph = None
        if outputs is not None:
            ph = (C.c_void_p * max(n, 1))(*[o.ctypes.data for o in outputs])
        lat = np.zeros(n, np.float64)
        st = np.zeros(n, np.int32)
        span = C.c_double(0)
        _check(_lib().cumodp_server_replay(self._h, n, arr.ctypes.data, kind.ctypes.data, pr.ctypes.data,
                                           la.ctypes.data, lb.ctypes.data, pa, pb, ph, threads,
                                           lat.ctypes.data, st.ctypes.data, C.byref(span)),
               "cumodp_server_replay")
        return st, lat, span.value

    def register(self, arr: np.ndarray) -> None:
        """Registers a C-contiguous host array (``cumodp_server_register``): requests whose operands or
        outputs lie in it skip the server's pinned staging copies.  Keep the array alive, and unchanged
        while requests read it, until unregister (or close)."""
        assert arr.flags["C_CONTIGUOUS"]
        _check(_lib().cumodp_server_register(self._h, arr.ctypes.data, arr.nbytes), "cumodp_server_register")
        self._regs.append(arr)

    def unregister(self, arr: np.ndarray) -> None:
        _check(_lib().cumodp_server_unregister(self._h, arr.ctypes.data), "cumodp_server_unregister")
        self._regs = [a for a in self._regs if a is not arr]

    def poll(self, rid: int) -> int:
        return int(_lib().cumodp_server_poll(self._h, rid))

    def wait(self, rid: int, timeout_us: int = -1) -> int:
        st = int(_lib().cumodp_server_wait(self._h, rid, timeout_us))
        if st != -2:
            self._outs.pop(rid, None)
        return st

    def stats(self) -> dict:
        s = ServerStats()
        _lib().cumodp_server_get_stats(self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def reset_stats(self) -> None:
        _lib().cumodp_server_reset_stats(self._h)

    def close(self) -> None:
        if self._h:
            _lib().cumodp_server_destroy(self._h)  # drains, then unregisters what is left
            self._h = None
            self._regs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def device_bytes_in_use() -> int:
    return int(_lib().cumodp_device_bytes_in_use())
