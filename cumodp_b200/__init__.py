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

# Fourier primes used by the reference (two-convolution).
P_469762049 = 469762049   # 7 * 2^26 + 1
P_754974721 = 754974721   # 45 * 2^24 + 1
TWOCONV_PRIMES = (962592769, 950009857, 940572673)


class CumodpError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = _lib().cumodp_error_string(code).decode() if _LIB is not None else ""
        super().__init__(f"{what}: cumodp_err 0x{code:03x} ({msg})")


_LIB = None

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
    a = np.asarray(x)
    if a.dtype == np.int32:
        return np.ascontiguousarray(a)
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


def device_bytes_in_use() -> int:
    return int(_lib().cumodp_device_bytes_in_use())
