// Field arithmetic over 32-bit Fourier primes p = c * 2^e + 1 < 2^30.
//
// Replaces the reference's fp64-quotient `mul_mod` (include/inlines.h:95-122)
// and its Montgomery-like `fourier_reduction` (include/montmulmod.h:52-140)
// with two integer-pipe products:
//   * Shoup's product for a constant multiplier w with a precomputed quotient
//     w' = floor(w * 2^32 / p): three 32-bit multiplies, result in [0, 2p)
//     for any 32-bit input;
//   * Montgomery's product with R = 2^32 for two variable operands:
//     a * b * 2^-32 mod p, result in [0, 2p) whenever a * b < 2^32 * p.
// Residues are kept lazily in [0, 2p) or [0, 4p); 4p < 2^32 because p < 2^30.
// Every result leaving the library is reduced to [0, p), so it is the
// canonical residue the reference returns.
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace cmb {

typedef uint32_t u32;
typedef uint64_t u64;

// Host-side prime description; computed once per prime.
struct PrimeInfo {
    u32 p;         // the prime, < 2^30
    u32 p2;        // 2p
    u32 pinv_neg;  // -p^-1 mod 2^32 (Montgomery)
    u32 r1;        // 2^32 mod p
    u32 r2;        // 2^64 mod p
    int two_adic;  // largest e with 2^e | p - 1
};

__host__ __device__ __forceinline__ u32 mulmod_exact(u32 a, u32 b, u32 p) {
    return (u32)(((u64)a * b) % p);
}

__host__ __device__ __forceinline__ u32 powmod_exact(u32 a, u64 e, u32 p) {
    u32 r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod_exact(r, a, p);
        a = mulmod_exact(a, a, p);
        e >>= 1;
    }
    return r;
}

// Shoup quotient floor(w * 2^32 / p) for w < p.
__host__ __device__ __forceinline__ u32 shoup_quot(u32 w, u32 p) {
    return (u32)(((u64)w << 32) / p);
}

#ifdef __CUDACC__
// a * w mod p in [0, 2p) for any a < 2^32; w < p, wq = shoup_quot(w, p).
__device__ __forceinline__ u32 mul_shoup(u32 a, u32 w, u32 wq, u32 p) {
    u32 q = __umulhi(a, wq);
    return a * w - q * p;
}

// a * b * 2^-32 mod p in [0, 2p), valid when a * b < 2^32 * p.
__device__ __forceinline__ u32 mul_mont(u32 a, u32 b, u32 p, u32 pinv_neg) {
    u32 lo = a * b;
    u32 hi = __umulhi(a, b);
    u32 m = lo * pinv_neg;  // lo + m*p == 0 (mod 2^32)
    u32 t = __umulhi(m, p);
    return hi + t + (lo != 0u);
}
#endif

// [0, 4p) -> [0, 2p) and [0, 2p) -> [0, p), branch-free (unsigned min).
__host__ __device__ __forceinline__ u32 red2(u32 a, u32 p2) {
    u32 b = a - p2;
    return a < b ? a : b;
}
__host__ __device__ __forceinline__ u32 red1(u32 a, u32 p) {
    u32 b = a - p;
    return a < b ? a : b;
}

// A twiddle in Shoup form, stored as one 8-byte word in tables.
struct __align__(8) Tw {
    u32 w, wq;
};

}  // namespace cmb
