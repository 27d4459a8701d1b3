/*
 * CPU oracle for the FFT-based polynomial product path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the arithmetic
 * of the reference library so that tests/ and bench.py's CPU baseline can
 * check the CUDA product path.  The shipped library (cumodp_b200/) never
 * links, loads or calls it.
 *
 * What is restated, with the reference file:line each piece follows:
 *   - field arithmetic: add/sub/mul/pow/inverse mod p
 *       (include/inlines.h:70-122, 137-167, 181-221);
 *   - deterministic primitive root: srand(1), rand() % p, r^((p-1)/n),
 *       reject while r^(n/2) == 1   (include/inlines.h:460-485);
 *   - the DFT the Stockham kernels compute: X[j] = sum_i x[i] w^(ij) in
 *       natural order (src/stockham.cu:413-434; inverse with w^-1 and n^-1
 *       scaling, src/stockham.cu:462-503);
 *   - schoolbook product mod p (src/fft_aux.cu:805-820, plain_polymul_uni_host);
 *   - FFT product mod p with the reference's size rule n = 2^ceil(log2(df+dg+1))
 *       (src/stockham.cu:562-611);
 *   - exact integer product by __int128 schoolbook (the two-convolution
 *       checker, unit_tests/test_two_convolution_poly_mul.cpp:112-193);
 *   - two-convolution helpers: coefficient bit width
 *       (src/two_convolution_poly_mul.cu:58-70), sign-magnitude limb split of
 *       a coefficient into K limbs of M bits mod a prime (:84-203),
 *       x-argument scaling by theta^(i mod K) (:207-245), and the 3-prime CRT
 *       lift to a signed integer (:292-385).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;
typedef __int128 i128;
typedef unsigned __int128 u128;

/* ---------------------------------------------------------------- field -- */

static inline u32 om_add(u32 a, u32 b, u32 p) { u32 r = a + b; return r >= p ? r - p : r; }
static inline u32 om_sub(u32 a, u32 b, u32 p) { return a >= b ? a - b : a + p - b; }
static inline u32 om_mul(u32 a, u32 b, u32 p) { return (u32)(((u64)a * b) % p); }

u32 or_pow(u32 a, u64 e, u32 p)
{
    u32 r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = om_mul(r, a, p);
        a = om_mul(a, a, p);
        e >>= 1;
    }
    return r;
}

/* Inverse by the extended Euclidean algorithm (include/inlines.h:137-167). */
u32 or_inv(u32 a, u32 p)
{
    i64 t = 0, nt = 1, r = p, nr = a % p;
    while (nr) {
        i64 q = r / nr, tmp;
        tmp = t - q * nt; t = nt; nt = tmp;
        tmp = r - q * nr; r = nr; nr = tmp;
    }
    if (t < 0) t += p;
    return (u32)t;
}

/* 2-adic order of p-1 (include/inlines.h:408-413). */
int or_fourier_degree(u32 p)
{
    u32 q = p - 1;
    int e = 0;
    while (q && !(q & 1)) { q >>= 1; ++e; }
    return e;
}

/* The reference's deterministic n-th primitive root, n = 2^e
 * (include/inlines.h:460-485): glibc srand(1) then rand() % p draws. */
u32 or_primitive_root(int e, u32 p)
{
    u32 k = (p - 1) >> e;
    u64 n2 = (u64)1 << (e - 1);
    u32 root = 0;
    srand(1);
    for (;;) {
        root = 1;
        while (root < 2) root = (u32)rand() % p;
        root = or_pow(root, k, p);
        if (or_pow(root, n2, p) != 1) break;
    }
    return root;
}

/* ------------------------------------------------------------ transforms -- */

/* Direct O(n^2) DFT: out[j] = sum_i x[i] w^(ij) mod p. */
void or_dft_naive(int n, const u32 *x, u32 w, u32 p, u32 *out)
{
    for (int j = 0; j < n; ++j) {
        u32 wj = or_pow(w, (u64)j, p), acc = 0, t = 1;
        for (int i = 0; i < n; ++i) {
            acc = om_add(acc, om_mul(x[i], t, p), p);
            t = om_mul(t, wj, p);
        }
        out[j] = acc;
    }
}

static void bit_reverse_perm(u32 *x, int k)
{
    u64 n = (u64)1 << k;
    for (u64 i = 1, j = 0; i < n; ++i) {
        u64 bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { u32 t = x[i]; x[i] = x[j]; x[j] = t; }
    }
}

/* In-place natural-order DFT of length 2^k with n-th root w: the same map as
 * the reference's stockham_dev (src/stockham.cu:413-434), computed here by a
 * textbook iterative radix-2 Cooley-Tukey pass structure. */
void or_ntt(u32 *x, int k, u32 w, u32 p)
{
    u64 n = (u64)1 << k;
    if (k == 0) return;
    bit_reverse_perm(x, k);
    u32 *pw = (u32 *)malloc(sizeof(u32) * (n / 2));
    for (u64 len = 2; len <= n; len <<= 1) {
        u32 wl = or_pow(w, n / len, p);
        u64 half = len / 2;
        pw[0] = 1;
        for (u64 j = 1; j < half; ++j) pw[j] = om_mul(pw[j - 1], wl, p);
        for (u64 i = 0; i < n; i += len)
            for (u64 j = 0; j < half; ++j) {
                u32 u = x[i + j], v = om_mul(x[i + j + half], pw[j], p);
                x[i + j] = om_add(u, v, p);
                x[i + j + half] = om_sub(u, v, p);
            }
    }
    free(pw);
}

/* Inverse: DFT with w^-1, then scale by n^-1 (src/stockham.cu:462-470). */
void or_intt(u32 *x, int k, u32 w, u32 p)
{
    u64 n = (u64)1 << k;
    or_ntt(x, k, or_inv(w, p), p);
    u32 ninv = or_inv((u32)(n % p), p);
    for (u64 i = 0; i < n; ++i) x[i] = om_mul(x[i], ninv, p);
}

/* --------------------------------------------------------------- products -- */

/* H[0..da+db] = A * B mod p, schoolbook (src/fft_aux.cu:805-820). */
void or_polymul_school(int da, const u32 *A, int db, const u32 *B, u32 *H, u32 p)
{
    int dh = da + db;
    u64 *acc = (u64 *)calloc((size_t)dh + 1, sizeof(u64));
    for (int i = 0; i <= da; ++i) {
        u64 a = A[i];
        for (int j = 0; j <= db; ++j) {
            acc[i + j] += a * B[j];
            if (acc[i + j] >= ((u64)1 << 63)) acc[i + j] %= p;
        }
    }
    for (int i = 0; i <= dh; ++i) H[i] = (u32)(acc[i] % p);
    free(acc);
}

/* H[0..da+db] = A * B mod p through transforms of size
 * n = 2^ceil(log2(da+db+1)) (src/stockham.cu:562-611).  Returns -1 when n
 * exceeds the prime's 2-adic order. */
int or_polymul_ntt(int da, const u32 *A, int db, const u32 *B, u32 *H, u32 p)
{
    u64 s = (u64)da + db + 1;
    int k = 0;
    while (((u64)1 << k) < s) ++k;
    if (k > or_fourier_degree(p)) return -1;
    u64 n = (u64)1 << k;
    u32 *F = (u32 *)calloc(n, sizeof(u32)), *G = (u32 *)calloc(n, sizeof(u32));
    memcpy(F, A, sizeof(u32) * ((size_t)da + 1));
    memcpy(G, B, sizeof(u32) * ((size_t)db + 1));
    /* any n-th primitive root gives the same product */
    u32 g = 3;
    while (k > 0 && or_pow(or_pow(g, (p - 1) >> k, p), n / 2, p) == 1) ++g;
    u32 w = k > 0 ? or_pow(g, (p - 1) >> k, p) : 1;
    or_ntt(F, k, w, p);
    or_ntt(G, k, w, p);
    for (u64 i = 0; i < n; ++i) F[i] = om_mul(F[i], G[i], p);
    or_intt(F, k, w, p);
    memcpy(H, F, sizeof(u32) * (size_t)s);
    free(F);
    free(G);
    return 0;
}

/* Exact product of int64 polynomials by __int128 schoolbook; H is written as
 * (lo, hi) 64-bit pairs, 2*(da+db+1) words. */
void or_polymul_i128(int da, const i64 *A, int db, const i64 *B, u64 *H)
{
    int dh = da + db;
    i128 *acc = (i128 *)calloc((size_t)dh + 1, sizeof(i128));
    for (int i = 0; i <= da; ++i) {
        i128 a = A[i];
        if (!a) continue;
        for (int j = 0; j <= db; ++j) acc[i + j] += a * (i128)B[j];
    }
    for (int i = 0; i <= dh; ++i) {
        u128 v = (u128)acc[i];
        H[2 * i] = (u64)v;
        H[2 * i + 1] = (u64)(v >> 64);
    }
    free(acc);
}

/* --------------------------------------------------- two-convolution parts -- */

/* Largest bit width of |c| over both inputs, with 0 counted as width 1 (the
 * behaviour of mpz_sizeinbase, src/two_convolution_poly_mul.cu:58-70). */
int or_bit_width(int na, const i64 *A, int nb, const i64 *B)
{
    int w = 0;
    for (int s = 0; s < 2; ++s) {
        const i64 *X = s ? B : A;
        int nx = s ? nb : na;
        for (int i = 0; i < nx; ++i) {
            u64 m = X[i] < 0 ? (u64)0 - (u64)X[i] : (u64)X[i];
            int b = m ? 64 - __builtin_clzll(m) : 1;
            if (b > w) w = b;
        }
    }
    return w;
}

/* Sign-magnitude limb split (src/two_convolution_poly_mul.cu:84-203): |c| is
 * cut into K limbs of M bits, least significant first; a negative c stores
 * p - limb for every non-zero limb.  out has n*K words, row i = coefficient i. */
void or_limb_split(int n, const i64 *A, int K, int M, u32 p, u32 *out)
{
    u64 mask = M >= 64 ? ~(u64)0 : (((u64)1 << M) - 1);
    for (int i = 0; i < n; ++i) {
        int neg = A[i] < 0;
        u64 m = neg ? (u64)0 - (u64)A[i] : (u64)A[i];
        for (int j = 0; j < K; ++j) {
            u64 limb = m & mask;
            m = M >= 64 ? 0 : m >> M;
            u32 r = (u32)(limb % p);
            out[(size_t)i * K + j] = (neg && r) ? p - r : r;
        }
    }
}

/* A[idx] *= theta^(idx mod K) mod p (src/two_convolution_poly_mul.cu:207-245). */
void or_scale_x(int size, u32 *A, int K, u32 theta, u32 p)
{
    for (int idx = 0; idx < size; ++idx)
        A[idx] = om_mul(A[idx], or_pow(theta, (u64)(idx % K), p), p);
}

/* Signed CRT lift of residues (r[0] mod p[0], ..., r[np-1] mod p[np-1]) to
 * the unique integer in (-P/2, P/2], P = prod p; returned as (lo, hi). Garner's
 * mixed-radix form, exact for np <= 3 primes below 2^31. */
void or_crt_signed(int np, const u32 *r, const u32 *p, u64 *lo, u64 *hi)
{
    /* mixed radix digits v0 + v1 p0 + v2 p0 p1 */
    u32 v[4];
    for (int i = 0; i < np; ++i) {
        u64 x = r[i] % p[i];
        /* subtract the digits found so far, in mod p[i] */
        u64 acc = 0, pr = 1;
        for (int j = 0; j < i; ++j) {
            acc = (acc + (u64)v[j] % p[i] * pr) % p[i];
            pr = pr * (p[j] % p[i]) % p[i];
        }
        x = (x + p[i] - acc) % p[i];
        v[i] = (u32)((u64)x * or_inv((u32)pr, p[i]) % p[i]);
    }
    u128 val = 0, P = 1;
    for (int i = 0; i < np; ++i) { val += (u128)v[i] * P; P *= p[i]; }
    i128 s = (i128)val;
    if (val > P / 2) s = (i128)val - (i128)P;
    *lo = (u64)(u128)s;
    *hi = (u64)((u128)s >> 64);
}
