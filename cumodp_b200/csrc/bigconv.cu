// Exact product of polynomials with big signed integer coefficients.
//
// Reference: the general two_convolution_poly_mul
// (src/two_convolution_poly_mul.cu:532-569) on std::vector<mpz_class>: the
// base table picks N-bit coefficients cut into K >= 32 limbs of M bits
// (determine_bivariate_base, :72-82; convert_to_modular_bivariate, :84-203),
// the x-direction is handled by a cyclic and a negacyclic convolution of
// length K (two_convolution_2d_dev, :431-530), three primes are lifted by
// CRT on the host with GMP (reconstruct_mpz_with_crt, :292-385) and the
// product is (u+v)(2^M)/2 + 2^N (u-v)(2^M)/2 (recover_product_host,
// :387-428).
//
// Here the coefficients travel as fixed-width two's-complement words (no GMP
// on either side of the boundary) and the whole computation stays on the
// GPU:
//   1. k_big_abs: |a_j| and its sign, one thread per coefficient;
//   2. k_big_split: per prime, the Kronecker layout A_p[j*(2K-1) + i] =
//      sign_j * limb_i(|a_j|) mod p for i < K and 0 for K <= i < 2K-1, one
//      thread per word.  The zero tail of every block keeps the
//      (2K-1)-coefficient linear x-convolution of two K-limb numbers inside
//      its block, so one univariate product per prime equals the bivariate
//      product (about the total transform length of a cyclic plus a
//      negacyclic convolution of length K);
//   3. one univariate product per prime (fused single-CTA or three-pass
//      kernels);
//   4. k_big_crt: per output coefficient, Garner's CRT of every x-coefficient
//      to a signed 128-bit integer and the sum of them shifted by M*i bits,
//      in separate positive and negative multiword accumulators, stored as
//      out_words two's-complement words.
// The planner picks the number of primes (3 or 4) and the limb width M with
// the cheapest transform such that every x-coefficient satisfies
// K * min(la, lb) * (2^M - 1)^2 < P / 2.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/cumodp.h"
#include "exact.cuh"

namespace cmb {

int batch_mul_dev(int count, const sfixn* df, const int64_t* f_off, const u32* F, const sfixn* dg,
                  const int64_t* g_off, const u32* G, const int64_t* h_off, u32* H, u32 p, cudaStream_t st);

namespace {

constexpr int kBigMaxInWords = 64;    // coefficients up to 4096 bits
constexpr int kBigMaxAccWords = 136;  // 2 * 4096 + 192 bits of accumulator
constexpr int kBigMaxPrimes = 4;

// Fourier primes below 2^30, largest first, with their 2-adic orders.
const u32 kBigPrimes[] = {998244353u, 897581057u, 880803841u, 754974721u, 645922817u,
                          595591169u, 469762049u, 377487361u, 167772161u};
const int kBigPrimeOrder[] = {23, 23, 23, 24, 23, 23, 26, 23, 25};

struct BigPlan {
    int K, M, nprimes, logn;
    u32 p[kBigMaxPrimes];
};

int ceil_log2_ll(long long v) {
    int l = 0;
    while ((1ll << l) < v) ++l;
    return l;
}

// log2 of a product of primes (a lower bound by a hair, for the bound test).
double log2_prod(const u32* p, int r) {
    double s = 0;
    for (int i = 0; i < r; ++i) s += std::log2((double)p[i]);
    return s;
}

int big_plan(int bw, long long na, long long nb, BigPlan* out) {
    if (bw < 0 || bw > 64 * kBigMaxInWords || na <= 0 || nb <= 0) return ASSUMPTION_ERROR;
    const int bits = std::max(bw, 1);
    const long long nmin = std::min(na, nb);
    bool found = false;
    BigPlan best{};
    double best_cost = 0;
    for (int r = 3; r <= kBigMaxPrimes; ++r) {
        for (int M = std::min(62, bits); M >= 1; --M) {
            const int K = (bits + M - 1) / M;
            const long long la = (2ll * K - 1) * (na - 1) + K, lb = (2ll * K - 1) * (nb - 1) + K;
            const int logn = ceil_log2_ll(la + lb - 1);
            if (logn > kMaxLog) continue;
            u32 p[kBigMaxPrimes];
            int k = 0;
            for (size_t i = 0; i < sizeof(kBigPrimes) / sizeof(kBigPrimes[0]) && k < r; ++i)
                if (kBigPrimeOrder[i] >= logn) p[k++] = kBigPrimes[i];
            if (k < r) continue;
            // |x-coefficient| <= K * nmin * (2^M - 1)^2 < 2^(2M + log2(K nmin)) < P / 2
            const double need = 2.0 * M + std::log2((double)K * (double)nmin) + 1.0;
            if (need >= log2_prod(p, r) - 0.01) continue;
            const double cost = (double)r * std::ldexp(1.0, logn) * logn;
            if (!found || cost < best_cost) {
                found = true;
                best_cost = cost;
                best.K = K;
                best.M = M;
                best.nprimes = r;
                best.logn = logn;
                for (int i = 0; i < r; ++i) best.p[i] = p[i];
            }
            break;  // the largest feasible M for this r
        }
    }
    if (!found) return FFT_SIZE_TOO_LARGE;
    *out = best;
    return OK;
}

// Words of a product coefficient: |c| <= min(na, nb) * (2^bw - 1)^2.
int big_out_words(long long na, long long nb, int bw) {
    const int bits = 2 * std::max(bw, 1) + ceil_log2_ll(std::min(na, nb) + 1) + 1;
    return (bits + 63) / 64;
}

// |x_j| (in_words words) and sign, one coefficient per thread and step of a
// grid-stride loop (the grid is capped by grid_of).
__global__ void k_big_abs(const unsigned long long* __restrict__ x, long long len, int words,
                          unsigned long long* __restrict__ mag, unsigned char* __restrict__ neg) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < len;
         j += (long long)gridDim.x * blockDim.x) {
        const unsigned long long* w = x + j * words;
        unsigned long long* m = mag + j * words;
        const bool s = (long long)w[words - 1] < 0;
        unsigned long long carry = 1;
        for (int i = 0; i < words; ++i) {
            if (s) {
                const unsigned long long v = ~w[i] + carry;
                carry = (carry && v == 0) ? 1 : 0;
                m[i] = v;
            } else {
                m[i] = w[i];
            }
        }
        neg[j] = s ? 1 : 0;
    }
}

struct BigSplitArgs {
    const unsigned long long* mag;
    const unsigned char* neg;
    long long len;  // coefficients
    int words, K, M, nprimes;
    u32 p[kBigMaxPrimes];
    u32* out[kBigMaxPrimes];  // (2K - 1)(len - 1) + K words each
};

// out_p[j*(2K-1) + i] = sign_j * (bits [M i, M i + M) of |x_j|) mod p, i < K;
// 0 for K <= i < 2K-1 (the last block is cut at K words).
__global__ void k_big_split(const __grid_constant__ BigSplitArgs A) {
    const int blk = 2 * A.K - 1;
    const long long total = (long long)blk * (A.len - 1) + A.K;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long j = t / blk;
        const int i = (int)(t % blk);
        unsigned long long limb = 0;
        if (i < A.K) {
            const long long s = (long long)A.M * i;
            const int w = (int)(s >> 6), b = (int)(s & 63);
            const unsigned long long* m = A.mag + j * A.words;
            if (w < A.words) {
                limb = m[w] >> b;
                if (b && w + 1 < A.words) limb |= m[w + 1] << (64 - b);
                if (A.M < 64) limb &= (1ull << A.M) - 1;
            }
        }
        const bool ng = A.neg[j] != 0;
        for (int k = 0; k < A.nprimes; ++k) {
            const u32 p = A.p[k];
            u32 r = (u32)(limb % p);
            if (ng && r) r = p - r;
            A.out[k][t] = r;
        }
    }
}

struct BigCrtArgs {
    const u32* prod[kBigMaxPrimes];  // (2K - 1) lc words each
    long long lc;                    // output coefficients
    int K, M, nprimes, out_words;
    u32 p[kBigMaxPrimes];
    u32 inv[kBigMaxPrimes][kBigMaxPrimes];  // inv[a][b] = p_a^-1 mod p_b (a < b)
    unsigned long long* c;
};

// Adds v (unsigned 128-bit) shifted left by s bits into acc (n words).
__device__ __forceinline__ void acc_add(unsigned long long* acc, int n, unsigned __int128 v, long long s) {
    const int w = (int)(s >> 6), b = (int)(s & 63);
    unsigned long long part[3];
    part[0] = (unsigned long long)v << b;
    part[1] = b ? (unsigned long long)(v >> (64 - b)) : (unsigned long long)(v >> 64);
    part[2] = b ? (unsigned long long)((v >> 64) >> (64 - b)) : 0ull;
    unsigned long long carry = 0;
    int i = 0;
    for (; i < 3 && w + i < n; ++i) {
        const unsigned long long a = acc[w + i];
        const unsigned long long t = a + part[i];
        const unsigned long long c1 = t < a;
        const unsigned long long u = t + carry;
        carry = c1 + (u < t);
        acc[w + i] = u;
    }
    for (int k = w + i; carry && k < n; ++k) {
        acc[k] += 1;
        carry = acc[k] == 0;
    }
}

__global__ void k_big_crt(const __grid_constant__ BigCrtArgs A) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= A.lc) return;
    const int nacc = min(kBigMaxAccWords, (int)((2ll * A.M * A.K + 192 + 63) / 64));
    unsigned long long pos[kBigMaxAccWords], negv[kBigMaxAccWords];
    for (int i = 0; i < nacc; ++i) pos[i] = negv[i] = 0;
    // P and P / 2 as unsigned 128-bit
    unsigned __int128 P = 1;
    for (int k = 0; k < A.nprimes; ++k) P *= A.p[k];
    const unsigned __int128 half = P >> 1;
    for (int i = 0; i < 2 * A.K - 1; ++i) {
        const long long idx = j * (2ll * A.K - 1) + i;
        // Garner: mixed-radix digits v_k with x = v_0 + v_1 p_0 + v_2 p_0 p_1 + ...
        u32 v[kBigMaxPrimes];
        for (int k = 0; k < A.nprimes; ++k) {
            u64 t = A.prod[k][idx];
            for (int a = 0; a < k; ++a) {
                // t = (t - v_a) * p_a^-1 mod p_k
                const u32 pk = A.p[k];
                const u64 d = (t + pk - (v[a] % pk)) % pk;
                t = (d * A.inv[a][k]) % pk;
            }
            v[k] = (u32)t;
        }
        unsigned __int128 x = 0, radix = 1;
        for (int k = 0; k < A.nprimes; ++k) {
            x += (unsigned __int128)v[k] * radix;
            radix *= A.p[k];
        }
        const long long s = (long long)A.M * i;
        if (x > half) acc_add(negv, nacc, P - x, s);
        else if (x) acc_add(pos, nacc, x, s);
    }
    // c = pos - neg, truncated to out_words
    unsigned long long* out = A.c + j * A.out_words;
    unsigned long long borrow = 0;
    for (int k = 0; k < A.out_words; ++k) {
        const unsigned long long a = k < nacc ? pos[k] : 0ull, b = k < nacc ? negv[k] : 0ull;
        const unsigned long long d = a - b;
        const unsigned long long b1 = a < b;
        const unsigned long long e = d - borrow;
        borrow = b1 + (d < borrow);
        out[k] = e;
    }
}

int grid_of(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 32)); }

}  // namespace

// Scratch of one product (bigconv_mul_dev with caller buffers): the
// magnitudes, signs, split operands and products per prime, then the
// products' workspace and job tables (as direct_batch takes them).
struct BigSizes {
    size_t mag_bytes, sign_bytes, words, ws_words, job_bytes;
};

BigSizes big_sizes(const BigPlan& pl, long long na, long long nb, int in_words) {
    const long long la = (2ll * pl.K - 1) * (na - 1) + pl.K, lb = (2ll * pl.K - 1) * (nb - 1) + pl.K;
    BigSizes z;
    z.mag_bytes = ((size_t)(na + nb) * in_words * 8 + 255) & ~(size_t)255;
    z.sign_bytes = ((size_t)(na + nb) + 255) & ~(size_t)255;
    z.words = (size_t)pl.nprimes * (la + lb + la + lb - 1);
    const long long LA[1] = {la}, LB[1] = {lb};
    z.ws_words = (size_t)pl.nprimes * direct_ws_words(1, LA, LB);
    z.job_bytes = (size_t)pl.nprimes * ((direct_job_bytes(1) + 255) & ~(size_t)255);
    return z;
}

// c (lc = na + nb - 1 coefficients of out_words words) = a * b exactly;
// device pointers, coefficients of in_words two's-complement words, bw the
// largest magnitude bit width of any coefficient.  bufs == nullptr: library
// workspace, one product per prime on side streams; else the caller's
// buffers (sizes from big_sizes), everything on st.
int bigconv_mul_dev(const unsigned long long* a, long long na, const unsigned long long* b, long long nb,
                    int in_words, unsigned long long* c, int out_words, int bw, cudaStream_t st, BigPlan* used,
                    const TwoConvBufs* bufs = nullptr) {
    if (in_words <= 0 || in_words > kBigMaxInWords || out_words <= 0 || na <= 0 || nb <= 0)
        return ASSUMPTION_ERROR;
    if (bw < 0 || bw > 64 * in_words) return ASSUMPTION_ERROR;
    BigPlan pl;
    int err = big_plan(bw, na, nb, &pl);
    if (err != OK) return err;
    if (used) *used = pl;
    const long long lc = na + nb - 1;
    const long long la = (2ll * pl.K - 1) * (na - 1) + pl.K, lb = (2ll * pl.K - 1) * (nb - 1) + pl.K;
    const long long lp = la + lb - 1;
    const int r = pl.nprimes;
    // scratch: |a|, |b| (64-bit words), signs, split operands and products per prime
    const BigSizes z = big_sizes(pl, na, nb, in_words);
    const size_t mag_bytes = z.mag_bytes, sign_bytes = z.sign_bytes, words = z.words;
    const int dev = current_device();
    char* ws = bufs ? (char*)bufs->eval : (char*)workspace(dev, kWsBig, mag_bytes + sign_bytes + words * 4, &err);
    if (!ws) return err;
    unsigned long long* mag = (unsigned long long*)ws;
    unsigned char* sg = (unsigned char*)(ws + mag_bytes);
    u32* w32 = (u32*)(ws + mag_bytes + sign_bytes);
    k_big_abs<<<grid_of(na), 256, 0, st>>>(a, na, in_words, mag, sg);
    k_big_abs<<<grid_of(nb), 256, 0, st>>>(b, nb, in_words, mag + (size_t)na * in_words, sg + na);
    u32 *ap[kBigMaxPrimes], *bp[kBigMaxPrimes], *cp[kBigMaxPrimes];
    for (int k = 0; k < r; ++k) {
        ap[k] = w32 + (size_t)k * (la + lb + lp);
        bp[k] = ap[k] + la;
        cp[k] = bp[k] + lb;
    }
    BigSplitArgs S;
    memset(&S, 0, sizeof(S));
    S.words = in_words;
    S.K = pl.K;
    S.M = pl.M;
    S.nprimes = r;
    for (int k = 0; k < r; ++k) S.p[k] = pl.p[k];
    S.mag = mag;
    S.neg = sg;
    S.len = na;
    for (int k = 0; k < r; ++k) S.out[k] = ap[k];
    k_big_split<<<grid_of(la), 256, 0, st>>>(S);
    S.mag = mag + (size_t)na * in_words;
    S.neg = sg + na;
    S.len = nb;
    for (int k = 0; k < r; ++k) S.out[k] = bp[k];
    k_big_split<<<grid_of(lb), 256, 0, st>>>(S);
    if ((err = cuda_err(cudaGetLastError())) != OK) return err;
    // one product per prime, on side streams (each batch plan owns its
    // workspace), joined before the CRT
    if (!bufs) {
        const sfixn df = (sfixn)(la - 1), dg = (sfixn)(lb - 1);
        const int64_t zero = 0;
        aux_fork(dev, st, r);
        for (int k = 0; k < r && err == OK; ++k)
            err = batch_mul_dev(1, &df, &zero, ap[k], &dg, &zero, bp[k], &zero, cp[k], pl.p[k], aux_stream(dev, k));
        aux_join(dev, st, r);
        if (err != OK) return err;
    } else {
        const long long LA[1] = {la}, LB[1] = {lb}, LH[1] = {lp};
        const size_t wsw = z.ws_words / r, jb = z.job_bytes / r;
        for (int k = 0; k < r; ++k) {
            const u32* pa[1] = {ap[k]};
            const u32* pb[1] = {bp[k]};
            u32* ph[1] = {cp[k]};
            err = direct_batch(1, pa, LA, pb, LB, ph, LH, pl.p[k], bufs->ws + k * wsw, (char*)bufs->djobs + k * jb,
                               (char*)bufs->hjobs + k * jb, st, false);
            if (err != OK) return err;
        }
    }
    BigCrtArgs C;
    memset(&C, 0, sizeof(C));
    for (int k = 0; k < r; ++k) {
        C.prod[k] = cp[k];
        C.p[k] = pl.p[k];
    }
    for (int x = 0; x < r; ++x)
        for (int y = x + 1; y < r; ++y) C.inv[x][y] = powmod_exact(pl.p[x] % pl.p[y], pl.p[y] - 2, pl.p[y]);
    C.lc = lc;
    C.K = pl.K;
    C.M = pl.M;
    C.nprimes = r;
    C.out_words = out_words;
    C.c = c;
    k_big_crt<<<(unsigned)((lc + 127) / 128), 128, 0, st>>>(C);
    return cuda_err(cudaGetLastError());
}

int exact_i64_long_dev_bufs(const long long* a, long long la, const long long* b, long long lb, long long* c, int bw,
                            cudaStream_t st, const TwoConvBufs* bufs) {
    return bigconv_mul_dev((const unsigned long long*)a, la, (const unsigned long long*)b, lb, 1,
                           (unsigned long long*)c, 2, bw, st, nullptr, bufs);
}

void exact_i64_long_sizes(long long la, long long lb, int bw, size_t* eval_words, size_t* ws_words,
                          size_t* job_bytes) {
    BigPlan pl;
    if (big_plan(bw, la, lb, &pl) != OK) {
        *eval_words = *ws_words = *job_bytes = 0;
        return;
    }
    const BigSizes z = big_sizes(pl, la, lb, 1);
    *eval_words = (z.mag_bytes + z.sign_bytes) / 4 + z.words;
    *ws_words = z.ws_words;
    *job_bytes = z.job_bytes;
}

int exact_i64_long_cost(long long la, long long lb, int bw, double* cost) {
    BigPlan pl;
    const int err = big_plan(bw, la, lb, &pl);
    if (err != OK) return err;
    *cost = (double)pl.nprimes * std::ldexp(1.0, pl.logn) * pl.logn;
    return OK;
}

int exact_i64_long_dev(const long long* a, long long la, const long long* b, long long lb, long long* c, int bw,
                       cudaStream_t st) {
    return bigconv_mul_dev((const unsigned long long*)a, la, (const unsigned long long*)b, lb, 1,
                           (unsigned long long*)c, 2, bw, st, nullptr);
}

// ------------------------------------------------- batches of one-limb products ----
// With one limb (K = 1) the split is the residue of the whole coefficient and
// the CRT of every output coefficient stands alone (no shifted sum across
// x-coefficients), so the products of a batch that share their three primes
// run as three elementwise kernels around one batched product per prime.

bool exact_i64_long_one_limb(int bw, long long la, long long lb, u32* primes) {
    BigPlan pl;
    if (big_plan(bw, la, lb, &pl) != OK || pl.K != 1 || pl.nprimes != 3) return false;
    for (int k = 0; k < 3; ++k) primes[k] = pl.p[k];
    return true;
}

namespace {

struct Prime3 {
    u32 p[3];
};

// r_k[j] = x[j] mod p_k in [0, p_k), one word per thread and step.
__global__ void k_i64_residues(const long long* __restrict__ x, long long n, Prime3 P, u32* __restrict__ r0,
                               u32* __restrict__ r1, u32* __restrict__ r2) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const long long v = x[j];
        const unsigned long long m = v < 0 ? 0ull - (unsigned long long)v : (unsigned long long)v;
        u32 r[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const u32 t = (u32)(m % P.p[k]);
            r[k] = (v < 0 && t) ? P.p[k] - t : t;
        }
        r0[j] = r[0];
        r1[j] = r[1];
        r2[j] = r[2];
    }
}

struct Crt3Args {
    const u32* prod[3];  // canonical residues of each output coefficient
    long long n;
    u32 p[3];
    u32 inv01, inv02, inv12;  // p0^-1 mod p1, p0^-1 mod p2, p1^-1 mod p2
    long long* c;             // lo, hi words of each signed 128-bit result
};

// Garner's CRT of three residues to the x in [0, P), stored as the signed
// value x - P when x > P / 2 (128-bit two's complement); one coefficient per
// thread and step.  The big-coefficient CRT (k_big_crt) with one limb.
__global__ void k_crt3_i128(const __grid_constant__ Crt3Args A) {
    const unsigned __int128 P01 = (unsigned __int128)A.p[0] * A.p[1];
    const unsigned __int128 P = P01 * A.p[2];
    const unsigned __int128 half = P >> 1;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < A.n;
         j += (long long)gridDim.x * blockDim.x) {
        const u32 v0 = A.prod[0][j];
        const u32 r1 = A.prod[1][j], r2 = A.prod[2][j];
        const u32 v1 = (u32)((u64)((r1 + A.p[1] - v0 % A.p[1]) % A.p[1]) * A.inv01 % A.p[1]);
        const u64 t2 = (u64)((r2 + A.p[2] - v0 % A.p[2]) % A.p[2]) * A.inv02 % A.p[2];
        const u32 v2 = (u32)((t2 + A.p[2] - v1 % A.p[2]) % A.p[2] * A.inv12 % A.p[2]);
        unsigned __int128 x = (unsigned __int128)v0 + (unsigned __int128)v1 * A.p[0] + (unsigned __int128)v2 * P01;
        if (x > half) x -= P;  // wraps to the two's complement of x - P
        A.c[2 * j] = (long long)(unsigned long long)x;
        A.c[2 * j + 1] = (long long)(unsigned long long)(x >> 64);
    }
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

void exact_i64_batch_sizes(int cnt, const long long* la, const long long* lb, size_t* eval_words, size_t* ws_words,
                           size_t* job_bytes) {
    long long nin = 0, nout = 0;
    for (int i = 0; i < cnt; ++i) {
        nin += la[i] + lb[i];
        nout += la[i] + lb[i] - 1;
    }
    *eval_words = 3 * (size_t)(nin + nout);
    *ws_words = direct_ws_words(cnt, la, lb);
    *job_bytes = 3 * round256(direct_job_bytes(cnt));
}

int exact_i64_long_batch(int cnt, const long long* x, const long long* la, const long long* lb, long long* c,
                         const u32* primes, cudaStream_t st, const TwoConvBufs& B) {
    if (cnt <= 0) return OK;
    long long nin = 0, nout = 0;
    std::vector<long long> lh(cnt), ia(cnt), ih(cnt);
    for (int i = 0; i < cnt; ++i) {
        if (la[i] <= 0 || lb[i] <= 0) return ASSUMPTION_ERROR;
        ia[i] = nin;
        ih[i] = nout;
        lh[i] = la[i] + lb[i] - 1;
        nin += la[i] + lb[i];
        nout += lh[i];
    }
    u32* res[3];
    u32* prod[3];
    for (int k = 0; k < 3; ++k) {
        res[k] = B.eval + (size_t)k * nin;
        prod[k] = B.eval + 3 * (size_t)nin + (size_t)k * nout;
    }
    Prime3 P3;
    for (int k = 0; k < 3; ++k) P3.p[k] = primes[k];
    k_i64_residues<<<grid_of(nin), 256, 0, st>>>(x, nin, P3, res[0], res[1], res[2]);
    int err = cuda_err(cudaGetLastError());
    if (err != OK) return err;
    const size_t jb = round256(direct_job_bytes(cnt));
    std::vector<const u32*> pa(cnt), pb(cnt);
    std::vector<u32*> ph(cnt);
    for (int k = 0; k < 3; ++k) {
        for (int i = 0; i < cnt; ++i) {
            pa[i] = res[k] + ia[i];
            pb[i] = res[k] + ia[i] + la[i];
            ph[i] = prod[k] + ih[i];
        }
        // one workspace (stream-ordered reuse), a job table region per prime
        // (the host writes each before its copy to the device has run)
        err = direct_batch(cnt, pa.data(), la, pb.data(), lb, ph.data(), lh.data(), primes[k], B.ws,
                           (char*)B.djobs + k * jb, (char*)B.hjobs + k * jb, st, false);
        if (err != OK) return err;
    }
    Crt3Args C;
    for (int k = 0; k < 3; ++k) {
        C.prod[k] = prod[k];
        C.p[k] = primes[k];
    }
    C.n = nout;
    C.inv01 = powmod_exact(primes[0] % primes[1], primes[1] - 2, primes[1]);
    C.inv02 = powmod_exact(primes[0] % primes[2], primes[2] - 2, primes[2]);
    C.inv12 = powmod_exact(primes[1] % primes[2], primes[2] - 2, primes[2]);
    C.c = c;
    k_crt3_i128<<<grid_of(nout), 256, 0, st>>>(C);
    return cuda_err(cudaGetLastError());
}

}  // namespace cmb

using namespace cmb;

namespace {

int bw_words(const uint64_t* x, long long n, int words) {
    int bw = 0;
    for (long long j = 0; j < n; ++j) {
        const uint64_t* w = x + j * words;
        const bool neg = (int64_t)w[words - 1] < 0;
        // magnitude bit width: for negative x, |x| = ~x + 1
        unsigned long long carry = 1;
        int top = 0;
        for (int i = 0; i < words; ++i) {
            unsigned long long v = w[i];
            if (neg) {
                v = ~v + carry;
                carry = (carry && v == 0) ? 1 : 0;
            }
            if (v) top = i * 64 + 64 - __builtin_clzll(v);
        }
        bw = std::max(bw, top);
    }
    return bw;
}

}  // namespace

extern "C" {

int cumodp_twoconv_big_out_words(long long na, long long nb, int bit_width) {
    if (na <= 0 || nb <= 0 || bit_width < 0) return 0;
    return big_out_words(na, nb, bit_width);
}

int cumodp_twoconv_big_bit_width(long long na, const uint64_t* a, long long nb, const uint64_t* b, int in_words) {
    if (na < 0 || nb < 0 || in_words <= 0 || (na && !a) || (nb && !b)) return -1;
    return std::max(bw_words(a, na, in_words), bw_words(b, nb, in_words));
}

cumodp_err cumodp_twoconv_big_plan(int bit_width, long long na, long long nb, int* K, int* M, int* nprimes,
                                   int* log_transform) {
    BigPlan pl;
    const int e = big_plan(bit_width, na, nb, &pl);
    if (e != OK) return (cumodp_err)e;
    if (K) *K = pl.K;
    if (M) *M = pl.M;
    if (nprimes) *nprimes = pl.nprimes;
    if (log_transform) *log_transform = pl.logn;
    return CUMODP_SUCCESS;
}

cumodp_err cumodp_twoconv_mul_big_dev(long long na, const uint64_t* a, long long nb, const uint64_t* b, int in_words,
                                      uint64_t* c, int out_words, int bit_width, void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (!a || !b || !c) return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = bigconv_mul_dev((const unsigned long long*)a, na, (const unsigned long long*)b, nb, in_words,
                            (unsigned long long*)c, out_words, bit_width, st, nullptr);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

cumodp_err cumodp_twoconv_mul_big(long long na, const uint64_t* a, long long nb, const uint64_t* b, int in_words,
                                  uint64_t* c, int out_words) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (na <= 0 || nb <= 0 || !a || !b || !c || in_words <= 0 || in_words > kBigMaxInWords || out_words <= 0)
        return CUMODP_ASSUMPTION_ERROR;
    const int bw = std::max(bw_words(a, na, in_words), bw_words(b, nb, in_words));
    std::lock_guard<std::mutex> g(lib_mutex());
    const int dev = current_device();
    cudaStream_t st = lib_stream(dev);
    const long long lc = na + nb - 1;
    int err = OK;
    const size_t in_bytes = (size_t)(na + nb) * in_words * 8, out_bytes = (size_t)lc * out_words * 8;
    char* d = (char*)workspace(dev, kWsStage, in_bytes + out_bytes, &err);
    if (!d) return (cumodp_err)err;
    unsigned long long* da = (unsigned long long*)d;
    unsigned long long* db = da + (size_t)na * in_words;
    unsigned long long* dc = (unsigned long long*)(d + in_bytes);
    cudaError_t ce = cudaMemcpyAsync(da, a, (size_t)na * in_words * 8, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(db, b, (size_t)nb * in_words * 8, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return (cumodp_err)cuda_err(ce);
    err = bigconv_mul_dev(da, na, db, nb, in_words, dc, out_words, bw, st, nullptr);
    if (err != OK) {
        cudaStreamSynchronize(st);
        return (cumodp_err)err;
    }
    ce = cudaMemcpyAsync(c, dc, out_bytes, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    return (cumodp_err)cuda_err(ce);
}

}  // extern "C"
