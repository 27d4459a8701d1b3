// Exact integer product of int64-coefficient polynomials by the
// two-convolution method over Fourier primes.
//
// Reference: two_convolution_poly_mul (src/two_convolution_poly_mul.cu:
// 532-569).  Each coefficient is cut into K limbs of M bits
// (convert_to_modular_bivariate, :84-203: sign-magnitude, a negative
// coefficient stores p - limb), so a(y) becomes a bivariate a(x, y) with
// a(2^M, y) = a(y).  The product is recovered from the cyclic convolution
// u = a*b mod (x^K - 1) and the negacyclic one v = a*b mod (x^K + 1)
// (the x-argument scaled by theta, :207-245), reduced mod several primes,
// lifted by CRT to signed integers (reconstruct_mpz_with_crt, :292-385) and
// recombined as (u+v)(2^M)/2 + 2^N (u-v)(2^M)/2 (recover_product_host,
// :387-428).
//
// B200 layout of the same computation:
//   1. k_split_eval: one pass over the int64 inputs; per prime it writes the
//      2K evaluations A_s(y) = sum_j limb_j(y) zeta^(js), zeta a primitive
//      2K-th root (even s: the cyclic points, odd s: theta-scaled negacyclic
//      points), so the x-convolutions become 2K independent y-products;
//   2. the y-products: one batched call per prime (fused single-CTA or
//      three-pass kernels, graph-launched);
//   3. k_crt_recombine: per output coefficient, the inverse 2K-point
//      x-transform, u and v, (u+v) and (u-v) mod each prime, the signed CRT
//      lift, evaluation at 2^M and the final shift, stored as a signed
//      128-bit integer (lo, hi words).
// K = 1 is the degenerate case with no limb split (u = v = the product).
// The planner picks the cheapest (K, M, primes) whose exactness bound holds.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/cumodp.h"
#include "exact.cuh"

namespace cmb {

int batch_mul_dev(int count, const sfixn* df, const int64_t* f_off, const u32* F, const sfixn* dg,
                  const int64_t* g_off, const u32* G, const int64_t* h_off, u32* H, u32 p, cudaStream_t st);

// The three primes of the reference (two_convolution_poly_mul.h:51-53).
static const u32 kTwoConvPrimes[3] = {962592769u, 950009857u, 940572673u};


struct SplitArgs {
    const long long* x;
    int len;
    int K, M;
    int npts;            // evaluation points: 2K, or 1 when K = 1
    int nprimes;
    u32 p[3];
    u32 zeta_pow[3][8];  // zeta^t, t < 2K (K <= 4)
    u32* out;            // [prime][s][len]
};

__global__ void k_split_eval(const __grid_constant__ SplitArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.len) return;
    const long long v = A.x[i];
    const bool neg = v < 0;
    const unsigned long long m = neg ? 0ull - (unsigned long long)v : (unsigned long long)v;
    const int twoK = 2 * A.K, npts = A.npts;
    const unsigned long long mask = A.M >= 64 ? ~0ull : ((1ull << A.M) - 1);
    for (int r = 0; r < A.nprimes; ++r) {
        const u32 p = A.p[r];
        u32 limb[4];
        for (int j = 0; j < A.K; ++j) {
            const unsigned long long l = (A.M * j >= 64) ? 0ull : ((m >> (A.M * j)) & mask);
            const u32 lr = (u32)(l % p);
            limb[j] = (neg && lr) ? p - lr : lr;
        }
        for (int s = 0; s < npts; ++s) {
            u64 acc = 0;
            for (int j = 0; j < A.K; ++j) acc += (u64)limb[j] * A.zeta_pow[r][(j * s) % twoK] % p;
            A.out[((size_t)r * npts + s) * A.len + i] = (u32)(acc % p);
        }
    }
}

struct CrtArgs {
    const u32* c;   // [prime][s][lc]
    int lc;
    int K, M, nprimes;
    int npts;
    u32 p[3];
    u32 zinv_pow[3][8];  // zeta^-t
    u32 inv2k[3];        // (2K)^-1 mod p
    u32 garner1;         // p0^-1 mod p1
    u32 garner2;         // (p0 p1)^-1 mod p2
    long long* out;      // (lo, hi) per coefficient
};

__device__ __forceinline__ __int128 crt_signed(const u32* r, const CrtArgs& A) {
    // Garner: x = v0 + v1 p0 + v2 p0 p1, then the symmetric lift
    const u64 p0 = A.p[0], p1 = A.p[1];
    const u64 v0 = r[0];
    if (A.nprimes == 1) {
        const long long x = (long long)v0;
        return (__int128)(2 * v0 > p0 ? x - (long long)p0 : x);
    }
    const u64 v1 = ((r[1] + p1 - v0 % p1) % p1) * A.garner1 % p1;
    unsigned __int128 x = (unsigned __int128)v0 + (unsigned __int128)v1 * p0;
    unsigned __int128 P = (unsigned __int128)p0 * p1;
    if (A.nprimes == 3) {
        const u64 p2 = A.p[2];
        const u64 t = (u64)(x % p2);
        const u64 v2 = ((r[2] + p2 - t) % p2) * A.garner2 % p2;
        x += (unsigned __int128)v2 * (unsigned __int128)(p0 * p1);
        P *= p2;
    }
    return (__int128)(x > P / 2 ? (__int128)x - (__int128)P : (__int128)x);
}

__global__ void k_crt_recombine(const __grid_constant__ CrtArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.lc) return;
    const int K = A.K, twoK = 2 * K, npts = A.npts;
    u32 S[3][4], D[3][4];
    for (int r = 0; r < A.nprimes; ++r) {
        const u32 p = A.p[r];
        u32 cs[8], c[8];
        for (int s = 0; s < npts; ++s) cs[s] = A.c[((size_t)r * npts + s) * A.lc + i];
        if (K == 1) {  // no limb split: the single product is c_0, and c_1 = 0
            c[0] = cs[0];
            c[1] = 0;
        } else {
            // inverse 2K-point x-transform: c_j = (2K)^-1 sum_s cs_s zeta^-js
            // (the acyclic x-product, degree 2K-2)
            for (int j = 0; j < twoK; ++j) {
                u64 acc = 0;
                for (int s = 0; s < twoK; ++s) acc += (u64)cs[s] * A.zinv_pow[r][(j * s) % twoK] % p;
                c[j] = (u32)((acc % p) * A.inv2k[r] % p);
            }
        }
        for (int j = 0; j < K; ++j) {
            // cyclic u_j = c_j + c_{j+K}, negacyclic v_j = c_j - c_{j+K};
            // (u+v) and (u-v) mod p as modular_sum_and_difference_dev does
            const u32 u = (u32)(((u64)c[j] + c[j + K]) % p);
            const u32 v = (u32)(((u64)c[j] + p - c[j + K]) % p);
            S[r][j] = (u32)(((u64)u + v) % p);
            D[r][j] = (u32)(((u64)u + p - v) % p);
        }
    }
    // (u+v)(2^M)/2 + 2^N (u-v)(2^M)/2 with N = K M: the 2K-1 lifted values
    // e_j = (u+v)_j (j < K) and (u-v)_(j-K) (j >= K) are the doubled limb
    // coefficients of the product, summed by Horner's rule from the top so
    // that no partial sum exceeds twice the final magnitude
    __int128 acc = 0;
    for (int j = 2 * K - 2; j >= 0; --j) {
        u32 rr[3];
        for (int r = 0; r < A.nprimes; ++r) rr[r] = j < K ? S[r][j] : D[r][j - K];
        acc = acc * ((__int128)1 << A.M) + crt_signed(rr, A);
    }
    const __int128 prod = acc / 2;  // exact: acc is even
    A.out[2 * (size_t)i] = (long long)(unsigned long long)(unsigned __int128)prod;
    A.out[2 * (size_t)i + 1] = (long long)(prod >> 64);
}

namespace {

// log2 of prod of the first k primes (floor)
double log2_prime_product(int k) {
    double s = 0;
    for (int i = 0; i < k; ++i) s += __builtin_log2((double)kTwoConvPrimes[i]);
    return s;
}

}  // namespace

// Chooses (K, M, primes) for coefficient bit widths ba, bb and lengths la, lb.
// Exactness: every CRT-lifted value (u+v or u-v, at most 2 * K * min(la, lb)
// * 2^(2M) in magnitude) must lie strictly inside half the prime product, and
// the product coefficients must fit in 127 bits.  `force_two_prime`
// requests the smallest limb split that needs only two primes.
int twoconv_plan(int ba, int bb, long long la, long long lb, bool force_two_prime, TwoConvPlan* out) {
    const long long mn = std::min(la, lb);
    const double lmin = __builtin_log2((double)mn);
    if (ba + bb + lmin + 1 > 127) return ASSUMPTION_ERROR;  // result would not fit in int128
    const int logn = product_logn(la, lb);
    const int bmax = std::max(ba, bb);
    TwoConvPlan best{0, 0, 0, 0};
    double best_cost = 1e300;
    for (int K : {1, 2, 4}) {
        const int M = (bmax + K - 1) / K;
        if (M > 62) continue;
        // magnitude bound of (u + v) = 2 c_j: 2 * K * min * 2^(2M)
        const double bound = 1.0 + __builtin_log2((double)K) + lmin + 2.0 * M;
        for (int np = 1; np <= 3; ++np) {
            if (bound + 1.0 >= log2_prime_product(np)) continue;  // need |x| < P/2
            if (logn > 20 && np == 3) continue;                    // 940572673 supports 2^20
            if (logn > 21) continue;
            if (force_two_prime && np != 2) continue;
            if (force_two_prime && K == 1) continue;
            const double cost = (double)np * (K == 1 ? 1 : 2 * K);
            if (cost < best_cost) {
                best_cost = cost;
                best = TwoConvPlan{K, M, np, logn};
            }
            break;  // more primes only cost more for this K
        }
    }
    if (!best.K) return FFT_SIZE_TOO_LARGE;
    *out = best;
    return OK;
}

void twoconv_buffer_sizes_plan(long long la, long long lb, const TwoConvPlan& pl, size_t* eval_words,
                               size_t* ws_words, size_t* job_bytes) {
    const int np = pl.nprimes, npts = pl.K == 1 ? 1 : 2 * pl.K;
    const long long lc = la + lb - 1;
    *eval_words = (size_t)np * npts * (la + lb + lc);
    std::vector<long long> A(npts, la), B(npts, lb);
    *ws_words = (size_t)np * direct_ws_words(npts, A.data(), B.data());
    *job_bytes = (size_t)np * direct_job_bytes(npts);
}

void twoconv_buffer_sizes(long long la, long long lb, size_t* eval_words, size_t* ws_words, size_t* job_bytes) {
    // worst case over plans: 3 primes x 8 points
    const int np = 3, npts = 8;
    const long long lc = la + lb - 1;
    *eval_words = (size_t)np * npts * (la + lb + lc);
    std::vector<long long> A(npts, la), B(npts, lb);
    *ws_words = (size_t)np * direct_ws_words(npts, A.data(), B.data());
    *job_bytes = (size_t)np * direct_job_bytes(npts);
}

// c (lo, hi pairs, la+lb-1 coefficients) = a * b exactly; device pointers.
// bufs == nullptr: library workspace and graph-launched batches.
int twoconv_mul_dev(const long long* a, long long la, const long long* b, long long lb, long long* c, int ba,
                    int bb, bool force_two_prime, cudaStream_t st, TwoConvPlan* used,
                    const TwoConvBufs* bufs) {
    if (la <= 0 || lb <= 0) return ASSUMPTION_ERROR;
    TwoConvPlan pl;
    int err = twoconv_plan(ba, bb, la, lb, force_two_prime, &pl);
    if (err != OK) return err;
    if (used) *used = pl;
    const int twoK = 2 * pl.K, np = pl.nprimes;
    const int npts = pl.K == 1 ? 1 : twoK;
    const long long lc = la + lb - 1;
    const int dev = current_device();
    // workspace: evaluations of a and b, and the products, per prime and point
    const size_t words = (size_t)np * npts * (la + lb + lc);
    u32* ws = bufs ? bufs->eval : (u32*)workspace(dev, kWsTwoConv, words * sizeof(u32), &err);
    if (!ws) return err;
    u32* ea = ws;
    u32* eb = ea + (size_t)np * npts * la;
    u32* ec = eb + (size_t)np * npts * lb;
    SplitArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.K = pl.K;
    sa.M = pl.M;
    sa.npts = npts;
    sa.nprimes = np;
    CrtArgs ca;
    memset(&ca, 0, sizeof(ca));
    ca.K = pl.K;
    ca.M = pl.M;
    ca.npts = npts;
    ca.nprimes = np;
    for (int r = 0; r < np; ++r) {
        const u32 p = kTwoConvPrimes[r];
        const PrimeCtx* pc = prime_ctx(p, &err);
        if (!pc) return err;
        const u32 zeta = canonical_root(*pc, twoK == 2 ? 1 : (twoK == 4 ? 2 : 3));
        const u32 zinv = powmod_exact(zeta, twoK - 1, p);
        sa.p[r] = ca.p[r] = p;
        for (int t = 0; t < twoK; ++t) {
            sa.zeta_pow[r][t] = powmod_exact(zeta, t, p);
            ca.zinv_pow[r][t] = powmod_exact(zinv, t, p);
        }
        ca.inv2k[r] = powmod_exact(twoK, p - 2, p);
    }
    ca.garner1 = powmod_exact(kTwoConvPrimes[0] % kTwoConvPrimes[1], kTwoConvPrimes[1] - 2, kTwoConvPrimes[1]);
    ca.garner2 = powmod_exact(
        (u32)((u64)kTwoConvPrimes[0] * kTwoConvPrimes[1] % kTwoConvPrimes[2]), kTwoConvPrimes[2] - 2,
        kTwoConvPrimes[2]);
    sa.x = a;
    sa.len = (int)la;
    sa.out = ea;
    k_split_eval<<<(unsigned)((la + 255) / 256), 256, 0, st>>>(sa);
    sa.x = b;
    sa.len = (int)lb;
    sa.out = eb;
    k_split_eval<<<(unsigned)((lb + 255) / 256), 256, 0, st>>>(sa);
    // y-products: one per evaluation point and prime
    std::vector<sfixn> df(npts, (sfixn)(la - 1)), dg(npts, (sfixn)(lb - 1));
    std::vector<int64_t> fo(npts), go(npts), ho(npts);
    for (int s = 0; s < npts; ++s) {
        fo[s] = (int64_t)s * la;
        go[s] = (int64_t)s * lb;
        ho[s] = (int64_t)s * lc;
    }
    if (!bufs) {
        // the primes are independent: one side stream each (each batch plan
        // owns its workspace), joined before the CRT
        aux_fork(dev, st, np);
        for (int r = 0; r < np; ++r) {
            err = batch_mul_dev(npts, df.data(), fo.data(), ea + (size_t)r * npts * la, dg.data(), go.data(),
                                eb + (size_t)r * npts * lb, ho.data(), ec + (size_t)r * npts * lc,
                                kTwoConvPrimes[r], aux_stream(dev, r));
            if (err != OK) {
                aux_join(dev, st, np);
                return err;
            }
        }
        aux_join(dev, st, np);
    } else {
        std::vector<long long> LA(npts, la), LB(npts, lb), LH(npts, lc);
        const size_t wsw = direct_ws_words(npts, LA.data(), LB.data());
        const size_t jb = direct_job_bytes(npts);
        for (int r = 0; r < np; ++r) {
            std::vector<const u32*> pa(npts), pb(npts);
            std::vector<u32*> ph(npts);
            for (int s2 = 0; s2 < npts; ++s2) {
                pa[s2] = ea + ((size_t)r * npts + s2) * la;
                pb[s2] = eb + ((size_t)r * npts + s2) * lb;
                ph[s2] = ec + ((size_t)r * npts + s2) * lc;
            }
            err = direct_batch(npts, pa.data(), LA.data(), pb.data(), LB.data(), ph.data(), LH.data(),
                               kTwoConvPrimes[r], bufs->ws + r * wsw, (char*)bufs->djobs + r * jb,
                               (char*)bufs->hjobs + r * jb, st, false);
            if (err != OK) return err;
        }
    }
    ca.c = ec;
    ca.lc = (int)lc;
    ca.out = c;
    k_crt_recombine<<<(unsigned)((lc + 127) / 128), 128, 0, st>>>(ca);
    return cuda_err(cudaGetLastError());
}

}  // namespace cmb

using namespace cmb;

namespace {

int bw_host(const int64_t* x, long long n) {
    unsigned long long m = 0;
    for (long long i = 0; i < n; ++i) {
        const unsigned long long v = x[i] < 0 ? 0ull - (unsigned long long)x[i] : (unsigned long long)x[i];
        m |= v;
    }
    return m ? 64 - __builtin_clzll(m) : 1;
}

}  // namespace

namespace cmb {

// Transforms past 2^21 points, which the reference's primes do not have, and
// 2^21-point products, where those primes need a limb split into 2 x 4
// transforms and primes of higher order 3, take the big-coefficient path
// (results are the same integers either way); ties keep the reference's
// primes.
bool exact_i64_prefers_long(int ba, int bb, long long la, long long lb) {
    TwoConvPlan pl;
    const int pe = twoconv_plan(ba, bb, la, lb, false, &pl);
    double big = 0;
    if (exact_i64_long_cost(la, lb, std::max(ba, bb), &big) != OK) return false;
    if (pe == FFT_SIZE_TOO_LARGE) return true;
    if (pe != OK) return false;
    const double tc = (double)pl.nprimes * (pl.K == 1 ? 1 : 2 * pl.K) * std::ldexp(1.0, pl.logn) * pl.logn;
    return big < tc;
}

namespace {

// The two-convolution product (the reference's primes, 962592769,
// 950009857, 940572673) where its plan exists and is the cheaper one; else
// the big-coefficient path over primes of higher 2-adic order (see
// exact_i64_prefers_long).  method 1 (the forced two-prime split of the
// reference's scheme) always takes the first.
int exact_i64_any_len(const int64_t* a, long long na, const int64_t* b, long long nb, int64_t* c, int ba, int bb,
                      int method, cudaStream_t st) {
    if (method != 1 && exact_i64_prefers_long(ba, bb, na, nb))
        return exact_i64_long_dev((const long long*)a, na, (const long long*)b, nb, (long long*)c, std::max(ba, bb),
                                  st);
    TwoConvPlan pl;
    const int pe = twoconv_plan(ba, bb, na, nb, method == 1, &pl);
    if (pe != OK) return pe;
    return twoconv_mul_dev((const long long*)a, na, (const long long*)b, nb, (long long*)c, ba, bb, method == 1, st,
                           nullptr, nullptr);
}

}  // namespace
}  // namespace cmb

extern "C" {

int cumodp_twoconv_bit_width(long long na, const int64_t* a, long long nb, const int64_t* b) {
    if (na < 0 || nb < 0 || (na && !a) || (nb && !b)) return -1;
    return std::max(bw_host(a, na), bw_host(b, nb));
}

cumodp_err cumodp_twoconv_plan(int bit_width_a, int bit_width_b, long long na, long long nb, int method, int* K,
                               int* M, int* nprimes) {
    TwoConvPlan pl;
    if (na <= 0 || nb <= 0 || bit_width_a <= 0 || bit_width_b <= 0) return CUMODP_ASSUMPTION_ERROR;
    const int e = twoconv_plan(bit_width_a, bit_width_b, na, nb, method == 1, &pl);
    if (e != OK) return (cumodp_err)e;
    if (K) *K = pl.K;
    if (M) *M = pl.M;
    if (nprimes) *nprimes = pl.nprimes;
    return CUMODP_SUCCESS;
}

cumodp_err cumodp_twoconv_mul_i64_dev(long long na, const int64_t* a, long long nb, const int64_t* b, int64_t* c,
                                      int bit_width, int method, void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (na <= 0 || nb <= 0 || !a || !b || !c || bit_width <= 0 || bit_width > 63 || na + nb - 1 > (1ll << 25))
        return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = exact_i64_any_len(a, na, b, nb, c, bit_width, bit_width, method, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

cumodp_err cumodp_twoconv_mul_i64(long long na, const int64_t* a, long long nb, const int64_t* b, int64_t* c,
                                  int method) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (na <= 0 || nb <= 0 || !a || !b || !c || na + nb - 1 > (1ll << 25)) return CUMODP_ASSUMPTION_ERROR;
    const int ba = bw_host(a, na), bb = bw_host(b, nb);
    std::lock_guard<std::mutex> g(lib_mutex());
    const int dev = current_device();
    cudaStream_t st = lib_stream(dev);
    const long long lc = na + nb - 1;
    const size_t in_bytes = (size_t)(na + nb) * 8, out_bytes = (size_t)lc * 16;
    int err = OK;
    long long* d = (long long*)workspace(dev, kWsStage, in_bytes + out_bytes, &err);
    if (!d) return (cumodp_err)err;
    // the operands and the result pass through pinned staging: one copy each way
    char* hs = (char*)pinned_workspace(kPinTwoConv, std::max(in_bytes, out_bytes), &err);
    if (!hs) return (cumodp_err)err;
    memcpy(hs, a, (size_t)na * 8);
    memcpy(hs + (size_t)na * 8, b, (size_t)nb * 8);
    long long *da = d, *db = d + na, *dc = d + na + nb;
    cudaError_t ce = cudaMemcpyAsync(da, hs, in_bytes, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return (cumodp_err)cuda_err(ce);
    err = exact_i64_any_len((const int64_t*)da, na, (const int64_t*)db, nb, (int64_t*)dc, ba, bb, method, st);
    if (err == OK) {
        ce = cudaMemcpyAsync(hs, dc, out_bytes, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        err = cuda_err(ce);
    } else {
        cudaStreamSynchronize(st);
    }
    if (err == OK) memcpy(c, hs, out_bytes);
    return (cumodp_err)err;
}

}  // extern "C"
