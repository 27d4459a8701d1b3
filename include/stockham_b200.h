/*
 * stockham_b200.h -- the C++ boundary of the reference's univariate
 * transforms and product (include/stockham.h:39-94, src/stockham.cu:413-611),
 * as inline forwarders to the C entry points of cumodp.h.
 *
 * Kept for the reference's internal callers (subresultants, scube and the
 * other C++ code that calls stockham_dev / stockham_poly_mul_dev directly).
 * Same arguments and meaning as the reference; the reference returns void,
 * these return the library's error code (callers that ignore it compile
 * unchanged).  X, F, G of the _dev functions are DEVICE pointers (16-byte
 * aligned when k >= 6, as cudaMalloc returns), the _host functions take HOST
 * arrays; everything is synchronous on the library's stream.
 *
 *   stockham_dev(X, n, k, w, p)          X <- DFT_n(X) with root w
 *                                        (src/stockham.cu:413-434)
 *   stockham_dev(X, n, k, W, p)          the same with the device table of
 *                                        powers W[i] = w^i (i < n/2); W[1] is
 *                                        the root (p - 1 for k = 1)
 *                                        (src/stockham.cu:437-453)
 *   inverse_stockham_dev(X, n, k, w, p)  X <- n^-1 DFT_n(X) with root w^-1
 *                                        (src/stockham.cu:462-467)
 *   inverse_stockham_dev(X, n, k, W, p)  the same with W holding the powers of
 *                                        the INVERSE root (src/stockham.cu:472-477)
 *   stockham_host / inverse_stockham_host   host-array versions
 *                                        (src/stockham.cu:479-503)
 *   stockham_poly_mul_dev(n, e, F, G, p) F <- DFT^-1(DFT F * DFT G), the cyclic
 *                                        convolution of length n = 2^e
 *                                        (src/stockham.cu:521-542); G is left
 *                                        unchanged
 *   stockham_poly_mul_host(dh, H, df, F, dg, G, p)   cumodp_fftmul_uni
 *                                        (src/stockham.cu:562-611)
 */
#ifndef STOCKHAM_B200_H
#define STOCKHAM_B200_H

#include "cumodp.h"

#ifdef __cplusplus
#include <cuda_runtime.h>

namespace cumodp_detail {
/* a^-1 mod p for 0 < a < p < 2^31 (Fermat). */
inline sfixn inv_mod_p(sfixn a, sfixn p) {
    unsigned long long r = 1, b = (unsigned long long)a % (unsigned long long)p;
    for (unsigned long long e = (unsigned long long)p - 2; e; e >>= 1) {
        if (e & 1) r = r * b % (unsigned long long)p;
        b = b * b % (unsigned long long)p;
    }
    return (sfixn)r;
}
/* The root of a device table of powers W[i] = w^i, i < n/2: W[1] for
 * k >= 2; for k = 1 the table holds only w^0 and the root is p - 1 (the only
 * primitive square root of unity); 1 for k = 0. */
inline cumodp_err root_from_table(const sfixn *W, sfixn k, sfixn p, sfixn *w) {
    *w = k == 1 ? p - 1 : 1;
    if (k >= 2 && cudaMemcpy(w, W + 1, sizeof(sfixn), cudaMemcpyDeviceToHost) != cudaSuccess)
        return CUMODP_FFT_ERROR;
    return CUMODP_SUCCESS;
}
inline bool length_ok(sfixn n, sfixn k) { return k >= 0 && k < 31 && n == ((sfixn)1 << k); }
}  // namespace cumodp_detail

inline cumodp_err stockham_dev(sfixn *X, sfixn n, sfixn k, sfixn w, sfixn p) {
    if (!cumodp_detail::length_ok(n, k)) return CUMODP_ASSUMPTION_ERROR;
    return cumodp_fft_uni_dev(X, n, k, w, p, 0, 0);
}

inline cumodp_err stockham_dev(sfixn *X, sfixn n, sfixn k, const sfixn *W, sfixn p) {
    if (!cumodp_detail::length_ok(n, k)) return CUMODP_ASSUMPTION_ERROR;
    sfixn w = 1;
    cumodp_err e = cumodp_detail::root_from_table(W, k, p, &w);
    return e != CUMODP_SUCCESS ? e : cumodp_fft_uni_dev(X, n, k, w, p, 0, 0);
}

inline cumodp_err inverse_stockham_dev(sfixn *X, sfixn n, sfixn k, sfixn w, sfixn p) {
    if (!cumodp_detail::length_ok(n, k)) return CUMODP_ASSUMPTION_ERROR;
    return cumodp_fft_uni_dev(X, n, k, w, p, 1, 0);
}

inline cumodp_err inverse_stockham_dev(sfixn *X, sfixn n, sfixn k, const sfixn *W, sfixn p) {
    if (!cumodp_detail::length_ok(n, k)) return CUMODP_ASSUMPTION_ERROR;
    sfixn wi = 1;
    cumodp_err e = cumodp_detail::root_from_table(W, k, p, &wi);
    if (e != CUMODP_SUCCESS) return e;
    if (wi <= 0 || wi >= p) return CUMODP_ASSUMPTION_ERROR;
    return cumodp_fft_uni_dev(X, n, k, cumodp_detail::inv_mod_p(wi, p), p, 1, 0);
}

inline cumodp_err stockham_host(sfixn *X, sfixn n, sfixn k, sfixn w, sfixn p) {
    return cumodp_fft_uni(X, n, k, w, p);
}

inline cumodp_err inverse_stockham_host(sfixn *X, sfixn n, sfixn k, sfixn w, sfixn p) {
    return cumodp_invfft_uni(X, n, k, w, p);
}

inline cumodp_err stockham_poly_mul_dev(sfixn n, sfixn e, sfixn *F, sfixn *G, sfixn p) {
    if (!cumodp_detail::length_ok(n, e)) return CUMODP_ASSUMPTION_ERROR;
    return cumodp_cyclic_mul_dev(e, F, G, p, 0);
}

inline cumodp_err stockham_poly_mul_host(sfixn dh, sfixn *H, sfixn df, const sfixn *F, sfixn dg, const sfixn *G,
                                         sfixn p) {
    return cumodp_fftmul_uni(dh, H, df, F, dg, G, p);
}
#endif

#endif
