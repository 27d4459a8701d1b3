/*
 * list_stockham_b200.h -- C++ signatures of the reference's list transform
 * and bivariate product, forwarding to cumodp_list_fft_dev and
 * cumodp_bivariate_mul_dev.
 *
 * Replaces list_stockham_dev (include/list_stockham.h:48-49,
 * src/list_stockham.cu:595-665): X = I_m (x) DFT_n(X) for a device array of m
 * rows of n = 2^k words, natural order.  The W overload takes the reference's
 * device table of powers W[i] = w^i and reads W[1] for the root.  Errors are
 * returned (the reference returns void and ignores them).
 */
#ifndef LIST_STOCKHAM_B200_H
#define LIST_STOCKHAM_B200_H

#include "cumodp.h"

#ifdef __cplusplus
#include <cuda_runtime.h>

inline cumodp_err list_stockham_dev(sfixn *X, sfixn m, sfixn k, sfixn w, sfixn p) {
    return cumodp_list_fft_dev(X, m, k, w, p, 0, 0);
}

inline cumodp_err list_stockham_dev(sfixn *X, sfixn m, sfixn k, const sfixn *W, sfixn p) {
    /* W[i] = w^i for i < n/2: W[1] is the root for k >= 2; for k = 1 the
     * table holds only w^0 and the root is p - 1 */
    sfixn w = k == 1 ? p - 1 : 1;
    if (k >= 2 && cudaMemcpy(&w, W + 1, sizeof(sfixn), cudaMemcpyDeviceToHost) != cudaSuccess)
        return CUMODP_FFT_ERROR;
    return cumodp_list_fft_dev(X, m, k, w, p, 0, 0);
}
// Replaces bi_stockham_poly_mul_dev (include/list_stockham.h:103-104,
// src/list_stockham.cu:1317-1348): F <- DFT^-1(DFT F * DFT G) on an m x n
// grid (m = 2^em rows in y, n = 2^en columns in x); G is overwritten.
inline cumodp_err bi_stockham_poly_mul_dev(sfixn m, sfixn em, sfixn n, sfixn en, sfixn *F, sfixn *G, sfixn p) {
    if (m != ((sfixn)1 << em) || n != ((sfixn)1 << en)) return CUMODP_ASSUMPTION_ERROR;
    return cumodp_bivariate_mul_dev(em, en, F, G, p, 0);
}
#endif

#endif
