/*
 * list_stockham_b200.h -- C++ signatures of the reference's list transform,
 * forwarding to cumodp_list_fft_dev.
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
    sfixn w = 1;
    if (k > 0 && cudaMemcpy(&w, W + 1, sizeof(sfixn), cudaMemcpyDeviceToHost) != cudaSuccess)
        return CUMODP_FFT_ERROR;
    return cumodp_list_fft_dev(X, m, k, w, p, 0, 0);
}
#endif

#endif
