/*
 * Driver for the reference's own GPU product path, compiled from the
 * reference sources as they lie (src/stockham.cu, src/fft_aux.cu; see
 * oracle/Makefile target ref_gpu).  It exposes C entry points that call the
 * reference's stockham_poly_mul_host (src/stockham.cu:562-611) -- the body of
 * cumodp_fftmul_uni (src/modpn.cu:249-261) -- so bench.py can time the
 * reference as shipped (radix-2 Stockham, one launch and one device sync per
 * step, per-call allocation) on the same GPU.
 *
 * Test/benchmark infrastructure only.
 */
#include <cstdio>
#include <cuda_runtime.h>
#include "stockham.h"

extern "C" int ref_gpu_fftmul(int dh, int *H, int df, const int *F, int dg, const int *G, int p)
{
    stockham_poly_mul_host(dh, H, df, F, dg, G, p);
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : (int)e;
}

// The reference's host-to-host transforms: stockham_host / inverse_stockham_host
// (src/stockham.cu:479-503), the bodies of cumodp_fft_uni / cumodp_invfft_uni.
extern "C" int ref_gpu_fft_host(int *X, int n, int k, int w, int p, int inverse)
{
    if (inverse) inverse_stockham_host(X, n, k, w, p);
    else stockham_host(X, n, k, w, p);
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : (int)e;
}

// Device-resident timing of the reference's stockham_dev (root overload,
// src/stockham.cu:413-434) on X_d (n = 2^k words, in place): reps calls
// bracketed by CUDA events on the default stream, which the reference uses;
// *ms receives the mean per call.
extern "C" int ref_gpu_time_fft_dev(int *X_d, int n, int k, int w, int p, int reps, float *ms)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    stockham_dev(X_d, n, k, w, p);  // warm-up
    cudaEventRecord(e0, 0);
    for (int i = 0; i < reps; ++i) stockham_dev(X_d, n, k, w, p);
    cudaEventRecord(e1, 0);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return e == cudaSuccess ? 0 : (int)e;
}

// Device-resident timing of the reference's stockham_poly_mul_dev
// (src/stockham.cu:521-542): F <- DFT^-1(DFT F * DFT G) on F_d, G_d of n = 2^e
// words, reps calls bracketed by CUDA events on the default stream.  F and G
// are overwritten (by the product and by DFT(G)); the work per call does not
// depend on the values.
extern "C" int ref_gpu_time_polymul_dev(int *F_d, int *G_d, int n, int e, int p, int reps, float *ms)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    stockham_poly_mul_dev(n, e, F_d, G_d, p);  // warm-up
    cudaEventRecord(e0, 0);
    for (int i = 0; i < reps; ++i) stockham_poly_mul_dev(n, e, F_d, G_d, p);
    cudaEventRecord(e1, 0);
    cudaError_t err = cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return err == cudaSuccess ? 0 : (int)err;
}
