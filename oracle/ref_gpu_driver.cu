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
