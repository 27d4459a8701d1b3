// Test driver: calls every C++ overload of include/stockham_b200.h and
// include/list_stockham_b200.h from compiled C++ (the way the reference's
// internal callers would), on host arrays staged through device memory here.
// Built and loaded by tests/test_cxx_boundary_gpu.py; each function returns
// the overload's error code (or -1 for a CUDA runtime failure in the driver).
#include <cuda_runtime.h>

#include <vector>

#include "list_stockham_b200.h"
#include "stockham_b200.h"

namespace {
sfixn powmod(sfixn a, long long e, sfixn p) {
    unsigned long long r = 1, b = (unsigned long long)a % (unsigned long long)p;
    for (; e; e >>= 1) {
        if (e & 1) r = r * b % (unsigned long long)p;
        b = b * b % (unsigned long long)p;
    }
    return (sfixn)r;
}
// device copy of powers table[i] = w^i, i < n/2 (the reference's W layout)
sfixn* device_powers(sfixn w, sfixn n, sfixn p) {
    std::vector<sfixn> t((size_t)(n > 1 ? n / 2 : 1));
    unsigned long long v = 1;
    for (size_t i = 0; i < t.size(); ++i) {
        t[i] = (sfixn)v;
        v = v * (unsigned long long)w % (unsigned long long)p;
    }
    sfixn* d = nullptr;
    if (cudaMalloc(&d, t.size() * sizeof(sfixn)) != cudaSuccess) return nullptr;
    cudaMemcpy(d, t.data(), t.size() * sizeof(sfixn), cudaMemcpyHostToDevice);
    return d;
}
}  // namespace

extern "C" {

// mode 0: stockham_dev(w); 1: stockham_dev(W); 2: inverse_stockham_dev(w);
// 3: inverse_stockham_dev(W, powers of w^-1); 4: stockham_host; 5: inverse_stockham_host
int cxx_transform(sfixn* X, sfixn n, sfixn k, sfixn w, sfixn p, int mode) {
    if (mode == 4) return stockham_host(X, n, k, w, p);
    if (mode == 5) return inverse_stockham_host(X, n, k, w, p);
    sfixn* d = nullptr;
    if (cudaMalloc(&d, (size_t)n * sizeof(sfixn)) != cudaSuccess) return -1;
    cudaMemcpy(d, X, (size_t)n * sizeof(sfixn), cudaMemcpyHostToDevice);
    int e = -1;
    sfixn* W = nullptr;
    if (mode == 0) e = stockham_dev(d, n, k, w, p);
    if (mode == 2) e = inverse_stockham_dev(d, n, k, w, p);
    if (mode == 1 || mode == 3) {
        W = device_powers(mode == 1 ? w : powmod(w, (long long)p - 2, p), n, p);
        if (!W) {
            cudaFree(d);
            return -1;
        }
        const sfixn* Wc = W;
        e = mode == 1 ? stockham_dev(d, n, k, Wc, p) : inverse_stockham_dev(d, n, k, Wc, p);
    }
    cudaMemcpy(X, d, (size_t)n * sizeof(sfixn), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (W) cudaFree(W);
    return e;
}

// stockham_poly_mul_dev(n, e, F, G, p) on copies of F and G; F receives the
// result, G the device G after the call (the library leaves it unchanged)
int cxx_poly_mul_dev(sfixn n, sfixn e, sfixn* F, sfixn* G, sfixn p) {
    sfixn *dF = nullptr, *dG = nullptr;
    if (cudaMalloc(&dF, (size_t)n * sizeof(sfixn)) != cudaSuccess) return -1;
    if (cudaMalloc(&dG, (size_t)n * sizeof(sfixn)) != cudaSuccess) {
        cudaFree(dF);
        return -1;
    }
    cudaMemcpy(dF, F, (size_t)n * sizeof(sfixn), cudaMemcpyHostToDevice);
    cudaMemcpy(dG, G, (size_t)n * sizeof(sfixn), cudaMemcpyHostToDevice);
    int r = stockham_poly_mul_dev(n, e, dF, dG, p);
    cudaMemcpy(F, dF, (size_t)n * sizeof(sfixn), cudaMemcpyDeviceToHost);
    cudaMemcpy(G, dG, (size_t)n * sizeof(sfixn), cudaMemcpyDeviceToHost);
    cudaFree(dF);
    cudaFree(dG);
    return r;
}

int cxx_poly_mul_host(sfixn dh, sfixn* H, sfixn df, const sfixn* F, sfixn dg, const sfixn* G, sfixn p) {
    return stockham_poly_mul_host(dh, H, df, F, dg, G, p);
}

// list_stockham_dev(X, m, k, w | W, p) on a copy of the m x 2^k host array
int cxx_list(sfixn* X, sfixn m, sfixn k, sfixn w, sfixn p, int use_table) {
    const size_t total = (size_t)m << k;
    sfixn* d = nullptr;
    if (cudaMalloc(&d, total * sizeof(sfixn)) != cudaSuccess) return -1;
    cudaMemcpy(d, X, total * sizeof(sfixn), cudaMemcpyHostToDevice);
    int e;
    if (use_table) {
        sfixn* W = device_powers(w, (sfixn)1 << k, p);
        const sfixn* Wc = W;
        e = W ? list_stockham_dev(d, m, k, Wc, p) : -1;
        if (W) cudaFree(W);
    } else {
        e = list_stockham_dev(d, m, k, w, p);
    }
    cudaMemcpy(X, d, total * sizeof(sfixn), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e;
}

// bi_stockham_poly_mul_dev on copies of two 2^em x 2^en grids; F receives the result
int cxx_bi_mul(sfixn em, sfixn en, sfixn* F, const sfixn* G, sfixn p) {
    const size_t total = (size_t)1 << (em + en);
    sfixn *dF = nullptr, *dG = nullptr;
    if (cudaMalloc(&dF, total * sizeof(sfixn)) != cudaSuccess) return -1;
    if (cudaMalloc(&dG, total * sizeof(sfixn)) != cudaSuccess) {
        cudaFree(dF);
        return -1;
    }
    cudaMemcpy(dF, F, total * sizeof(sfixn), cudaMemcpyHostToDevice);
    cudaMemcpy(dG, G, total * sizeof(sfixn), cudaMemcpyHostToDevice);
    int e = bi_stockham_poly_mul_dev((sfixn)1 << em, em, (sfixn)1 << en, en, dF, dG, p);
    cudaMemcpy(F, dF, total * sizeof(sfixn), cudaMemcpyDeviceToHost);
    cudaFree(dF);
    cudaFree(dG);
    return e;
}

}  // extern "C"
