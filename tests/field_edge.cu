// Test driver: runs the library's field primitives (cumodp_b200/csrc/field.cuh)
// and register DFTs (ntt_engine.cuh) on the GPU for operands chosen by the
// test, so their stated ranges can be checked against exact integer
// arithmetic at the edges (2^32 - 1, 4p - 1, 2p - 1, p - 1, the Montgomery
// bound a b < 2^32 p).  Built and loaded by tests/test_field_edge_gpu.py.
#include <cuda_runtime.h>

#include <cstdint>

#include "../cumodp_b200/csrc/ntt_engine.cuh"

using namespace cmb;

__global__ void k_field(const u32* a, const u32* b, int n, u32 p, u32 pinv_neg, u32* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 x = a[i], y = b[i];
    out[4 * i] = mul_shoup(x, y, shoup_quot(y, p), p);  // needs y < p
    out[4 * i + 1] = mul_mont(x, y, p, pinv_neg);        // needs x y < 2^32 p
    out[4 * i + 2] = red2(x, 2 * p);                     // needs x < 4p
    out[4 * i + 3] = red1(x, p);                         // needs x < 2p
}

// one 32-point DIF (dir 0, then also the TW variant's outputs: dir 2) or
// DIT (dir 1, and dir 3: the PRE variant) per thread, on 32 inputs each
template <int DIR>
__global__ void k_dft32(const u32* x, int nvec, u32 p, const Tw* rc, u32* y) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvec) return;
    u32 r[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = x[32 * v + j];
    if (DIR == 0) dif_regs<32>(r, rc, p, 2 * p);
    if (DIR == 2) dif_regs<32, true>(r, rc, p, 2 * p);
    if (DIR == 1) dit_regs<32>(r, rc, p, 2 * p);
    if (DIR == 3) dit_regs<32, true>(r, rc, p, 2 * p);
#pragma unroll
    for (int j = 0; j < 32; ++j) y[32 * v + j] = r[j];
}

extern "C" {

// out[4 i .. 4 i + 3] = mul_shoup(a_i, b_i), mul_mont(a_i, b_i), red2(a_i), red1(a_i)
int field_edge(const uint32_t* a, const uint32_t* b, int n, uint32_t p, uint32_t pinv_neg, uint32_t* out) {
    u32 *d = nullptr;
    if (cudaMalloc(&d, (size_t)6 * n * sizeof(u32)) != cudaSuccess) return -1;
    cudaMemcpy(d, a, (size_t)n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d + n, b, (size_t)n * 4, cudaMemcpyHostToDevice);
    k_field<<<(n + 127) / 128, 128>>>(d, d + n, n, p, pinv_neg, d + 2 * n);
    cudaError_t e = cudaMemcpy(out, d + 2 * n, (size_t)4 * n * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -1;
}

// y = 32-point register DFTs of x (nvec vectors); roots[j] = w_32^j (j < 16) of
// the direction's root; dir: 0 DIF, 1 DIT, 2 DIF with TW, 3 DIT with PRE
int dft32(const uint32_t* x, int nvec, uint32_t p, const uint32_t* roots, int dir, uint32_t* y) {
    Tw rc[16];
    for (int j = 0; j < 16; ++j) rc[j] = Tw{roots[j], shoup_quot(roots[j], p)};
    u32* d = nullptr;
    Tw* drc = nullptr;
    if (cudaMalloc(&d, (size_t)64 * nvec * sizeof(u32)) != cudaSuccess) return -1;
    if (cudaMalloc(&drc, sizeof(rc)) != cudaSuccess) {
        cudaFree(d);
        return -1;
    }
    cudaMemcpy(drc, rc, sizeof(rc), cudaMemcpyHostToDevice);
    cudaMemcpy(d, x, (size_t)32 * nvec * 4, cudaMemcpyHostToDevice);
    const int g = (nvec + 63) / 64;
    if (dir == 0) k_dft32<0><<<g, 64>>>(d, nvec, p, drc, d + 32 * nvec);
    if (dir == 1) k_dft32<1><<<g, 64>>>(d, nvec, p, drc, d + 32 * nvec);
    if (dir == 2) k_dft32<2><<<g, 64>>>(d, nvec, p, drc, d + 32 * nvec);
    if (dir == 3) k_dft32<3><<<g, 64>>>(d, nvec, p, drc, d + 32 * nvec);
    cudaError_t e = cudaMemcpy(y, d + 32 * nvec, (size_t)32 * nvec * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    cudaFree(drc);
    return e == cudaSuccess ? 0 : -1;
}

}  // extern "C"
