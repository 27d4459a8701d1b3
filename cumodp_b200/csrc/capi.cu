// C entry points (include/cumodp.h): device queries, the univariate product
// and the out-of-scope stubs.  Reference interface: src/modpn.cu:47-408.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "../../include/cumodp.h"
#include "product.cuh"

using namespace cmb;

namespace {

cumodp_err to_err(int e) { return (cumodp_err)e; }

bool have_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return n > 0;
}

}  // namespace

extern "C" {

void cumodp_inject_alloc_failures(int count) { inject_alloc_failures(count); }


int is_cuda_enabled(void) { return have_device() ? 1 : 0; }

int num_of_cuda_devices(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int is_double_float_enabled(void) { return have_device() ? 1 : 0; }

unsigned int global_memory_in_bytes(void) {
    if (!have_device()) return 0;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, current_device());
    size_t m = prop.totalGlobalMem;
    return m > 0xffffffffull ? 0xffffffffu : (unsigned int)m;
}

float global_memory_in_megabytes(void) {
    if (!have_device()) return 0.0f;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, current_device());
    return (float)(prop.totalGlobalMem >> 20);
}

int can_call_fftmul_uni(sfixn df, sfixn dg) {
    if (!have_device() || df < 0 || dg < 0) return 0;
    const int logn = product_logn((long long)df + 1, (long long)dg + 1);
    if (logn > kMaxSplitLog) return 0;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    // staging (F, G, H) plus the product's workspace
    const size_t need = ((size_t)df + dg + 2 + ((size_t)df + dg + 1) + mul_ws_words(logn)) * 4;
    return need < tot / 2 ? 1 : 0;
}

int can_call_subres2(sfixn, sfixn, sfixn) { return 0; }
int can_call_subres3(sfixn, sfixn, sfixn, sfixn) { return 0; }

cumodp_err cumodp_fftmul_uni_dev(sfixn lh, sfixn* H, sfixn df, const sfixn* F, sfixn dg, const sfixn* G,
                                 sfixn p, void* stream) {
    if (!have_device()) return CUMODP_NO_CUDA_DEVICE;
    if (df < 0 || dg < 0 || lh < 0 || !F || !G || (lh > 0 && !H)) return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = mul_dev((const u32*)F, (long long)df + 1, (const u32*)G, (long long)dg + 1, (u32*)H, lh, (u32)p, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return to_err(e);
}

cumodp_err cumodp_cyclic_mul_dev(sfixn e, sfixn* F, const sfixn* G, sfixn p, void* stream) {
    if (!have_device()) return CUMODP_NO_CUDA_DEVICE;
    if (e < 0 || !F || !G) return CUMODP_ASSUMPTION_ERROR;
    if (e < 31) {
        const size_t n = (size_t)1 << e;
        const char *f = (const char*)F, *g = (const char*)G;
        if (f < g + 4 * n && g < f + 4 * n) return CUMODP_ASSUMPTION_ERROR;  // F and G overlap
    }
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int err = cyclic_mul_dev((u32*)F, (const u32*)G, (int)e, (u32)p, st);
    if (err == OK && !stream) err = cuda_err(cudaStreamSynchronize(st));
    return to_err(err);
}

cumodp_err cumodp_fftmul_uni(sfixn dh, sfixn* H, sfixn df, const sfixn* F, sfixn dg, const sfixn* G, sfixn p) {
    if (!have_device()) return CUMODP_NO_CUDA_DEVICE;
    if (df < 0 || dg < 0 || dh < 0 || !F || !G || !H) return CUMODP_ASSUMPTION_ERROR;
    NvtxRange range("cumodp_fftmul_uni");
    std::lock_guard<std::mutex> g(lib_mutex());
    const int dev = current_device();
    cudaStream_t st = lib_stream(dev);
    const size_t la = (size_t)df + 1, lb = (size_t)dg + 1, lh = (size_t)dh + 1;
    int err = OK;
    u32* d = (u32*)workspace(dev, kWsStage, (la + lb + lh) * sizeof(u32), &err);
    if (!d) return to_err(err);
    u32 *dA = d, *dB = d + la, *dH = d + la + lb;
    cudaError_t ce = cudaMemcpyAsync(dA, F, la * 4, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(dB, G, lb * 4, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return to_err(cuda_err(ce));
    err = mul_dev(dA, (long long)la, dB, (long long)lb, dH, (long long)lh, (u32)p, st);
    if (err != OK) {
        cudaStreamSynchronize(st);
        return to_err(err);
    }
    ce = cudaMemcpyAsync(H, dH, lh * 4, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    return to_err(cuda_err(ce));
}

// ------------------------------------------------------------- stubs ----
sfixn cumodp_subres_chain2_fine(sfixn*, sfixn, sfixn, sfixn, sfixn, const sfixn*, sfixn, sfixn, const sfixn*,
                                sfixn) { return -1; }
sfixn cumodp_subres_chain2_coarse(sfixn*, sfixn, sfixn, sfixn, sfixn, const sfixn*, sfixn, sfixn, const sfixn*,
                                  sfixn) { return -1; }
sfixn cumodp_subres_chain3_fine(sfixn*, sfixn, sfixn, sfixn, sfixn, sfixn, sfixn, sfixn, const sfixn*, sfixn,
                                sfixn, sfixn, const sfixn*, sfixn) { return -1; }
sfixn cumodp_subres_chain3_coarse(sfixn*, sfixn, sfixn, sfixn, sfixn, sfixn, sfixn, sfixn, const sfixn*,
                                  sfixn, sfixn, sfixn, const sfixn*, sfixn) { return -1; }
// NULL is the reference's own "use the CPU" answer (src/modpn.cu:321-341).
void* init_cuda_scube(sfixn, const sfixn*, const sfixn*, sfixn) { return nullptr; }
void free_cuda_scube(void*) {}
void print_cuda_scube(const void*) {}
cumodp_err build_cuda_scube(void*, const sfixn*, const sfixn*, const sfixn*, const sfixn*) {
    return CUMODP_FAILURE;
}
const sfixn* interp_subres_coeff2(sfixn*, void*, sfixn, sfixn) { return nullptr; }
const sfixn* interp_subres_coeff3(sfixn*, sfixn*, void*, sfixn, sfixn) { return nullptr; }

size_t cumodp_device_bytes_in_use(void) { return bytes_in_use(); }

void cumodp_trace_passes(int enable) { pass_timing_enable(enable != 0); }

size_t cumodp_trace_report(char* buf, size_t len, int reset) {
    const std::string r = pass_timing_report(reset != 0);
    if (buf && len) {
        const size_t n = std::min(len - 1, r.size());
        memcpy(buf, r.data(), n);
        buf[n] = 0;
    }
    return r.size();
}

cumodp_err cumodp_select_device(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || dev < 0 || dev >= n) {
        cudaGetLastError();
        return n ? CUMODP_ASSUMPTION_ERROR : CUMODP_NO_CUDA_DEVICE;
    }
    return cudaSetDevice(dev) == cudaSuccess ? CUMODP_SUCCESS : CUMODP_FAILURE;
}

const char* cumodp_error_string(cumodp_err e) {
    switch (e) {
        case CUMODP_SUCCESS: return "success";
        case CUMODP_FAILURE: return "failure";
        case CUMODP_ASSUMPTION_ERROR: return "invalid argument (prime, size, root or pointer)";
        case CUMODP_NO_CUDA_DEVICE: return "no CUDA device";
        case CUMODP_HAS_CUDA_DEVICE: return "has CUDA device";
        case CUMODP_FFT_ERROR: return "CUDA error during FFT";
        case CUMODP_FOURIER_DEGREE_TOO_SMALL: return "prime's 2-adic order too small";
        case CUMODP_FFT_SIZE_TOO_LARGE: return "transform size too large";
        case CUMODP_FFT_SIZE_TOO_SMALL: return "transform size too small";
        case CUMODP_OUT_OF_MEMORY: return "out of device memory";
        default: return "unknown error";
    }
}

}  // extern "C"
