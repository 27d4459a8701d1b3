// Host runtime shared by every entry point: prime set-up, resident twiddle
// tables, per-device workspace and the error convention.
#pragma once
#include <nvtx3/nvToolsExt.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "ntt_engine.cuh"
#include "plans.cuh"

namespace cmb {

// Numeric codes of the reference's cumodp_err (include/types.h:123-146).
enum Err : int {
    OK = 0x000,
    FAILURE = 0x001,
    ASSUMPTION_ERROR = 0x002,
    NO_CUDA_DEVICE = 0x100,
    FFT_ERROR = 0x200,
    FOURIER_DEGREE_TOO_SMALL = 0x201,
    FFT_SIZE_TOO_LARGE = 0x202,
    FFT_SIZE_TOO_SMALL = 0x203,
    OUT_OF_MEMORY = 0x401,
};

// Everything the kernels need to know about one prime (and one root family).
struct PrimeCtx {
    PrimeInfo info;
    u32 root_max;  // canonical primitive 2^two_adic-th root
    PrimeK pk;     // kernel constants for the canonical roots
};

// Validates p (odd prime < 2^30 with 2-adic order >= 5) and returns the
// cached context, or nullptr with *err set.
const PrimeCtx* prime_ctx(u32 p, int* err);

// Root helpers (exact host arithmetic).
u32 canonical_root(const PrimeCtx& pc, int logn);  // primitive 2^logn-th root
PrimeK make_prime_k(const PrimeInfo& pi, u32 w32);  // w32: a primitive 32nd root
// Constants for register DFTs of a transform of length 2^logl with the
// primitive root `root`; below length 32 only the entries radix-2^logl
// butterflies read are filled.
PrimeK make_prime_k_for(const PrimeInfo& pi, u32 root, int logl);
Tw tw_of(u32 w, u32 p);

// Device-resident tables for the row (contiguous) plan of length 2^logl
// built from the primitive 2^logl-th root `root`; forward tables first, the
// inverse tables start at plan_tw_entries(row_plan(logl), logl).
const Tw* row_tables(int dev, u32 p, u32 root, int logl, int* err);
// Same for the interleaved-column plan.
const Tw* col_tables(int dev, u32 p, u32 root, int logl, int* err);
// Inter-pass twiddle seeds for a two-pass transform of length 2^logn:
// lo[e] = w^e (e < 2^12) and hi[e] = w^(e << 12) (e < 2^(logn-12)), both in
// Montgomery form times R (w^e * 2^64 mod p) so that one Montgomery product
// of two entries yields w^(lo+hi) * 2^32.
const u32* seed_tables(int dev, u32 p, u32 root, int logn, int* err);

// The same tables written into caller storage (no allocation):
// level_tables_entries / seed_words give the sizes.
size_t level_tables_entries(int kind, int logl);  // kind 0: row plan, 1: column plan
int level_tables_into(int kind, u32 p, u32 root, int logl, Tw* out, size_t cap);
size_t seed_words(int logn);
int seeds_into(u32 p, u32 root, int logn, u32* out, size_t cap);

// Per-device scratch that grows on demand (never shrinks while the process
// lives).  Each call site names a slot so concurrent users do not collide.
void* workspace(int dev, int slot, size_t bytes, int* err);

// Pinned host staging that grows on demand (shared by every device; the
// caller holds lib_mutex and keeps no copy from it in flight past its call).
void* pinned_workspace(int slot, size_t bytes, int* err);

// The stream every synchronous entry point issues its work on.
cudaStream_t lib_stream(int dev);

// Serialises host entry points that share workspace and caches.
std::mutex& lib_mutex();

// NVTX range (host timeline) around a library operation: visible in Nsight
// Systems / ncu range filters, a few nanoseconds when no tool is attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Every device allocation of the library goes through dev_malloc, which
// honours the host-side fault injection of inject_alloc_failures.
cudaError_t dev_malloc(void** p, size_t bytes);
// Stream-ordered allocation (cudaMallocAsync) with the same fault injection.
cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t st);
void inject_alloc_failures(int n);

// Side streams of the library (per device) for independent pieces of one
// call: aux_fork makes streams 0..n-1 wait for `st`'s work so far,
// aux_stream(dev, i) is stream i, aux_join makes `st` wait for all of them.
// Calls are serialised by lib_mutex, so the side streams are never shared by
// two calls at once.
constexpr int kAuxStreams = 4;
cudaStream_t aux_fork(int dev, cudaStream_t st, int n);
cudaStream_t aux_stream(int dev, int i);
void aux_join(int dev, cudaStream_t st, int n);

int current_device();

// Device bytes held by the caches and workspace of this process.
size_t bytes_in_use();
// Records an allocation made outside the caches (plans, server pools).
void account_bytes(long long delta);

// Per-pass tracing: when enabled, launches that are not being captured into
// a graph are bracketed by CUDA events on their stream; the totals per
// kernel name are aggregated on demand (events are read after a sync).
bool pass_timing_on();
void pass_timing_enable(bool on);
// Returns an event pair from the pool, or false when tracing is off or the
// stream is capturing.
bool pass_timing_begin(cudaStream_t st, cudaEvent_t* e0);
void pass_timing_end(cudaStream_t st, const char* name, cudaEvent_t e0);
// "name launches total_ms" lines for every kernel seen since the last reset.
std::string pass_timing_report(bool reset);

// Copies the last CUDA error (if any) into a library code.
int cuda_err(cudaError_t e);

}  // namespace cmb
