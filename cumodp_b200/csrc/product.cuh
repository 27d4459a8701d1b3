// Host-side product dispatch shared by the C entry points.
#pragma once
#include "large_product.cuh"
#include "runtime.cuh"

namespace cmb {

constexpr int kMinLog = 5;        // smallest transform: one radix-32 row
constexpr int kMaxSmallLog = 14;  // largest single-CTA product (2 x 64 KiB of shared memory)
constexpr int kMaxColLog = 11;    // 16-column tile of 2^11 rows = 136 KiB of shared memory
constexpr int kMaxRowLog = 14;
constexpr int kMinRowLog = 6;
constexpr int kMaxLog = 25;        // largest transform of the three-pass kernels (2^11 x 2^14)
constexpr int kMaxSplitLog = 29;   // longer single products and transforms, up to the prime's 2-adic
                                   // order (at most 29 for p < 2^30), are split into 2^25 pieces
constexpr int kDefaultColLog = 10;  // column length of the default split (rows of 2^14)

// workspace slots (runtime.cuh: workspace)
enum WsSlot { kWsSingle = 0, kWsBatch = 1, kWsStage = 2, kWsNtt = 3, kWsTwoConv = 4, kWsServer = 5,
              kWsBiv = 6, kWsBivHost = 7, kWsBig = 8, kWsSplitProd = 9, kWsSplitIn = 10,
              kWsSplitNtt = 11 /* + (k - kMaxLog - 1) for a 2^k transform: 11..14 */, kWsBivT = 15,
              kWsListJobs = 16, kWsCyclic = 17 };
// pinned host staging slots (runtime.cuh: pinned_workspace)
enum PinSlot { kPinTwoConv = 0 };

// SMs of device dev (cached per device).
int sm_count(int dev);

// Transform length log2 for a product of la and lb coefficients.
int product_logn(long long la, long long lb);
// Default row length log2 of the three-pass split.
int default_row_log(int logn);

int small_args(const PrimeCtx& pc, u32 root, int logn, int dev, SmallArgs* a);
int large_args(const PrimeCtx& pc, u32 root_n, int logn, int l2, int dev, LargeArgs* a);
// A product's pass A through the persistent pipelined kernel when the column
// length has one (2^9, 2^10 rows); false when the caller must launch k_col_fwd.
bool launch_col_fwd_pipe(const LargeArgs& a, int njobs, cudaStream_t st);
// A natural-order transform's column pass (operand a of each job, over wa)
// through k_col_fwd_pipe1 when the columns have 2^10 rows; false otherwise.
bool launch_col_fwd_pipe1(const LargeArgs& a, int njobs, cudaStream_t st);
void launch_small(int logn, const SmallArgs& a, int njobs, cudaStream_t st);
void launch_large(const LargeArgs& a, int njobs, cudaStream_t st);

// Sets the shared-memory limits of every product kernel once (must run
// before any launch is captured into a graph).
void ensure_kernel_attrs();

// Batched products on caller-owned buffers, direct launches (batch.cu).
size_t direct_ws_words(int count, const long long* la, const long long* lb);
size_t direct_job_bytes(int count);
// allow_tuning: a size class seen for the first time may be autotuned
// (synchronous timing runs); otherwise cached choices or the default split.
int direct_batch(int count, const u32* const* a, const long long* la, const u32* const* b, const long long* lb,
                 u32* const* h, const long long* lh, u32 p, u32* ws, void* djobs, void* hjobs,
                 cudaStream_t st, bool allow_tuning);

// Device words of workspace a single product of transform length 2^logn
// takes (mul_dev), beside its operands and result.
size_t mul_ws_words(int logn);

// h[0..lh) = a[0..la) * b[0..lb) mod p on device pointers, on stream st.
int mul_dev(const u32* a, long long la, const u32* b, long long lb, u32* h, long long lh, u32 p,
            cudaStream_t st);

// f <- f * g mod (x^(2^e) - 1, p), the length-2^e cyclic convolution, on
// device arrays of 2^e words (f may not overlap g): the product kernels on
// one transform of length 2^e for kMinLog <= e <= kMaxLog, otherwise
// natural-order transforms around a pointwise product (cyclic_mul_compose,
// which needs 16-byte aligned arrays when e >= 6).
int cyclic_mul_dev(u32* f, const u32* g, int e, u32 p, cudaStream_t st);
int cyclic_mul_compose(u32* f, const u32* g, int e, u32 p, cudaStream_t st);

}  // namespace cmb
