// Exact integer products (two-convolution path), shared declarations.
#pragma once
#include "product.cuh"

namespace cmb {

struct TwoConvPlan {
    int K, M, nprimes;
    int logn;  // y-transform length
};

// Caller-owned buffers for an exact product (the serving loop runs several
// at once on different streams); sizes from twoconv_buffer_sizes.
struct TwoConvBufs {
    u32* eval;    // evaluations and products
    u32* ws;      // product workspace
    void* djobs;  // device job tables
    void* hjobs;  // pinned host job tables (untouched until the stream passes)
};

void twoconv_buffer_sizes(long long la, long long lb, size_t* eval_words, size_t* ws_words, size_t* job_bytes);
// The same for the plan the product will use (exact, not the worst case).
void twoconv_buffer_sizes_plan(long long la, long long lb, const TwoConvPlan& pl, size_t* eval_words,
                               size_t* ws_words, size_t* job_bytes);
int twoconv_plan(int ba, int bb, long long la, long long lb, bool force_two_prime, TwoConvPlan* out);
// c (lo, hi pairs, la+lb-1 coefficients) = a * b exactly, device pointers;
// bufs == nullptr uses the library workspace and graph-launched batches.
int twoconv_mul_dev(const long long* a, long long la, const long long* b, long long lb, long long* c, int ba,
                    int bb, bool force_two_prime, cudaStream_t st, TwoConvPlan* used, const TwoConvBufs* bufs);

// The same product for lengths past the reference primes' transforms
// (twoconv_plan: FFT_SIZE_TOO_LARGE): the big-coefficient path with one
// 64-bit word per input coefficient and two per output coefficient, over
// Fourier primes of 2-adic order >= 22 (bigconv.cu); library workspace.
int exact_i64_long_dev(const long long* a, long long la, const long long* b, long long lb, long long* c, int bw,
                       cudaStream_t st);
// Transform work of that path (primes x 2^logn x logn), or its planner's error.
int exact_i64_long_cost(long long la, long long lb, int bw, double* cost);
// The same on caller buffers (bufs->eval holds eval_words, bufs->ws ws_words,
// the job tables job_bytes; exact_i64_long_sizes), everything on st.
int exact_i64_long_dev_bufs(const long long* a, long long la, const long long* b, long long lb, long long* c, int bw,
                            cudaStream_t st, const TwoConvBufs* bufs);
void exact_i64_long_sizes(long long la, long long lb, int bw, size_t* eval_words, size_t* ws_words,
                          size_t* job_bytes);
// Whether the big-coefficient plan of (la, lb, bw) has one limb and three
// primes (written to primes[0..3)): the plan exact_i64_long_batch runs.
bool exact_i64_long_one_limb(int bw, long long la, long long lb, u32* primes);
// Buffers of exact_i64_long_batch for cnt products of lengths la, lb.
void exact_i64_batch_sizes(int cnt, const long long* la, const long long* lb, size_t* eval_words, size_t* ws_words,
                           size_t* job_bytes);
// cnt exact products whose one-limb plans share the three primes, together:
// x holds each product's a then b (la[i] + lb[i] words, products in order),
// c receives each product's la[i] + lb[i] - 1 coefficients as (lo, hi)
// pairs, in order; one residue kernel, one batched product per prime, one
// CRT kernel, all on st and on the caller's buffers.
int exact_i64_long_batch(int cnt, const long long* x, const long long* la, const long long* lb, long long* c,
                         const u32* primes, cudaStream_t st, const TwoConvBufs& B);
// Whether the exact product of (la, lb) with bit widths (ba, bb) takes the
// big-coefficient path (method 0): no two-convolution plan, or a dearer one.
bool exact_i64_prefers_long(int ba, int bb, long long la, long long lb);

}  // namespace cmb
