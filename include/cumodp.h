/*
 * cumodp.h -- C entry points of the B200 polynomial-product library.
 *
 * Drop-in for the reference's include/cumodp.h (FFT / FFT-multiplication
 * part).  Every reference entry point keeps its name, argument meaning and
 * numeric error codes; where the reference silently misbehaved the deviation
 * is listed at the function.  Functions marked "addition" have no
 * counterpart in the reference.
 *
 * Coefficients are sfixn = 32-bit int holding residues in [0, p); p is an
 * odd "Fourier" prime p = c * 2^e + 1 below 2^30.  Unless noted, pointers
 * are HOST pointers and results are complete when the call returns.  All
 * entry points are thread-safe (calls are serialised per process).
 */
#ifndef CUMODP_B200_H
#define CUMODP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; everything declared here is
 * exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* include/types.h:45-53 under LINUXINTEL64 */
typedef int32_t sfixn;

/* Same numeric values as the reference enum (include/types.h:123-146). */
typedef enum {
    CUMODP_SUCCESS = 0x000,
    CUMODP_FAILURE = 0x001,
    CUMODP_ASSUMPTION_ERROR = 0x002,
    CUMODP_NO_CUDA_DEVICE = 0x100,
    CUMODP_HAS_CUDA_DEVICE = 0x101,
    CUMODP_FFT_ERROR = 0x200,
    CUMODP_FOURIER_DEGREE_TOO_SMALL = 0x201,
    CUMODP_FFT_SIZE_TOO_LARGE = 0x202,
    CUMODP_FFT_SIZE_TOO_SMALL = 0x203,
    CUMODP_SUBRES_ERROR = 0x300,
    CUMODP_SUBRES_COARSE_ERROR = 0x301,
    CUMODP_SUBRES_FINE_ERROR = 0x302,
    CUMODP_SUBRES_NON_REGULAR = 0x303,
    CUMODP_RES2_ERROR = 0x304,
    CUMODP_RES3_ERROR = 0x305,
    CUMODP_OUT_OF_MEMORY = 0x401,
    CUMODP_UNKNOWN_ERROR = 0x999
} cumodp_err;

/* ------------------------------------------------------ device queries -- */
/* Replace src/modpn.cu:51-57. */
int is_cuda_enabled(void);
/* Replaces src/modpn.cu:62-67. */
int num_of_cuda_devices(void);
/* Replaces src/modpn.cu:72-88 (every sm_100 device has fp64: 1 with a device). */
int is_double_float_enabled(void);
/* Replaces src/modpn.cu:93-98; saturates at 4 GiB - 1 like the reference's
 * unsigned int return type truncates. */
unsigned int global_memory_in_bytes(void);
/* Replaces src/modpn.cu:103-108. */
float global_memory_in_megabytes(void);
/* Replaces src/modpn.cu:113-126: nonzero when a product of degrees df, dg
 * fits this library's transform limits (2^29; the prime's 2-adic order is
 * checked by the product itself, as the reference's stockham path leaves it
 * to the caller) and the device's memory. */
int can_call_fftmul_uni(sfixn df, sfixn dg);
/* Replace src/modpn.cu:142-173.  The subresultant GPU path is not part of
 * this library: always 0, so modpn keeps its CPU subresultant code. */
int can_call_subres2(sfixn dx, sfixn d1, sfixn d2);
int can_call_subres3(sfixn dx, sfixn dy, sfixn d1, sfixn d2);

/* ------------------------------------------- FFT and FFT multiplication -- */
/* In-place natural-order DFT of X (n = 2^k words): X[j] <- sum_i X[i] w^(ij)
 * mod p, w a primitive n-th root.  Replaces src/modpn.cu:181-192
 * (stockham_host, src/stockham.cu:479-487).  Deviation: invalid p, n != 2^k,
 * or a w that is not a primitive n-th root return CUMODP_ASSUMPTION_ERROR;
 * n above the prime's 2-adic order returns CUMODP_FFT_SIZE_TOO_LARGE (the
 * reference computes garbage); n < 256 is supported (the reference's grid
 * arithmetic breaks below k = 8).  n up to 2^25 runs as one four-step
 * transform; longer ones take one radix-2 step over HBM first. */
cumodp_err cumodp_fft_uni(sfixn *X, sfixn n, sfixn k, sfixn w, sfixn p);
/* Inverse: DFT with w^-1 then scaling by n^-1.  Replaces src/modpn.cu:197-210
 * (inverse_stockham_host, src/stockham.cu:489-503). */
cumodp_err cumodp_invfft_uni(sfixn *X, sfixn n, sfixn k, sfixn w, sfixn p);
/* 2-D DFT of a row-major 2^em x 2^en array X: w_m-DFT down the columns
 * (length 2^em) and w_n-DFT along the rows (length 2^en).  Replaces
 * src/modpn.cu:215-244 (bivariate_stockham_host, src/list_stockham.cu).
 * Deviation: em != en is computed correctly (the reference is square-only).
 * Rows of 2^6 words or more, em + en <= 30; columns up to 2^11 with rows up to
 * 2^14 run as one column pass and one row pass, larger shapes as row
 * transforms and transposed column transforms. */
cumodp_err cumodp_fft_bivariate(sfixn *X, sfixn em, sfixn wm, sfixn en, sfixn wn, sfixn p);
cumodp_err cumodp_invfft_bivariate(sfixn *X, sfixn em, sfixn wm, sfixn en, sfixn wn, sfixn p);
/* H = F * G mod p: F has df+1 coefficients, G dg+1, H receives dh+1 words.
 * Replaces src/modpn.cu:249-261 (stockham_poly_mul_host, src/stockham.cu:
 * 562-611).  H may alias F or G (modpn multiplies in place, FMUL.c:1949).
 * Every transform length up to the prime's 2-adic order is computed: up to
 * 2^25 directly, beyond that as 2^25-point products of 2^24-coefficient
 * pieces added at their offsets.
 * Deviations (documented fixes): every size is computed (the reference
 * returns SUCCESS with H untouched below transform size 256); exactly dh+1
 * words are written, zero beyond df+dg (the reference writes 2^ceil(log2
 * (df+dg+1)) words whenever dh >= df+dg+1); nothing is printed. */
cumodp_err cumodp_fftmul_uni(sfixn dh, sfixn *H, sfixn df, const sfixn *F,
                             sfixn dg, const sfixn *G, sfixn p);

/* --------------------------------------------------- out-of-scope stubs -- */
/* The subresultant-chain and scube GPU code of the reference
 * (src/modpn.cu:272-408) is not part of this library.  These symbols exist
 * so that modpn links unchanged; each reports "not available" the way the
 * reference does for unsupported cases, and modpn falls back to its CPU
 * code (modpn/src/IteratedResultant.c:421-1253). */
sfixn cumodp_subres_chain2_fine(sfixn *S, sfixn B, sfixn w, sfixn npx, sfixn npy, const sfixn *P,
                                sfixn nqx, sfixn nqy, const sfixn *Q, sfixn p);
sfixn cumodp_subres_chain2_coarse(sfixn *S, sfixn B, sfixn w, sfixn npx, sfixn npy, const sfixn *P,
                                  sfixn nqx, sfixn nqy, const sfixn *Q, sfixn p);
sfixn cumodp_subres_chain3_fine(sfixn *S, sfixn Bx, sfixn By, sfixn wx, sfixn wy, sfixn npx, sfixn npy,
                                sfixn npz, const sfixn *P, sfixn nqx, sfixn nqy, sfixn nqz,
                                const sfixn *Q, sfixn p);
sfixn cumodp_subres_chain3_coarse(sfixn *S, sfixn Bx, sfixn By, sfixn wx, sfixn wy, sfixn npx,
                                  sfixn npy, sfixn npz, const sfixn *P, sfixn nqx, sfixn nqy,
                                  sfixn nqz, const sfixn *Q, sfixn p);
void *init_cuda_scube(sfixn N, const sfixn *sz_p, const sfixn *sz_q, sfixn fp);
void free_cuda_scube(void *scb);
void print_cuda_scube(const void *scb);
cumodp_err build_cuda_scube(void *scb, const sfixn *sz_p, const sfixn *P, const sfixn *sz_q,
                            const sfixn *Q);
const sfixn *interp_subres_coeff2(sfixn *nx, void *scb, sfixn i, sfixn j);
const sfixn *interp_subres_coeff3(sfixn *nx, sfixn *ny, void *scb, sfixn i, sfixn j);

/* ------------------------------------------------------------ additions -- */
/* Addition.  Device-pointer product on a caller stream (0 = the library's
 * stream, then synchronised).  F, G, H are DEVICE pointers; lh words of H
 * are written.  Counterpart of the reference's C++ stockham_poly_mul_dev
 * (src/stockham.cu:521-542) without its size-padding contract: inputs need
 * no padding and are not modified. */
cumodp_err cumodp_fftmul_uni_dev(sfixn lh, sfixn *H, sfixn df, const sfixn *F,
                                 sfixn dg, const sfixn *G, sfixn p, void *stream);

/* Addition.  Cyclic convolution on DEVICE arrays of n = 2^e words:
 * F <- DFT^-1(DFT F * DFT G) = F * G mod (x^n - 1, p), the operation of the
 * reference's C++ stockham_poly_mul_dev(n, e, F, G, p)
 * (src/stockham.cu:521-542), which is the polynomial product when F and G are
 * zero-padded so that deg F + deg G < n.  Inputs in [0, p).  G is left
 * unchanged (the reference overwrites it with its transform); F and G must
 * not overlap.  Lengths 2^5..2^25 run on the product kernels (one transform
 * of length n, no padding), others as natural-order transforms around a
 * pointwise product (then F and G 16-byte aligned when e >= 6).  e up to the
 * prime's 2-adic order.  stream 0 = the library's stream, then synchronised. */
cumodp_err cumodp_cyclic_mul_dev(sfixn e, sfixn *F, const sfixn *G, sfixn p, void *stream);

/* Addition (no counterpart in the reference).  The device-pointer product of
 * cumodp_fftmul_uni_dev for callers that cannot allocate device memory --
 * services whose device memory belongs to their own pool allocator, plugins
 * loaded after the host partitioned all device memory, latency-critical code
 * that cannot afford cudaMalloc's implicit synchronisation.  It calls no
 * cudaMalloc/cudaFree and no allocating library routine: its scratch
 * (workspace and twiddle tables) is one fixed ~8.4 MiB array in the
 * library's device data segment, held by every GPU that loads the library
 * until exit.  Limit: df + dg + 1 <= 2^20 (CUMODP_FFT_SIZE_TOO_LARGE
 * beyond).  Every call first writes the twiddle tables of its prime and size
 * into the array (a small kernel on `stream`), so no state passes from one
 * call to the next.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture, and do not cudaDeviceReset that device afterwards.  All calls
 * share the array: calls whose GPU work overlaps race.  stream 0 runs on the
 * default stream and synchronises before returning. */
cumodp_err cumodp_fftmul_uni_dev_noalloc(sfixn lh, sfixn *H, sfixn df, const sfixn *F,
                                         sfixn dg, const sfixn *G, sfixn p, void *stream);

/* Addition.  Batched products mod one prime, all on the device: product i is
 * H_i = F_i * G_i with F_i = F + f_off[i] (df[i]+1 words), G_i = G + g_off[i]
 * (dg[i]+1 words), H_i = H + h_off[i] (df[i]+dg[i]+1 words).  f_off, g_off,
 * h_off, df, dg are HOST arrays of length count; F, G, H are DEVICE
 * pointers.  Products are grouped by transform size and run as one
 * CUDA-graph launch; the plan (grouping, job tables, workspace) is cached
 * per batch shape.  Transforms up to 2^25 (CUMODP_FFT_SIZE_TOO_LARGE beyond:
 * longer products go through cumodp_fftmul_uni_dev).  stream: 0 = library
 * stream, then synchronised. */
cumodp_err cumodp_fftmul_batch_dev(int count, const sfixn *df, const int64_t *f_off, const sfixn *F,
                                   const sfixn *dg, const int64_t *g_off, const sfixn *G,
                                   const int64_t *h_off, sfixn *H, sfixn p, void *stream);

/* Addition.  Same as cumodp_fftmul_batch_dev with HOST F, G, H: copies in,
 * computes and copies out (pinned staging, one H2D and one D2H copy). */
cumodp_err cumodp_fftmul_batch(int count, const sfixn *df, const int64_t *f_off, const sfixn *F,
                               const sfixn *dg, const int64_t *g_off, const sfixn *G,
                               const int64_t *h_off, sfixn *H, sfixn p);

/* Addition.  Exact product of int64-coefficient polynomials: c = a * b in Z[y]
 * with c written as signed 128-bit integers, two int64 words per
 * coefficient (low word first), na+nb-1 coefficients.  Counterpart of the
 * reference's C++ two_convolution_poly_mul (src/two_convolution_poly_mul.cu:
 * 532-569) for coefficients that fit int64 (the reference takes GMP mpz).
 * Same algorithm: limb split (K limbs of M bits, sign-magnitude), cyclic and
 * negacyclic x-convolutions mod Fourier primes 962592769, 950009857,
 * 940572673, CRT, (u+v)/2 + 2^N (u-v)/2.  method 0 picks the cheapest exact
 * (K, M, primes); method 1 forces the smallest limb split that needs only
 * two primes.  With method 0, products longer than those primes'
 * transforms allow (past 2^21 coefficients) or that they make dearer (2^21
 * points, which need 2 x 4 transforms there against 3 over primes of
 * higher order) run on the big-coefficient path (cumodp_twoconv_mul_big's
 * planner, Fourier primes of 2-adic order >= 22), up to 2^25 coefficients:
 * the same integers, fewer transforms.  Host
 * arrays pass through pinned staging (one copy each way).  Returns
 * CUMODP_ASSUMPTION_ERROR when the exact product does not fit 127 bits or
 * na + nb - 1 > 2^25, CUMODP_FFT_SIZE_TOO_LARGE when no plan exists. */
cumodp_err cumodp_twoconv_mul_i64(long long na, const int64_t *a, long long nb, const int64_t *b, int64_t *c,
                                  int method);
/* Addition.  Same on DEVICE pointers, on a caller stream (0 = library stream,
 * then synchronised); bit_width is max over both inputs of the bit length of
 * |coefficient| (cumodp_twoconv_bit_width on host data). */
cumodp_err cumodp_twoconv_mul_i64_dev(long long na, const int64_t *a, long long nb, const int64_t *b, int64_t *c,
                                      int bit_width, int method, void *stream);
/* Addition.  Bit width of the largest |coefficient| (0 counts as width 1),
 * as find_largest_bit_width_of_coefficients (src/two_convolution_poly_mul.cu:
 * 58-70); -1 on bad arguments. */
int cumodp_twoconv_bit_width(long long na, const int64_t *a, long long nb, const int64_t *b);
/* Addition.  The (K, M, number of primes) the product of two inputs of the
 * given bit widths and lengths uses (determine_bivariate_base,
 * src/two_convolution_poly_mul.cu:72-82, re-derived from an exactness bound
 * instead of the reference's fixed table). */
cumodp_err cumodp_twoconv_plan(int bit_width_a, int bit_width_b, long long na, long long nb, int method, int *K,
                               int *M, int *nprimes);

/* ---------------------------------------------------- serving (addition) -- */
/* A request loop with continuous batching.  Requests (modular products, or
 * exact int64 products) are copied at submission; a batcher thread admits
 * them in arrival order while the device-memory budget allows, groups them
 * by (kind, prime) and runs each group as one batch (at most max_batch
 * requests and 1 GiB of device buffers, or one larger request) on a free
 * lane (stream plus device buffers); batches on different lanes overlap on the GPU, and
 * requests arriving meanwhile join the next batch.  Operands are copied at
 * submission into pinned memory owned by the server; the result is copied
 * into the caller's output buffer by cumodp_server_wait, which must be
 * called once per request (the buffer must stay valid until then).  Memory
 * the caller registers (cumodp_server_register) skips both copies: operands
 * go to the device from it and results come back into it.  No counterpart in
 * the reference. */
typedef struct cumodp_server cumodp_server;
typedef struct {
    int device;              /* CUDA device ordinal */
    size_t memory_budget;    /* device bytes for requests in flight (0: a quarter of free memory) */
    int max_batch;           /* requests per batch (default 512) */
    int batch_window_us;     /* wait for more arrivals once work is queued (default 50) */
    int lanes;               /* batches in flight at once (default 4) */
    int inject_fault_batch;  /* tests: the n-th batch fails on the host before launching (0 = off) */
    size_t host_budget;      /* pinned host memory for the operand and result slabs of unfinished
                                requests (power-of-two slabs carved from chunks pinned when the
                                server is created); a submission that finds no room completes at
                                once with CUMODP_OUT_OF_MEMORY (load shedding).  Requests in
                                registered memory count against it too.  0 = 2 GiB */
} cumodp_server_config;
typedef struct {
    long long completed, failed, batches, pending;
    size_t inflight_bytes;
    double p50_us, p99_us, max_us;  /* submission-to-result latency of completed requests */
    double products_per_s;          /* completed / (last completion - first submission) */
} cumodp_server_stats;
void cumodp_server_default_config(cumodp_server_config *cfg);
cumodp_server *cumodp_server_create(const cumodp_server_config *cfg);
/* H receives df+dg+1 words.  Returns the request id (> 0), -1 on bad arguments. */
long long cumodp_server_submit_mod(cumodp_server *s, sfixn p, sfixn df, const sfixn *F, sfixn dg, const sfixn *G,
                                   sfixn *H);
/* c receives na+nb-1 signed 128-bit coefficients as (lo, hi) int64 pairs. */
long long cumodp_server_submit_i64(cumodp_server *s, long long na, const int64_t *a, long long nb, const int64_t *b,
                                   int64_t *c);
/* 1 done, 0 pending, -1 unknown id. */
int cumodp_server_poll(cumodp_server *s, long long id);
/* Waits (timeout_us < 0: forever) and returns the request's cumodp_err, -2
 * on timeout, -1 for an unknown id; a waited-for id is forgotten. */
int cumodp_server_wait(cumodp_server *s, long long id, long long timeout_us);
/* Addition.  Open-loop replay of a timed request trace against a server,
 * driven by native threads (a load generator for capacity planning).
 * Request i is submitted arrival_us[i] microseconds after the call starts
 * (a submitter that falls behind submits at once): kind[i] = 0 is the
 * product mod p[i] of la[i] and lb[i] sfixn coefficients a[i], b[i] into
 * h[i] (la+lb-1 words); kind[i] = 1 the exact product of int64 operands into
 * h[i] (2(la+lb-1) int64 words).  h may be NULL (each result then lands in
 * the server's pinned slab and is dropped when collected: no host copy).
 * `threads` submitters share the
 * trace round-robin, each with a collector thread.  On return status[i] is
 * the request's cumodp_err (-1: refused by the server), lat_us[i] the time
 * from the scheduled arrival to the result in the output buffer, and
 * *span_us the time from the start to the last result. */
cumodp_err cumodp_server_replay(cumodp_server *s, long long count, const double *arrival_us, const int *kind,
                                const sfixn *p, const long long *la, const long long *lb, const void *const *a,
                                const void *const *b, void *const *h, int threads, double *lat_us, int *status,
                                double *span_us);
/* Addition.  Registers the caller's host memory [ptr, ptr + bytes) with the
 * server (page-locked in place and mapped into the device's address space,
 * cudaHostRegister with cudaHostRegisterMapped).  A request whose two
 * operands lie in registered memory is copied to the device straight from
 * there, and a result buffer that lies in registered memory receives the
 * result straight from the device: no copy through the server's pinned slabs
 * and no host memcpy on either side.  Copies under 512 KiB are made by one
 * kernel per batch that reads or writes the mapped memory (a copy-engine
 * transfer costs about 4 us of its own, whatever its size); larger ones by
 * the copy engines.  The caller leaves such operands
 * unchanged until the request completes.  Unfinished requests still count
 * their operand and result bytes against host_budget, which keeps bounding
 * the backlog (shedding beyond it).  Ranges may not overlap.  Unregister only
 * when no unfinished request uses the range; cumodp_server_destroy
 * unregisters what is left. */
cumodp_err cumodp_server_register(cumodp_server *s, void *ptr, size_t bytes);
cumodp_err cumodp_server_unregister(cumodp_server *s, void *ptr);
void cumodp_server_get_stats(cumodp_server *s, cumodp_server_stats *out);
void cumodp_server_reset_stats(cumodp_server *s);
/* Drains queued and in-flight work, then frees everything. */
void cumodp_server_destroy(cumodp_server *s);

/* Addition.  Device-pointer natural-order transform on a caller stream (0 =
 * the library's stream, then synchronised): forward as cumodp_fft_uni, or
 * the inverse of it when `inverse` is nonzero.  X is a DEVICE pointer,
 * 16-byte aligned (as cudaMalloc returns) when k >= 6. */
cumodp_err cumodp_fft_uni_dev(sfixn *X, sfixn n, sfixn k, sfixn w, sfixn p, int inverse, void *stream);

/* Addition.  Device-pointer 2-D transform on a caller stream (0 = the
 * library's stream, then synchronised): cumodp_fft_bivariate, or
 * cumodp_invfft_bivariate when `inverse` is nonzero, in place on the DEVICE
 * array X (16-byte aligned).  Counterpart of the reference's C++
 * bivariate_stockham_dev / inverse_bivariate_stockham_dev
 * (src/list_stockham.cu:1161-1204, 1251-1263), given the roots wm, wn
 * instead of their power tables. */
cumodp_err cumodp_fft_bivariate_dev(sfixn *X, sfixn em, sfixn wm, sfixn en, sfixn wn, sfixn p, int inverse,
                                    void *stream);

/* Addition.  The list transform I_m (x) DFT_n: m independent natural-order
 * transforms of length n = 2^k of the DEVICE array X (row i at X + i n), in
 * place, root w (inverse: w^-1 and scaling by n^-1); X 16-byte aligned when
 * k >= 6.  Counterpart of the
 * reference's C++ list_stockham_dev (src/list_stockham.cu:595-665, declared
 * in include/list_stockham.h:48-49; include/list_stockham_b200.h here gives
 * the same C++ signatures) without its grid bug for m * n / 128 > 2^15 and
 * without its __constant__ globals.  stream: 0 = library stream, then
 * synchronised. */
cumodp_err cumodp_list_fft_dev(sfixn *X, sfixn m, sfixn k, sfixn w, sfixn p, int inverse, void *stream);

/* Addition.  Bivariate product on a 2^em x 2^en grid of DEVICE words (row
 * j, of 2^en words, holds the coefficients of y^j; x^i at column i):
 * F <- DFT^-1(DFT F * DFT G), the 2-D cyclic convolution, which is the
 * bivariate product when both operands are zero-padded to the product's
 * size.  G is overwritten; F and G 16-byte aligned.  Counterpart of the reference's C++
 * bi_stockham_poly_mul_dev (src/list_stockham.cu:1317-1348, declared in
 * include/list_stockham.h:103-104; include/list_stockham_b200.h gives that
 * signature), for any em, en within the prime's 2-adic order (em + en <= 30).
 * stream: 0 = library stream, then synchronised. */
cumodp_err cumodp_bivariate_mul_dev(sfixn em, sfixn en, sfixn *F, sfixn *G, sfixn p, void *stream);

/* Addition.  Bivariate product of HOST operands in the (nx, ny) dense layout
 * (coefficient of x^i y^j at j * nx + i): H receives
 * (nxf + nxg - 1) * (nyf + nyg - 1) words in the (nxf + nxg - 1,
 * nyf + nyg - 1) layout.  Counterpart of the reference's
 * bi_stockham_poly_mul_host (src/list_stockham.cu:1352-1390, with
 * expand_to_fft2_dev / extract_from_fft2_dev, src/fft_aux.cu:630-681), on
 * plain arrays instead of its rdr_poly class. */
cumodp_err cumodp_bivariate_mul(sfixn nxf, sfixn nyf, const sfixn *F, sfixn nxg, sfixn nyg, const sfixn *G,
                                sfixn *H, sfixn p);

/* Addition.  One level of a subproduct tree, as one call on DEVICE arrays:
 * M_in holds 2*npairs monic polynomials of degree l stored without their
 * leading coefficient (l words each, constant term first, polynomial j at
 * M_in + j*l); M_out (not overlapping M_in) receives the npairs products
 * M_in[2j] * M_in[2j+1], monic of degree 2l, likewise without the leading
 * coefficient (2l words each, at M_out + 2*j*l).  Replaces the reference's
 * level step of subProductTree (src/fastPolyEvaluation.cu:604-650:
 * zeroInbetween, list_stockham_dev, pointMul, inverse transform, scalarMul,
 * pointAdd2 and pointAdd, whose kernels are at :83-160) for any l >= 1 and
 * any number of pairs (the reference: powers of two).
 * stream: 0 = library stream, then synchronised. */
cumodp_err cumodp_subproduct_level_dev(sfixn l, sfixn npairs, const sfixn *M_in, sfixn *M_out, sfixn p,
                                       void *stream);

/* Addition.  Exact product of polynomials with big signed integer
 * coefficients: the general two_convolution_poly_mul
 * (src/two_convolution_poly_mul.cu:532-569, std::vector<mpz_class>) without
 * GMP at the boundary.  Every coefficient of a and b is `in_words`
 * little-endian 64-bit words in two's complement (in_words <= 64: up to 4096
 * bits); c receives na+nb-1 coefficients of `out_words` words in two's
 * complement, truncated to out_words (cumodp_twoconv_big_out_words gives the
 * width that always holds the product).  Host arrays.  The whole computation
 * (limb split, one univariate product per prime, CRT and recombination) runs
 * on the GPU; cumodp_twoconv_big_plan reports the limb split and primes. */
cumodp_err cumodp_twoconv_mul_big(long long na, const uint64_t *a, long long nb, const uint64_t *b, int in_words,
                                  uint64_t *c, int out_words);
/* The same on DEVICE arrays; bit_width bounds the magnitude bit width of
 * every coefficient (cumodp_twoconv_big_bit_width computes it on the host). */
cumodp_err cumodp_twoconv_mul_big_dev(long long na, const uint64_t *a, long long nb, const uint64_t *b, int in_words,
                                      uint64_t *c, int out_words, int bit_width, void *stream);
int cumodp_twoconv_big_bit_width(long long na, const uint64_t *a, long long nb, const uint64_t *b, int in_words);
int cumodp_twoconv_big_out_words(long long na, long long nb, int bit_width);
/* K limbs of M bits per coefficient, `nprimes` Fourier primes, transform
 * length 2^log_transform: the cheapest split whose CRT bound
 * K * min(na, nb) * (2^M - 1)^2 < P/2 holds (the reference picks from
 * base_table with K >= 32, include/two_convolution_poly_mul.h:94-527). */
cumodp_err cumodp_twoconv_big_plan(int bit_width, long long na, long long nb, int *K, int *M, int *nprimes,
                                   int *log_transform);

/* Addition (testing).  Host-side fault injection: the next `count` device
 * allocations the library makes fail as if the device were out of memory
 * (the calls that needed them return CUMODP_OUT_OF_MEMORY; nothing is left
 * half-built, so the same call succeeds once the injection is used up).
 * 0 cancels.  Nothing touches the GPU. */
void cumodp_inject_alloc_failures(int count);

/* Addition.  Makes `dev` the current device of the calling thread for the
 * library's own CUDA runtime (one process per GPU). */
cumodp_err cumodp_select_device(int dev);

/* Addition.  Per-pass tracing: when enabled, every kernel launch that is not
 * being captured into a graph is bracketed by CUDA events on its stream.
 * cumodp_trace_report writes "kernel launches total_ms" lines (NUL
 * terminated, truncated to len) and returns the full report length;
 * `reset` clears the totals. */
void cumodp_trace_passes(int enable);
size_t cumodp_trace_report(char *buf, size_t len, int reset);

/* Addition.  Bytes of device memory the library currently holds (tables,
 * workspace, plans). */
size_t cumodp_device_bytes_in_use(void);

/* Addition.  Human-readable text of an error code. */
const char *cumodp_error_string(cumodp_err e);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* CUMODP_B200_H */
