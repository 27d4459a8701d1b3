// A product entry point that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: a service whose device
// memory is owned by its own pool allocator and may not be allocated behind
// its back, a plugin loaded into a host that has already partitioned all
// device memory, or code on a latency-critical path where cudaMalloc's
// implicit device synchronisation is not acceptable.
// cumodp_fftmul_uni_dev_noalloc serves them: the caller passes device buffers
// for the operands and the result, and everything else the product needs --
// the three-pass workspace and the twiddle tables -- lives in one fixed array
// in the library's own device data segment (g_noalloc_scratch below, about
// 8.4 MiB), which every GPU that loads the library holds until the process
// exits.
//
// Limits and sharing:
//   * products with df + dg + 1 <= 2^20 (transform length <= 2^20); larger
//     requests are rejected with CUMODP_FFT_SIZE_TOO_LARGE;
//   * every call writes the twiddle tables of its (prime, size) into the
//     array with a small kernel on the caller's stream, then runs the
//     product: no state is carried from one call to the next, and nothing in
//     the array has to start at zero, because each call writes every word it
//     reads before reading it;
//   * every call uses the same array, which keeps the last call's contents:
//     calls whose work overlaps on the GPU (different streams, or other host
//     threads' calls still running) race on the array;
//   * the array's device address is looked up once per device (the first
//     call on that device, with that device current); cudaDeviceReset after
//     that first call is not supported, as for the library's other
//     per-device state.
#include <cstring>
#include <mutex>

#include "../../include/cumodp.h"
#include "product.cuh"

namespace cmb {

namespace {

constexpr int kNaMaxLog = 20;
constexpr size_t kNaAlign = 64;  // words: keeps every region 256-byte aligned
constexpr size_t align_up(size_t x) { return (x + kNaAlign - 1) / kNaAlign * kNaAlign; }
constexpr size_t kNaWs = 2ull << kNaMaxLog;          // two transform-length buffers
constexpr size_t kNaRowTw = 2 * (16384 + 4096 + 512) + 2;  // row plan 2^14, both directions
constexpr size_t kNaColTw = 2 * (1024 + 128) + 2;          // column plan 2^10, both directions
constexpr size_t kNaSeeds = 2 * (4096 + 256);              // inter-pass seeds of a 2^20 transform
constexpr size_t kNaOffRow = align_up(kNaWs);
constexpr size_t kNaOffCol = align_up(kNaOffRow + 2 * kNaRowTw);
constexpr size_t kNaOffSeeds = align_up(kNaOffCol + 2 * kNaColTw);
constexpr size_t kNaWords = align_up(kNaOffSeeds + kNaSeeds);

// The scratch array.  In host code this name is only a stand-in for the
// symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) u32 g_noalloc_scratch[kNaWords];

struct NaDevice {
    u32* base = nullptr;  // device address of g_noalloc_scratch on this device
};

std::mutex g_na_m;
NaDevice g_na[64];

// One plan's level tables (the layout of level_tables_into: per level i,
// task o and slot j at off_i + o R_i + j hold w_B^(o bitrev(j)) in Shoup
// form, the forward tables first and the inverse ones nf entries later, then
// two zero words), with w_B and w_B^-1 of every level in Montgomery form.
struct NaPlan {
    Tw* out;
    LevelPlan pl;
    int logl, nf;
    u32 wb[6], wbi[6];
};

// x^e * 2^32 mod p from the Montgomery form xm = x 2^32 (lazy, in [0, 2p)).
__device__ __forceinline__ u32 na_pow_m(u32 xm, u64 e, u32 one_m, u32 p, u32 pinv) {
    u32 acc = one_m;
    for (int b = 63 - __clzll((long long)(e | 1)); b >= 0; --b) {
        acc = mul_mont(acc, acc, p, pinv);
        if ((e >> b) & 1) acc = mul_mont(acc, xm, p, pinv);
    }
    return acc;
}

__device__ __forceinline__ Tw na_level_entry(const NaPlan& P, int t, u32 one_m, u32 p, u32 pinv) {
    const bool inv = t >= P.nf;
    if (inv) t -= P.nf;
    int off = 0, lb = P.logl;
    for (int i = 0; i + 1 < P.pl.nlev; ++i) {
        const int r = P.pl.logr[i];
        if (t < off + (1 << lb)) {
            const int q = t - off, o = q >> r, j = q & ((1 << r) - 1);
            const u32 m = na_pow_m(inv ? P.wbi[i] : P.wb[i], (u64)o * rev_bits((u32)j, r), one_m, p, pinv);
            const u32 v = red1(mul_mont(m, 1u, p, pinv), p);
            return Tw{v, shoup_quot(v, p)};
        }
        off += 1 << lb;
        lb -= r;
    }
    return Tw{0u, 0u};  // the two padding entries after the inverse tables
}

// Every table one product reads, into the scratch array: the row plan's
// level tables, and for a three-pass product the column plan's and the
// inter-pass seeds (seeds_into's layout: lo[e] = w^e 2^32 for e < nlo, then
// hi[e] = w^(4096 e) 2^32 for e < nhi, forward then inverse; wm, wim, w4m,
// wi4m: w, w^-1, w^4096, w^-4096 in Montgomery form).
__global__ void k_na_tables(const NaPlan row, const NaPlan col, u32* seeds, u32 nlo, u32 nhi, u32 wm, u32 wim,
                            u32 w4m, u32 wi4m, u32 p, u32 pinv, u32 one_m) {
    const int nr = row.out ? 2 * row.nf + 2 : 0, nc = col.out ? 2 * col.nf + 2 : 0;
    const int ns = seeds ? (int)(2 * (nlo + nhi)) : 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr + nc + ns; t += gridDim.x * blockDim.x) {
        if (t < nr) {
            row.out[t] = na_level_entry(row, t, one_m, p, pinv);
        } else if (t < nr + nc) {
            col.out[t - nr] = na_level_entry(col, t - nr, one_m, p, pinv);
        } else {
            const u32 s = (u32)(t - nr - nc);
            const bool inv = s >= nlo + nhi;
            const u32 u = inv ? s - (nlo + nhi) : s;
            const u32 base = u < nlo ? (inv ? wim : wm) : (inv ? wi4m : w4m);
            seeds[s] = red1(na_pow_m(base, u < nlo ? u : u - nlo, one_m, p, pinv), p);
        }
    }
}

// The host side of k_na_tables' arguments for one plan (scalars only).
NaPlan na_plan(Tw* out, const LevelPlan& pl, int logl, u32 root, const PrimeInfo& pi) {
    NaPlan P;
    memset(&P, 0, sizeof(P));
    P.out = out;
    P.pl = pl;
    P.logl = logl;
    P.nf = plan_tw_entries(pl, logl);
    const u32 p = pi.p;
    const u32 rinv = powmod_exact(root, (1ull << logl) - 1, p);
    int lb = logl;
    for (int i = 0; i + 1 < pl.nlev; ++i) {
        P.wb[i] = mulmod_exact(powmod_exact(root, 1ull << (logl - lb), p), pi.r1, p);
        P.wbi[i] = mulmod_exact(powmod_exact(rinv, 1ull << (logl - lb), p), pi.r1, p);
        lb -= pl.logr[i];
    }
    return P;
}

}  // namespace

int mul_dev_noalloc(const u32* a, long long la, const u32* b, long long lb, u32* h, long long lh, u32 p,
                    cudaStream_t st) {
    if (la <= 0 || lb <= 0 || lh < 0) return ASSUMPTION_ERROR;
    if (lh == 0) return OK;
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    const int logn = product_logn(la, lb);
    if (logn > kNaMaxLog || logn > pc->info.two_adic) return FFT_SIZE_TOO_LARGE;
    const int dev = current_device();
    if (dev < 0 || dev >= 64) return ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(g_na_m);
    NaDevice& D = g_na[dev];
    if (!D.base) {
        // once per device, with that device current
        cudaError_t ce = cudaGetSymbolAddress((void**)&D.base, g_noalloc_scratch);
        if (ce != cudaSuccess) {
            D.base = nullptr;
            return cuda_err(ce);
        }
    }
    ensure_kernel_attrs();
    const long long n = 1ll << logn;
    const u32 root = canonical_root(*pc, logn);
    const bool large = logn > kMaxSmallLog;
    const int l2 = large ? default_row_log(logn) : logn, l1 = large ? logn - l2 : 0;
    const u32 root_r = large ? powmod_exact(root, 1ull << l1, p) : root;
    Tw* d_row = reinterpret_cast<Tw*>(D.base + kNaOffRow);
    Tw* d_col = reinterpret_cast<Tw*>(D.base + kNaOffCol);
    u32* d_seeds = D.base + kNaOffSeeds;
    // the tables of this (prime, size), written on the caller's stream ahead
    // of the product's kernels (nothing is carried over from earlier calls)
    {
        const PrimeInfo& pi = pc->info;
        const NaPlan rowp = na_plan(d_row, row_plan(l2), l2, root_r, pi);
        NaPlan colp;
        memset(&colp, 0, sizeof(colp));
        u32 nlo = 0, nhi = 0, wm = 0, wim = 0, w4m = 0, wi4m = 0;
        if ((size_t)(2 * rowp.nf + 2) > kNaRowTw) return ASSUMPTION_ERROR;  // the array's row-table region
        if (large) {
            colp = na_plan(d_col, col_plan(l1), l1, powmod_exact(root, 1ull << l2, p), pi);
            if ((size_t)(2 * colp.nf + 2) > kNaColTw || seed_words(logn) > kNaSeeds) return ASSUMPTION_ERROR;
            nlo = (u32)std::min<long long>(n, 4096);
            nhi = (u32)std::max<long long>(1, n / 4096);
            const u32 rinv = powmod_exact(root, (u64)n - 1, p);
            wm = mulmod_exact(root, pi.r1, p);
            wim = mulmod_exact(rinv, pi.r1, p);
            w4m = mulmod_exact(powmod_exact(root, 4096, p), pi.r1, p);
            wi4m = mulmod_exact(powmod_exact(rinv, 4096, p), pi.r1, p);
        }
        k_na_tables<<<2 * sm_count(dev), 256, 0, st>>>(rowp, colp, large ? d_seeds : nullptr, nlo, nhi, wm, wim, w4m,
                                                       wi4m, p, pi.pinv_neg, pi.r1);
        if (cudaError_t ce = cudaGetLastError(); ce != cudaSuccess) return cuda_err(ce);
    }
    if (lh > n) {  // coefficients beyond the transform length are zero
        cudaError_t ce = cudaMemsetAsync(h + n, 0, (size_t)(lh - n) * sizeof(u32), st);
        if (ce != cudaSuccess) return cuda_err(ce);
        lh = n;
    }
    if (!large) {
        SmallArgs A;
        memset(&A, 0, sizeof(A));
        A.pk = pc->pk;
        const u32 linv = powmod_exact((u32)(n % p), p - 2, p);
        A.scale = tw_of(mulmod_exact(linv, pc->info.r1, p), p);
        A.tw = d_row;
        A.tw_inv_off = plan_tw_entries(row_plan(logn), logn);
        A.job0 = ProdJob{a, b, h, (int)la, (int)lb, (int)lh, 0};
        A.njobs = 1;
        launch_small(logn, A, 1, st);
    } else {
        LargeArgs A;
        memset(&A, 0, sizeof(A));
        A.pk = A.pkc = pc->pk;
        A.twr = d_row;
        A.twc = d_col;
        A.twr_inv = plan_tw_entries(row_plan(l2), l2);
        A.twc_inv = plan_tw_entries(col_plan(l1), l1);
        A.seeds = d_seeds;
        A.nlo = (int)std::min<long long>(n, 4096);
        A.nhi = (int)std::max<long long>(1, n / 4096);
        const u32 ninv = powmod_exact((u32)(n % p), p - 2, p);
        A.scale_rn = mulmod_exact(ninv, pc->info.r1, p);
        A.l1 = l1;
        A.l2 = l2;
        A.colpl = col_plan(l1);
        A.r32p = 4294967296.0 / (double)p;
        u32* ws = D.base;  // workspace: the first 2n words of the array
        A.job0 = LargeJob{a, b, h, (int)la, (int)lb, (int)lh, 0, ws, ws + n};
        A.njobs = 1;
        launch_large(A, 1, st);
    }
    return cuda_err(cudaGetLastError());
}

}  // namespace cmb

using namespace cmb;

extern "C" {

cumodp_err cumodp_fftmul_uni_dev_noalloc(sfixn lh, sfixn* H, sfixn df, const sfixn* F, sfixn dg, const sfixn* G,
                                         sfixn p, void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (df < 0 || dg < 0 || lh < 0 || !F || !G || (lh > 0 && !H)) return CUMODP_ASSUMPTION_ERROR;
    cudaStream_t st = (cudaStream_t)stream;
    int e = mul_dev_noalloc((const u32*)F, (long long)df + 1, (const u32*)G, (long long)dg + 1, (u32*)H, lh,
                            (u32)p, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

}  // extern "C"
