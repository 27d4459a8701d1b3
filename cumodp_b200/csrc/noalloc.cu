// A product entry point that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: code that runs while
// another component is capturing the device's work into a CUDA graph, a
// service whose device memory is owned by its own pool allocator and may not
// be allocated behind its back, or a plugin loaded into a host that has
// already partitioned all device memory.  cumodp_fftmul_uni_dev_noalloc
// serves them: the caller passes device buffers for the operands and the
// result, and everything else the product needs -- the three-pass workspace
// and the twiddle tables -- lives in one fixed array in the library's own
// device data segment (g_noalloc_scratch below, about 8.4 MiB), which every
// GPU that loads the library holds until the process exits.
//
// Limits and sharing:
//   * products with df + dg + 1 <= 2^20 (transform length <= 2^20); larger
//     requests are rejected with CUMODP_FFT_SIZE_TOO_LARGE;
//   * every call uses the same array, which keeps the last call's contents
//     (the workspace of the last product and the tables of the last
//     (prime, size)); nothing in it has to start at zero because each call
//     writes every word it reads;
//   * calls whose work overlaps on the GPU (different streams, or other host
//     threads' calls still running) race on the array.
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
    u32 key_p = 0;        // (prime, size) whose tables the array holds
    int key_logn = -1;
};

std::mutex g_na_m;
NaDevice g_na[64];

// Host staging for the tables: fixed storage, nothing allocated per call.
Tw g_host_row[kNaRowTw];
Tw g_host_col[kNaColTw];
u32 g_host_seeds[kNaSeeds];

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
    if (D.key_p != p || D.key_logn != logn) {
        // tables of this (prime, size) into the array; the pageable source
        // is staged by the copy before the call returns
        if ((err = level_tables_into(0, p, root_r, l2, g_host_row, kNaRowTw)) != OK) return err;
        cudaError_t ce = cudaMemcpyAsync(d_row, g_host_row, level_tables_entries(0, l2) * sizeof(Tw),
                                         cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess && large) {
            const u32 root_c = powmod_exact(root, 1ull << l2, p);
            if ((err = level_tables_into(1, p, root_c, l1, g_host_col, kNaColTw)) != OK) return err;
            if ((err = seeds_into(p, root, logn, g_host_seeds, kNaSeeds)) != OK) return err;
            ce = cudaMemcpyAsync(d_col, g_host_col, level_tables_entries(1, l1) * sizeof(Tw),
                                 cudaMemcpyHostToDevice, st);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(d_seeds, g_host_seeds, seed_words(logn) * sizeof(u32), cudaMemcpyHostToDevice,
                                     st);
        }
        if (ce != cudaSuccess) {
            D.key_logn = -1;
            return cuda_err(ce);
        }
        D.key_p = p;
        D.key_logn = logn;
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
