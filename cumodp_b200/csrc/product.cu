// Product dispatch: size classes, kernel instantiation tables, launches.
#include "product.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdlib>
#include <cstring>

namespace cmb {

namespace {

template <int LOGL>
void launch_small_t(const SmallArgs& a, int nctas, cudaStream_t st) {
    constexpr int L = 1 << LOGL;
    const size_t smem = (size_t)small_ppc(LOGL) * 2 * L * sizeof(u32);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_small_product<LOGL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_small_product<LOGL><<<nctas, small_threads(LOGL), smem, st>>>(a);
}

typedef void (*SmallFn)(const SmallArgs&, int, cudaStream_t);
const SmallFn kSmall[15] = {nullptr, nullptr, nullptr, nullptr, nullptr,
                            launch_small_t<5>, launch_small_t<6>, launch_small_t<7>,
                            launch_small_t<8>, launch_small_t<9>, launch_small_t<10>,
                            launch_small_t<11>, launch_small_t<12>, launch_small_t<13>,
                            launch_small_t<14>};


// Launch with programmatic stream serialization: the kernel may start while
// the previous kernel of the stream finishes (it calls pdl_wait before
// reading that kernel's results).
template <class K>
void launch_pdl(K kernel, dim3 grid, int threads, size_t smem, cudaStream_t st, const LargeArgs& a) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, a);
}

template <int L1>
void launch_col_fwd_t(const LargeArgs& a, dim3 grid, cudaStream_t st) {
    const size_t smem = col_smem_bytes(L1, false);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_col_fwd<L1, col_warps(L1, false)>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_col_fwd<L1, col_warps(L1, false)><<<grid, col_warps(L1, false) * 32, smem, st>>>(a);
}
}  // namespace

int sm_count(int dev) {
    static int cache[64] = {0};
    if (dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = v > 0 ? v : 148;
    }
    return cache[dev];
}

namespace {

// Whether pass A uses the persistent pipelined kernel where it applies
// (CUMODP_COL_PIPE=0 selects the one-tile-per-CTA kernel, for comparison).
bool col_pipe_enabled() {
    static const bool on = [] {
        const char* e = getenv("CUMODP_COL_PIPE");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <int L1>
void launch_col_fwd_pipe_t(const LargeArgs& a, int ntiles, cudaStream_t st) {
    constexpr int smem = col_pipe_smem_bytes(L1);
    const int grid = std::min(ntiles, sm_count(current_device()) * col_pipe_ctas(L1));
    k_col_fwd_pipe<L1, col_pipe_kind(L1), col_pipe_warps(L1)><<<grid, col_pipe_warps(L1) * 32, smem, st>>>(a);
}

template <int L1>
void launch_col_inv_pipe_t(const LargeArgs& a, int ntiles, cudaStream_t st) {
    const int grid = std::min(ntiles, sm_count(current_device()));
    launch_pdl(k_col_inv_pipe<L1, col_inv_pipe_warps(L1)>, dim3(grid), col_inv_pipe_warps(L1) * 32,
               (size_t)col_inv_pipe_smem_bytes(L1), st, a);
}

template <int L1>
void launch_col_inv_t(const LargeArgs& a, dim3 grid, cudaStream_t st) {
    const size_t smem = col_smem_bytes(L1, true);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_col_inv<L1, col_warps(L1, true)>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    launch_pdl(k_col_inv<L1, col_warps(L1, true)>, grid, col_warps(L1, true) * 32, smem, st, a);
}
template <int L2>
void launch_row_t(const LargeArgs& a, dim3 grid, cudaStream_t st) {
    const size_t smem = (size_t)2 * (1 << L2) * sizeof(u32);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_row_fused<L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_row_fused<L2><<<grid, row_threads(L2), smem, st>>>(a);
}

// Dynamic shared memory of the split row kernels: the row, its level-0
// factor table and the scratch to build the table in place.
template <int L2>
constexpr size_t rowsplit_smem() {
    return (size_t)(1 << L2) * sizeof(u32) + (size_t)RowTab<L2>::TABW * sizeof(Tw) +
           (size_t)RowTab<L2>::NPOW * sizeof(u32);
}

template <int L2>
void launch_rowtab_t(const LargeArgs& a, Tw* out, cudaStream_t st) {
    k_rowtab_build<L2><<<dim3(1u << a.l1, 2), rowsplit_threads(L2), 0, st>>>(a, out);
}
typedef void (*RowTabFn)(const LargeArgs&, Tw*, cudaStream_t);
RowTabFn rowtab_fn(int l2) {
    switch (l2) {
        case 11: return launch_rowtab_t<11>;
        case 12: return launch_rowtab_t<12>;
        case 13: return launch_rowtab_t<13>;
        case 14: return launch_rowtab_t<14>;
        default: return nullptr;
    }
}
size_t rowtab_words(int l2) {
    switch (l2) {
        case 11: return RowTab<11>::TABW;
        case 12: return RowTab<12>::TABW;
        case 13: return RowTab<13>::TABW;
        case 14: return RowTab<14>::TABW;
        default: return 0;
    }
}

// Every slot's level-0 factor tables (both directions) for the transform
// shape of `a`, built once on the device and kept for the process; nullptr
// (the row kernels then build each table themselves) for rows without
// tables or when the memory is not there.
const Tw* row_factor_tables(const LargeArgs& a, int dev, u32 p, u32 root_n, int logn) {
    const RowTabFn fn = rowtab_fn(a.l2);
    if (!fn) return nullptr;
    static const bool off = [] {  // CUMODP_ROWTAB=0: kernels build their tables (for comparison)
        const char* e = getenv("CUMODP_ROWTAB");
        return e && e[0] == '0';
    }();
    if (off) return nullptr;
    static std::mutex m;
    static std::map<std::tuple<int, u32, u32, int, int>, Tw*> cache;
    std::lock_guard<std::mutex> g(m);
    const auto key = std::make_tuple(dev, p, root_n, logn, a.l2);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const size_t bytes = (size_t)2 * ((size_t)1 << a.l1) * rowtab_words(a.l2) * sizeof(Tw);
    Tw* d = nullptr;
    if (dev_malloc((void**)&d, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    const cudaStream_t st = lib_stream(dev);
    fn(a, d, st);
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    account_bytes((long long)bytes);
    cache[key] = d;
    return d;
}
template <int L2>
void launch_row_g_t(const LargeArgs& a, dim3 grid, cudaStream_t st) {
    launch_pdl(k_row_fwd_g<L2>, grid, rowsplit_threads(L2), rowsplit_smem<L2>(), st, a);
}
template <int L2>
void launch_row_f_t(const LargeArgs& a, dim3 grid, cudaStream_t st) {
    launch_pdl(k_row_mul_f<L2>, grid, rowsplit_threads(L2), rowsplit_smem<L2>(), st, a);
}

typedef void (*PassFn)(const LargeArgs&, dim3, cudaStream_t);
const PassFn kColFwd[12] = {nullptr, launch_col_fwd_t<1>, launch_col_fwd_t<2>, launch_col_fwd_t<3>,
                            launch_col_fwd_t<4>, launch_col_fwd_t<5>, launch_col_fwd_t<6>,
                            launch_col_fwd_t<7>, launch_col_fwd_t<8>, launch_col_fwd_t<9>,
                            launch_col_fwd_t<10>, launch_col_fwd_t<11>};
const PassFn kColInv[12] = {nullptr, launch_col_inv_t<1>, launch_col_inv_t<2>, launch_col_inv_t<3>,
                            launch_col_inv_t<4>, launch_col_inv_t<5>, launch_col_inv_t<6>,
                            launch_col_inv_t<7>, launch_col_inv_t<8>, launch_col_inv_t<9>,
                            launch_col_inv_t<10>, launch_col_inv_t<11>};
const PassFn kRow[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                         launch_row_t<6>, launch_row_t<7>, launch_row_t<8>, launch_row_t<9>,
                         launch_row_t<10>, launch_row_t<11>, launch_row_t<12>, launch_row_t<13>,
                         launch_row_t<14>};

template <int LOGL>
void attr_small() {
    cudaFuncSetAttribute(k_small_product<LOGL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)((size_t)small_ppc(LOGL) * 2 * (1 << LOGL) * sizeof(u32)));
}
template <int L1>
void attr_col() {
    cudaFuncSetAttribute(k_col_fwd<L1, col_warps(L1, false)>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         col_smem_bytes(L1, false));
    cudaFuncSetAttribute(k_col_inv<L1, col_warps(L1, true)>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         col_smem_bytes(L1, true));
}
void attr_col_pipe1() {
    cudaFuncSetAttribute(k_col_fwd_pipe1<10, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         col_pipe1_smem_bytes(10));
}
template <int L1>
void attr_col_pipe() {
    cudaFuncSetAttribute(k_col_fwd_pipe<L1, col_pipe_kind(L1), col_pipe_warps(L1)>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         col_pipe_smem_bytes(L1));
    cudaFuncSetAttribute(k_col_inv_pipe<L1, col_inv_pipe_warps(L1)>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         col_inv_pipe_smem_bytes(L1));
}
template <int L2>
void attr_row() {
    cudaFuncSetAttribute(k_row_fused<L2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         2 * (1 << L2) * (int)sizeof(u32));
}

template <int L2>
void attr_rowsplit() {
    const int smem = (int)rowsplit_smem<L2>();
    cudaFuncSetAttribute(k_row_fwd_g<L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_row_mul_f<L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

const PassFn kRowG[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                          launch_row_g_t<6>, launch_row_g_t<7>, launch_row_g_t<8>, launch_row_g_t<9>,
                          launch_row_g_t<10>, launch_row_g_t<11>, launch_row_g_t<12>, launch_row_g_t<13>,
                          launch_row_g_t<14>};
const PassFn kRowF[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                          launch_row_f_t<6>, launch_row_f_t<7>, launch_row_f_t<8>, launch_row_f_t<9>,
                          launch_row_f_t<10>, launch_row_f_t<11>, launch_row_f_t<12>, launch_row_f_t<13>,
                          launch_row_f_t<14>};

int ceil_log2(long long s) {
    int k = 0;
    while ((1ll << k) < s) ++k;
    return k;
}

}  // namespace

void ensure_kernel_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        attr_small<5>(); attr_small<6>(); attr_small<7>(); attr_small<8>(); attr_small<9>();
        attr_small<10>(); attr_small<11>(); attr_small<12>(); attr_small<13>(); attr_small<14>();
        attr_col<1>(); attr_col<2>(); attr_col<3>(); attr_col<4>(); attr_col<5>();
        attr_col<6>(); attr_col<7>(); attr_col<8>(); attr_col<9>(); attr_col<10>(); attr_col<11>();
        attr_col_pipe<9>(); attr_col_pipe<10>(); attr_col_pipe1();
        attr_row<6>(); attr_row<7>(); attr_row<8>(); attr_row<9>(); attr_row<10>();
        attr_row<11>(); attr_row<12>(); attr_row<13>(); attr_row<14>();
        attr_rowsplit<6>(); attr_rowsplit<7>(); attr_rowsplit<8>(); attr_rowsplit<9>(); attr_rowsplit<10>();
        attr_rowsplit<11>(); attr_rowsplit<12>(); attr_rowsplit<13>(); attr_rowsplit<14>();
    });
}

int product_logn(long long la, long long lb) {
    return std::max(kMinLog, ceil_log2(la + lb - 1));
}

int default_row_log(int logn) {
    // rows of 2^l2 words, columns of 2^(logn-l2): the split with the shortest
    // single-product time measured on B200 for each length 2^15..2^24 (a
    // batch's own splits come from the autotuner)
    static const int kBest[25] = {7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7,
                                  7, 11, 12, 13, 14, 10, 11, 12, 14, 14};
    if (logn >= 0 && logn <= 24) return kBest[logn];
    int l2 = std::max(logn - kDefaultColLog, 7);
    return std::min(l2, kMaxRowLog);
}

int small_args(const PrimeCtx& pc, u32 root, int logn, int dev, SmallArgs* a) {
    int err = OK;
    const Tw* tw = row_tables(dev, pc.info.p, root, logn, &err);
    if (!tw) return err;
    const u32 p = pc.info.p;
    memset(a, 0, sizeof(*a));
    a->pk = pc.pk;
    // 2^32 / L: undoes the Montgomery 2^-32 of the pointwise product and
    // the factor L of the unnormalised inverse
    const u32 linv = powmod_exact((u32)((1ull << logn) % p), p - 2, p);
    a->scale = tw_of(mulmod_exact(linv, pc.info.r1, p), p);
    a->tw = tw;
    a->tw_inv_off = plan_tw_entries(row_plan(logn), logn);
    return OK;
}

int large_args(const PrimeCtx& pc, u32 root_n, int logn, int l2, int dev, LargeArgs* a) {
    int err = OK;
    const u32 p = pc.info.p;
    const int l1 = logn - l2;
    const u32 root_r = powmod_exact(root_n, 1ull << l1, p);  // w_n2
    const u32 root_c = powmod_exact(root_n, 1ull << l2, p);  // w_n1
    const Tw* twr = row_tables(dev, p, root_r, l2, &err);
    const Tw* twc = col_tables(dev, p, root_c, l1, &err);
    const u32* seeds = seed_tables(dev, p, root_n, logn, &err);
    if (!twr || !twc || !seeds) return err ? err : OUT_OF_MEMORY;
    memset(a, 0, sizeof(*a));
    a->pk = pc.pk;
    a->pkc = pc.pk;
    a->twr = twr;
    a->twc = twc;
    a->twr_inv = plan_tw_entries(row_plan(l2), l2);
    a->twc_inv = plan_tw_entries(col_plan(l1), l1);
    a->seeds = seeds;
    a->nlo = (int)std::min<long long>(1ll << logn, 4096);
    a->nhi = (int)std::max<long long>(1, (1ll << logn) / 4096);
    const u32 ninv = powmod_exact((u32)((1ull << logn) % p), p - 2, p);
    a->scale_rn = mulmod_exact(ninv, pc.info.r1, p);
    a->l1 = l1;
    a->l2 = l2;
    a->colpl = col_plan(l1);
    a->r32p = 4294967296.0 / (double)p;
    const char* rf = getenv("CUMODP_ROW_FUSED");
    a->row_fused = rf && rf[0] == '1';
    a->rowtab = row_factor_tables(*a, dev, p, root_n, logn);
    return OK;
}

// Pass-timing names: kernel and the log2 of its transform dimension.
static const char* kSmallName[15] = {"", "", "", "", "", "small_product_5", "small_product_6",
    "small_product_7", "small_product_8", "small_product_9", "small_product_10", "small_product_11",
    "small_product_12", "small_product_13", "small_product_14"};
static const char* kColFwdName[12] = {"", "col_fwd_1", "col_fwd_2", "col_fwd_3", "col_fwd_4", "col_fwd_5",
    "col_fwd_6", "col_fwd_7", "col_fwd_8", "col_fwd_9", "col_fwd_10", "col_fwd_11"};
static const char* kColInvName[12] = {"", "col_inv_1", "col_inv_2", "col_inv_3", "col_inv_4", "col_inv_5",
    "col_inv_6", "col_inv_7", "col_inv_8", "col_inv_9", "col_inv_10", "col_inv_11"};
static const char* kRowGName[15] = {"", "", "", "", "", "", "row_fwd_g_6", "row_fwd_g_7", "row_fwd_g_8",
    "row_fwd_g_9", "row_fwd_g_10", "row_fwd_g_11", "row_fwd_g_12", "row_fwd_g_13", "row_fwd_g_14"};
static const char* kRowFName[15] = {"", "", "", "", "", "", "row_mul_f_6", "row_mul_f_7", "row_mul_f_8",
    "row_mul_f_9", "row_mul_f_10", "row_mul_f_11", "row_mul_f_12", "row_mul_f_13", "row_mul_f_14"};
static const char* kRowName[15] = {"", "", "", "", "", "", "row_fused_6", "row_fused_7", "row_fused_8",
    "row_fused_9", "row_fused_10", "row_fused_11", "row_fused_12", "row_fused_13", "row_fused_14"};

void launch_small(int logn, const SmallArgs& a, int njobs, cudaStream_t st) {
    const int ppc = small_ppc(logn);
    NvtxRange range(kSmallName[logn]);
    cudaEvent_t e0;
    const bool tr = pass_timing_begin(st, &e0);
    kSmall[logn](a, (njobs + ppc - 1) / ppc, st);
    if (tr) pass_timing_end(st, kSmallName[logn], e0);
}

bool launch_col_fwd_pipe(const LargeArgs& a, int njobs, cudaStream_t st) {
    if (!col_pipe_ok(a.l1) || !col_pipe_enabled()) return false;
    const int ntiles = ((1 << a.l2) / col_tile_cols_rt(a.l1, col_pipe_kind(a.l1))) * 2 * njobs;
    if (a.l1 == 10) launch_col_fwd_pipe_t<10>(a, ntiles, st);
    else launch_col_fwd_pipe_t<9>(a, ntiles, st);
    return true;
}

bool launch_col_fwd_pipe1(const LargeArgs& a, int njobs, cudaStream_t st) {
    if (a.l1 != 10 || !col_pipe_enabled()) return false;
    ensure_kernel_attrs();
    const int ntiles = ((1 << a.l2) / col_tile_cols_rt(10, 2)) * njobs;
    const int grid = std::min(ntiles, sm_count(current_device()));
    k_col_fwd_pipe1<10, 16><<<grid, 16 * 32, col_pipe1_smem_bytes(10), st>>>(a);
    return true;
}

void launch_large(const LargeArgs& a, int njobs, cudaStream_t st) {
    const int n1 = 1 << a.l1, n2 = 1 << a.l2;
    NvtxRange range(kRowFName[a.l2]);  // the product's three passes, named by its dominant kernel
    cudaEvent_t e0;
    bool tr = pass_timing_begin(st, &e0);
    if (!launch_col_fwd_pipe(a, njobs, st)) kColFwd[a.l1](a, dim3(n2 / col_tile_cols_rt(a.l1, false), 2, njobs), st);
    if (tr) pass_timing_end(st, kColFwdName[a.l1], e0);
    if (a.row_fused) {
        tr = pass_timing_begin(st, &e0);
        kRow[a.l2](a, dim3(n1, njobs, 1), st);
        if (tr) pass_timing_end(st, kRowName[a.l2], e0);
    } else {
        tr = pass_timing_begin(st, &e0);
        kRowG[a.l2](a, dim3(n1, njobs, 1), st);
        if (tr) pass_timing_end(st, kRowGName[a.l2], e0);
        tr = pass_timing_begin(st, &e0);
        kRowF[a.l2](a, dim3(n1, njobs, 1), st);
        if (tr) pass_timing_end(st, kRowFName[a.l2], e0);
    }
    tr = pass_timing_begin(st, &e0);
    if (col_pipe_ok(a.l1) && col_pipe_enabled()) {
        const int ntiles = (n2 / col_tile_cols_rt(a.l1, true)) * njobs;
        if (a.l1 == 10) launch_col_inv_pipe_t<10>(a, ntiles, st);
        else launch_col_inv_pipe_t<9>(a, ntiles, st);
    } else {
        kColInv[a.l1](a, dim3(n2 / col_tile_cols_rt(a.l1, true), 1, njobs), st);
    }
    if (tr) pass_timing_end(st, kColInvName[a.l1], e0);
}

// h[i] = (h[i] + t[i]) mod p for i < len; both in [0, p).
__global__ void k_add_mod(u32* __restrict__ h, const u32* __restrict__ t, long long len, u32 p) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
         i += (long long)gridDim.x * blockDim.x)
        h[i] = red1(h[i] + t[i], p);
}

size_t mul_ws_words(int logn) {
    // direct: the two n-word arrays of the three passes; split: those of a
    // 2^kMaxLog piece plus the piece's product
    return logn <= kMaxLog ? (size_t)2 << logn : (size_t)3 << kMaxLog;
}

namespace {

// A product whose transform is longer than 2^kMaxLog.  Each operand is cut
// into pieces of 2^(kMaxLog-1) coefficients; every pair of pieces (i, j)
// is multiplied by the three-pass kernels (a transform of at most
// 2^kMaxLog) and added into h at offset i + j.  At most four pairs for
// balanced operands of a 2^26 product.  An operand that overlaps h is first
// copied aside (h is cleared before the pieces are added).
int mul_split_dev(const u32* a, long long la, const u32* b, long long lb, u32* h, long long lh, u32 p,
                  cudaStream_t st) {
    const long long C = 1ll << (kMaxLog - 1);
    const int dev = current_device();
    int err = OK;
    auto overlaps = [&](const u32* x, long long lx) { return x < h + lh && h < x + lx; };
    if (overlaps(a, la) || overlaps(b, lb)) {
        u32* in = (u32*)workspace(dev, kWsSplitIn, (size_t)(la + lb) * sizeof(u32), &err);
        if (!in) return err;
        cudaError_t e = cudaMemcpyAsync(in, a, (size_t)la * sizeof(u32), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(in + la, b, (size_t)lb * sizeof(u32), cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_err(e);
        a = in;
        b = in + la;
    }
    u32* t = (u32*)workspace(dev, kWsSplitProd, (size_t)(2 * C) * sizeof(u32), &err);
    if (!t) return err;
    cudaError_t e = cudaMemsetAsync(h, 0, (size_t)lh * sizeof(u32), st);
    if (e != cudaSuccess) return cuda_err(e);
    const int grid = 4 * sm_count(dev);
    for (long long i = 0; i < la; i += C)
        for (long long j = 0; j < lb; j += C) {
            const long long off = i + j;
            if (off >= lh) continue;
            const long long li = std::min(C, la - i), lj = std::min(C, lb - j);
            const long long lt = std::min(li + lj - 1, lh - off);
            if ((err = mul_dev(a + i, li, b + j, lj, t, lt, p, st)) != OK) return err;
            k_add_mod<<<grid, 256, 0, st>>>(h + off, t, lt, p);
        }
    return cuda_err(cudaGetLastError());
}

}  // namespace

namespace {

// h[0..lh) = a * b mod (x^n - 1, p) with n = 2^logn (kMinLog <= logn <=
// kMaxLog, la, lb <= n): one forward transform of each operand, the
// pointwise product and the inverse transform -- the linear product when
// la + lb - 1 <= n, the cyclic convolution otherwise (the forward column
// passes take operands of any length up to n).
int mul_dev_len(const u32* a, long long la, const u32* b, long long lb, u32* h, long long lh, u32 p, int logn,
                const PrimeCtx& pc, cudaStream_t st) {
    int err = OK;
    const long long n = 1ll << logn;
    const int dev = current_device();
    ensure_kernel_attrs();
    if (lh > n) {  // coefficients beyond the transform length are zero
        cudaError_t e = cudaMemsetAsync(h + n, 0, (size_t)(lh - n) * sizeof(u32), st);
        if (e != cudaSuccess) return cuda_err(e);
        lh = n;
    }
    const u32 root = canonical_root(pc, logn);
    if (logn <= kMaxSmallLog && logn < single_large_min_log()) {
        SmallArgs A;
        if ((err = small_args(pc, root, logn, dev, &A)) != OK) return err;
        A.job0 = ProdJob{a, b, h, (int)la, (int)lb, (int)lh, 0};
        A.njobs = 1;
        launch_small(logn, A, 1, st);
    } else {
        const int l2 = default_row_log(logn);
        LargeArgs A;
        if ((err = large_args(pc, root, logn, l2, dev, &A)) != OK) return err;
        u32* ws = (u32*)workspace(dev, kWsSingle, (size_t)2 * n * sizeof(u32), &err);
        if (!ws) return err;
        A.job0 = LargeJob{a, b, h, (int)la, (int)lb, (int)lh, 0, ws, ws + n};
        A.njobs = 1;
        launch_large(A, 1, st);
    }
    return cuda_err(cudaGetLastError());
}

}  // namespace

int mul_dev(const u32* a, long long la, const u32* b, long long lb, u32* h, long long lh, u32 p,
            cudaStream_t st) {
    if (la <= 0 || lb <= 0 || lh < 0) return ASSUMPTION_ERROR;
    if (lh == 0) return OK;
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    const int logn = product_logn(la, lb);
    if (logn > pc->info.two_adic) return FFT_SIZE_TOO_LARGE;
    if (logn > kMaxSplitLog) return FFT_SIZE_TOO_LARGE;
    if (logn > kMaxLog) return mul_split_dev(a, la, b, lb, h, lh, p, st);
    return mul_dev_len(a, la, b, lb, h, lh, p, logn, *pc, st);
}

int cyclic_mul_dev(u32* f, const u32* g, int e, u32 p, cudaStream_t st) {
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    if (e < 0) return ASSUMPTION_ERROR;
    if (e > pc->info.two_adic || e > kMaxSplitLog) return FFT_SIZE_TOO_LARGE;
    if (e < kMinLog || e > kMaxLog) return cyclic_mul_compose(f, g, e, p, st);
    const long long n = 1ll << e;
    return mul_dev_len(f, n, g, n, f, n, p, e, *pc, st);
}

}  // namespace cmb
