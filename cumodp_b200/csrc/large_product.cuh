// Three-pass product for transform lengths n = n1 * n2 > 2^14.
//
// The reference runs log2(n) radix-2 Stockham steps, each three HBM round
// trips (src/stockham.cu:437-453).  Here the length-n transform is the
// four-step split x[r*n2 + c]: a length-n1 DFT down every column, a twiddle
// w_n^(c*k1), and a length-n2 DFT along every row.  The whole product needs
// three passes over HBM:
//   A  k_col_fwd    column DFTs of both operands (tile of 32 columns x n1
//                   rows in shared memory; the zero pad is never read);
//   B  k_row_fused  per row: twiddle, row DFT of both operands, pointwise
//                   product, inverse row DFT, inverse twiddle with the 1/n
//                   scale folded in;
//   C  k_col_inv    inverse column DFTs, truncation, canonical residues.
// Rows leave pass A in digit-reversed order of k1 and are consumed in that
// order by passes B and C, so nothing is ever permuted.
#pragma once
#include "small_product.cuh"

namespace cmb {

struct LargeJob {
    const u32* a;
    const u32* b;
    u32* h;
    int la, lb, lh;
    int pad;
    u32* wa;  // workspace, n words: column spectra of a, then the row pass output
    u32* wb;  // workspace, n words: column spectra of b
};

struct LargeArgs {
    PrimeK pk;                   // row transform constants (root w_n2)
    PrimeK pkc;                  // column transform constants (root w_n1)
    const Tw* __restrict__ twr;  // row plan tables (length n2)
    const Tw* __restrict__ twc;  // column plan tables (length n1)
    int twr_inv, twc_inv;        // inverse table offsets
    const u32* __restrict__ seeds;  // w_n^e * 2^32 mod p: lo_f, hi_f, lo_i, hi_i
    int nlo, nhi;
    u32 scale_rn;                // 2^32 / n mod p
    int l1, l2;                  // n1 = 2^l1 (columns), n2 = 2^l2 (rows)
    const LargeJob* __restrict__ jobs;  // device job table, or nullptr: use job0
    int njobs;
    LevelPlan colpl;             // column plan (row slot -> k1 map)
    int row_fused;               // 1: one fused row kernel; 0: the split pair
    LargeJob job0;
};

#ifdef __CUDACC__

template <int LOGL, int LEV>
struct ColLevel {
    static constexpr LevelPlan PL = col_plan(LOGL);
    static constexpr int R = 1 << PL.logr[LEV];
    static constexpr int LOGB = [] {
        int lb = LOGL;
        for (int i = 0; i < LEV; ++i) lb -= PL.logr[i];
        return lb;
    }();
    static constexpr int B = 1 << LOGB;
    static constexpr int TB = B / R;
    static constexpr int TWOFF = [] {
        int n = 0, lb = LOGL;
        for (int i = 0; i < LEV; ++i) { n += 1 << lb; lb -= PL.logr[i]; }
        return n;
    }();
};

// Row slot -> frequency index k1 of the column transform (digit reversal of
// the column plan).
__host__ __device__ __forceinline__ u32 col_slot_to_k1(u32 s, const LevelPlan& PL, int L1) {
    u32 k = 0, mul = 1;
    int lb = L1;
    for (int i = 0; i < PL.nlev; ++i) {
        const int r = PL.logr[i];
        lb -= r;
        const u32 j = (s >> lb) & ((1u << r) - 1);
        k += rev_bits(j, r) * mul;
        mul <<= r;
    }
    return k;
}

// ------------------------------------------------------ column tiles ----
// A column CTA owns a tile of TC = col_tile_cols(L1, INV) adjacent columns x n1
// rows, stored row-major in shared memory (tile_row gives a row's offset).
// The tile is loaded and stored with 16-byte accesses by all threads at
// once, so every load of the tile is in flight together; the levels then run
// on shared memory with lane = column (32-column tiles) or half-warp = task,
// lane % 16 = column (16-column tiles): conflict-free, and every twiddle is a
// broadcast to the (half-)warp.

// Word offset of tile row r.
template <int L1, int INV>
__host__ __device__ __forceinline__ int tile_row(int r) {
    constexpr int TC = col_tile_cols(L1, INV);
    if constexpr (TC == 32) return r * 32;
    else return (r + (r >> col_pad_log(L1))) * TC;
}

// tile_row(row0 + TB * m) - tile_row(row0) for element m of a level task
// with TB rows between its elements (row0 = a multiple of the block size plus
// the task index): a constant.  Every non-last level of a column plan has TB
// a multiple of the padding period; the last level has TB = 1 and blocks of
// exactly one period.
template <int L1, int INV, int TB>
__host__ __device__ __forceinline__ constexpr int tile_step(int m) {
    constexpr int TC = col_tile_cols(L1, INV), PAD = 1 << col_pad_log(L1);
    if constexpr (TC == 32) return TB * m * 32;
    else if constexpr (TB % PAD == 0) return TB * m * TC + (TB / PAD) * m * TC;
    else return m * TC;
}

// Bulk-loads rows [0, n1) x columns [c0, c0 + TC) of src (row stride n2),
// zero beyond `len` elements, reducing every word to [0, 2p) when `reduce`.
// Rows entirely inside `len` take a branch-free 16-byte path when src is
// 16-byte aligned; only the boundary row checks elements one by one, and
// rows entirely past `len` are zero-filled without loads.
// With ASYNC (and no reduction) the full rows are copied with cp.async,
// global to shared without a register round trip.
template <int L1, int INV, int T, bool ASYNC = false>
__device__ __forceinline__ void tile_load(u32* tile, const u32* __restrict__ src, long long len, int c0, int n2,
                                          bool reduce, const PrimeK& pk) {
    constexpr int n1 = 1 << L1, TC = col_tile_cols(L1, INV), QR = TC / 4;
    constexpr int Q = n1 * QR;  // 16-byte quads in the tile
    const bool vec = ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
    // rows [0, rf) lie fully below len; rows [re, n1) fully at or above it
    const long long lc = len - c0;
    const int rf = vec ? (int)(lc >= TC ? min((long long)n1, (lc - TC) / n2 + 1) : 0) : 0;
    const int re = (int)(lc > 0 ? min((long long)n1, (lc - 1) / n2 + 1) : 0);
    if constexpr (ASYNC) {
#pragma unroll 4
        for (int idx = threadIdx.x; idx < rf * QR; idx += T) {
            const int r = idx / QR, q = idx % QR;
            const unsigned dst = (unsigned)__cvta_generic_to_shared(tile + tile_row<L1, INV>(r) + 4 * q);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst),
                         "l"(src + (long long)r * n2 + c0 + 4 * q) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
#pragma unroll 4
    for (int idx = threadIdx.x; idx < (ASYNC ? 0 : rf * QR); idx += T) {
        const int r = idx / QR, q = idx % QR;
        uint4 v = __ldg(reinterpret_cast<const uint4*>(src + (long long)r * n2 + c0 + 4 * q));
        if (reduce) {
            v.x = mul_shoup(v.x, 1u, pk.one_q, pk.p);
            v.y = mul_shoup(v.y, 1u, pk.one_q, pk.p);
            v.z = mul_shoup(v.z, 1u, pk.one_q, pk.p);
            v.w = mul_shoup(v.w, 1u, pk.one_q, pk.p);
        }
        *reinterpret_cast<uint4*>(tile + tile_row<L1, INV>(r) + 4 * q) = v;
    }
    for (int idx = rf * QR + threadIdx.x; idx < re * QR; idx += T) {
        const int r = idx / QR, q = idx % QR;
        const long long gi = (long long)r * n2 + c0 + 4 * q;
        uint4 v;
        v.x = gi < len ? __ldg(src + gi) : 0u;
        v.y = gi + 1 < len ? __ldg(src + gi + 1) : 0u;
        v.z = gi + 2 < len ? __ldg(src + gi + 2) : 0u;
        v.w = gi + 3 < len ? __ldg(src + gi + 3) : 0u;
        if (reduce) {
            v.x = mul_shoup(v.x, 1u, pk.one_q, pk.p);
            v.y = mul_shoup(v.y, 1u, pk.one_q, pk.p);
            v.z = mul_shoup(v.z, 1u, pk.one_q, pk.p);
            v.w = mul_shoup(v.w, 1u, pk.one_q, pk.p);
        }
        *reinterpret_cast<uint4*>(tile + tile_row<L1, INV>(r) + 4 * q) = v;
    }
    for (int idx = re * QR + threadIdx.x; idx < Q; idx += T)
        *reinterpret_cast<uint4*>(tile + tile_row<L1, INV>(idx / QR) + 4 * (idx % QR)) = make_uint4(0u, 0u, 0u, 0u);
    if constexpr (ASYNC) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Bulk-stores the tile; `final` reduces to [0, p) and stops at `len`.
template <int L1, int INV, int T>
__device__ __forceinline__ void tile_store(const u32* tile, u32* __restrict__ dst, long long len, int c0, int n2,
                                           bool final, const PrimeK& pk) {
    constexpr int n1 = 1 << L1, TC = col_tile_cols(L1, INV), QR = TC / 4;
    const bool vec = ((reinterpret_cast<uintptr_t>(dst) & 15) == 0);
    const long long lc = len - c0;
    const int rf = vec ? (int)(lc >= TC ? min((long long)n1, (lc - TC) / n2 + 1) : 0) : 0;
    const int re = (int)(lc > 0 ? min((long long)n1, (lc - 1) / n2 + 1) : 0);
#pragma unroll 4
    for (int idx = threadIdx.x; idx < rf * QR; idx += T) {
        const int r = idx / QR, q = idx % QR;
        uint4 v = *reinterpret_cast<const uint4*>(tile + tile_row<L1, INV>(r) + 4 * q);
        if (final) {
            v.x = red1(red2(v.x, pk.p2), pk.p);
            v.y = red1(red2(v.y, pk.p2), pk.p);
            v.z = red1(red2(v.z, pk.p2), pk.p);
            v.w = red1(red2(v.w, pk.p2), pk.p);
        }
        *reinterpret_cast<uint4*>(dst + (long long)r * n2 + c0 + 4 * q) = v;
    }
    for (int idx = rf * QR + threadIdx.x; idx < re * QR; idx += T) {
        const int r = idx / QR, q = idx % QR;
        const long long gi = (long long)r * n2 + c0 + 4 * q;
        uint4 v = *reinterpret_cast<const uint4*>(tile + tile_row<L1, INV>(r) + 4 * q);
        if (final) {
            v.x = red1(red2(v.x, pk.p2), pk.p);
            v.y = red1(red2(v.y, pk.p2), pk.p);
            v.z = red1(red2(v.z, pk.p2), pk.p);
            v.w = red1(red2(v.w, pk.p2), pk.p);
        }
        if (gi < len) dst[gi] = v.x;
        if (gi + 1 < len) dst[gi + 1] = v.y;
        if (gi + 2 < len) dst[gi + 2] = v.z;
        if (gi + 3 < len) dst[gi + 3] = v.w;
    }
}

// Forward column level LEV, shared memory to shared memory, on a tile of
// kind KIND (col_tile_cols).
template <int L1, int LEV, int NW, int KIND = 0>
__device__ __forceinline__ void col_fwd_level(u32* tile, const PrimeK& pk, const Tw* __restrict__ twc) {
    using LV = ColLevel<L1, LEV>;
    constexpr LevelPlan PL = col_plan(L1);
    constexpr int R = LV::R, TB = LV::TB, B = LV::B;
    constexpr bool LAST = LEV + 1 == PL.nlev;
    constexpr int TASKS = (1 << L1) / R;
    constexpr int INV = KIND;
    constexpr int TC = col_tile_cols(L1, INV), SUB = 32 / TC;
    const u32 p = pk.p, p2 = pk.p2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % TC;
    for (int id = warp * SUB + lane / TC; id < TASKS; id += NW * SUB) {
        const int blk = id / TB, o = id % TB;
        const int row0 = blk * B + o;
        u32 x[R];
        u32* base = tile + tile_row<L1, INV>(row0) + col;
#pragma unroll
        for (int m = 0; m < R; ++m) x[m] = base[tile_step<L1, INV, TB>(m)];
        dif_regs<R, !LAST>(x, pk.rc.f, p, p2);
        if constexpr (!LAST) {
            const Tw* t = twc + LV::TWOFF + o * R;
#pragma unroll
            for (int j = 1; j < R; ++j) {
                const Tw w = t[j];  // uniform across the (half-)warp: broadcast
                x[j] = mul_shoup(x[j], w.w, w.wq, p);
            }
        }
#pragma unroll
        for (int m = 0; m < R; ++m) base[tile_step<L1, INV, TB>(m)] = x[m];
    }
}

template <int L1, int LEV, int NW, int KIND = 0>
__device__ __forceinline__ void col_fwd_levels(u32* tile, const PrimeK& pk, const Tw* __restrict__ twc) {
    constexpr LevelPlan PL = col_plan(L1);
    if constexpr (LEV < PL.nlev) {
        col_fwd_level<L1, LEV, NW, KIND>(tile, pk, twc);
        __syncthreads();
        col_fwd_levels<L1, LEV + 1, NW, KIND>(tile, pk, twc);
    }
}

// Inverse column level LEV (pre-twiddle, DIT), shared memory to shared memory.
template <int L1, int LEV, int NW>
__device__ __forceinline__ void col_inv_level(u32* tile, const PrimeK& pk, const Tw* __restrict__ twci) {
    using LV = ColLevel<L1, LEV>;
    constexpr LevelPlan PL = col_plan(L1);
    constexpr int R = LV::R, TB = LV::TB, B = LV::B;
    constexpr bool DEEPEST = LEV + 1 == PL.nlev;
    constexpr int TASKS = (1 << L1) / R;
    constexpr int INV = 1;
    constexpr int TC = col_tile_cols(L1, INV), SUB = 32 / TC;
    const u32 p = pk.p, p2 = pk.p2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % TC;
    for (int id = warp * SUB + lane / TC; id < TASKS; id += NW * SUB) {
        const int blk = id / TB, o = id % TB;
        const int row0 = blk * B + o;
        u32 x[R];
        u32* base = tile + tile_row<L1, INV>(row0) + col;
#pragma unroll
        for (int m = 0; m < R; ++m) x[m] = base[tile_step<L1, INV, TB>(m)];
        if constexpr (!DEEPEST) {
            const Tw* t = twci + LV::TWOFF + o * R;
#pragma unroll
            for (int j = 1; j < R; ++j) {
                const Tw w = t[j];
                x[j] = mul_shoup(x[j], w.w, w.wq, p);
            }
        }
        dit_regs<R, !DEEPEST>(x, pk.rc.i, p, p2);
#pragma unroll
        for (int m = 0; m < R; ++m) base[tile_step<L1, INV, TB>(m)] = x[m];
    }
}

template <int L1, int LEV, int NW>
__device__ __forceinline__ void col_inv_levels(u32* tile, const PrimeK& pk, const Tw* __restrict__ twci) {
    if constexpr (LEV >= 0) {
        col_inv_level<L1, LEV, NW>(tile, pk, twci);
        __syncthreads();
        col_inv_levels<L1, LEV - 1, NW>(tile, pk, twci);
    }
}

// pass A, grid: (n2/TC column tiles, operands, jobs); KIND 0 for a product's
// operands, 2 for the forward pass of a natural-order transform
template <int L1, int NW, int KIND = 0>
__global__ void __launch_bounds__(NW * 32, col_ctas(L1, KIND)) k_col_fwd(const __grid_constant__ LargeArgs A) {
    extern __shared__ __align__(16) u32 tile[];
    const LargeJob& J = A.jobs ? A.jobs[blockIdx.z] : A.job0;
    const int op = blockIdx.y;
    const u32* src = op ? J.b : J.a;
    const int len = op ? J.lb : J.la;
    u32* dst = op ? J.wb : J.wa;
    const int n2 = 1 << A.l2;
    const int c0 = blockIdx.x * col_tile_cols(L1, KIND);
    // the plan's twiddles (broadcast reads) next to the tile
    constexpr int NTW = col_tw_entries(L1);
    Tw* tws = reinterpret_cast<Tw*>(tile + col_tile_words(L1, KIND));
    for (int i = threadIdx.x; i < NTW; i += NW * 32) tws[i] = A.twc[i];
    // reduced while loaded (an input row half made of padding costs nothing)
    tile_load<L1, KIND, NW * 32>(tile, src, len, c0, n2, true, A.pkc);
    __syncthreads();
    col_fwd_levels<L1, 0, NW, KIND>(tile, A.pkc, tws);
    tile_store<L1, KIND, NW * 32>(tile, dst, 1ll << (L1 + A.l2), c0, n2, false, A.pkc);
}

// pass C, grid: (n2/TC column tiles, 1, jobs)
template <int L1, int NW>
__global__ void __launch_bounds__(NW * 32, col_ctas(L1, true)) k_col_inv(const __grid_constant__ LargeArgs A) {
    extern __shared__ __align__(16) u32 tile[];
    const LargeJob& J = A.jobs ? A.jobs[blockIdx.z] : A.job0;
    const int n2 = 1 << A.l2;
    const int c0 = blockIdx.x * col_tile_cols(L1, true);
    constexpr int NTW = col_tw_entries(L1);
    Tw* tws = reinterpret_cast<Tw*>(tile + col_tile_words(L1, true));
    for (int i = threadIdx.x; i < NTW; i += NW * 32) tws[i] = A.twc[A.twc_inv + i];
    pdl_wait();  // pass B's output
    tile_load<L1, true, NW * 32, true>(tile, J.wa, 1ll << (L1 + A.l2), c0, n2, false, A.pkc);
    __syncthreads();
    col_inv_levels<L1, col_plan(L1).nlev - 1, NW>(tile, A.pkc, tws);
    tile_store<L1, true, NW * 32>(tile, J.h, J.lh, c0, n2, true, A.pkc);
}

// ------------------------------------------------------------- pass B ----
// Shoup pair of w_n^(+-e) (times an optional extra factor) from the seeds.
__device__ __forceinline__ u32 seed_mont(const LargeArgs& A, u32 e, bool inv) {
    const u32* s = A.seeds + (inv ? (A.nlo + A.nhi) : 0);
    return mul_mont(__ldg(s + (e & 4095u)), __ldg(s + A.nlo + (e >> 12)), A.pk.p, A.pk.pinv_neg);
}

template <int L2>
__global__ void __launch_bounds__(row_threads(L2), 1) k_row_fused(const __grid_constant__ LargeArgs A) {
    constexpr int n2 = 1 << L2;
    constexpr int T = row_threads(L2);
    constexpr LevelPlan PL = row_plan(L2);
    static_assert(PL.nlev >= 2, "row pass needs at least two levels");
    using LV0 = SmallLevel<L2, 0>;
    constexpr int R0 = LV0::R, TB0 = LV0::TB;  // level 0: tasks o < TB0 = n2 / R0
    extern __shared__ __align__(16) u32 sm[];   // [F row | G row], swizzled
    __shared__ Tw bf[R0], bi[R0];

    const LargeJob& J = A.jobs ? A.jobs[blockIdx.y] : A.job0;
    const u32 s = blockIdx.x;
    const u32 k1 = col_slot_to_k1(s, A.colpl, A.l1);
    const u32 nmask = (1u << (A.l1 + L2)) - 1;
    const u32 p = A.pk.p, p2 = A.pk.p2, pinv = A.pk.pinv_neg;

    // slot factors w^(+-k1*TB0*m), the inverse one carrying 2^32/n
    if (threadIdx.x < 2 * R0) {
        const bool inv = threadIdx.x >= R0;
        const u32 m = threadIdx.x % R0;
        const u32 e = (k1 * (u32)TB0 * m) & nmask;
        u32 v = red1(mul_mont(seed_mont(A, e, inv), 1u, p, pinv), p);  // plain w^(+-e)
        if (inv) v = (u32)(((u64)v * A.scale_rn) % p);
        const Tw t{v, (u32)(((u64)v << 32) / p)};
        if (inv) bi[m] = t; else bf[m] = t;
    }
    __syncthreads();

    const u32* rowF = J.wa + (size_t)s * n2;
    const u32* rowG = J.wb + (size_t)s * n2;
    RowCtx ctx{A.pk, A.twr, A.twr_inv};

    // both rows into shared memory with 16-byte loads, all in flight at once
#pragma unroll 8
    for (int i = threadIdx.x * 4; i < n2; i += T * 4) {
        const uint4 f = __ldg(reinterpret_cast<const uint4*>(rowF + i));
        const uint4 g = __ldg(reinterpret_cast<const uint4*>(rowG + i));
        *reinterpret_cast<uint4*>(sm + swz(i)) = f;
        *reinterpret_cast<uint4*>(sm + swz(n2 + i)) = g;
    }
    __syncthreads();

    // level 0 forward with the inter-pass twiddle
    for (int o = threadIdx.x; o < TB0; o += T) {
        const u32 mo = seed_mont(A, (k1 * (u32)o) & nmask, false);  // w^(k1 o) * 2^32
        u32 xf[R0], xg[R0];
#pragma unroll
        for (int m = 0; m < R0; ++m) {
            const u32 cm = mul_shoup(mo, bf[m].w, bf[m].wq, p);  // w^(k1 (o + TB0 m)) * 2^32
            xf[m] = mul_mont(sm[swz_task<TB0, n2>(o, swz(o), m)], cm, p, pinv);
            xg[m] = mul_mont(sm[swz_task<TB0, n2>(n2 + o, swz(n2 + o), m)], cm, p, pinv);
        }
        dif_regs<R0, true>(xf, A.pk.rc.f, p, p2);
        dif_regs<R0, true>(xg, A.pk.rc.f, p, p2);
        Tw t[R0];
        load_tw<R0>(t, A.twr + o * R0);
#pragma unroll
        for (int j = 1; j < R0; ++j) {
            xf[j] = mul_shoup(xf[j], t[j].w, t[j].wq, p);
            xg[j] = mul_shoup(xg[j], t[j].w, t[j].wq, p);
        }
#pragma unroll
        for (int m = 0; m < R0; ++m) {
            sm[swz_task<TB0, n2>(o, swz(o), m)] = xf[m];
            sm[swz_task<TB0, n2>(n2 + o, swz(n2 + o), m)] = xg[m];
        }
    }
    __syncthreads();
    small_fwd_levels<L2, 1, T, 1>(sm, ctx);

    // last level: forward DIF of every 32-word row of both operands, then
    // per row the pointwise product (Montgomery; its 2^-32 is undone by the
    // inverse twiddle) and the inverse DIT of that level
    for (int row = threadIdx.x; row < n2 / 16; row += T) {
        u32 x[32];
        load_row32(x, sm, row * 32);  // rows [0, n2/32): F, then G
        dif_regs<32>(x, A.pk.rc.f, p, p2);
        store_row32(sm, row * 32, x);
    }
    __syncthreads();
    for (int row = threadIdx.x; row < n2 / 32; row += T) {
        u32 x[32];
        load_row32(x, sm, row * 32);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const uint4 g = *reinterpret_cast<const uint4*>(sm + swz(n2 + row * 32 + 4 * c));
            x[4 * c] = mul_mont(x[4 * c], g.x, p, pinv);
            x[4 * c + 1] = mul_mont(x[4 * c + 1], g.y, p, pinv);
            x[4 * c + 2] = mul_mont(x[4 * c + 2], g.z, p, pinv);
            x[4 * c + 3] = mul_mont(x[4 * c + 3], g.w, p, pinv);
        }
        dit_regs<32>(x, A.pk.rc.i, p, p2);
        store_row32(sm, row * 32, x);
    }
    __syncthreads();
    small_inv_levels<L2, PL.nlev - 2, T, 1, 1>(sm, ctx);

    // level 0 inverse, inverse twiddle and scale, to global memory
    u32* rowH = J.wa + (size_t)s * n2;
    for (int o = threadIdx.x; o < TB0; o += T) {
        u32 x[R0];
#pragma unroll
        for (int m = 0; m < R0; ++m) x[m] = sm[swz_task<TB0, n2>(o, swz(o), m)];
        Tw t[R0];
        load_tw<R0>(t, A.twr + A.twr_inv + o * R0);
#pragma unroll
        for (int j = 1; j < R0; ++j) x[j] = mul_shoup(x[j], t[j].w, t[j].wq, p);
        dit_regs<R0, true>(x, A.pk.rc.i, p, p2);
        const u32 mo = seed_mont(A, (k1 * (u32)o) & nmask, true);  // w^-(k1 o) * 2^32
#pragma unroll
        for (int m = 0; m < R0; ++m) {
            const u32 d = mul_shoup(mo, bi[m].w, bi[m].wq, p);  // w^-(k1 c) * 2^64 / n
            rowH[o + TB0 * m] = mul_mont(red2(x[m], p2), d, p, pinv);
        }
    }
}


// ------------------------------------------------------------ pass B' ----
// The row pass as two kernels of one operand each, so a CTA needs half the
// shared memory (one 2^14-word row = 64 KiB) and two CTAs share an SM:
//   k_row_fwd_g   row DFT of G' (inter-pass twiddle, all forward levels),
//                 result written over G' in digit-reversed row order;
//   k_row_mul_f   row DFT of F', pointwise product with that row of G^
//                 read from global memory in the same order, inverse row
//                 DFT, inverse twiddle with 2^64/n, result over F'.
// Costs one extra n-word write and read of HBM against the fused pass.

template <int L2>
__device__ __forceinline__ void row_slot_factors(const LargeArgs& A, u32 k1, Tw* bf, Tw* bi) {
    using LV0 = SmallLevel<L2, 0>;
    constexpr int R0 = LV0::R, TB0 = LV0::TB;
    const u32 nmask = (1u << (A.l1 + L2)) - 1;
    const u32 p = A.pk.p, pinv = A.pk.pinv_neg;
    if (threadIdx.x < 2 * R0) {
        const bool inv = threadIdx.x >= R0;
        if (inv && !bi) return;
        const u32 m = threadIdx.x % R0;
        const u32 e = (k1 * (u32)TB0 * m) & nmask;
        u32 v = red1(mul_mont(seed_mont(A, e, inv), 1u, p, pinv), p);  // plain w^(+-e)
        if (inv) v = (u32)(((u64)v * A.scale_rn) % p);
        const Tw t{v, (u32)(((u64)v << 32) / p)};
        if (inv) bi[m] = t; else bf[m] = t;
    }
}

// Loads one row into swizzled shared memory with 16-byte asynchronous
// copies (cp.async: global to shared without a register round trip, all of
// a thread's copies in flight at once); the caller's __syncthreads follows
// the wait.
template <int L2, int T>
__device__ __forceinline__ void row_load(u32* sm, const u32* __restrict__ row) {
    constexpr int n2 = 1 << L2;
#pragma unroll 8
    for (int i = threadIdx.x * 4; i < n2; i += T * 4) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(sm + swz(i));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(row + i) : "memory");
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Level 0 forward of one operand with the inter-pass twiddle w_n^(k1 c).
template <int L2, int T>
__device__ __forceinline__ void row_level0_fwd(u32* sm, const LargeArgs& A, u32 k1, const Tw* bf) {
    using LV0 = SmallLevel<L2, 0>;
    constexpr int R0 = LV0::R, TB0 = LV0::TB;
    const u32 nmask = (1u << (A.l1 + L2)) - 1;
    const u32 p = A.pk.p, p2 = A.pk.p2, pinv = A.pk.pinv_neg;
    for (int o = threadIdx.x; o < TB0; o += T) {
        Tw t[R0];
        load_tw<R0>(t, A.twr + o * R0);
        const u32 mo = seed_mont(A, (k1 * (u32)o) & nmask, false);  // w^(k1 o) * 2^32
        u32 x[R0];
#pragma unroll
        for (int m = 0; m < R0; ++m)
            x[m] = mul_mont(sm[swz_task<TB0, (1 << L2)>(o, swz(o), m)], mul_shoup(mo, bf[m].w, bf[m].wq, p), p, pinv);
        dif_regs<R0, true>(x, A.pk.rc.f, p, p2);
#pragma unroll
        for (int j = 1; j < R0; ++j) x[j] = mul_shoup(x[j], t[j].w, t[j].wq, p);
#pragma unroll
        for (int m = 0; m < R0; ++m) sm[swz_task<TB0, (1 << L2)>(o, swz(o), m)] = x[m];
    }
}

template <int L2>
__global__ void __launch_bounds__(rowsplit_threads(L2), rowsplit_ctas(L2)) k_row_fwd_g(const __grid_constant__ LargeArgs A) {
    constexpr int n2 = 1 << L2;
    constexpr int T = rowsplit_threads(L2);
    constexpr LevelPlan PL = row_plan(L2);
    static_assert(PL.nlev >= 2, "row pass needs at least two levels");
    constexpr int R0 = SmallLevel<L2, 0>::R;
    extern __shared__ __align__(16) u32 sm[];
    __shared__ Tw bf[R0];
    const LargeJob& J = A.jobs ? A.jobs[blockIdx.y] : A.job0;
    const u32 s = blockIdx.x;
    const u32 k1 = col_slot_to_k1(s, A.colpl, A.l1);
    const u32 p = A.pk.p, p2 = A.pk.p2;
    u32* row = J.wb + (size_t)s * n2;
    pdl_trigger();
    row_slot_factors<L2>(A, k1, bf, nullptr);
    pdl_wait();  // pass A's columns of G
    row_load<L2, T>(sm, row);
    __syncthreads();
    row_level0_fwd<L2, T>(sm, A, k1, bf);
    __syncthreads();
    fwd1_levels<L2, 1, T>(sm, A.pk, A.twr);
    for (int r = threadIdx.x; r < n2 / 32; r += T) {
        u32 x[32];
        load_row32(x, sm, r * 32);
        dif_regs<32>(x, A.pk.rc.f, p, p2);
        // store this 32-word row of the spectrum straight to global memory
#pragma unroll
        for (int c = 0; c < 8; ++c)
            *reinterpret_cast<uint4*>(row + r * 32 + 4 * c) =
                make_uint4(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);
    }
}

template <int L2>
__global__ void __launch_bounds__(rowsplit_threads(L2), rowsplit_ctas(L2)) k_row_mul_f(const __grid_constant__ LargeArgs A) {
    constexpr int n2 = 1 << L2;
    constexpr int T = rowsplit_threads(L2);
    constexpr LevelPlan PL = row_plan(L2);
    static_assert(PL.nlev >= 2, "row pass needs at least two levels");
    using LV0 = SmallLevel<L2, 0>;
    constexpr int R0 = LV0::R, TB0 = LV0::TB;
    extern __shared__ __align__(16) u32 sm[];
    __shared__ Tw bf[R0], bi[R0];
    const LargeJob& J = A.jobs ? A.jobs[blockIdx.y] : A.job0;
    const u32 s = blockIdx.x;
    const u32 k1 = col_slot_to_k1(s, A.colpl, A.l1);
    const u32 nmask = (1u << (A.l1 + L2)) - 1;
    const u32 p = A.pk.p, p2 = A.pk.p2, pinv = A.pk.pinv_neg;
    u32* rowF = J.wa + (size_t)s * n2;
    const u32* rowG = J.wb + (size_t)s * n2;
    RowCtx ctx{A.pk, A.twr, A.twr_inv};
    pdl_trigger();
    // F's forward row pass depends only on pass A (complete before the
    // previous kernel, G's row pass, started), so it runs while that kernel
    // finishes; G's spectrum is read after pdl_wait
    row_slot_factors<L2>(A, k1, bf, bi);
    row_load<L2, T>(sm, rowF);
    __syncthreads();
    row_level0_fwd<L2, T>(sm, A, k1, bf);
    __syncthreads();
    fwd1_levels<L2, 1, T>(sm, A.pk, A.twr);
    pdl_wait();
    for (int r = threadIdx.x; r < n2 / 32; r += T) {
        u32 x[32];
        load_row32(x, sm, r * 32);
        dif_regs<32>(x, A.pk.rc.f, p, p2);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const uint4 g = __ldg(reinterpret_cast<const uint4*>(rowG + r * 32 + 4 * c));
            x[4 * c] = mul_mont(x[4 * c], g.x, p, pinv);
            x[4 * c + 1] = mul_mont(x[4 * c + 1], g.y, p, pinv);
            x[4 * c + 2] = mul_mont(x[4 * c + 2], g.z, p, pinv);
            x[4 * c + 3] = mul_mont(x[4 * c + 3], g.w, p, pinv);
        }
        dit_regs<32>(x, A.pk.rc.i, p, p2);
        store_row32(sm, r * 32, x);
    }
    __syncthreads();
    small_inv_levels<L2, PL.nlev - 2, T, 1, 1>(sm, ctx);
    for (int o = threadIdx.x; o < TB0; o += T) {
        u32 x[R0];
#pragma unroll
        for (int m = 0; m < R0; ++m) x[m] = sm[swz_task<TB0, n2>(o, swz(o), m)];
        Tw t[R0];
        load_tw<R0>(t, A.twr + A.twr_inv + o * R0);
#pragma unroll
        for (int j = 1; j < R0; ++j) x[j] = mul_shoup(x[j], t[j].w, t[j].wq, p);
        dit_regs<R0, true>(x, A.pk.rc.i, p, p2);
        const u32 mo = seed_mont(A, (k1 * (u32)o) & nmask, true);  // w^-(k1 o) * 2^32
#pragma unroll
        for (int m = 0; m < R0; ++m) {
            const u32 d = mul_shoup(mo, bi[m].w, bi[m].wq, p);  // w^-(k1 c) * 2^64 / n
            rowF[o + TB0 * m] = mul_mont(red2(x[m], p2), d, p, pinv);
        }
    }
}

#endif  // __CUDACC__

}  // namespace cmb
