// Three-pass product for transform lengths n = n1 * n2 > 2^14.
//
// The reference runs log2(n) radix-2 Stockham steps, each three HBM round
// trips (src/stockham.cu:437-453).  Here the length-n transform is the
// four-step split x[r*n2 + c]: a length-n1 DFT down every column, a twiddle
// w_n^(c*k1), and a length-n2 DFT along every row.  The whole product needs
// three passes over HBM:
//   A  column DFTs of both operands: k_col_fwd_pipe (persistent, the next
//      tile staged while the current one is transformed) for 2^9- and
//      2^10-row columns, k_col_fwd (one tile per CTA) otherwise; the zero
//      pad is never read;
//   B  per row: twiddle, row DFT of both operands, pointwise product,
//      inverse row DFT, inverse twiddle with the 1/n scale folded in: the
//      split pair k_row_fwd_g + k_row_mul_f (one operand row per CTA; level
//      0 reads per-slot factor tables built once by k_rowtab_build), or
//      k_row_fused (both rows in one CTA, for comparison);
//   C  inverse column DFTs, truncation, canonical residues: k_col_inv_pipe
//      or k_col_inv, as for pass A.
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
    double r32p;                 // 2^32 / p (estimate for Shoup quotients on the device)
    const Tw* __restrict__ rowtab;  // per-slot level-0 factor tables (RowTab), or nullptr
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

// Pass A as a persistent, software-pipelined kernel for the two-level
// column plans (n1 = 2^9, 2^10), on tiles of the layout `KIND` (0: 32
// columns, one per lane; 2: 16 columns, one task per half-warp, padded rows).
// Each CTA walks the tiles gridDim.x apart; while it transforms one tile,
// rows [0, n1/2) of its next tile are already on their way into a staging
// buffer (cp.async, zero-filled past the operand's end), so the SM does not
// wait for HBM between tiles.  A product's operands are usually at most n/2
// words long: their rows [n1/2, n1) are zero and the first level skips that
// half.  Level 0 reads the stage and writes the tile; the last level reads
// the tile and stores its outputs straight to HBM (each warp store covers
// whole row segments).  A longer operand also has rows [n1/2, n1) copied
// into the tile before level 0, which then reads them there.  Sources that
// are not 16-byte aligned are copied word by word.  Results are those of
// k_col_fwd (same levels, same output layout).
template <int L1, int KIND, int NW>
__global__ void __launch_bounds__(NW * 32, col_pipe_ctas(L1)) k_col_fwd_pipe(const __grid_constant__ LargeArgs A) {
    constexpr LevelPlan PL = col_plan(L1);
    static_assert(PL.nlev == 2, "two-level column plans only");
    constexpr int n1 = 1 << L1, HALF = n1 / 2, T = NW * 32;
    constexpr int R0 = 1 << PL.logr[0], R1 = 1 << PL.logr[1];  // n1 = R0 * R1; level-0 tasks: R1
    constexpr int TC = col_tile_cols(L1, KIND), SUB = 32 / TC, QR = TC / 4;
    extern __shared__ __align__(16) u32 smem[];
    u32* tile = smem;                                                   // n1 rows
    u32* stage = smem + col_tile_words(L1, KIND);                       // rows [0, HALF)
    Tw* tws = reinterpret_cast<Tw*>(stage + tile_row<L1, KIND>(HALF));  // level-0 twiddles (n1 entries)
    const int n2 = 1 << A.l2, ct = n2 / TC;
    const int ntiles = ct * 2 * A.njobs;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % TC;
    const u32 p = A.pkc.p, p2 = A.pkc.p2, oneq = A.pkc.one_q;
    for (int i = threadIdx.x; i < n1; i += T) tws[i] = A.twc[i];

    // tile t -> job, operand, first column
    auto decode = [&](int t, const u32*& src, long long& len, u32*& dst, int& c0) {
        const LargeJob& J = A.jobs ? A.jobs[t / (2 * ct)] : A.job0;
        const int op = (t / ct) & 1;
        src = op ? J.b : J.a;
        len = op ? J.lb : J.la;
        dst = op ? J.wb : J.wa;
        c0 = (t % ct) * TC;
    };
    // rows [r0, r1) x TC columns of the operand into buf at the tile layout
    // (one commit group); words at or past len read as 0
    auto rows_issue = [&](u32* buf, const u32* src, long long len, int c0, int r0, int r1) {
        if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
            // a thread keeps one quad column q and walks rows T / QR apart
            // (running index: 64-bit adds, no multiply per copy)
            static_assert(T % QR == 0, "whole rows per thread round");
            const int q = threadIdx.x % QR;
            const long long step = (long long)(T / QR) * n2;
            long long gi = (long long)(r0 + threadIdx.x / QR) * n2 + c0 + 4 * q;
#pragma unroll 4
            for (int r = r0 + threadIdx.x / QR; r < r1; r += T / QR, gi += step) {
                const long long rem = len - gi;
                const int bytes = rem >= 4 ? 16 : (rem > 0 ? (int)rem * 4 : 0);
                const u32* g = bytes ? src + gi : src;
                const unsigned d = (unsigned)__cvta_generic_to_shared(buf + tile_row<L1, KIND>(r) + 4 * q);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(g), "r"(bytes) : "memory");
            }
        } else {
            for (int idx = r0 * TC + threadIdx.x; idx < r1 * TC; idx += T) {
                const int r = idx / TC, c = idx % TC;
                const long long gi = (long long)r * n2 + c0 + c;
                const int bytes = gi < len ? 4 : 0;
                const u32* g = bytes ? src + gi : src;
                const unsigned d = (unsigned)__cvta_generic_to_shared(buf + tile_row<L1, KIND>(r) + c);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(g), "r"(bytes) : "memory");
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    int t = blockIdx.x;
    if (t < ntiles) {
        const u32* src; long long len; u32* dst; int c0;
        decode(t, src, len, dst, c0);
        rows_issue(stage, src, len, c0, 0, HALF);
    }
    for (; t < ntiles; t += gridDim.x) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();  // stage and twiddles visible; the previous tile's last level is done with `tile`
        bool full;
        {
            const u32* src; long long len; u32* dst; int c0;
            decode(t, src, len, dst, c0);
            full = len > (long long)HALF * n2;
            if (full) {  // the upper rows of a long operand, into the tile
                rows_issue(tile, src, len, c0, HALF, n1);
                asm volatile("cp.async.wait_group 0;\n" ::: "memory");
                __syncthreads();
            }
        }

        // level 0: task o (rows o + R1 m)
        for (int o = warp * SUB + lane / TC; o < R1; o += NW * SUB) {
            u32 x[R0];
            const int off = tile_row<L1, KIND>(o) + col;
#pragma unroll
            for (int m = 0; m < R0 / 2; ++m) x[m] = stage[off + tile_step<L1, KIND, R1>(m)];
            if (!full) {
                dif_regs_halfzero<R0, true>(x, A.pkc.rc.f, p, p2, oneq);
            } else {
#pragma unroll
                for (int m = 0; m < R0; ++m)
                    x[m] = mul_shoup(m < R0 / 2 ? x[m] : tile[off + tile_step<L1, KIND, R1>(m)], 1u, oneq, p);
                dif_regs<R0, true>(x, A.pkc.rc.f, p, p2);
            }
#pragma unroll
            for (int j = 1; j < R0; ++j) {
                const Tw w = tws[o * R0 + j];  // broadcast to the (half-)warp
                x[j] = mul_shoup(x[j], w.w, w.wq, p);
            }
#pragma unroll
            for (int m = 0; m < R0; ++m) tile[off + tile_step<L1, KIND, R1>(m)] = x[m];
        }
        __syncthreads();  // tile complete; the stage is free

        if (t + (int)gridDim.x < ntiles) {
            const u32* src; long long len; u32* dst; int c0;
            decode(t + gridDim.x, src, len, dst, c0);
            rows_issue(stage, src, len, c0, 0, HALF);
        }

        // level 1 (last): block blk = rows blk * R1 + m, straight to HBM
        const u32* src; long long len; u32* dst; int c0;
        decode(t, src, len, dst, c0);
        for (int blk = warp * SUB + lane / TC; blk < R0; blk += NW * SUB) {
            u32 x[R1];
            const int off = tile_row<L1, KIND>(blk * R1) + col;
#pragma unroll
            for (int m = 0; m < R1; ++m) x[m] = tile[off + tile_step<L1, KIND, 1>(m)];
            dif_regs<R1>(x, A.pkc.rc.f, p, p2);
            // running pointer: 64-bit adds on the ALU pipe, not a multiply per store
            u32* out = dst + (size_t)(blk * R1) * n2 + c0 + col;
#pragma unroll
            for (int m = 0; m < R1; ++m, out += n2) *out = x[m];
        }
    }
}

// Pass A of a natural-order transform (one full-length operand per job,
// written over wa) as a persistent, software-pipelined kernel for 2^10-row
// columns on 16-column tiles: the whole next tile is staged by cp.async
// (zero-filled past the operand's end; word by word for an unaligned
// source) while the current one is transformed.  Level 0 reads and reduces
// the stage and writes the tile; level 1 stores straight to HBM.  Results
// are those of k_col_fwd<L1, NW, 2>.
template <int L1, int NW>
__global__ void __launch_bounds__(NW * 32, 1) k_col_fwd_pipe1(const __grid_constant__ LargeArgs A) {
    constexpr LevelPlan PL = col_plan(L1);
    static_assert(PL.nlev == 2, "two-level column plans only");
    constexpr int KIND = 2, n1 = 1 << L1, T = NW * 32;
    constexpr int R0 = 1 << PL.logr[0], R1 = 1 << PL.logr[1];  // n1 = R0 * R1
    constexpr int TC = col_tile_cols(L1, KIND), SUB = 32 / TC, QR = TC / 4;
    constexpr int TW = col_tile_words(L1, KIND);
    extern __shared__ __align__(16) u32 smem[];
    u32* tile = smem;
    u32* stage = smem + TW;
    Tw* tws = reinterpret_cast<Tw*>(stage + TW);  // level-0 twiddles (n1 entries)
    const int n2 = 1 << A.l2, ct = n2 / TC;
    const int ntiles = ct * A.njobs;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % TC;
    const u32 p = A.pkc.p, p2 = A.pkc.p2, oneq = A.pkc.one_q;
    for (int i = threadIdx.x; i < n1; i += T) tws[i] = A.twc[i];

    // all n1 rows x TC columns of tile t into the stage (one commit group);
    // words at or past the operand's length read as 0
    auto stage_issue = [&](int t) {
        const LargeJob& J = A.jobs ? A.jobs[t / ct] : A.job0;
        const u32* src = J.a;
        const long long len = J.la;
        const int c0 = (t % ct) * TC;
        if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
            static_assert(T % QR == 0, "whole rows per thread round");
            const int q = threadIdx.x % QR;
            const long long step = (long long)(T / QR) * n2;
            long long gi = (long long)(threadIdx.x / QR) * n2 + c0 + 4 * q;
#pragma unroll 4
            for (int r = threadIdx.x / QR; r < n1; r += T / QR, gi += step) {
                const long long rem = len - gi;
                const int bytes = rem >= 4 ? 16 : (rem > 0 ? (int)rem * 4 : 0);
                const u32* g = bytes ? src + gi : src;
                const unsigned d = (unsigned)__cvta_generic_to_shared(stage + tile_row<L1, KIND>(r) + 4 * q);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(g), "r"(bytes) : "memory");
            }
        } else {
            for (int idx = threadIdx.x; idx < n1 * TC; idx += T) {
                const int r = idx / TC, c = idx % TC;
                const long long gi = (long long)r * n2 + c0 + c;
                const int bytes = gi < len ? 4 : 0;
                const u32* g = bytes ? src + gi : src;
                const unsigned d = (unsigned)__cvta_generic_to_shared(stage + tile_row<L1, KIND>(r) + c);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(g), "r"(bytes) : "memory");
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    int t = blockIdx.x;
    if (t < ntiles) stage_issue(t);
    for (; t < ntiles; t += gridDim.x) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();  // stage and twiddles visible; the previous tile's level 1 is done with `tile`

        // level 0: task o (rows o + R1 m), inputs reduced, DIF, twiddles, stage -> tile
        for (int o = warp * SUB + lane / TC; o < R1; o += NW * SUB) {
            u32 x[R0];
            const int off = tile_row<L1, KIND>(o) + col;
#pragma unroll
            for (int m = 0; m < R0; ++m) x[m] = mul_shoup(stage[off + tile_step<L1, KIND, R1>(m)], 1u, oneq, p);
            dif_regs<R0, true>(x, A.pkc.rc.f, p, p2);
#pragma unroll
            for (int j = 1; j < R0; ++j) {
                const Tw w = tws[o * R0 + j];
                x[j] = mul_shoup(x[j], w.w, w.wq, p);
            }
#pragma unroll
            for (int m = 0; m < R0; ++m) tile[off + tile_step<L1, KIND, R1>(m)] = x[m];
        }
        __syncthreads();  // tile complete; the stage is free
        if (t + (int)gridDim.x < ntiles) stage_issue(t + gridDim.x);

        // level 1 (last): block blk = rows blk * R1 + m, straight to HBM
        const LargeJob& J = A.jobs ? A.jobs[t / ct] : A.job0;
        const int c0 = (t % ct) * TC;
        for (int blk = warp * SUB + lane / TC; blk < R0; blk += NW * SUB) {
            u32 x[R1];
            const int off = tile_row<L1, KIND>(blk * R1) + col;
#pragma unroll
            for (int m = 0; m < R1; ++m) x[m] = tile[off + tile_step<L1, KIND, 1>(m)];
            dif_regs<R1>(x, A.pkc.rc.f, p, p2);
            u32* out = J.wa + (size_t)(blk * R1) * n2 + c0 + col;
#pragma unroll
            for (int m = 0; m < R1; ++m, out += n2) *out = x[m];
        }
    }
}

// Pass C as a persistent, software-pipelined kernel for the two-level
// column plans (n1 = 2^9: 32-column tiles, n1 = 2^10: 16-column tiles, the
// inverse pass's layouts).  Each CTA walks the tiles gridDim.x apart; the
// whole next tile is copied into a stage buffer (cp.async) while the current
// one is transformed: each warp refills the stage rows of its own blocks as
// soon as its deepest-level tasks have consumed them.  The deepest level
// reads the stage and writes the tile; level 0 reads the tile and stores the
// canonical residues straight to the output, truncated at lh.  Results are
// those of k_col_inv.
template <int L1, int NW>
__global__ void __launch_bounds__(NW * 32, 1) k_col_inv_pipe(const __grid_constant__ LargeArgs A) {
    constexpr LevelPlan PL = col_plan(L1);
    static_assert(PL.nlev == 2, "two-level column plans only");
    constexpr int INV = 1, T = NW * 32;
    constexpr int TC = col_tile_cols(L1, INV), SUB = 32 / TC, QR = TC / 4;
    constexpr int n1 = 1 << L1, R0 = 1 << PL.logr[0], R1 = 1 << PL.logr[1];  // n1 = R0 * R1
    constexpr int TW = col_tile_words(L1, INV);
    extern __shared__ __align__(16) u32 smem[];
    u32* tile = smem;
    u32* stage = smem + TW;
    Tw* tws = reinterpret_cast<Tw*>(stage + TW);  // inverse level-0 twiddles (n1 entries)
    const int n2 = 1 << A.l2, ct = n2 / TC;
    const int ntiles = ct * A.njobs;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = lane % TC;
    const u32 p = A.pkc.p, p2 = A.pkc.p2;
    for (int i = threadIdx.x; i < n1; i += T) tws[i] = A.twc[A.twc_inv + i];

    // the whole tile t (all n1 rows of the row pass's output) into the stage
    // (the first tile; later ones are refilled per warp)
    auto stage_issue = [&](int t) {
        const LargeJob& J = A.jobs ? A.jobs[t / ct] : A.job0;
        // a thread keeps one quad column q and walks rows T / QR apart
        static_assert(T % QR == 0, "whole rows per thread round");
        const int q = threadIdx.x % QR;
        const u32* src = J.wa + (t % ct) * TC + (size_t)(threadIdx.x / QR) * n2 + 4 * q;
        const size_t step = (size_t)(T / QR) * n2;
#pragma unroll 4
        for (int r = threadIdx.x / QR; r < n1; r += T / QR, src += step) {
            const unsigned d = (unsigned)__cvta_generic_to_shared(stage + tile_row<L1, INV>(r) + 4 * q);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    pdl_wait();  // pass B's output
    int t = blockIdx.x;
    if (t < ntiles) stage_issue(t);
    for (; t < ntiles; t += gridDim.x) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();  // stage and twiddles visible; the previous tile's level 0 is done with `tile`

        // deepest level: blocks of R1 consecutive rows, DIT, stage -> tile
        for (int id = warp * SUB + lane / TC; id < R0; id += NW * SUB) {
            u32 x[R1];
            const int off = tile_row<L1, INV>(id * R1) + col;
#pragma unroll
            for (int m = 0; m < R1; ++m) x[m] = stage[off + tile_step<L1, INV, 1>(m)];
            dit_regs<R1, false>(x, A.pkc.rc.i, p, p2);
#pragma unroll
            for (int m = 0; m < R1; ++m) tile[off + tile_step<L1, INV, 1>(m)] = x[m];
        }
        // this warp's blocks (rows [warp SUB R1, (warp + 1) SUB R1)) have been
        // read (their words reached the tile), so the warp refills those stage
        // rows with the next tile's at once, half a tile earlier than a
        // CTA-wide refill after the barrier
        static_assert(NW * SUB == R0, "one block set per warp");
        __syncwarp();
        if (t + (int)gridDim.x < ntiles) {
            const int tn = t + gridDim.x;
            const LargeJob& Jn = A.jobs ? A.jobs[tn / ct] : A.job0;
            const int q = lane % QR;
            const int r0 = warp * SUB * R1 + lane / QR;
            const u32* src = Jn.wa + (tn % ct) * TC + (size_t)r0 * n2 + 4 * q;
            const size_t step = (size_t)(32 / QR) * n2;
#pragma unroll 4
            for (int r = r0; r < (warp + 1) * SUB * R1; r += 32 / QR, src += step) {
                const unsigned d = (unsigned)__cvta_generic_to_shared(stage + tile_row<L1, INV>(r) + 4 * q);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        __syncthreads();  // tile complete

        // level 0: task o (rows o + R1 m), pre-twiddle, DIT, canonical residues out
        const LargeJob& J = A.jobs ? A.jobs[t / ct] : A.job0;
        const long long lh = J.lh;
        const int c0 = (t % ct) * TC;
        for (int o = warp * SUB + lane / TC; o < R1; o += NW * SUB) {
            u32 x[R0];
            const int off = tile_row<L1, INV>(o) + col;
#pragma unroll
            for (int m = 0; m < R0; ++m) x[m] = tile[off + tile_step<L1, INV, R1>(m)];
#pragma unroll
            for (int j = 1; j < R0; ++j) {
                const Tw w = tws[o * R0 + j];
                x[j] = mul_shoup(x[j], w.w, w.wq, p);
            }
            dit_regs<R0, true>(x, A.pkc.rc.i, p, p2);
            // running index and pointer (64-bit adds on the ALU pipe)
            long long gi = (long long)o * n2 + c0 + col;
            u32* out = J.h + gi;
            const long long step = (long long)R1 * n2;
#pragma unroll
            for (int m = 0; m < R0; ++m, gi += step, out += step)
                if (gi < lh) *out = red1(red2(x[m], p2), p);
        }
    }
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
//                 result written over G' in digit-reversed row order, its
//                 32-word groups quad-interleaved (coalesced both ways);
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
__device__ __forceinline__ void row_load_issue(u32* sm, const u32* __restrict__ row) {
    constexpr int n2 = 1 << L2;
#pragma unroll 8
    for (int i = threadIdx.x * 4; i < n2; i += T * 4) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(sm + swz(i));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(row + i) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void row_load_wait() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <int L2, int T>
__device__ __forceinline__ void row_load(u32* sm, const u32* __restrict__ row) {
    row_load_issue<L2, T>(sm, row);
    row_load_wait();
}

// floor(w * 2^32 / p) for w < p < 2^30 (the Shoup quotient of w): a
// double-precision estimate, off by at most one, corrected with exact
// 64-bit integer arithmetic.
__host__ __device__ __forceinline__ u32 shoup_quot_dev(u32 w, u32 p, double r32p) {
    u32 q = (u32)((double)w * r32p);
    const long long r = (long long)(((u64)w << 32) - (u64)q * p);
    if (r < 0) --q;
    else if (r >= (long long)p) ++q;
    return q;
}

// Per-row factor tables of the split row kernels' level 0.
//
// Level 0 of the row DFT of slot s (column frequency k1, W = w_n^k1) takes
// task o's inputs c = o + TB0 m times the inter-pass twiddle W^c, runs a
// radix-R0 DIF and multiplies output j by the level twiddle w_n2^(o rev(j)).
// W^c = W^o * W^(TB0 m), and the common factor W^o of a task commutes with
// the DIF, so the level is: inputs times V_m = W^(TB0 m) (the slot factors),
// DIF, outputs times U_j^o with U_j = W w_n2^rev(j).  U_j^o is the product
// of two table entries, U_j^(o mod NA) and U_j^(NA (o div NA)), so no
// twiddle of level 0 is read from L2 inside the level.  An entry
// U_j^e = W^e * w_n2^(e rev(j)) is a power of W (from the seed tables) times
// the level-0 twiddle table entry (e, j).  The inverse level uses the
// inverse factors: inputs times U_j^-o, DIT, outputs times W^-(TB0 m) with
// the 2^32/n scale.  A slot's table (one direction: the U entries, then the
// R0 slot factors) depends only on the prime and the transform shape: it is
// built once into HBM (k_rowtab_build) and copied into shared memory next to
// the row; without it (rowtab == nullptr) each CTA builds its own.  Rows
// shorter than 2^11 words keep computing W^c from the seeds per task: there
// the table would cost more than it saves.
template <int L2>
struct RowTab {
    using LV0 = SmallLevel<L2, 0>;
    static constexpr bool USE = L2 >= 11;
    static constexpr int R0 = LV0::R, TB0 = LV0::TB;
    static constexpr int LOGTB = LV0::LOGB - LV0::PL.logr[0];
    static constexpr int LA = (LOGTB + 1) / 2;
    static constexpr int NA = 1 << LA, NB = TB0 >> LA;
    static constexpr int ENTRIES = USE ? R0 * (NA + NB) : 0;  // [j][NA] then [j][NB]
    static constexpr int TABW = USE ? ENTRIES + R0 : 0;        // + the slot factors
    static constexpr int NPOW = USE ? NA + NB : 0;             // W^e: e < NA, then e = NA k
};

// Slot factors of one direction into f[0, R0): W^(TB0 m), or W^-(TB0 m)
// times 2^32/n (the inverse's output factors).
template <int L2>
__device__ __forceinline__ void row_slot_entries(Tw* f, const LargeArgs& A, u32 k1, bool inv) {
    using LV0 = SmallLevel<L2, 0>;
    const u32 nmask = (1u << (A.l1 + L2)) - 1;
    const u32 p = A.pk.p, pinv = A.pk.pinv_neg;
    if (threadIdx.x < LV0::R) {
        const u32 m = threadIdx.x;
        u32 v = red1(mul_mont(seed_mont(A, (k1 * (u32)LV0::TB * m) & nmask, inv), 1u, p, pinv), p);
        if (inv) v = (u32)(((u64)v * A.scale_rn) % p);
        f[m] = Tw{v, shoup_quot_dev(v, p, A.r32p)};
    }
}

// W^(+-e) * 2^32 for the table's exponents (e < NA, then e = NA k).
template <int L2, int T>
__device__ __forceinline__ void row_wpow_build(u32* wp, const LargeArgs& A, u32 k1, bool inv) {
    using RT = RowTab<L2>;
    const u32 nmask = (1u << (A.l1 + L2)) - 1;
    for (int i = threadIdx.x; i < RT::NPOW; i += T) {
        const u32 e = i < RT::NA ? (u32)i : (u32)(i - RT::NA) * RT::NA;
        wp[i] = seed_mont(A, (k1 * e) & nmask, inv);
    }
}

// The U entries of one direction from the powers wp and that direction's
// level-0 twiddles twl (entry e R0 + j = w_n2^(+-e rev(j))).  The loop runs
// j fastest so the twiddle reads are coalesced.
template <int L2, int T>
__device__ __forceinline__ void row_tab_build(Tw* tab, const u32* wp, const Tw* __restrict__ twl, const LargeArgs& A) {
    using RT = RowTab<L2>;
    const u32 p = A.pk.p, pinv = A.pk.pinv_neg;
    for (int q = threadIdx.x; q < RT::ENTRIES; q += T) {
        const int j = q % RT::R0;
        int e, w, at;
        if (q < RT::R0 * RT::NA) {
            const int a = q / RT::R0;
            e = a; w = a; at = j * RT::NA + a;
        } else {
            const int k = (q - RT::R0 * RT::NA) / RT::R0;
            e = k * RT::NA; w = RT::NA + k; at = RT::R0 * RT::NA + j * RT::NB + k;
        }
        const u32 v = red1(mul_mont(wp[w], __ldg(&twl[e * RT::R0 + j].w), p, pinv), p);
        tab[at] = Tw{v, shoup_quot_dev(v, p, A.r32p)};
    }
}

// One slot's table of one direction into tab (shared or global memory):
// from HBM when the prebuilt tables exist (cp.async, one commit group; the
// caller waits), else built here (wp: NPOW words of shared scratch; the
// caller's barrier must separate this from the table's first read).
template <int L2, int T>
__device__ __forceinline__ void row_tab_fetch(Tw* tab, u32* wp, const LargeArgs& A, u32 s, u32 k1, bool inv) {
    using RT = RowTab<L2>;
    if (A.rowtab) {
        const Tw* src = A.rowtab + ((size_t)(inv ? 1 : 0) * (1u << A.l1) + s) * RT::TABW;
        for (int i = threadIdx.x; i < RT::TABW / 2; i += T) {
            const unsigned d = (unsigned)__cvta_generic_to_shared(tab + 2 * i);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 2 * i) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    } else {
        row_slot_entries<L2>(tab + RT::ENTRIES, A, k1, inv);
        row_wpow_build<L2, T>(wp, A, k1, inv);
        __syncthreads();
        row_tab_build<L2, T>(tab, wp, inv ? A.twr + A.twr_inv : A.twr, A);
    }
}

// Builds every slot's tables into HBM: grid (n1 slots, 2 directions).
template <int L2>
__global__ void __launch_bounds__(rowsplit_threads(L2)) k_rowtab_build(const __grid_constant__ LargeArgs A, Tw* out) {
    using RT = RowTab<L2>;
    __shared__ u32 wp[RT::NPOW > 0 ? RT::NPOW : 1];
    const u32 s = blockIdx.x;
    const bool inv = blockIdx.y != 0;
    const u32 k1 = col_slot_to_k1(s, A.colpl, A.l1);
    Tw* dst = out + ((size_t)blockIdx.y * gridDim.x + s) * RT::TABW;
    row_slot_entries<L2>(dst + RT::ENTRIES, A, k1, inv);
    row_wpow_build<L2, rowsplit_threads(L2)>(wp, A, k1, inv);
    __syncthreads();
    row_tab_build<L2, rowsplit_threads(L2)>(dst, wp, inv ? A.twr + A.twr_inv : A.twr, A);
}

// Level 0 forward of one operand computing the inter-pass twiddle W^c per
// task from the seeds (short rows).
template <int L2, int T>
__device__ __forceinline__ void row_level0_fwd_seeds(u32* sm, const LargeArgs& A, u32 k1, const Tw* bf) {
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

// Level 0 forward of one operand: slot factors on the inputs, DIF, the
// per-row factors U_j^o on the outputs.
template <int L2, int T>
__device__ __forceinline__ void row_level0_fwd(u32* sm, const LargeArgs& A, const Tw* tab) {
    using RT = RowTab<L2>;
    constexpr int R0 = RT::R0, TB0 = RT::TB0;
    static_assert(T % RT::NA == 0, "the tasks of a thread share o mod NA");
    const u32 p = A.pk.p, p2 = A.pk.p2;
    // the slot factors and this thread's U_j^(o mod NA) are the same for all
    // of its tasks: kept in registers
    Tw vf[R0], af[R0];
#pragma unroll
    for (int j = 0; j < R0; ++j) {
        vf[j] = tab[RT::ENTRIES + j];
        af[j] = tab[j * RT::NA + threadIdx.x % RT::NA];
    }
    for (int o = threadIdx.x; o < TB0; o += T) {
        u32 x[R0];
#pragma unroll
        for (int m = 0; m < R0; ++m) {
            const u32 v = sm[swz_task<TB0, (1 << L2)>(o, swz(o), m)];
            x[m] = m == 0 ? v : mul_shoup(v, vf[m].w, vf[m].wq, p);
        }
        dif_regs<R0, true>(x, A.pk.rc.f, p, p2);
        const Tw* tb = tab + RT::R0 * RT::NA + o / RT::NA;
#pragma unroll
        for (int j = 0; j < R0; ++j) {
            const Tw b = tb[j * RT::NB];
            x[j] = mul_shoup(mul_shoup(x[j], af[j].w, af[j].wq, p), b.w, b.wq, p);
        }
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
    // the row, then the level-0 factor table (and scratch to build it)
    extern __shared__ __align__(16) u32 sm[];
    __shared__ Tw bf[R0];
    Tw* tab = reinterpret_cast<Tw*>(sm + n2);
    u32* wp = reinterpret_cast<u32*>(tab + RowTab<L2>::TABW);
    const LargeJob& J = A.jobs ? A.jobs[blockIdx.y] : A.job0;
    const u32 s = blockIdx.x;
    const u32 k1 = col_slot_to_k1(s, A.colpl, A.l1);
    const u32 p = A.pk.p, p2 = A.pk.p2;
    u32* row = J.wb + (size_t)s * n2;
    pdl_trigger();
    if constexpr (RowTab<L2>::USE) row_tab_fetch<L2, T>(tab, wp, A, s, k1, false);
    else row_slot_factors<L2>(A, k1, bf, nullptr);
    pdl_wait();  // pass A's columns of G
    row_load_issue<L2, T>(sm, row);
    row_load_wait();
    __syncthreads();
    if constexpr (RowTab<L2>::USE) row_level0_fwd<L2, T>(sm, A, tab);
    else row_level0_fwd_seeds<L2, T>(sm, A, k1, bf);
    __syncthreads();
    fwd1_levels<L2, 1, T>(sm, A.pk, A.twr);
    for (int r = threadIdx.x; r < n2 / 32; r += T) {
        u32 x[32];
        load_row32(x, sm, r * 32);
        dif_regs<32>(x, A.pk.rc.f, p, p2);
        // store this 32-word group of the spectrum straight to global memory,
        // quad-interleaved (quad c of group r at c * n2/8 + 4 r): the lanes of
        // a warp write one contiguous 512-byte run per store, and k_row_mul_f
        // reads it back the same way
#pragma unroll
        for (int c = 0; c < 8; ++c)
            *reinterpret_cast<uint4*>(row + c * (n2 / 8) + 4 * r) =
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
    // the row, then the level-0 factor table (and scratch to build it)
    extern __shared__ __align__(16) u32 sm[];
    __shared__ Tw bf[R0], bi[R0];
    Tw* tab = reinterpret_cast<Tw*>(sm + n2);
    u32* wp = reinterpret_cast<u32*>(tab + RowTab<L2>::TABW);
    const LargeJob& J = A.jobs ? A.jobs[blockIdx.y] : A.job0;
    const u32 s = blockIdx.x;
    const u32 k1 = col_slot_to_k1(s, A.colpl, A.l1);
    const u32 p = A.pk.p, p2 = A.pk.p2, pinv = A.pk.pinv_neg;
    u32* rowF = J.wa + (size_t)s * n2;
    const u32* rowG = J.wb + (size_t)s * n2;
    RowCtx ctx{A.pk, A.twr, A.twr_inv};
    pdl_trigger();
    // F's forward row pass depends only on pass A (complete before the
    // previous kernel, G's row pass, started), so it runs while that kernel
    // finishes; G's spectrum is read after pdl_wait
    row_load_issue<L2, T>(sm, rowF);
    if constexpr (RowTab<L2>::USE) row_tab_fetch<L2, T>(tab, wp, A, s, k1, false);
    else row_slot_factors<L2>(A, k1, bf, bi);
    row_load_wait();
    __syncthreads();
    if constexpr (RowTab<L2>::USE) row_level0_fwd<L2, T>(sm, A, tab);
    else row_level0_fwd_seeds<L2, T>(sm, A, k1, bf);
    __syncthreads();
    // level 0's inverse factors replace the forward ones; they are waited
    // for (prebuilt) or visible (built here) after the barriers below
    if constexpr (RowTab<L2>::USE) row_tab_fetch<L2, T>(tab, wp, A, s, k1, true);
    fwd1_levels<L2, 1, T>(sm, A.pk, A.twr);
    pdl_wait();
    for (int r = threadIdx.x; r < n2 / 32; r += T) {
        u32 x[32];
        load_row32(x, sm, r * 32);
        dif_regs<32>(x, A.pk.rc.f, p, p2);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const uint4 g = __ldg(reinterpret_cast<const uint4*>(rowG + c * (n2 / 8) + 4 * r));  // quad-interleaved
            x[4 * c] = mul_mont(x[4 * c], g.x, p, pinv);
            x[4 * c + 1] = mul_mont(x[4 * c + 1], g.y, p, pinv);
            x[4 * c + 2] = mul_mont(x[4 * c + 2], g.z, p, pinv);
            x[4 * c + 3] = mul_mont(x[4 * c + 3], g.w, p, pinv);
        }
        dit_regs<32>(x, A.pk.rc.i, p, p2);
        store_row32(sm, r * 32, x);
    }
    row_load_wait();  // the inverse factor table
    __syncthreads();
    small_inv_levels<L2, PL.nlev - 2, T, 1, 1>(sm, ctx);
    // level 0 inverse: inputs times U_j^-o, DIT, outputs times W^-(TB0 m) 2^32/n
    using RT = RowTab<L2>;
    if constexpr (RT::USE) {
        const Tw* bo = tab + RT::ENTRIES;
        Tw af[R0];  // this thread's U_j^-(o mod NA), the same for all of its tasks
#pragma unroll
        for (int j = 0; j < R0; ++j) af[j] = tab[j * RT::NA + threadIdx.x % RT::NA];
        for (int o = threadIdx.x; o < TB0; o += T) {
            u32 x[R0];
            const Tw* tb = tab + RT::R0 * RT::NA + o / RT::NA;
#pragma unroll
            for (int j = 0; j < R0; ++j) {
                const Tw b = tb[j * RT::NB];
                x[j] = mul_shoup(mul_shoup(sm[swz_task<TB0, n2>(o, swz(o), j)], af[j].w, af[j].wq, p), b.w, b.wq, p);
            }
            dit_regs<R0, true>(x, A.pk.rc.i, p, p2);
#pragma unroll
            for (int m = 0; m < R0; ++m) rowF[o + TB0 * m] = mul_shoup(x[m], bo[m].w, bo[m].wq, p);
        }
    } else {  // short rows: level twiddles from the table, W^-c from the seeds
        const u32 nmask = (1u << (A.l1 + L2)) - 1;
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
}

#endif  // __CUDACC__

}  // namespace cmb
