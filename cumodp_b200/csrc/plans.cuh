// Compile-time level plans for the shared-memory transforms.
#pragma once
#include "ntt_engine.cuh"

namespace cmb {

// Plan for a contiguous transform of length 2^logl held in shared memory.
// The last level always has radix 32: every earlier level then has at least
// 32 tasks per block, so 32 lanes touch 32 consecutive words (no bank
// conflicts), and the last level reads whole 32-word rows with 16-byte
// accesses through the swizzle.  Earlier levels use radix <= 16 so that a
// thread can hold both operands of a product (2 x 16 registers).
__host__ __device__ constexpr LevelPlan row_plan(int logl) {
    switch (logl) {
        case 5: return LevelPlan{1, {5}};
        case 6: return LevelPlan{2, {1, 5}};
        case 7: return LevelPlan{2, {2, 5}};
        case 8: return LevelPlan{2, {3, 5}};
        case 9: return LevelPlan{2, {4, 5}};
        case 10: return LevelPlan{3, {2, 3, 5}};
        case 11: return LevelPlan{3, {3, 3, 5}};
        case 12: return LevelPlan{4, {2, 2, 3, 5}};
        case 13: return LevelPlan{4, {2, 3, 3, 5}};
        case 14: return LevelPlan{4, {3, 3, 3, 5}};
        default: return LevelPlan{0, {0}};
    }
}

// Plan for a batch of interleaved columns (lane = column): bank conflicts do
// not depend on the radix, so fewer, wider levels are used (two levels up to
// 2^10 rows: every element goes through shared memory twice).
__host__ __device__ constexpr LevelPlan col_plan(int logl) {
    switch (logl) {
        case 1: return LevelPlan{1, {1}};
        case 2: return LevelPlan{1, {2}};
        case 3: return LevelPlan{1, {3}};
        case 4: return LevelPlan{1, {4}};
        case 5: return LevelPlan{2, {2, 3}};
        case 6: return LevelPlan{2, {3, 3}};
        case 7: return LevelPlan{2, {3, 4}};
        case 8: return LevelPlan{2, {4, 4}};
        case 9: return LevelPlan{2, {4, 5}};
        case 10: return LevelPlan{2, {5, 5}};
        case 11: return LevelPlan{3, {3, 4, 4}};
        case 12: return LevelPlan{3, {4, 4, 4}};
        default: return LevelPlan{0, {0}};
    }
}

// Twiddle entries (one direction) of the column plan of length 2^logl.
__host__ __device__ constexpr int col_tw_entries(int logl) {
    int n = 0, lb = logl;
    const LevelPlan pl = col_plan(logl);
    for (int i = 0; i + 1 < pl.nlev; ++i) { n += 1 << lb; lb -= pl.logr[i]; }
    return n;
}
// Column tiles: col_tile_cols adjacent columns x 2^logl rows in shared
// memory, processed by col_warps warps, col_ctas resident CTAs per SM, each
// chosen per kind of pass (0: the product's forward pass, whose operands are
// half zero padding; 1: the inverse pass; 2: the forward pass of a
// natural-order transform).  32-column tiles put
// one column on each lane; 16-column tiles put two tasks on each warp (one
// per half-warp) and insert a 16-word pad after every 2^col_pad_log rows (the
// plan's last radix), so that the two half-warps always read opposite halves
// of the banks.  Short tiles (2^5, 2^6 rows: the column side of products of
// 2^15-2^17) run on one or two warps, so many CTAs share an SM.  Kinds 1 and
// 2 over 2^10-row tiles use 16 columns and two
// CTAs per SM (their load, compute and store phases overlap); kind 0 keeps
// 32 columns (its loads skip the zero-padded half).
__host__ __device__ constexpr int col_tile_cols(int logl, int kind) { return (kind != 0 && logl == 10) || logl >= 11 ? 16 : 32; }
__host__ __device__ constexpr int col_warps(int logl, int kind) { return logl == 10 && kind == 0 ? 32 : (logl <= 5 ? 1 : (logl <= 6 ? 2 : 16)); }
__host__ __device__ constexpr int col_ctas(int logl, int kind) { return kind != 0 && logl == 10 ? 2 : 1; }
__host__ __device__ constexpr int col_pad_log(int logl) { return col_plan(logl).logr[col_plan(logl).nlev - 1]; }
__host__ __device__ constexpr int col_tile_words(int logl, int kind) {
    return col_tile_cols(logl, kind) == 32
               ? (32 << logl)
               : ((1 << logl) + ((1 << logl) >> col_pad_log(logl))) * col_tile_cols(logl, kind);
}
// Whether a column CTA stages its twiddles in shared memory next to the
// tile (else the levels read them from global memory, as broadcasts).
__host__ __device__ constexpr bool col_tw_smem(int logl, int kind) { return true; }
// col_tile_cols for a run-time logl.
__host__ __device__ inline int col_tile_cols_rt(int logl, int kind) {
    constexpr int t[3][13] = {
        {col_tile_cols(0, 0), col_tile_cols(1, 0), col_tile_cols(2, 0), col_tile_cols(3, 0), col_tile_cols(4, 0),
         col_tile_cols(5, 0), col_tile_cols(6, 0), col_tile_cols(7, 0), col_tile_cols(8, 0), col_tile_cols(9, 0),
         col_tile_cols(10, 0), col_tile_cols(11, 0), col_tile_cols(12, 0)},
        {col_tile_cols(0, 1), col_tile_cols(1, 1), col_tile_cols(2, 1), col_tile_cols(3, 1), col_tile_cols(4, 1),
         col_tile_cols(5, 1), col_tile_cols(6, 1), col_tile_cols(7, 1), col_tile_cols(8, 1), col_tile_cols(9, 1),
         col_tile_cols(10, 1), col_tile_cols(11, 1), col_tile_cols(12, 1)},
        {col_tile_cols(0, 2), col_tile_cols(1, 2), col_tile_cols(2, 2), col_tile_cols(3, 2), col_tile_cols(4, 2),
         col_tile_cols(5, 2), col_tile_cols(6, 2), col_tile_cols(7, 2), col_tile_cols(8, 2), col_tile_cols(9, 2),
         col_tile_cols(10, 2), col_tile_cols(11, 2), col_tile_cols(12, 2)}};
    return t[kind][logl];
}
// Dynamic shared memory of a column CTA: the tile and its twiddles.
__host__ __device__ constexpr int col_smem_bytes(int logl, int kind) {
    return col_tile_words(logl, kind) * 4 + (col_tw_smem(logl, kind) ? col_tw_entries(logl) * 8 : 0);
}

// Persistent pass A (k_col_fwd_pipe) for the two-level column plans, up to
// 128 registers a thread (1024 threads at 64 registers spill): 2^10-row
// columns in 16-column tiles (the layout of kind 2), two 256-thread CTAs per
// SM, whose barriers and phases then overlap (measured 8 % faster than one
// 512-thread CTA on 32-column tiles); 2^9-row columns in 32-column tiles,
// one 512-thread CTA per SM (two per SM measured slower).  Shared memory:
// the tile, a stage of its first n1/2 rows and the level-0 twiddles.
__host__ __device__ constexpr bool col_pipe_ok(int logl) { return logl == 9 || logl == 10; }
__host__ __device__ constexpr int col_pipe_kind(int logl) { return logl == 10 ? 2 : 0; }  // tile layout (col_tile_cols)
__host__ __device__ constexpr int col_pipe_warps(int logl) { return logl == 10 ? 8 : 16; }
__host__ __device__ constexpr int col_pipe_ctas(int logl) { return logl == 10 ? 2 : 1; }
__host__ __device__ constexpr int col_pipe_smem_bytes(int logl) {
    // tile, stage (the tile layout's first n1/2 rows), level-0 twiddles
    return col_tile_words(logl, col_pipe_kind(logl)) * 4 +
           (col_tile_cols(logl, col_pipe_kind(logl)) == 32
                ? (16 << logl)
                : ((1 << logl) / 2 + ((1 << logl) / 2 >> col_pad_log(logl))) * col_tile_cols(logl, col_pipe_kind(logl))) * 4 +
           (1 << logl) * 8;
}

// Persistent pass C (k_col_inv_pipe) for the same column lengths: one
// 512-thread CTA per SM holding the tile, a stage for the whole next tile
// and the level-0 twiddles (two 256-thread CTAs per SM with a half-tile
// stage measured 9 % slower: the unstaged half's load is exposed).
__host__ __device__ constexpr int col_inv_pipe_warps(int logl) { return 16; }
__host__ __device__ constexpr int col_inv_pipe_smem_bytes(int logl) {
    return 2 * col_tile_words(logl, 1) * 4 + (1 << logl) * 8;
}

// Persistent pass A of a natural-order transform (k_col_fwd_pipe1): 2^10-row
// columns, one 512-thread CTA per SM holding the tile, a stage for the whole
// next tile and the level-0 twiddles.
__host__ __device__ constexpr int col_pipe1_smem_bytes(int logl) {
    return 2 * col_tile_words(logl, 2) * 4 + (1 << logl) * 8;
}

// A single product (no batch) of transform length 2^logn uses the three-pass
// kernels from this length on, even where one CTA could hold it: spread over
// many CTAs it finishes sooner than on one SM.
__host__ __device__ constexpr int single_large_min_log() { return 13; }

// Threads of the three-pass row kernel: 2^14-word rows use 1024 threads with
// at most 64 registers each (32 warps per SM; the plan's twiddled levels
// have radix <= 8 so both operands fit), shorter rows the single-CTA count.
__host__ __device__ constexpr int row_threads(int logl);

// Threads and products per CTA for the fused single-CTA product of length L.
__host__ __device__ constexpr int small_threads(int logl) { return logl >= 12 ? (1 << (logl - 5)) : 128; }
__host__ __device__ constexpr int small_ppc(int logl) { return logl >= 12 ? 1 : (1 << (12 - logl)); }
// Resident CTAs per SM the fused single-CTA product is compiled for: six
// 32 KiB CTAs of 128 threads (80 registers) for lengths <= 2^12, three
// 64 KiB CTAs for 2^13, one 128 KiB CTA for 2^14.
__host__ __device__ constexpr int small_ctas(int logl) { return logl <= 12 ? 6 : logl == 13 ? 3 : 1; }
__host__ __device__ constexpr int row_threads(int logl) { return logl == 14 ? 1024 : small_threads(logl); }
// Threads of the split row kernels (one operand row per CTA): one per
// 32-word row of the last level, two CTAs per SM; 2^14-word rows use 256
// threads (up to 85 registers each) and three CTAs per SM, so that the load,
// compute and store phases of three rows overlap on every SM.
__host__ __device__ constexpr int rowsplit_threads(int logl) { return logl == 14 ? 256 : logl >= 10 ? (1 << (logl - 5)) : 32; }
// Natural-order row transforms (k_row_ntt): one thread per 32-word group of
// the last level (at least a warp), one row of shared memory per CTA, 1024
// threads per SM.
__host__ __device__ constexpr int ntt_row_threads(int logl) { return logl >= 10 ? (1 << (logl - 5)) : 32; }
__host__ __device__ constexpr int ntt_row_ctas(int logl) { return 1024 / ntt_row_threads(logl) < 32 ? 1024 / ntt_row_threads(logl) : 32; }

// Resident CTAs per SM the split row kernels are compiled for: three for
// 2^14-word rows, else enough for 1024 threads per SM (64 registers).
__host__ __device__ constexpr int rowsplit_ctas(int logl) { return logl == 14 ? 3 : (1024 / rowsplit_threads(logl) < 32 ? 1024 / rowsplit_threads(logl) : 32); }

}  // namespace cmb
