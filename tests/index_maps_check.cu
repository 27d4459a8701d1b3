// Host-side check of every shared-memory and table index map the kernels use,
// for every plan the library instantiates.  The maps are the kernels' own
// __host__ __device__ functions (compiled here for the host), so an
// out-of-bounds or colliding index shows up here instead of on a GPU.
//
//   rows:    every non-last level of every row plan (lengths 2^5..2^14,
//            products of one and of several operand pairs per CTA) touches
//            each word of its buffer exactly once, swz_task equals the plain
//            swizzle, the last level's 16-byte quads tile the buffer, and the
//            twiddle reads stay inside the plan's table;
//   columns: for every tile kind and 2^1..2^11 rows, tile_row is injective and
//            in bounds, tile_step equals tile_row differences for every level
//            task, and the two half-warps of a 16-column tile read opposite
//            halves of the banks;
//   orders:  col_slot_to_k1 and row_pos_to_freq are permutations;
//   row factor tables (rows of 2^11..2^14 words): every level-0 task reads
//            its two entries inside the table, the two digits recompose the
//            task index, and the row kernels' shared memory fits the SM;
//   pipelined column pass: stage, tile and twiddle indexes in bounds;
//   Shoup quotients from the double estimate equal floor(w 2^32 / p);
//   the quad-interleaved row spectrum is a permutation with warp-contiguous runs;
//   the natural-order reorder buffer's swizzle is a bijection without store conflicts.
#include <cstdio>
#include <set>
#include <vector>

#include "../cumodp_b200/csrc/large_product.cuh"

using namespace cmb;

static int failures = 0;
#define CHECK(c, ...)                          \
    do {                                       \
        if (!(c)) {                            \
            if (failures < 20) {               \
                std::printf("FAIL: " __VA_ARGS__); \
                std::printf("\n");             \
            }                                  \
            ++failures;                        \
        }                                      \
    } while (0)

template <int LOGL, int LEV>
void row_level(int ppc) {
    using LV = SmallLevel<LOGL, LEV>;
    constexpr int L = 1 << LOGL, R = LV::R, TB = LV::TB, B = LV::B;
    std::vector<int> seen((size_t)ppc * 2 * L, 0);
    for (int q = 0; q < ppc; ++q)
        for (int op = 0; op < 2; ++op)
            for (int rest = 0; rest < L / R; ++rest) {
                const int blk = rest / TB, o = rest % TB;
                const int base = q * 2 * L + op * L + blk * B + o;
                const int bs = swz(base);
                for (int m = 0; m < R; ++m) {
                    const int a = swz_task<TB, B>(base, bs, m);
                    CHECK((a == swz(base + TB * m)), "row L=%d lev=%d swz_task", LOGL, LEV);
                    CHECK(a >= 0 && a < (int)seen.size(), "row L=%d lev=%d out of range", LOGL, LEV);
                    if (a >= 0 && a < (int)seen.size()) seen[a]++;
                }
                // twiddles of this task: o * R + j < the level's B entries
                CHECK(LV::TWOFF + o * R + R - 1 < plan_tw_entries(row_plan(LOGL), LOGL),
                      "row L=%d lev=%d twiddle index", LOGL, LEV);
            }
    for (size_t i = 0; i < seen.size(); ++i) CHECK(seen[i] == 1, "row L=%d lev=%d word %zu hit %d", LOGL, LEV, i, seen[i]);
}

template <int LOGL, int LEV>
void row_levels(int ppc) {
    constexpr LevelPlan PL = row_plan(LOGL);
    if constexpr (LEV + 1 < PL.nlev) {
        row_level<LOGL, LEV>(ppc);
        row_levels<LOGL, LEV + 1>(ppc);
    }
}

template <int LOGL>
void row_plan_check() {
    constexpr int L = 1 << LOGL;
    row_levels<LOGL, 0>(1);
    if (small_ppc(LOGL) > 1) row_levels<LOGL, 0>(small_ppc(LOGL));
    // last level: 32-word groups read as 8 quads through the swizzle
    std::vector<int> seen(L, 0);
    for (int r = 0; r < L / 32; ++r)
        for (int c = 0; c < 8; ++c) {
            const int a = swz(r * 32 + 4 * c);
            CHECK(a % 4 == 0 && a >= 0 && a + 3 < L, "row L=%d quad", LOGL);
            for (int k = 0; k < 4; ++k)
                if (a + k >= 0 && a + k < L) seen[a + k]++;
        }
    for (int i = 0; i < L; ++i) CHECK(seen[i] == 1, "row L=%d last level word %d", LOGL, i);
    // natural order after the row plan: a permutation
    if constexpr (LOGL >= 6) {
        std::vector<int> f(L, 0);
        for (int P = 0; P < L; ++P) {
            const u32 v = row_pos_to_freq<LOGL>((u32)P);
            CHECK(v < (u32)L, "row_pos_to_freq L=%d", LOGL);
            if (v < (u32)L) f[v]++;
        }
        for (int i = 0; i < L; ++i) CHECK(f[i] == 1, "row_pos_to_freq L=%d not a permutation", LOGL);
    }
}

template <int L1, int INV, int LEV>
void col_level() {
    using LV = ColLevel<L1, LEV>;
    constexpr int R = LV::R, TB = LV::TB, B = LV::B;
    constexpr int TC = col_tile_cols(L1, INV);
    constexpr int TASKS = (1 << L1) / R;
    for (int id = 0; id < TASKS; ++id) {
        const int blk = id / TB, o = id % TB;
        const int row0 = blk * B + o;
        for (int m = 0; m < R; ++m)
            CHECK((tile_row<L1, INV>(row0) + tile_step<L1, INV, TB>(m) == tile_row<L1, INV>(row0 + TB * m)),
                  "col L1=%d kind=%d lev=%d tile_step", L1, INV, LEV);
        // a 16-column tile puts tasks id (even) and id + 1 on the two half-warps
        if (TC == 16 && id % 2 == 0 && id + 1 < TASKS) {
            const int blk2 = (id + 1) / TB, o2 = (id + 1) % TB;
            const int row1 = blk2 * B + o2;
            for (int m = 0; m < R; ++m) {
                const int a = tile_row<L1, INV>(row0 + TB * m), b = tile_row<L1, INV>(row1 + TB * m);
                CHECK(((a - b) % 32 + 32) % 32 == 16, "col L1=%d kind=%d lev=%d half-warp banks", L1, INV, LEV);
            }
        }
    }
}

template <int L1, int INV, int LEV>
void col_levels() {
    constexpr LevelPlan PL = col_plan(L1);
    if constexpr (LEV < PL.nlev) {
        col_level<L1, INV, LEV>();
        col_levels<L1, INV, LEV + 1>();
    }
}

template <int L1, int INV>
void col_kind_check() {
    constexpr int n1 = 1 << L1, TC = col_tile_cols(L1, INV);
    std::set<int> used;
    for (int r = 0; r < n1; ++r)
        for (int c = 0; c < TC; ++c) {
            const int a = tile_row<L1, INV>(r) + c;
            CHECK((a >= 0 && a < col_tile_words(L1, INV)), "col L1=%d kind=%d out of tile", L1, INV);
            CHECK(used.insert(a).second, "col L1=%d kind=%d collision", L1, INV);
        }
    // 16-byte quads of a row stay inside the row and 16-byte aligned
    for (int r = 0; r < n1; ++r) CHECK((tile_row<L1, INV>(r) % 4 == 0), "col L1=%d kind=%d quad alignment", L1, INV);
    CHECK((col_smem_bytes(L1, INV) <= 227 * 1024), "col L1=%d kind=%d shared memory", L1, INV);
    col_levels<L1, INV, 0>();
}

template <int L1>
void col_plan_check() {
    col_kind_check<L1, 0>();
    col_kind_check<L1, 1>();
    col_kind_check<L1, 2>();
    const LevelPlan PL = col_plan(L1);
    std::vector<int> k(1 << L1, 0);
    for (u32 s = 0; s < (1u << L1); ++s) {
        const u32 v = col_slot_to_k1(s, PL, L1);
        CHECK(v < (1u << L1), "col_slot_to_k1 L1=%d", L1);
        if (v < (1u << L1)) k[v]++;
    }
    for (int i = 0; i < (1 << L1); ++i) CHECK(k[i] == 1, "col_slot_to_k1 L1=%d not a permutation", L1);
}

// Natural-order reorder of k_row_ntt: swz_nat is a bijection, and the
// stores of one step (lanes r = 32 w + lane, output j) hit distinct banks.
template <int L2>
void ntt_reorder_check() {
    constexpr int n2 = 1 << L2;
    std::vector<int> hit(n2, 0);
    for (int f = 0; f < n2; ++f) {
        const int a = swz_nat(f);
        CHECK((a >= 0 && a < n2), "reorder L2=%d range", L2);
        if (a >= 0 && a < n2) hit[a]++;
    }
    for (int i = 0; i < n2; ++i) CHECK(hit[i] == 1, "reorder L2=%d bijection", L2);
    for (int w = 0; w * 32 < n2 / 32; ++w)
        for (int j = 0; j < 32; ++j) {
            int banks[32] = {0};
            for (int l = 0; l < 32 && w * 32 + l < n2 / 32; ++l)
                banks[swz_nat((int)row_pos_to_freq<L2>((u32)((w * 32 + l) * 32 + j))) % 32]++;
            for (int b = 0; b < 32; ++b) CHECK(banks[b] <= 1, "reorder L2=%d bank conflict", L2);
        }
}

// G's row spectrum between the row kernels: quad c of 32-word group r at
// c * n2/8 + 4 r, a permutation of the row's quads; the lanes of a warp
// (consecutive r) cover one contiguous 512-byte run per quad index.
template <int L2>
void spectrum_layout_check() {
    constexpr int n2 = 1 << L2, G = n2 / 32;
    std::vector<int> hit(n2 / 4, 0);
    for (int r = 0; r < G; ++r)
        for (int c = 0; c < 8; ++c) {
            const int w = c * (n2 / 8) + 4 * r;
            CHECK((w % 4 == 0 && w + 3 < n2), "spectrum L2=%d quad in row", L2);
            if (w % 4 == 0 && w + 3 < n2) hit[w / 4]++;
            if (r % 32 != 0) CHECK(w == c * (n2 / 8) + 4 * (r - 1) + 4, "spectrum L2=%d warp run", L2);
        }
    for (int q = 0; q < n2 / 4; ++q) CHECK(hit[q] == 1, "spectrum L2=%d quad %d hit %d", L2, q, hit[q]);
}

template <int L2>
void row_tab_check() {
    using RT = RowTab<L2>;
    CHECK(RT::NA * RT::NB == RT::TB0, "rowtab L2=%d digits", L2);
    for (int o = 0; o < RT::TB0; ++o) {
        CHECK((o % RT::NA) + RT::NA * (o / RT::NA) == o, "rowtab L2=%d recompose", L2);
        for (int j = 0; j < RT::R0; ++j) {
            const int ia = (o % RT::NA) + j * RT::NA;
            const int ib = RT::R0 * RT::NA + o / RT::NA + j * RT::NB;
            CHECK(ia >= 0 && ia < RT::R0 * RT::NA, "rowtab L2=%d A index", L2);
            CHECK(ib >= RT::R0 * RT::NA && ib < RT::ENTRIES, "rowtab L2=%d B index", L2);
        }
    }
    // build loop (row_tab_build's decode): every table slot written once, the
    // power and twiddle read for it in bounds and of the slot's exponent
    std::vector<int> hit(RT::ENTRIES, 0);
    for (int q = 0; q < RT::ENTRIES; ++q) {
        const int j = q % RT::R0;
        int e, w, at;
        if (q < RT::R0 * RT::NA) { const int a = q / RT::R0; e = a; w = a; at = j * RT::NA + a; }
        else { const int k = (q - RT::R0 * RT::NA) / RT::R0; e = k * RT::NA; w = RT::NA + k; at = RT::R0 * RT::NA + j * RT::NB + k; }
        CHECK(at >= 0 && at < RT::ENTRIES, "rowtab L2=%d build slot", L2);
        if (at >= 0 && at < RT::ENTRIES) hit[at]++;
        CHECK(w >= 0 && w < RT::NPOW, "rowtab L2=%d build power", L2);
        CHECK(e * RT::R0 + j < plan_tw_entries(row_plan(L2), L2), "rowtab L2=%d build twiddle", L2);
        // the slot the level reads for (o, j) has exponent o mod NA, resp. NA (o div NA)
        if (q < RT::R0 * RT::NA) CHECK(at % RT::NA == e && at / RT::NA == j, "rowtab L2=%d A exponent", L2);
        else CHECK((at - RT::R0 * RT::NA) % RT::NB * RT::NA == e, "rowtab L2=%d B exponent", L2);
    }
    for (int i = 0; i < RT::ENTRIES; ++i) CHECK(hit[i] == 1, "rowtab L2=%d slot %d written %d times", L2, i, hit[i]);
    // shared memory of the split row kernels (+1 KiB reserved per CTA)
    const long long smem = (long long)(1 << L2) * 4 + (long long)RT::TABW * 8 + (long long)RT::NPOW * 4 + 2 * RT::R0 * 8;
    CHECK((RT::TABW * 8) % 16 == 0, "rowtab L2=%d table not a whole number of 16-byte copies", L2);
    // the natural-order row kernel holds the row and the forward table
    CHECK(((long long)(1 << L2) * 4 + (long long)RT::TABW * 8 + RT::R0 * 8 + 1024) * ntt_row_ctas(L2) <= 228 * 1024,
          "ntt row L2=%d shared memory", L2);
    CHECK((smem + 1024) * rowsplit_ctas(L2) <= 228 * 1024, "rowsplit L2=%d shared memory", L2);
}

template <int L1, int KIND>
void col_pipe_check() {
    constexpr LevelPlan PL = col_plan(L1);
    constexpr int n1 = 1 << L1, HALF = n1 / 2, R0 = 1 << PL.logr[0], R1 = 1 << PL.logr[1];
    constexpr int TC = col_tile_cols(L1, KIND), QR = TC / 4;
    constexpr int TW = col_tile_words(L1, KIND);
    const int SW = tile_row<L1, KIND>(HALF);
    CHECK(PL.nlev == 2 && R0 * R1 == n1, "colpipe L1=%d plan", L1);
    // stage copies of rows [0, HALF) and tile copies of rows [HALF, n1)
    for (int idx = 0; idx < n1 * QR; ++idx) {
        const int r = idx / QR, q = idx % QR;
        const int a = tile_row<L1, KIND>(r) + 4 * q;
        CHECK((a % 4 == 0 && a + 3 < (r < HALF ? SW : TW)), "colpipe L1=%d kind=%d copy", L1, KIND);
    }
    for (int o = 0; o < R1; ++o)
        for (int m = 0; m < R0; ++m) {
            const int row = o + R1 * m;
            CHECK((tile_row<L1, KIND>(o) + tile_step<L1, KIND, R1>(m) == tile_row<L1, KIND>(row)), "colpipe L1=%d level-0 step", L1);
            if (m < R0 / 2) CHECK((row < HALF && tile_row<L1, KIND>(row) + TC <= SW), "colpipe L1=%d stage row", L1);
            else CHECK(row >= HALF, "colpipe L1=%d upper row", L1);
            CHECK(o * R0 + m < col_tw_entries(L1), "colpipe L1=%d twiddle", L1);
        }
    for (int blk = 0; blk < R0; ++blk)
        for (int m = 0; m < R1; ++m)
            CHECK((tile_row<L1, KIND>(blk * R1) + tile_step<L1, KIND, 1>(m) == tile_row<L1, KIND>(blk * R1 + m)), "colpipe L1=%d level-1 step", L1);
    if (KIND == col_pipe_kind(L1)) {
        CHECK(col_pipe_smem_bytes(L1) == TW * 4 + SW * 4 + col_tw_entries(L1) * 8, "colpipe L1=%d layout", L1);
        CHECK((col_pipe_smem_bytes(L1) + 1024) * col_pipe_ctas(L1) <= 228 * 1024, "colpipe L1=%d shared memory", L1);
    }
}

template <int L1>
void col_inv_pipe_check() {
    constexpr LevelPlan PL = col_plan(L1);
    constexpr int n1 = 1 << L1, R0 = 1 << PL.logr[0], R1 = 1 << PL.logr[1];
    constexpr int TC = col_tile_cols(L1, 1), QR = TC / 4, TW = col_tile_words(L1, 1);
    // stage copies: every 16-byte quad of every row inside the stage, aligned
    for (int idx = 0; idx < n1 * QR; ++idx) {
        const int r = idx / QR, q = idx % QR;
        const int a = tile_row<L1, 1>(r) + 4 * q;
        CHECK((a % 4 == 0 && a + 3 < TW), "colinvpipe L1=%d stage quad", L1);
    }
    // deepest level (blocks of R1 rows) and level 0 (rows o + R1 m): in the tile
    for (int id = 0; id < R0; ++id)
        for (int m = 0; m < R1; ++m)
            CHECK((tile_row<L1, 1>(id * R1) + tile_step<L1, 1, 1>(m) == tile_row<L1, 1>(id * R1 + m)), "colinvpipe L1=%d deep", L1);
    for (int o = 0; o < R1; ++o)
        for (int m = 0; m < R0; ++m) {
            CHECK((tile_row<L1, 1>(o) + tile_step<L1, 1, R1>(m) == tile_row<L1, 1>(o + R1 * m)), "colinvpipe L1=%d lvl0", L1);
            CHECK(o * R0 + m < n1, "colinvpipe L1=%d twiddle", L1);
        }
    CHECK(col_inv_pipe_smem_bytes(L1) + 1024 <= 228 * 1024, "colinvpipe L1=%d shared memory", L1);
    // per-warp refill: warp w's deepest-level blocks are exactly the rows it
    // copies, [w SUB R1, (w + 1) SUB R1), and the warps cover all n1 rows once
    constexpr int NW = col_inv_pipe_warps(L1), SUB = 32 / TC;
    CHECK(NW * SUB == R0, "colinvpipe L1=%d one block set per warp", L1);
    std::vector<int> rows(n1, 0);
    for (int w = 0; w < NW; ++w)
        for (int l = 0; l < 32; ++l) {
            const int blk = w * SUB + l / TC;
            CHECK((blk * R1 >= w * SUB * R1 && (blk + 1) * R1 <= (w + 1) * SUB * R1), "colinvpipe L1=%d warp blocks", L1);
            for (int r = w * SUB * R1 + l / QR; r < (w + 1) * SUB * R1; r += 32 / QR)
                if (l % QR == 0) rows[r]++;
        }
    for (int r = 0; r < n1; ++r) CHECK(rows[r] == 1, "colinvpipe L1=%d refill row %d copied %d times", L1, r, rows[r]);
}

void shoup_quot_check() {
    const u32 primes[] = {469762049u, 754974721u, 962592769u, 950009857u, 940572673u, 998244353u,
                          257u, 7681u, 12289u, 40961u, 1073479681u};
    unsigned long long st = 0x9E3779B97F4A7C15ull;
    for (u32 p : primes) {
        const double r = 4294967296.0 / (double)p;
        for (int k = 0; k < 200000; ++k) {
            st ^= st << 13; st ^= st >> 7; st ^= st << 17;
            u32 w = (u32)(st % p);
            if (k < 4) w = k < 2 ? (u32)k : p - (u32)(k - 1);
            const u32 want = (u32)(((unsigned long long)w << 32) / p);
            CHECK(shoup_quot_dev(w, p, r) == want, "shoup quotient p=%u w=%u", p, w);
        }
    }
}

int main() {
    row_plan_check<5>();
    row_plan_check<6>();
    row_plan_check<7>();
    row_plan_check<8>();
    row_plan_check<9>();
    row_plan_check<10>();
    row_plan_check<11>();
    row_plan_check<12>();
    row_plan_check<13>();
    row_plan_check<14>();
    col_plan_check<1>();
    col_plan_check<2>();
    col_plan_check<3>();
    col_plan_check<4>();
    col_plan_check<5>();
    col_plan_check<6>();
    col_plan_check<7>();
    col_plan_check<8>();
    col_plan_check<9>();
    col_plan_check<10>();
    col_plan_check<11>();
    ntt_reorder_check<10>();
    ntt_reorder_check<11>();
    ntt_reorder_check<12>();
    ntt_reorder_check<13>();
    ntt_reorder_check<14>();
    spectrum_layout_check<6>();
    spectrum_layout_check<10>();
    spectrum_layout_check<14>();
    row_tab_check<11>();
    row_tab_check<12>();
    row_tab_check<13>();
    row_tab_check<14>();
    col_pipe_check<9, 0>();
    col_pipe_check<10, 0>();
    col_pipe_check<10, 2>();
    CHECK(col_pipe1_smem_bytes(10) + 1024 <= 228 * 1024, "colpipe1 shared memory");
    CHECK(col_pipe1_smem_bytes(10) == 2 * col_tile_words(10, 2) * 4 + 1024 * 8, "colpipe1 layout");
    col_inv_pipe_check<9>();
    col_inv_pipe_check<10>();
    shoup_quot_check();
    std::printf("%s: %d failures\n", failures ? "FAILED" : "OK", failures);
    return failures ? 1 : 0;
}
