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
//   orders:  col_slot_to_k1 and row_pos_to_freq are permutations.
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
    std::printf("%s: %d failures\n", failures ? "FAILED" : "OK", failures);
    return failures ? 1 : 0;
}
