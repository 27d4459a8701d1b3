// Natural-order transforms behind cumodp_fft_uni / cumodp_invfft_uni and
// the bivariate entry points.
//
// Reference behaviour: stockham_host / inverse_stockham_host
// (src/stockham.cu:479-503) compute X[j] = sum_i X[i] w^(ij) in natural
// order with the caller's root; bivariate_stockham_host
// (src/list_stockham.cu:1224-1245) computes the row-column 2-D DFT
// (DFT_m (x) I_n)(I_m (x) DFT_n) of a row-major 2^em x 2^en array.
//
// Here a transform of length <= 2^14 is one CTA (levels in shared memory,
// then an in-CTA reorder to natural order).  Longer 1-D transforms use the
// four-step split of the product path: a column pass (k_col_fwd), a row
// pass that applies w_n^(k1*c), transforms the row and writes it back in
// natural order as row k1, and a tiled transpose.  The 2-D transform is the
// column pass plus the row pass with no inter-pass twiddle: its rows land
// directly in natural order.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/cumodp.h"
#include "product.cuh"

namespace cmb {

struct RowNttArgs {
    PrimeK pk;
    const Tw* __restrict__ twr;
    const u32* __restrict__ seeds;  // inter-pass twiddles w_n^(k1 c) (nullptr: none)
    int nlo, nhi;
    int l1;                         // rows come from a column pass of length 2^l1 (0: none)
    LevelPlan colpl;
    const u32* src;                 // row slot s at src + s * n2
    u32* dst;                       // natural row k1 at dst + k1 * n2
    Tw scale;                       // applied to every output (folded into level 0's input factors)
    int rows_in_place;              // 1: independent rows, row s written to dst row s
    const Tw* __restrict__ rowtab;  // per-slot level-0 factor tables (RowTab, forward direction), or nullptr
    long long job_stride;           // words between the transforms of grid row blockIdx.y (list transforms)
};

__device__ __forceinline__ u32 seed_mont_at(const u32* __restrict__ seeds, int nlo, u32 e, u32 p, u32 pinv) {
    return mul_mont(__ldg(seeds + (e & 4095u)), __ldg(seeds + nlo + (e >> 12)), p, pinv);
}


// One row of the natural-order transform per CTA: the row (a column-pass
// output row, or an independent row) is copied into shared memory with
// cp.async, level 0 applies the inter-pass twiddle w_n^(k1 c) (or reduces
// the input), the remaining levels run as in the product kernels, and the
// last level leaves each thread one 32-word group in registers; after a
// barrier the groups are written back at their natural positions in the same
// buffer, and the row is stored with 16-byte accesses.  With the prebuilt
// per-slot factor tables (rows of 2^11-2^14 words) level 0 is that of the
// product's row kernels: inputs times W^(TB0 m), DIF, outputs times the two
// shared-memory factors of U_j^o.  The output scale (the inverse transform's
// 2^-k) is folded into level 0's input factors, so a transform is linear in
// it at no cost per word: the last level only reduces to [0, p).
//
// QOUT (rows of a four-step transform that a permuting transpose,
// k_transpose64_q, puts in natural order): the in-row reorder is skipped and
// each thread stores its last-level groups straight from registers in the
// layout of the product's row spectra -- digit-reversed positions, quad c of
// 32-word group r at c n2/8 + 4r, so a warp store covers one contiguous
// 512-byte run -- with the split row kernels' CTA shape (256 threads, three
// CTAs per SM for 2^14-word rows).
template <int L2, bool QOUT = false>
__global__ void __launch_bounds__(QOUT ? rowsplit_threads(L2) : ntt_row_threads(L2),
                                  QOUT ? rowsplit_ctas(L2) : ntt_row_ctas(L2))
    k_row_ntt(const __grid_constant__ RowNttArgs A) {
    constexpr int n2 = 1 << L2;
    constexpr int T = QOUT ? rowsplit_threads(L2) : ntt_row_threads(L2);
    constexpr LevelPlan PL = row_plan(L2);
    static_assert(PL.nlev >= 2, "row transform needs two levels");
    static_assert(QOUT || T * 32 >= n2, "one last-level group per thread");
    using LV0 = SmallLevel<L2, 0>;
    constexpr int R0 = LV0::R, TB0 = LV0::TB;
    extern __shared__ __align__(16) u32 sm[];
    __shared__ Tw bf[R0];

    const u32 s = blockIdx.x;
    const u32 k1 = A.l1 ? col_slot_to_k1(s, A.colpl, A.l1) : 0u;
    const u32 out_row = A.rows_in_place ? s : k1;
    const bool twid = A.seeds != nullptr;
    const u32 nmask = (1u << (A.l1 + L2)) - 1;
    const u32 p = A.pk.p, p2 = A.pk.p2, pinv = A.pk.pinv_neg;
    using RT = RowTab<L2>;
    const bool tabbed = RT::USE && twid && A.rowtab;
    const bool scaled = A.scale.w != 1u;
    Tw* tab = reinterpret_cast<Tw*>(sm + n2);
    const size_t joff = (size_t)blockIdx.y * (size_t)A.job_stride;
    row_load_issue<L2, T>(sm, A.src + joff + (size_t)s * n2);
    if (tabbed) {
        const Tw* src = A.rowtab + (size_t)s * RT::TABW;  // forward direction
        for (int i = threadIdx.x; i < RT::TABW / 2; i += T) {
            const unsigned d = (unsigned)__cvta_generic_to_shared(tab + 2 * i);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 2 * i) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    } else if (twid && threadIdx.x < R0) {
        const u32 e = (k1 * (u32)TB0 * threadIdx.x) & nmask;
        u32 v = red1(mul_mont(seed_mont_at(A.seeds, A.nlo, e, p, pinv), 1u, p, pinv), p);
        if (scaled) v = mulmod_exact(v, A.scale.w, p);
        bf[threadIdx.x] = Tw{v, shoup_quot(v, p)};
    }
    row_load_wait();
    __syncthreads();
    if (tabbed && scaled) {  // the slot factors times the scale (factor 0 becomes the scale)
        if (threadIdx.x < R0) {
            Tw* vf = tab + RT::ENTRIES;
            const u32 v = threadIdx.x == 0 ? A.scale.w : mulmod_exact(vf[threadIdx.x].w, A.scale.w, p);
            vf[threadIdx.x] = Tw{v, shoup_quot(v, p)};
        }
        __syncthreads();
    }

    if constexpr (RT::USE) {
        if (tabbed) {
            const Tw* vf = tab + RT::ENTRIES;
            for (int o = threadIdx.x; o < TB0; o += T) {
                u32 x[R0];
                const int bs = swz(o);
#pragma unroll
                for (int m = 0; m < R0; ++m) {
                    const u32 v = sm[swz_task<TB0, n2>(o, bs, m)];
                    x[m] = m == 0 && !scaled ? v : mul_shoup(v, vf[m].w, vf[m].wq, p);
                }
                dif_regs<R0, true>(x, A.pk.rc.f, p, p2);
                const Tw* ta = tab + (o % RT::NA);
                const Tw* tb = tab + RT::R0 * RT::NA + o / RT::NA;
#pragma unroll
                for (int j = 0; j < R0; ++j) {
                    const Tw a = ta[j * RT::NA], b = tb[j * RT::NB];
                    x[j] = mul_shoup(mul_shoup(x[j], a.w, a.wq, p), b.w, b.wq, p);
                }
#pragma unroll
                for (int m = 0; m < R0; ++m) sm[swz_task<TB0, n2>(o, bs, m)] = x[m];
            }
        }
    }
    for (int o = threadIdx.x; o < (tabbed ? 0 : TB0); o += T) {
        u32 x[R0];
        const u32 mo = twid ? seed_mont_at(A.seeds, A.nlo, (k1 * (u32)o) & nmask, p, pinv) : 0u;
        const int bs = swz(o);
#pragma unroll
        for (int m = 0; m < R0; ++m) {
            const u32 v = sm[swz_task<TB0, n2>(o, bs, m)];
            if (twid) x[m] = mul_mont(v, mul_shoup(mo, bf[m].w, bf[m].wq, p), p, pinv);
            else if (scaled) x[m] = mul_shoup(v, A.scale.w, A.scale.wq, p);
            else x[m] = mul_shoup(v, 1u, A.pk.one_q, p);
        }
        dif_regs<R0, true>(x, A.pk.rc.f, p, p2);
        Tw t[R0];
        load_tw<R0>(t, A.twr + o * R0);
#pragma unroll
        for (int j = 1; j < R0; ++j) x[j] = mul_shoup(x[j], t[j].w, t[j].wq, p);
#pragma unroll
        for (int m = 0; m < R0; ++m) sm[swz_task<TB0, n2>(o, bs, m)] = x[m];
    }
    __syncthreads();
    fwd1_levels<L2, 1, T>(sm, A.pk, A.twr);

    if constexpr (QOUT) {
        u32* out = A.dst + joff + (size_t)out_row * n2;
        for (int r = threadIdx.x; r < n2 / 32; r += T) {
            u32 x[32];
            load_row32(x, sm, r * 32);
            dif_regs<32>(x, A.pk.rc.f, p, p2);
#pragma unroll
            for (int c = 0; c < 8; ++c)
                *reinterpret_cast<uint4*>(out + c * (n2 / 8) + 4 * r) =
                    make_uint4(red1(x[4 * c], p), red1(x[4 * c + 1], p), red1(x[4 * c + 2], p), red1(x[4 * c + 3], p));
        }
        return;
    }
    const int r = threadIdx.x;
    const bool has = r < n2 / 32;
    u32 x[32];
    if (has) {
        load_row32(x, sm, r * 32);
        dif_regs<32>(x, A.pk.rc.f, p, p2);
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] = red1(x[j], p);
    }
    __syncthreads();
    // natural order through shared memory (swz_nat layout: the reorder's
    // stores are conflict-free), read out word by word, consecutive lanes on
    // consecutive words
    if (has) {
#pragma unroll
        for (int j = 0; j < 32; ++j) sm[swz_nat((int)row_pos_to_freq<L2>((u32)(r * 32 + j)))] = x[j];
    }
    __syncthreads();
    u32* out = A.dst + joff + (size_t)out_row * n2;
#pragma unroll 4
    for (int i = threadIdx.x; i < n2; i += T) out[i] = sm[swz_nat(i)];
}

// out[c * rows + r] = in[r * cols + c] for rows and cols multiples of 64:
// 64 x 64 tiles through shared memory, 16-byte loads and stores, 256
// threads (16 x 16, four 4-word groups each).
__global__ void __launch_bounds__(256) k_transpose64(const u32* __restrict__ in, u32* __restrict__ out, int rows,
                                                     int cols) {
    __shared__ u32 t[64][65];
    in += (size_t)blockIdx.z * rows * cols;  // transform blockIdx.z of a list
    out += (size_t)blockIdx.z * rows * cols;
    const size_t c0 = (size_t)blockIdx.x * 64, r0 = (size_t)blockIdx.y * 64;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const u32* src = in + r0 * cols + c0 + 4 * tx;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int rr = ty + 16 * k;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(src + (size_t)rr * cols));
        t[rr][4 * tx] = v.x;
        t[rr][4 * tx + 1] = v.y;
        t[rr][4 * tx + 2] = v.z;
        t[rr][4 * tx + 3] = v.w;
    }
    __syncthreads();
    u32* dst = out + c0 * rows + r0 + 4 * tx;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int cc = ty + 16 * k;
        const uint4 v = make_uint4(t[4 * tx][cc], t[4 * tx + 1][cc], t[4 * tx + 2][cc], t[4 * tx + 3][cc]);
        *reinterpret_cast<uint4*>(dst + (size_t)cc * rows) = v;
    }
}

// out[f(c) * rows + r] = in[r * n2 + c] for rows a multiple of 64, where row
// r of `in` is a row spectrum in the layout k_row_ntt<L2, true> stores and
// f(c) is the frequency word c holds: word c = q n2/8 + 4 g + e (e < 4,
// g < n2/32) holds digit-reversed position P = 32 g + 4 q + e, whose
// frequency is row_pos_to_freq<L2>(P).  64 x 64 tiles through shared
// memory, 16-byte loads and stores (each of a tile's 64 words is one
// frequency, whose 64 rows are one 256-byte run of the output).
template <int L2>
__global__ void __launch_bounds__(256) k_transpose64_q(const u32* __restrict__ in, u32* __restrict__ out, int rows) {
    constexpr int n2 = 1 << L2;
    __shared__ u32 t[64][65];
    in += (size_t)blockIdx.z * rows * n2;  // transform blockIdx.z of a list
    out += (size_t)blockIdx.z * rows * n2;
    const int c0 = blockIdx.x * 64;
    const size_t r0 = (size_t)blockIdx.y * 64;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const u32* src = in + r0 * n2 + c0 + 4 * tx;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int rr = ty + 16 * k;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(src + (size_t)rr * n2));
        t[rr][4 * tx] = v.x;
        t[rr][4 * tx + 1] = v.y;
        t[rr][4 * tx + 2] = v.z;
        t[rr][4 * tx + 3] = v.w;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int cc = ty + 16 * k;
        const u32 c = (u32)(c0 + cc), q = c / (n2 / 8), g = (c % (n2 / 8)) / 4, e = c % 4;
        const u32 f = row_pos_to_freq<L2>(32 * g + 4 * q + e);
        const uint4 v = make_uint4(t[4 * tx][cc], t[4 * tx + 1][cc], t[4 * tx + 2][cc], t[4 * tx + 3][cc]);
        *reinterpret_cast<uint4*>(out + (size_t)f * rows + r0 + 4 * tx) = v;
    }
}

// out[c * rows + r] = in[r * cols + c]: 32 x 32 tiles through shared memory.
__global__ void k_transpose(const u32* __restrict__ in, u32* __restrict__ out, int rows, int cols) {
    __shared__ u32 t[32][33];
    in += (size_t)blockIdx.z * rows * cols;  // transform blockIdx.z of a list
    out += (size_t)blockIdx.z * rows * cols;
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
        t[y][threadIdx.x] = in[(size_t)(r0 + y) * cols + c0 + threadIdx.x];
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
        out[(size_t)(c0 + y) * rows + r0 + threadIdx.x] = t[threadIdx.x][y];
}

// Direct DFT for n <= 32, one CTA of n threads per vector (vector b at
// offset b * n): out[j] = scale * sum x_i w^(ij).
__global__ void k_tiny_dft(const u32* __restrict__ x, u32* __restrict__ y, int n, u32 w, u32 p, u32 scale) {
    __shared__ u32 xs[32], pw[32];
    const int j = threadIdx.x;
    x += (size_t)blockIdx.x * n;
    y += (size_t)blockIdx.x * n;
    xs[j] = x[j] % p;
    u32 t = 1;
    for (int i = 0; i < j; ++i) t = (u32)(((u64)t * w) % p);
    pw[j] = t;
    __syncthreads();
    u64 acc = 0;
    for (int i = 0; i < n; ++i) acc = (acc + (u64)xs[i] * pw[(i * j) & (n - 1)]) % p;
    y[j] = (u32)((acc * scale) % p);
}

namespace {

template <int L2>
void launch_row_ntt_t(const RowNttArgs& a, int rows, cudaStream_t st, int jobs) {
    const size_t smem = (size_t)(1 << L2) * sizeof(u32) + (size_t)RowTab<L2>::TABW * sizeof(Tw);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_row_ntt<L2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_row_ntt<L2><<<dim3(rows, jobs), ntt_row_threads(L2), smem, st>>>(a);
}

// The rows of a four-step transform with 2^14-word rows and at least 64 of
// them: k_row_ntt<14, true> then the permuting transpose into x_out (jobs
// transforms of rows x 2^14 words, w2 and x_out job_stride words apart).
void row_ntt_q_and_transpose(const RowNttArgs& a, int rows, u32* x_out, cudaStream_t st, int jobs) {
    constexpr int L2 = kMaxRowLog;
    const size_t smem = (size_t)(1 << L2) * sizeof(u32) + (size_t)RowTab<L2>::TABW * sizeof(Tw);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_row_ntt<L2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    cudaEvent_t e0;
    bool tr = pass_timing_begin(st, &e0);
    k_row_ntt<L2, true><<<dim3(rows, jobs), rowsplit_threads(L2), smem, st>>>(a);
    if (tr) pass_timing_end(st, "ntt_row", e0);
    tr = pass_timing_begin(st, &e0);
    k_transpose64_q<L2><<<dim3((1 << L2) / 64, rows / 64, jobs), 256, 0, st>>>(a.dst, x_out, rows);
    if (tr) pass_timing_end(st, "ntt_transpose", e0);
}
typedef void (*RowNttFn)(const RowNttArgs&, int, cudaStream_t, int);
const RowNttFn kRowNtt[15] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                              launch_row_ntt_t<6>, launch_row_ntt_t<7>, launch_row_ntt_t<8>,
                              launch_row_ntt_t<9>, launch_row_ntt_t<10>, launch_row_ntt_t<11>,
                              launch_row_ntt_t<12>, launch_row_ntt_t<13>, launch_row_ntt_t<14>};

// Forward-column launchers shared with the product path (single operand).
template <int L1>
void launch_colfwd1_t(const LargeArgs& a, int tiles, cudaStream_t st) {
    const size_t smem = col_smem_bytes(L1, 2);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_col_fwd<L1, col_warps(L1, 2), 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        attr = true;
    }
    k_col_fwd<L1, col_warps(L1, 2), 2><<<dim3(tiles, 1, a.njobs), col_warps(L1, 2) * 32, smem, st>>>(a);
}
typedef void (*ColFn)(const LargeArgs&, int, cudaStream_t);
const ColFn kColFwd1[12] = {nullptr, launch_colfwd1_t<1>, launch_colfwd1_t<2>, launch_colfwd1_t<3>,
                            launch_colfwd1_t<4>, launch_colfwd1_t<5>, launch_colfwd1_t<6>,
                            launch_colfwd1_t<7>, launch_colfwd1_t<8>, launch_colfwd1_t<9>,
                            launch_colfwd1_t<10>, launch_colfwd1_t<11>};

// w is a primitive 2^k-th root of unity mod p.
bool root_has_order(u32 w, int k, u32 p) {
    if (w == 0 || w >= p) return false;
    if (k == 0) return w == 1;
    return powmod_exact(w, 1ull << k, p) == 1 && powmod_exact(w, 1ull << (k - 1), p) == p - 1;
}

u32 inv_of(u32 a, u32 p) { return powmod_exact(a, p - 2, p); }

// Column pass of a single array (rows of n2 words, 2^l1 rows) into dst.
int column_pass(const PrimeCtx& pc, u32 root_c, int l1, int l2, const u32* src, long long len, u32* dst,
                int dev, cudaStream_t st, const LargeJob* djobs = nullptr, int njobs = 1) {
    int err = OK;
    const u32 p = pc.info.p;
    const Tw* twc = col_tables(dev, p, root_c, l1, &err);
    if (!twc) return err;
    LargeArgs A;
    memset(&A, 0, sizeof(A));
    A.pk = A.pkc = make_prime_k_for(pc.info, root_c, l1);
    A.twc = twc;
    A.twc_inv = plan_tw_entries(col_plan(l1), l1);
    A.l1 = l1;
    A.l2 = l2;
    A.colpl = col_plan(l1);
    A.job0 = LargeJob{src, nullptr, nullptr, (int)std::min<long long>(len, 1ll << 30), 0, 0, 0, dst, nullptr};
    A.jobs = djobs;  // a device job table (a list of transforms), or nullptr: job0
    A.njobs = njobs;
    if (!launch_col_fwd_pipe1(A, njobs, st)) kColFwd1[l1](A, (1 << l2) / col_tile_cols_rt(l1, 2), st);
    return OK;
}

// First radix-2 (decimation-in-frequency) step of a transform of n = 2h
// words with root w: y0[j] = s (x[j] + x[j+h]) and y1[j] = s (x[j] - x[j+h])
// w^j for j < h, written over x_out[j] and x_out[j+h] (x_out may be x_in:
// each thread reads and writes the same four pairs).  Then the even outputs
// are DFT_h(y0; w^2) and the odd ones DFT_h(y1; w^2).  w^j * 2^32 is the
// Montgomery product of the seed-table words w^(j mod 4096) 2^32 and
// w^(4096 floor(j / 4096)) 2^32.  Inputs are any 32-bit words (reduced
// here); s = 1 (scaled = 0) or the inverse transform's 2^-k.
__global__ void __launch_bounds__(256) k_split_dif(const u32* x_in, u32* x_out, long long h,
                                                   const u32* __restrict__ seeds, int nlo, PrimeK pk, Tw s,
                                                   int scaled) {
    const u32 p = pk.p;
    const uint4* a4 = reinterpret_cast<const uint4*>(x_in);
    const uint4* b4 = reinterpret_cast<const uint4*>(x_in + h);
    uint4* y0 = reinterpret_cast<uint4*>(x_out);
    uint4* y1 = reinterpret_cast<uint4*>(x_out + h);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < h / 4;
         q += (long long)gridDim.x * blockDim.x) {
        const uint4 av = a4[q], bv = b4[q];
        u32 a[4] = {av.x, av.y, av.z, av.w}, b[4] = {bv.x, bv.y, bv.z, bv.w}, u[4], v[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const u32 ra = red1(mul_shoup(a[t], 1u, pk.one_q, p), p);
            const u32 rb = red1(mul_shoup(b[t], 1u, pk.one_q, p), p);
            const u32 e = (u32)(4 * q + t);  // j < h <= 2^28
            const u32 wj = seed_mont_at(seeds, nlo, e, p, pk.pinv_neg);  // w^j 2^32, [0, 2p)
            u32 s0 = red1(ra + rb, p);
            u32 s1 = red1(mul_mont(ra - rb + p, wj, p, pk.pinv_neg), p);
            if (scaled) {
                s0 = red1(mul_shoup(s0, s.w, s.wq, p), p);
                s1 = red1(mul_shoup(s1, s.w, s.wq, p), p);
            }
            u[t] = s0;
            v[t] = s1;
        }
        y0[q] = make_uint4(u[0], u[1], u[2], u[3]);
        y1[q] = make_uint4(v[0], v[1], v[2], v[3]);
    }
}

// x[2m] = s0[m], x[2m+1] = s1[m] for m < h (the even and odd outputs of the
// split transform back in natural order).
__global__ void __launch_bounds__(256) k_interleave2(const u32* __restrict__ s0, const u32* __restrict__ s1,
                                                     u32* __restrict__ x, long long h) {
    const uint4* a4 = reinterpret_cast<const uint4*>(s0);
    const uint4* b4 = reinterpret_cast<const uint4*>(s1);
    uint4* x4 = reinterpret_cast<uint4*>(x);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < h / 4;
         q += (long long)gridDim.x * blockDim.x) {
        const uint4 a = a4[q], b = b4[q];
        x4[2 * q] = make_uint4(a.x, b.x, a.y, b.y);
        x4[2 * q + 1] = make_uint4(a.z, b.z, a.w, b.w);
    }
}

}  // namespace

int ntt_natural_dev(const u32* x_in, u32* x_out, int k, u32 w, u32 p, bool inverse, cudaStream_t st);

namespace {

// A transform longer than the four-step kernels' 2^kMaxLog: one radix-2
// step over HBM (k_split_dif, which also applies the inverse's scaling),
// the two half-length transforms with root^2 (recursively), and the
// interleave of their outputs.  root is the transform's own root (already
// inverted for an inverse transform).
int ntt_split_dev(const PrimeCtx& pc, const u32* x_in, u32* x_out, int k, u32 root, u32 sc, cudaStream_t st) {
    int err = OK;
    const u32 p = pc.info.p;
    const long long n = 1ll << k, h = n / 2;
    const int dev = current_device();
    const u32* seeds = seed_tables(dev, p, root, k, &err);
    if (!seeds) return err ? err : OUT_OF_MEMORY;
    u32* S = (u32*)workspace(dev, kWsSplitNtt + (k - kMaxLog - 1), (size_t)n * sizeof(u32), &err);
    if (!S) return err;
    const int grid = 4 * sm_count(dev);
    k_split_dif<<<grid, 256, 0, st>>>(x_in, x_out, h, seeds, (int)std::min<long long>(n, 4096), pc.pk,
                                      tw_of(sc, p), sc != 1u);
    const u32 root2 = mulmod_exact(root, root, p);
    if ((err = ntt_natural_dev(x_out, S, k - 1, root2, p, false, st)) != OK) return err;
    if ((err = ntt_natural_dev(x_out + h, S + h, k - 1, root2, p, false, st)) != OK) return err;
    k_interleave2<<<grid, 256, 0, st>>>(S, S + h, x_out, h);
    return cuda_err(cudaGetLastError());
}

}  // namespace

// x_out = DFT(x_in) with root w (inverse: root w^-1 and scaling by 2^-k).
int ntt_natural_dev(const u32* x_in, u32* x_out, int k, u32 w, u32 p, bool inverse, cudaStream_t st) {
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    if (k < 0) return ASSUMPTION_ERROR;
    if (k >= 6 && (((uintptr_t)x_in | (uintptr_t)x_out) & 15)) return ASSUMPTION_ERROR;  // 16-byte rows
    if (k > pc->info.two_adic) return FFT_SIZE_TOO_LARGE;
    if (!root_has_order(w, k, p)) return ASSUMPTION_ERROR;
    if (k > kMaxSplitLog) return FFT_SIZE_TOO_LARGE;
    const int dev = current_device();
    const u32 root = inverse ? inv_of(w, p) : w;
    const u32 sc = inverse ? inv_of((u32)((1ull << k) % p), p) : 1u;
    if (k > kMaxLog) return ntt_split_dev(*pc, x_in, x_out, k, root, sc, st);
    if (k <= 5) {
        k_tiny_dft<<<1, 1 << k, 0, st>>>(x_in, x_out, 1 << k, root, p, sc);
        return cuda_err(cudaGetLastError());
    }
    if (k <= kMaxSmallLog) {
        RowNttArgs A;
        memset(&A, 0, sizeof(A));
        const Tw* twr = row_tables(dev, p, root, k, &err);
        if (!twr) return err;
        A.pk = make_prime_k_for(pc->info, root, k);
        A.twr = twr;
        A.src = x_in;
        A.dst = x_out;
        A.scale = tw_of(sc, p);
        cudaEvent_t e0;
        const bool tr = pass_timing_begin(st, &e0);
        kRowNtt[k](A, 1, st, 1);
        if (tr) pass_timing_end(st, "ntt_row", e0);
        return cuda_err(cudaGetLastError());
    }
    const int l1 = std::max(5, k - kMaxRowLog), l2 = k - l1;
    const long long n = 1ll << k;
    u32* ws = (u32*)workspace(dev, kWsNtt, (size_t)2 * n * sizeof(u32), &err);
    if (!ws) return err;
    u32 *w1 = ws, *w2 = ws + n;
    const u32 root_c = powmod_exact(root, 1ull << l2, p), root_r = powmod_exact(root, 1ull << l1, p);
    cudaEvent_t e0;
    bool tr = pass_timing_begin(st, &e0);
    if ((err = column_pass(*pc, root_c, l1, l2, x_in, n, w1, dev, st)) != OK) return err;
    if (tr) pass_timing_end(st, "ntt_col", e0);
    RowNttArgs A;
    memset(&A, 0, sizeof(A));
    const Tw* twr = row_tables(dev, p, root_r, l2, &err);
    const u32* seeds = seed_tables(dev, p, root, k, &err);
    if (!twr || !seeds) return err ? err : OUT_OF_MEMORY;
    A.pk = make_prime_k_for(pc->info, root_r, l2);
    A.twr = twr;
    A.seeds = seeds;
    A.nlo = (int)std::min<long long>(n, 4096);
    A.nhi = (int)std::max<long long>(1, n / 4096);
    A.l1 = l1;
    A.colpl = col_plan(l1);
    A.src = w1;
    A.dst = w2;
    A.scale = tw_of(sc, p);
    {
        LargeArgs LA;  // the level-0 factor tables of this root and shape (built once, cached)
        if (large_args(*pc, root, k, l2, dev, &LA) == OK) A.rowtab = LA.rowtab;
    }
    if (l1 >= 6 && l2 == kMaxRowLog) {
        row_ntt_q_and_transpose(A, 1 << l1, x_out, st, 1);
        return cuda_err(cudaGetLastError());
    }
    tr = pass_timing_begin(st, &e0);
    kRowNtt[l2](A, 1 << l1, st, 1);
    if (tr) pass_timing_end(st, "ntt_row", e0);
    tr = pass_timing_begin(st, &e0);
    if (l1 >= 6)
        k_transpose64<<<dim3((1 << l2) / 64, (1 << l1) / 64), 256, 0, st>>>(w2, x_out, 1 << l1, 1 << l2);
    else
        k_transpose<<<dim3((1 << l2) / 32, (1 << l1) / 32), dim3(32, 8), 0, st>>>(w2, x_out, 1 << l1, 1 << l2);
    if (tr) pass_timing_end(st, "ntt_transpose", e0);
    return cuda_err(cudaGetLastError());
}

namespace {

// m transforms of 2^k words (kMaxSmallLog < k <= kMaxLog), in place: the
// four-step passes of ntt_natural_dev, each launch covering up to
// min(2^16 - 1, 2^26 / 2^k) transforms (the column pass reads them from a
// job table, the row pass and the transpose take them from a grid
// dimension).  root is already inverted for an inverse transform.
int list_ntt_four_step(const PrimeCtx& pc, u32* x, long long m, int k, u32 root, u32 sc, cudaStream_t st) {
    int err = OK;
    const u32 p = pc.info.p;
    const int dev = current_device();
    const int l1 = std::max(5, k - kMaxRowLog), l2 = k - l1;
    const long long n = 1ll << k;
    const long long cm = std::min<long long>(m, std::max<long long>(1, std::min<long long>(65535, (1ll << 26) >> k)));
    u32* ws = (u32*)workspace(dev, kWsNtt, (size_t)2 * cm * n * sizeof(u32), &err);
    if (!ws) return err;
    LargeJob* dj = (LargeJob*)workspace(dev, kWsListJobs, (size_t)cm * sizeof(LargeJob), &err);
    if (!dj) return err;
    u32 *w1 = ws, *w2 = ws + cm * n;
    const u32 root_c = powmod_exact(root, 1ull << l2, p), root_r = powmod_exact(root, 1ull << l1, p);
    RowNttArgs A;
    memset(&A, 0, sizeof(A));
    const Tw* twr = row_tables(dev, p, root_r, l2, &err);
    const u32* seeds = seed_tables(dev, p, root, k, &err);
    if (!twr || !seeds) return err ? err : OUT_OF_MEMORY;
    A.pk = make_prime_k_for(pc.info, root_r, l2);
    A.twr = twr;
    A.seeds = seeds;
    A.nlo = (int)std::min<long long>(n, 4096);
    A.nhi = (int)std::max<long long>(1, n / 4096);
    A.l1 = l1;
    A.colpl = col_plan(l1);
    A.src = w1;
    A.dst = w2;
    A.scale = tw_of(sc, p);
    A.job_stride = n;
    {
        LargeArgs LA;
        if (large_args(pc, root, k, l2, dev, &LA) == OK) A.rowtab = LA.rowtab;
    }
    std::vector<LargeJob> hj((size_t)cm);
    for (long long r0 = 0; r0 < m; r0 += cm) {
        const int cnt = (int)std::min(cm, m - r0);
        for (int t = 0; t < cnt; ++t)
            hj[t] = LargeJob{x + (r0 + t) * n, nullptr, nullptr, (int)n, 0, 0, 0, w1 + (long long)t * n, nullptr};
        // pageable source: staged before the call returns, so hj is free to refill
        cudaError_t e = cudaMemcpyAsync(dj, hj.data(), (size_t)cnt * sizeof(LargeJob), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_err(e);
        if ((err = column_pass(pc, root_c, l1, l2, nullptr, n, nullptr, dev, st, dj, cnt)) != OK) return err;
        u32* out = x + r0 * n;
        if (l1 >= 6 && l2 == kMaxRowLog) {
            row_ntt_q_and_transpose(A, 1 << l1, out, st, cnt);
            continue;
        }
        kRowNtt[l2](A, 1 << l1, st, cnt);
        if (l1 >= 6)
            k_transpose64<<<dim3((1 << l2) / 64, (1 << l1) / 64, cnt), 256, 0, st>>>(w2, out, 1 << l1, 1 << l2);
        else
            k_transpose<<<dim3((1 << l2) / 32, (1 << l1) / 32, cnt), dim3(32, 8), 0, st>>>(w2, out, 1 << l1,
                                                                                          1 << l2);
    }
    return cuda_err(cudaGetLastError());
}

}  // namespace

// m independent natural-order transforms of length 2^k (row i at x + i 2^k),
// in place: the list transform I_m (x) DFT_n.
int list_ntt_dev(u32* x, long long m, int k, u32 w, u32 p, bool inverse, cudaStream_t st) {
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    if (m < 0 || k < 0) return ASSUMPTION_ERROR;
    if (k >= 6 && ((uintptr_t)x & 15)) return ASSUMPTION_ERROR;  // 16-byte rows
    if (m == 0) return OK;
    if (k > pc->info.two_adic) return FFT_SIZE_TOO_LARGE;
    if (!root_has_order(w, k, p)) return ASSUMPTION_ERROR;
    const u32 root = inverse ? inv_of(w, p) : w;
    const u32 sc = inverse ? inv_of((u32)((1ull << k) % p), p) : 1u;
    if (k <= 5) {
        for (long long r0 = 0; r0 < m; r0 += 65535) {
            const unsigned nb = (unsigned)std::min<long long>(65535, m - r0);
            k_tiny_dft<<<nb, 1 << k, 0, st>>>(x + (r0 << k), x + (r0 << k), 1 << k, root, p, sc);
        }
        return cuda_err(cudaGetLastError());
    }
    if (k <= kMaxSmallLog) {
        const int dev = current_device();
        const Tw* twr = row_tables(dev, p, root, k, &err);
        if (!twr) return err;
        RowNttArgs A;
        memset(&A, 0, sizeof(A));
        A.pk = make_prime_k_for(pc->info, root, k);
        A.twr = twr;
        A.scale = tw_of(sc, p);
        A.rows_in_place = 1;
        for (long long r0 = 0; r0 < m; r0 += (1ll << 30)) {
            A.src = x + (r0 << k);
            A.dst = x + (r0 << k);
            kRowNtt[k](A, (int)std::min<long long>(1ll << 30, m - r0), st, 1);
        }
        return cuda_err(cudaGetLastError());
    }
    if (k <= kMaxLog) return list_ntt_four_step(*pc, x, m, k, root, sc, st);
    for (long long r = 0; r < m; ++r)
        if ((err = ntt_natural_dev(x + (r << k), x + (r << k), k, w, p, inverse, st)) != OK) return err;
    return OK;
}

namespace {

// out[c * rows + r] = in[r * cols + c]: 32 x 32 tiles through shared memory,
// bounds-checked.  blockIdx.x runs over the longer side (rows_on_x), so any
// shape with rows * cols <= 2^30 fits the grid (the shorter side is then at
// most 2^15 long).
__global__ void k_transpose_long(const u32* __restrict__ in, u32* __restrict__ out, long long rows, long long cols,
                                 int rows_on_x) {
    __shared__ u32 t[32][33];
    const long long r0 = 32ll * (rows_on_x ? blockIdx.x : blockIdx.y);
    const long long c0 = 32ll * (rows_on_x ? blockIdx.y : blockIdx.x);
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
        if (r0 + y < rows && c0 + threadIdx.x < cols) t[y][threadIdx.x] = in[(r0 + y) * cols + c0 + threadIdx.x];
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
        if (c0 + y < cols && r0 + threadIdx.x < rows) out[(c0 + y) * rows + r0 + threadIdx.x] = t[threadIdx.x][y];
}

void transpose_long(const u32* in, u32* out, long long rows, long long cols, cudaStream_t st) {
    const unsigned tr = (unsigned)((rows + 31) / 32), tc = (unsigned)((cols + 31) / 32);
    const bool rx = tr >= tc;
    k_transpose_long<<<rx ? dim3(tr, tc) : dim3(tc, tr), dim3(32, 8), 0, st>>>(in, out, rows, cols, rx ? 1 : 0);
}

// A 2-D transform past the fused path's limits (columns longer than
// 2^kMaxColLog or rows longer than 2^kMaxRowLog): the rows as a list
// transform in place, then the columns as a list transform of the
// transposed array, transposed back.  Each list transform applies its own
// inverse scaling (2^-en, 2^-em).
int bivariate_general(u32* x, int em, u32 wm, int en, u32 wn, u32 p, bool inverse, cudaStream_t st) {
    int err = OK;
    if (em + en > 30) return FFT_SIZE_TOO_LARGE;
    const long long rows = 1ll << em, cols = 1ll << en;
    if ((err = list_ntt_dev(x, rows, en, wn, p, inverse, st)) != OK) return err;
    if (em == 0) return OK;
    u32* t = (u32*)workspace(current_device(), kWsBivT, (size_t)(rows * cols) * sizeof(u32), &err);
    if (!t) return err;
    transpose_long(x, t, rows, cols, st);
    if ((err = list_ntt_dev(t, cols, em, wm, p, inverse, st)) != OK) return err;
    transpose_long(t, x, cols, rows, st);
    return cuda_err(cudaGetLastError());
}

}  // namespace

// 2-D DFT of a row-major 2^em x 2^en array, in place.
int bivariate_dev(u32* x, int em, u32 wm, int en, u32 wn, u32 p, bool inverse, cudaStream_t st) {
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    if (em < 0 || en < 0) return ASSUMPTION_ERROR;
    if ((uintptr_t)x & 15) return ASSUMPTION_ERROR;  // 16-byte rows
    if (em > pc->info.two_adic || en > pc->info.two_adic) return FFT_SIZE_TOO_LARGE;
    if (!root_has_order(wm, em, p) || !root_has_order(wn, en, p)) return ASSUMPTION_ERROR;
    if (en < 6) return FFT_SIZE_TOO_SMALL;
    if (en > kMaxRowLog || em > kMaxColLog) return bivariate_general(x, em, wm, en, wn, p, inverse, st);
    const int dev = current_device();
    const u32 rm = inverse ? inv_of(wm, p) : wm, rn = inverse ? inv_of(wn, p) : wn;
    const u32 sc = inverse ? inv_of((u32)((1ull << (em + en)) % p), p) : 1u;
    const long long total = 1ll << (em + en);
    const Tw* twr = row_tables(dev, p, rn, en, &err);
    if (!twr) return err;
    RowNttArgs A;
    memset(&A, 0, sizeof(A));
    A.pk = make_prime_k_for(pc->info, rn, en);
    A.twr = twr;
    A.scale = tw_of(sc, p);
    A.dst = x;
    if (em == 0) {
        A.src = x;
        kRowNtt[en](A, 1, st, 1);
        return cuda_err(cudaGetLastError());
    }
    u32* w1 = (u32*)workspace(dev, kWsNtt, (size_t)total * sizeof(u32), &err);
    if (!w1) return err;
    if ((err = column_pass(*pc, rm, em, en, x, total, w1, dev, st)) != OK) return err;
    A.l1 = em;
    A.colpl = col_plan(em);
    A.src = w1;
    kRowNtt[en](A, 1 << em, st, 1);
    return cuda_err(cudaGetLastError());
}

// a[i] = a[i] * b[i] mod p (inputs in [0, p)): a Montgomery product
// (a b 2^-32) times r2 = 2^64 mod p by a second one, then one reduction.
__global__ void k_pointwise_mod(u32* __restrict__ a, const u32* __restrict__ b, long long n, u32 p, u32 pinv_neg,
                                u32 r2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = red1(mul_mont(mul_mont(a[i], b[i], p, pinv_neg), r2, p, pinv_neg), p);
}

// dst (2^ey2 rows of 2^ex2) = src (ny1 rows of nx1) zero-padded, reduced mod p.
__global__ void k_expand2(const u32* __restrict__ src, int nx1, int ny1, u32* __restrict__ dst, int ex2, int ey2,
                          u32 p) {
    const long long total = 1ll << (ex2 + ey2);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long y = i >> ex2, x = i & ((1ll << ex2) - 1);
        dst[i] = (x < nx1 && y < ny1) ? src[y * nx1 + x] % p : 0u;
    }
}

// dst (ny1 rows of nx1) = the top-left corner of src (rows of 2^ex2).
__global__ void k_extract2(const u32* __restrict__ src, int ex2, u32* __restrict__ dst, int nx1, int ny1) {
    const long long total = (long long)nx1 * ny1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long y = i / nx1, x = i % nx1;
        dst[i] = src[(y << ex2) + x];
    }
}

int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); }

// f <- f * g mod (x^n - 1, p), n = 2^e, for the lengths the product kernels
// do not cover (e < 5 or e > 25): natural-order transforms of f (in place)
// and of g (into workspace, so g is left as it is), the pointwise product and
// the inverse transform of f.
int cyclic_mul_compose(u32* f, const u32* g, int e, u32 p, cudaStream_t st) {
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    const long long n = 1ll << e;
    const u32 w = canonical_root(*pc, e);
    u32* gt = (u32*)workspace(current_device(), kWsCyclic, (size_t)n * sizeof(u32), &err);
    if (!gt) return err;
    if ((err = ntt_natural_dev(g, gt, e, w, p, false, st)) != OK) return err;
    if ((err = ntt_natural_dev(f, f, e, w, p, false, st)) != OK) return err;
    k_pointwise_mod<<<grid_for(n), 256, 0, st>>>(f, gt, n, p, pc->info.pinv_neg, pc->info.r2);
    if ((err = cuda_err(cudaGetLastError())) != OK) return err;
    return ntt_natural_dev(f, f, e, w, p, true, st);
}

// F <- DFT^-1(DFT F * DFT G) on a 2^em x 2^en row-major grid (rows: y, of
// length 2^en in x): the 2-D cyclic convolution, i.e. the bivariate product
// when both operands are zero-padded to the product's size.  Grids within
// the fused 2-D transform's limits use it (column pass + row pass per
// transform).  Otherwise: row transforms,
// a transpose, column transforms (as rows) give both spectra in transposed
// order; the pointwise product and the inverse steps run in that order, so
// nothing is permuted back before the last transpose.  G is overwritten.
int bivariate_mul_dev(u32* F, u32* G, int em, int en, u32 p, cudaStream_t st) {
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    if (em < 0 || en < 0) return ASSUMPTION_ERROR;
    if ((em >= 6 || en >= 6) && (((uintptr_t)F | (uintptr_t)G) & 15)) return ASSUMPTION_ERROR;  // 16-byte rows
    if (em > pc->info.two_adic || en > pc->info.two_adic || em + en > 30) return FFT_SIZE_TOO_LARGE;
    const long long m = 1ll << em, n = 1ll << en, total = m * n;
    const u32 wm = em ? canonical_root(*pc, em) : 1u, wn = en ? canonical_root(*pc, en) : 1u;
    if (en >= 6 && en <= kMaxRowLog && em <= kMaxColLog) {
        // grids the fused 2-D transform covers: two passes per transform, no transposes
        if ((err = bivariate_dev(F, em, wm, en, wn, p, false, st)) != OK) return err;
        if ((err = bivariate_dev(G, em, wm, en, wn, p, false, st)) != OK) return err;
        k_pointwise_mod<<<grid_for(total), 256, 0, st>>>(F, G, total, p, pc->info.pinv_neg, pc->info.r2);
        if ((err = bivariate_dev(F, em, wm, en, wn, p, true, st)) != OK) return err;
        return cuda_err(cudaGetLastError());
    }
    const int dev = current_device();
    const long long tpad = (total + 3) & ~3ll;  // 16-byte aligned halves
    u32* ws = (u32*)workspace(dev, kWsBiv, (size_t)2 * tpad * sizeof(u32), &err);
    if (!ws) return err;
    u32 *W1 = ws, *W2 = ws + tpad;
    u32* src[2] = {F, G};
    u32* spec[2] = {W1, W2};
    for (int o = 0; o < 2; ++o) {
        if ((err = list_ntt_dev(src[o], m, en, wn, p, false, st)) != OK) return err;
        transpose_long(src[o], spec[o], m, n, st);
        if ((err = list_ntt_dev(spec[o], n, em, wm, p, false, st)) != OK) return err;
    }
    k_pointwise_mod<<<grid_for(total), 256, 0, st>>>(W1, W2, total, p, pc->info.pinv_neg, pc->info.r2);
    if ((err = list_ntt_dev(W1, n, em, wm, p, true, st)) != OK) return err;
    transpose_long(W1, F, n, m, st);
    if ((err = list_ntt_dev(F, m, en, wn, p, true, st)) != OK) return err;
    return cuda_err(cudaGetLastError());
}

// Bivariate product of (nx, ny)-dense operands (coefficient of x^i y^j at
// j * nx + i), device buffers: H gets (nxf + nxg - 1) x (nyf + nyg - 1).
int bivariate_product_dev(const u32* F, int nxf, int nyf, const u32* G, int nxg, int nyg, u32* H, u32 p,
                          cudaStream_t st) {
    int err = OK;
    const long long lx = (long long)nxf + nxg - 1, ly = (long long)nyf + nyg - 1;
    int ex = 0, ey = 0;
    while ((1ll << ex) < lx) ++ex;
    while ((1ll << ey) < ly) ++ey;
    if (ex + ey > 30) return FFT_SIZE_TOO_LARGE;
    const long long total = 1ll << (ex + ey);
    const long long tpad = (total + 3) & ~3ll;  // 16-byte aligned halves
    u32* ws = (u32*)workspace(current_device(), kWsBivHost, (size_t)2 * tpad * sizeof(u32), &err);
    if (!ws) return err;
    u32 *F2 = ws, *G2 = ws + tpad;
    k_expand2<<<grid_for(total), 256, 0, st>>>(F, nxf, nyf, F2, ex, ey, p);
    k_expand2<<<grid_for(total), 256, 0, st>>>(G, nxg, nyg, G2, ex, ey, p);
    if ((err = bivariate_mul_dev(F2, G2, ey, ex, p, st)) != OK) return err;
    k_extract2<<<grid_for(lx * ly), 256, 0, st>>>(F2, ex, H, (int)lx, (int)ly);
    return cuda_err(cudaGetLastError());
}

}  // namespace cmb

using namespace cmb;

namespace {

cumodp_err host_ntt(sfixn* X, sfixn n, sfixn k, sfixn w, sfixn p, bool inverse) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (!X || k < 0 || k > 30 || n != (sfixn)(1u << k) || p <= 0) return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    const int dev = current_device();
    cudaStream_t st = lib_stream(dev);
    int err = OK;
    u32* d = (u32*)workspace(dev, kWsStage, (size_t)n * sizeof(u32), &err);
    if (!d) return (cumodp_err)err;
    cudaError_t ce = cudaMemcpyAsync(d, X, (size_t)n * 4, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return (cumodp_err)cuda_err(ce);
    err = ntt_natural_dev(d, d, k, (u32)w, (u32)p, inverse, st);
    if (err != OK) {
        cudaStreamSynchronize(st);
        return (cumodp_err)err;
    }
    ce = cudaMemcpyAsync(X, d, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    return (cumodp_err)cuda_err(ce);
}

cumodp_err host_bivariate(sfixn* X, sfixn em, sfixn wm, sfixn en, sfixn wn, sfixn p, bool inverse) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (!X || em < 0 || en < 0 || em + en > 30 || p <= 0) return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    const int dev = current_device();
    cudaStream_t st = lib_stream(dev);
    const size_t total = (size_t)1 << (em + en);
    int err = OK;
    u32* d = (u32*)workspace(dev, kWsStage, total * sizeof(u32), &err);
    if (!d) return (cumodp_err)err;
    cudaError_t ce = cudaMemcpyAsync(d, X, total * 4, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return (cumodp_err)cuda_err(ce);
    err = bivariate_dev(d, em, (u32)wm, en, (u32)wn, (u32)p, inverse, st);
    if (err != OK) {
        cudaStreamSynchronize(st);
        return (cumodp_err)err;
    }
    ce = cudaMemcpyAsync(X, d, total * 4, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    return (cumodp_err)cuda_err(ce);
}

}  // namespace

extern "C" {

cumodp_err cumodp_fft_uni_dev(sfixn* X, sfixn n, sfixn k, sfixn w, sfixn p, int inverse, void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (!X || k < 0 || k > 30 || n != (sfixn)(1u << k) || p <= 0) return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = ntt_natural_dev((const u32*)X, (u32*)X, k, (u32)w, (u32)p, inverse != 0, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

cumodp_err cumodp_fft_bivariate_dev(sfixn* X, sfixn em, sfixn wm, sfixn en, sfixn wn, sfixn p, int inverse,
                                    void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (!X || em < 0 || en < 0 || em + en > 30 || p <= 0) return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = bivariate_dev((u32*)X, em, (u32)wm, en, (u32)wn, (u32)p, inverse != 0, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

cumodp_err cumodp_list_fft_dev(sfixn* X, sfixn m, sfixn k, sfixn w, sfixn p, int inverse, void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (!X || m < 0 || k < 0 || k > 30 || p <= 0) return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = list_ntt_dev((u32*)X, m, k, (u32)w, (u32)p, inverse != 0, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

cumodp_err cumodp_bivariate_mul_dev(sfixn em, sfixn en, sfixn* F, sfixn* G, sfixn p, void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (!F || !G || em < 0 || en < 0 || p <= 0) return CUMODP_ASSUMPTION_ERROR;
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = bivariate_mul_dev((u32*)F, (u32*)G, em, en, (u32)p, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

cumodp_err cumodp_bivariate_mul(sfixn nxf, sfixn nyf, const sfixn* F, sfixn nxg, sfixn nyg, const sfixn* G,
                                sfixn* H, sfixn p) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (!F || !G || !H || nxf <= 0 || nyf <= 0 || nxg <= 0 || nyg <= 0 || p <= 0) return CUMODP_ASSUMPTION_ERROR;
    const long long nf = (long long)nxf * nyf, ng = (long long)nxg * nyg;
    const long long nh = ((long long)nxf + nxg - 1) * ((long long)nyf + nyg - 1);
    if (nh > (1ll << 30)) return CUMODP_FFT_SIZE_TOO_LARGE;
    std::lock_guard<std::mutex> g(lib_mutex());
    const int dev = current_device();
    cudaStream_t st = lib_stream(dev);
    int err = OK;
    u32* d = (u32*)workspace(dev, kWsStage, (size_t)(nf + ng + nh) * sizeof(u32), &err);
    if (!d) return (cumodp_err)err;
    cudaError_t ce = cudaMemcpyAsync(d, F, nf * 4, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(d + nf, G, ng * 4, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return (cumodp_err)cuda_err(ce);
    err = bivariate_product_dev(d, nxf, nyf, d + nf, nxg, nyg, d + nf + ng, (u32)p, st);
    if (err != OK) {
        cudaStreamSynchronize(st);
        return (cumodp_err)err;
    }
    ce = cudaMemcpyAsync(H, d + nf + ng, nh * 4, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    return (cumodp_err)cuda_err(ce);
}

cumodp_err cumodp_fft_uni(sfixn* X, sfixn n, sfixn k, sfixn w, sfixn p) { return host_ntt(X, n, k, w, p, false); }

cumodp_err cumodp_invfft_uni(sfixn* X, sfixn n, sfixn k, sfixn w, sfixn p) { return host_ntt(X, n, k, w, p, true); }

cumodp_err cumodp_fft_bivariate(sfixn* X, sfixn em, sfixn wm, sfixn en, sfixn wn, sfixn p) {
    return host_bivariate(X, em, wm, en, wn, p, false);
}

cumodp_err cumodp_invfft_bivariate(sfixn* X, sfixn em, sfixn wm, sfixn en, sfixn wn, sfixn p) {
    return host_bivariate(X, em, wm, en, wn, p, true);
}

}  // extern "C"
