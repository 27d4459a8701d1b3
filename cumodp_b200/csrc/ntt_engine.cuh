// CTA-level NTT building blocks for sm_100a.
//
// The reference computes every radix-2 Stockham step as three separate
// kernels over HBM (butterfly, stride permutation, twiddle;
// src/stockham.cu:75-397).  Here a transform of length L <= 2^14 lives in
// shared memory and is computed in a few "levels".  A level of radix
// R = 2^r splits each current block of size B into R strided sub-sequences
// (task o in [0, B/R) owns elements o + (B/R)*m, m < R), runs an R-point DFT
// in registers (r radix-2 stages, constants only), and multiplies output k
// of task o by w_B^(o*k) (four-step / Gentleman-Sande decomposition).  The
// forward transform is DIF (natural order in, digit-reversed order out); the
// inverse runs the transposed levels (DIT with inverse roots, digit-reversed
// in, natural out).  A product never needs natural-order spectra, so the
// forward/inverse pair needs no permutation at all.
//
// Butterflies follow Harvey's lazy reduction ("Faster arithmetic for
// number-theoretic transforms", J. Symb. Comp. 2014): forward values stay in
// [0, 2p), inverse values in [0, 4p).
#pragma once
#include "field.cuh"

namespace cmb {

// Root constants shared by every register DFT of radix <= 32:
// c[j] = w_32^j (forward) or w_32^-j (inverse) for j < 16, in Shoup form.
struct RootConsts {
    Tw f[16];
    Tw i[16];
};

// Per-prime constants passed by value to kernels (live in the constant bank).
struct PrimeK {
    u32 p, p2, pinv_neg;
    u32 one_q;  // shoup_quot(1, p): reduces any u32 to [0, 2p)
    RootConsts rc;
};

#ifdef __CUDACC__

// Shared-memory word index swizzle: the 16-byte quad inside each 32-word row
// is XOR-ed with (row & 7).  Scalar accesses by 32 lanes to 32 consecutive
// words and 16-byte accesses by lanes to consecutive 32-word rows (or to
// consecutive 16/8/4-word groups) are both bank-conflict free.
__host__ __device__ __forceinline__ int swz(int i) { return i ^ (((i >> 5) & 7) << 2); }

// swz(base + TB * m) for the m-th element of a level task, where base is a
// multiple of the block size B plus the task index o < TB, and m is an
// unrolled constant.  With TB a multiple of 256 words the row bits that feed
// the XOR do not change with m: the address is swz(base) + TB * m (an
// immediate offset).  With TB = 32 and B a multiple of 256, base lies in a
// row that is a multiple of 8, so the XOR is the constant (m & 7) << 2.
template <int TB, int B>
__host__ __device__ __forceinline__ int swz_task(int base, int bswz, int m) {
    if constexpr (TB % 256 == 0) return bswz + TB * m;
    else if constexpr (TB == 32 && B % 256 == 0) return (base ^ ((m & 7) << 2)) + 32 * m;
    else return swz(base + TB * m);
}

// The low r bits of j in reverse order.
// Word index swizzle of the natural-order reorder buffer: bits 0-3 XOR bits
// 5-8.  When the lanes of a warp each store one last-level output at its
// frequency, those frequencies share their low bits; the XOR spreads them
// over all 32 banks (for every row plan of 2^10-2^14 words).  A bijection
// on each 512-word block, and a permutation of every 32-word row, so a
// read-out of consecutive words by consecutive lanes is conflict-free too.
__host__ __device__ __forceinline__ int swz_nat(int f) { return f ^ ((f >> 5) & 15); }

__host__ __device__ __forceinline__ u32 rev_bits(u32 j, int r) {
#ifdef __CUDA_ARCH__
    return __brev(j) >> (32 - r);
#else
    u32 v = 0;
    for (int i = 0; i < r; ++i) v |= ((j >> i) & 1u) << (r - 1 - i);
    return v;
#endif
}

// Forward R-point DIF on registers; x[j] ends holding X[bitrev_r(j)].
// Inputs in [0, 2p).  Outputs in [0, 2p), except that with TW (the caller
// multiplies every output j >= 1 by a Shoup twiddle next, which accepts any
// 32-bit input) the last stage leaves outputs j >= 1 in [0, 4p).  H0 < R/2
// runs only the stages of butterfly span H0, H0/2, ..., 1 (the caller did
// the earlier ones).
template <int R, bool TW = false, int H0 = R / 2>
__device__ __forceinline__ void dif_regs(u32 (&x)[R], const Tw* __restrict__ c, u32 p, u32 p2) {
#pragma unroll
    for (int half = H0; half >= 1; half >>= 1) {
#pragma unroll
        for (int g = 0; g < R; g += 2 * half) {
#pragma unroll
            for (int j = 0; j < half; ++j) {
                const int e = j * (32 / (2 * half));  // w_{2half}^j = w_32^e
                const bool lazy = TW && half == 1;
                u32 a = x[g + j], b = x[g + j + half];
                u32 s = a + b;
                u32 d = a - b + p2;
                x[g + j] = (lazy && g + j != 0) ? s : red2(s, p2);
                x[g + j + half] = (e == 0) ? (lazy ? d : red2(d, p2)) : mul_shoup(d, c[e].w, c[e].wq, p);
            }
        }
    }
}

// Forward R-point DIF whose inputs R/2 .. R-1 are zero: x[0 .. R/2) hold
// raw words (any 32-bit value, reduced here) and x[R/2 .. R) are ignored.
// The first stage reduces to x[j] = v, x[j + R/2] = v * w_R^j; the rest is
// dif_regs.  Same output ranges as dif_regs<R, TW>.
template <int R, bool TW = false>
__device__ __forceinline__ void dif_regs_halfzero(u32 (&x)[R], const Tw* __restrict__ c, u32 p, u32 p2,
                                                  u32 one_q) {
#pragma unroll
    for (int j = 0; j < R / 2; ++j) {
        const int e = j * (32 / R);
        const u32 v = x[j];
        const u32 r = mul_shoup(v, 1u, one_q, p);
        x[j] = r;
        x[j + R / 2] = e == 0 ? r : mul_shoup(v, c[e].w, c[e].wq, p);
    }
    dif_regs<R, TW, R / 4>(x, c, p, p2);
}

// Inverse R-point DIT on registers (roots c = w_32^-j); x[j] holds Y[bitrev(j)]
// on entry and R * y[j] on exit.  Inputs and outputs in [0, 4p).  With PRE
// (the caller multiplied every input j >= 1 by a Shoup twiddle, so those are
// already in [0, 2p)) the first stage skips their reductions.
template <int R, bool PRE = false>
__device__ __forceinline__ void dit_regs(u32 (&x)[R], const Tw* __restrict__ c, u32 p, u32 p2) {
#pragma unroll
    for (int half = 1; half < R; half <<= 1) {
#pragma unroll
        for (int g = 0; g < R; g += 2 * half) {
#pragma unroll
            for (int j = 0; j < half; ++j) {
                const int e = j * (32 / (2 * half));
                const bool small_in = PRE && half == 1;
                u32 a = (small_in && g + j != 0) ? x[g + j] : red2(x[g + j], p2);
                u32 b = x[g + j + half];
                u32 t = (e == 0) ? (small_in ? b : red2(b, p2)) : mul_shoup(b, c[e].w, c[e].wq, p);
                x[g + j] = a + t;
                x[g + j + half] = a - t + p2;
            }
        }
    }
}

// Programmatic dependent launch: pdl_trigger lets the next kernel of the
// stream (launched with programmatic stream serialization) be scheduled as
// this grid's CTAs retire, to run its independent prologue; pdl_wait blocks
// until the previous kernel of the stream has completed and its writes are
// visible.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <int R>
__device__ __forceinline__ void load_tw(Tw (&t)[R], const Tw* __restrict__ src) {
    const uint4* s4 = reinterpret_cast<const uint4*>(src);
#pragma unroll
    for (int j = 0; j < R / 2; ++j) {
        uint4 v = __ldg(s4 + j);
        t[2 * j] = Tw{v.x, v.y};
        t[2 * j + 1] = Tw{v.z, v.w};
    }
}

#endif  // __CUDACC__

// --------------------------------------------------------------------------
// Level plans.  A plan is a list of log-radices r_1..r_m with sum = log2 L.
// Level i acts on blocks of size B_i = L >> (r_1 + ... + r_{i-1}).  Its
// twiddle table holds, for each task o < B_i / R_i and register slot j < R_i,
// w_{B_i}^(o * bitrev(j)) (forward) and the inverse root power (inverse), as
// Tw pairs; the last level needs none (B_m = R_m).
// --------------------------------------------------------------------------
struct LevelPlan {
    int nlev;
    int logr[6];
};

// Number of Tw entries one direction of a plan's tables needs.
__host__ __device__ inline int plan_tw_entries(const LevelPlan& pl, int logl) {
    int n = 0, lb = logl;
    for (int i = 0; i + 1 < pl.nlev; ++i) {
        n += 1 << lb;  // (B/R) * R entries
        lb -= pl.logr[i];
    }
    return n;
}

}  // namespace cmb
