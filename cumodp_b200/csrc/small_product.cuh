// Fused single-CTA polynomial product for transform lengths L = 2^5 .. 2^14.
//
// One kernel does what the reference spreads over ~110 synchronised launches
// for one product (src/stockham.cu:521-611: expand_to_fft_dev x2,
// stockham_dev x3, get_powers_binary x2, pointwise_mul_dev,
// scale_vector_dev): load both operands with the zero pad, forward DIF of
// both (sharing every twiddle load), pointwise Montgomery product with the
// 1/L scale folded in, inverse DIT, truncation and store of the canonical
// residues.  Products of one size class are batched: each CTA holds
// `small_ppc` products and the grid covers the whole class.
#pragma once
#include "plans.cuh"

namespace cmb {

// One product job: h[0..lh) = (a[0..la) * b[0..lb)) mod p, coefficient
// order; a, b, h are device pointers (h may alias a or b only when the job
// is the sole job reading them).
struct ProdJob {
    const u32* a;
    const u32* b;
    u32* h;
    int la, lb, lh;
    int pad;
};

// A job as the single-CTA kernels keep it in shared memory: 32 bytes
// instead of 40 (operand lengths are at most 2^14 there), so that the job
// slots of a 128-product CTA take 4 KiB and six 32 KiB CTAs fit an SM.
struct SmemJob {
    const u32* a;
    const u32* b;
    u32* h;
    unsigned short la, lb;
    int lh;
};

// What the shared-memory row levels need: prime constants and the plan's
// twiddle tables.
struct RowCtx {
    PrimeK pk;
    const Tw* __restrict__ tw;  // forward level tables, then inverse tables
    int tw_inv_off;
};

struct SmallArgs {
    PrimeK pk;
    Tw scale;               // 2^32 / L mod p in Shoup form (undoes Montgomery R and 1/L)
    const Tw* __restrict__ tw;  // plan tables: forward levels then inverse levels
    const ProdJob* __restrict__ jobs;  // device job table, or nullptr: use job0
    int njobs;
    int tw_inv_off;         // entries before the inverse tables
    ProdJob job0;           // the single job when jobs == nullptr
};

#ifdef __CUDACC__

template <int LOGL, int LEV>
struct SmallLevel {
    static constexpr LevelPlan PL = row_plan(LOGL);
    static constexpr int R = 1 << PL.logr[LEV];
    // block size and table offset of this level
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

// Position in a row after the row plan's DIF levels -> frequency index.
template <int L2>
__host__ __device__ __forceinline__ u32 row_pos_to_freq(u32 P) {
    constexpr LevelPlan PL = row_plan(L2);
    u32 f = 0, mul = 1;
    int lb = L2;
#pragma unroll
    for (int i = 0; i < PL.nlev; ++i) {
        const int r = PL.logr[i];
        lb -= r;
        const u32 j = (P >> lb) & ((1u << r) - 1);
        f += rev_bits(j, r) * mul;
        mul <<= r;
    }
    return f;
}

// Forward non-last level on both operands of every product in the CTA.
template <int LOGL, int LEV, int T, int PPC, class Ctx>
__device__ __forceinline__ void small_fwd_level(u32* sm, const Ctx& A) {
    using LV = SmallLevel<LOGL, LEV>;
    constexpr int L = 1 << LOGL, R = LV::R, TB = LV::TB, B = LV::B;
    constexpr int TASKS = PPC * (L / R);
    const u32 p = A.pk.p, p2 = A.pk.p2;
    for (int id = threadIdx.x; id < TASKS; id += T) {
        const int q = id / (L / R);
        const int rest = id % (L / R);
        const int blk = rest / TB, o = rest % TB;
        const int base = q * 2 * L + blk * B + o;
        const int bs = swz(base), bsg = swz(base + L);
        u32 xf[R], xg[R];
#pragma unroll
        for (int m = 0; m < R; ++m) {
            xf[m] = sm[swz_task<TB, B>(base, bs, m)];
            xg[m] = sm[swz_task<TB, B>(base + L, bsg, m)];
        }
        dif_regs<R, true>(xf, A.pk.rc.f, p, p2);
        dif_regs<R, true>(xg, A.pk.rc.f, p, p2);
        Tw t[R];
        load_tw<R>(t, A.tw + LV::TWOFF + o * R);
#pragma unroll
        for (int j = 1; j < R; ++j) {
            xf[j] = mul_shoup(xf[j], t[j].w, t[j].wq, p);
            xg[j] = mul_shoup(xg[j], t[j].w, t[j].wq, p);
        }
#pragma unroll
        for (int m = 0; m < R; ++m) {
            sm[swz_task<TB, B>(base, bs, m)] = xf[m];
            sm[swz_task<TB, B>(base + L, bsg, m)] = xg[m];
        }
    }
}

// Inverse non-last level on the product held in the first operand slot.
template <int LOGL, int LEV, int T, int PPC, class Ctx>
__device__ __forceinline__ void small_inv_level(u32* sm, const Ctx& A) {
    using LV = SmallLevel<LOGL, LEV>;
    constexpr int L = 1 << LOGL, R = LV::R, TB = LV::TB, B = LV::B;
    constexpr int TASKS = PPC * (L / R);
    const u32 p = A.pk.p, p2 = A.pk.p2;
    for (int id = threadIdx.x; id < TASKS; id += T) {
        const int q = id / (L / R);
        const int rest = id % (L / R);
        const int blk = rest / TB, o = rest % TB;
        const int base = q * 2 * L + blk * B + o;
        const int bs = swz(base);
        u32 x[R];
#pragma unroll
        for (int m = 0; m < R; ++m) x[m] = sm[swz_task<TB, B>(base, bs, m)];
        Tw t[R];
        load_tw<R>(t, A.tw + A.tw_inv_off + LV::TWOFF + o * R);
#pragma unroll
        for (int j = 1; j < R; ++j) x[j] = mul_shoup(x[j], t[j].w, t[j].wq, p);
        dit_regs<R, true>(x, A.pk.rc.i, p, p2);
#pragma unroll
        for (int m = 0; m < R; ++m) sm[swz_task<TB, B>(base, bs, m)] = x[m];
    }
}

// Forward levels LEV .. nlev-2 (every level but the last).
template <int LOGL, int LEV, int T, int PPC, class Ctx>
__device__ __forceinline__ void small_fwd_levels(u32* sm, const Ctx& A) {
    constexpr LevelPlan PL = row_plan(LOGL);
    if constexpr (LEV + 1 < PL.nlev) {
        small_fwd_level<LOGL, LEV, T, PPC>(sm, A);
        __syncthreads();
        small_fwd_levels<LOGL, LEV + 1, T, PPC>(sm, A);
    }
}

// Inverse levels LEV, LEV-1, ..., STOP.
template <int LOGL, int LEV, int T, int PPC, int STOP, class Ctx>
__device__ __forceinline__ void small_inv_levels(u32* sm, const Ctx& A) {
    if constexpr (LEV >= STOP) {
        small_inv_level<LOGL, LEV, T, PPC>(sm, A);
        __syncthreads();
        small_inv_levels<LOGL, LEV - 1, T, PPC, STOP>(sm, A);
    }
}

// Single-operand forward level LEV (not the last) on a row in shared memory.
template <int LOGL, int LEV, int T>
__device__ __forceinline__ void fwd1_level(u32* sm, const PrimeK& pk, const Tw* __restrict__ tw) {
    using LV = SmallLevel<LOGL, LEV>;
    constexpr int L = 1 << LOGL, R = LV::R, TB = LV::TB, B = LV::B;
    const u32 p = pk.p, p2 = pk.p2;
    for (int id = threadIdx.x; id < L / R; id += T) {
        const int blk = id / TB, o = id % TB;
        const int base = blk * B + o;
        const int bs = swz(base);
        u32 x[R];
#pragma unroll
        for (int m = 0; m < R; ++m) x[m] = sm[swz_task<TB, B>(base, bs, m)];
        dif_regs<R, true>(x, pk.rc.f, p, p2);
        Tw t[R];
        load_tw<R>(t, tw + LV::TWOFF + o * R);
#pragma unroll
        for (int j = 1; j < R; ++j) x[j] = mul_shoup(x[j], t[j].w, t[j].wq, p);
#pragma unroll
        for (int m = 0; m < R; ++m) sm[swz_task<TB, B>(base, bs, m)] = x[m];
    }
}

template <int LOGL, int LEV, int T>
__device__ __forceinline__ void fwd1_levels(u32* sm, const PrimeK& pk, const Tw* __restrict__ tw) {
    constexpr LevelPlan PL = row_plan(LOGL);
    if constexpr (LEV + 1 < PL.nlev) {
        fwd1_level<LOGL, LEV, T>(sm, pk, tw);
        __syncthreads();
        fwd1_levels<LOGL, LEV + 1, T>(sm, pk, tw);
    }
}

__device__ __forceinline__ void load_row32(u32 (&x)[32], const u32* sm, int base) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint4 v = *reinterpret_cast<const uint4*>(sm + swz(base + 4 * c));
        x[4 * c] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
    }
}
__device__ __forceinline__ void store_row32(u32* sm, int base, const u32 (&x)[32]) {
#pragma unroll
    for (int c = 0; c < 8; ++c)
        *reinterpret_cast<uint4*>(sm + swz(base + 4 * c)) =
            make_uint4(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);
}

// The whole product of up to PPC jobs of one size class in one CTA of T =
// small_threads(LOGL) threads: gjobs[0, njobs) (device job table), shared
// memory sm (PPC * 2 * L words) and jobs (PPC entries).  C gives the prime
// constants and the plan tables (pk, tw, tw_inv_off); scale = 2^32 / L.
template <int LOGL, class Ctx>
__device__ __forceinline__ void small_product_body(const Ctx& C, Tw scale, const ProdJob* __restrict__ gjobs,
                                                   int njobs, u32* sm, SmemJob* jobs) {
    constexpr int L = 1 << LOGL;
    constexpr int T = small_threads(LOGL);
    constexpr int PPC = small_ppc(LOGL);
    constexpr LevelPlan PL = row_plan(LOGL);
    for (int q = threadIdx.x; q < PPC; q += T) {
        if (q < njobs) {
            const ProdJob g = gjobs[q];
            jobs[q] = SmemJob{g.a, g.b, g.h, (unsigned short)g.la, (unsigned short)g.lb, g.lh};
        } else {
            jobs[q] = SmemJob{nullptr, nullptr, nullptr, 0, 0, 0};
        }
    }
    __syncthreads();

    const u32 p = C.pk.p, p2 = C.pk.p2, oneq = C.pk.one_q;
    // load + zero pad + reduce to [0, 2p), kLoadBatch independent loads in
    // flight per thread before any is stored (one at a time, a thread waited
    // out a global-load latency per word)
    constexpr int TOT = PPC * 2 * L, kLoadBatch = 8;
    for (int base = threadIdx.x; base < TOT; base += kLoadBatch * T) {
        u32 v[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int idx = base + u * T;
            v[u] = 0u;
            if (idx < TOT) {
                const int q = idx / (2 * L);
                const int op = (idx / L) & 1;
                const int i = idx % L;
                const SmemJob& J = jobs[q];
                const u32* src = op ? J.b : J.a;
                const int len = op ? J.lb : J.la;
                if (i < len) v[u] = __ldg(src + i);
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int idx = base + u * T;
            if (idx < TOT) sm[swz(idx)] = mul_shoup(v[u], 1u, oneq, p);
        }
    }
    __syncthreads();

    small_fwd_levels<LOGL, 0, T, PPC>(sm, C);

    // last level (radix 32) forward on both operands, pointwise, inverse
    for (int id = threadIdx.x; id < PPC * (L / 32); id += T) {
        const int q = id / (L / 32);
        const int row = id % (L / 32);
        const int base = q * 2 * L + row * 32;
        u32 xf[32], xg[32];
        load_row32(xf, sm, base);
        load_row32(xg, sm, base + L);
        dif_regs<32>(xf, C.pk.rc.f, p, p2);
        dif_regs<32>(xg, C.pk.rc.f, p, p2);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            u32 h = mul_mont(xf[j], xg[j], p, C.pk.pinv_neg);
            xf[j] = mul_shoup(h, scale.w, scale.wq, p);
        }
        dit_regs<32>(xf, C.pk.rc.i, p, p2);
        store_row32(sm, base, xf);
    }
    __syncthreads();

    small_inv_levels<LOGL, PL.nlev - 2, T, PPC, 0>(sm, C);

    // truncate + canonical residues
    for (int idx = threadIdx.x; idx < PPC * L; idx += T) {
        const int q = idx / L, i = idx % L;
        const SmemJob& J = jobs[q];
        if (i < J.lh) J.h[i] = red1(red2(sm[swz(q * 2 * L + i)], p2), p);
    }
}

template <int LOGL>
__global__ void __launch_bounds__(small_threads(LOGL), small_ctas(LOGL))
k_small_product(const __grid_constant__ SmallArgs A) {
    constexpr int PPC = small_ppc(LOGL);
    extern __shared__ __align__(16) u32 sm[];
    __shared__ SmemJob jobs[PPC];
    const int job0 = blockIdx.x * PPC;
    if (A.jobs) {
        small_product_body<LOGL>(A, A.scale, A.jobs + job0, A.njobs - job0, sm, jobs);
    } else {
        small_product_body<LOGL>(A, A.scale, &A.job0, 1, sm, jobs);
    }
}

// ------------------------------------------------------------ work queue --
// All the small size classes of a batch (transforms of 2^5 .. 2^12 words:
// the classes whose CTA is 128 threads with 32 KiB of products in shared
// memory) in ONE persistent launch: each CTA takes the next work item -- up
// to small_ppc(logn) products of one class -- from a device counter until
// the queue is empty, so the classes share the SMs with no launch or tail
// per class, larger items first.
constexpr int kQueueMinLog = 5, kQueueMaxLog = 12;
constexpr int kQueueThreads = 128;  // small_threads(logn) for every queued class
constexpr int kQueueCtas = 6;       // small_ctas(logn) for every queued class
constexpr int kQueueSmemWords = 2 << kQueueMaxLog;  // small_ppc(logn) * 2 * 2^logn for every queued class

struct SmallItem {
    const ProdJob* jobs;  // the item's jobs (device job table of its class)
    int logn, njobs;      // njobs <= small_ppc(logn)
};

struct SmallQueueArgs {
    PrimeK pk;
    const Tw* tw[kQueueMaxLog + 1];  // plan tables of each class (forward then inverse)
    int tw_inv_off[kQueueMaxLog + 1];
    Tw scale[kQueueMaxLog + 1];      // 2^32 / 2^logn
    const SmallItem* __restrict__ items;
    int nitems;
    int* counter;                    // next item; zero before the launch
};

// The level functions' view of one class: the prime constants stay in the
// kernel parameters, the tables are the class's.
struct SmallQueueCtx {
    const PrimeK& pk;
    const Tw* __restrict__ tw;
    int tw_inv_off;
};

template <int LOGL>
__device__ __forceinline__ void small_queue_item(const SmallQueueArgs& Q, const SmallItem& I, u32* sm,
                                                 SmemJob* jobs) {
    static_assert(small_threads(LOGL) == kQueueThreads, "queued classes run on 128 threads");
    static_assert(small_ppc(LOGL) * 2 * (1 << LOGL) == kQueueSmemWords, "queued classes fill 32 KiB");
    const SmallQueueCtx C{Q.pk, Q.tw[LOGL], Q.tw_inv_off[LOGL]};
    small_product_body<LOGL>(C, Q.scale[LOGL], I.jobs, I.njobs, sm, jobs);
}

// (a template only so that every file including this header shares one kernel)
template <int MAXLOG>
__global__ void __launch_bounds__(kQueueThreads, kQueueCtas) k_small_queue(const __grid_constant__ SmallQueueArgs Q) {
    static_assert(MAXLOG == kQueueMaxLog, "the queued classes");
    extern __shared__ __align__(16) u32 sm[];
    __shared__ SmemJob jobs[small_ppc(kQueueMinLog)];
    __shared__ int item;
    for (;;) {
        if (threadIdx.x == 0) item = atomicAdd(Q.counter, 1);
        __syncthreads();
        const int it = item;
        if (it >= Q.nitems) return;
        const SmallItem I = Q.items[it];
        switch (I.logn) {
            case 5: small_queue_item<5>(Q, I, sm, jobs); break;
            case 6: small_queue_item<6>(Q, I, sm, jobs); break;
            case 7: small_queue_item<7>(Q, I, sm, jobs); break;
            case 8: small_queue_item<8>(Q, I, sm, jobs); break;
            case 9: small_queue_item<9>(Q, I, sm, jobs); break;
            case 10: small_queue_item<10>(Q, I, sm, jobs); break;
            case 11: small_queue_item<11>(Q, I, sm, jobs); break;
            case 12: small_queue_item<12>(Q, I, sm, jobs); break;
            default: break;
        }
        __syncthreads();  // the item's shared memory, jobs and `item` are free again
    }
}

#endif  // __CUDACC__

}  // namespace cmb
