// Batched products of uneven degree: size classes, autotuned splits, and one
// CUDA-graph launch per batch.
//
// The reference batches only same-size items (list_stockham_dev,
// src/list_stockham.cu:595-630, one root and one n for all m items, with the
// geometry in __constant__ globals), and a list product is explicit pad +
// list NTTs + list_pointwise_mul + list inverse + shrink
// (src/list_pointwise_mul.cu:43-194), each a separate synchronised launch.
// Here a batch of any degrees is planned once per shape:
//   * products are grouped by transform length n = 2^ceil(log2(la+lb-1));
//   * all classes with n <= 2^12 run in ONE persistent launch of the fused
//     kernel (k_small_queue): CTAs pull work items (up to small_ppc(n)
//     products of one class) from a device counter until none is left;
//   * a class of 2^13 or 2^14 runs on the fused single-CTA kernel or on the
//     three-pass kernels, as the autotuner measured faster for its size;
//   * a larger class is the three-pass product over all its jobs at once,
//     with the column/row split chosen by the autotuner;
//   * the queue and every other class run on their own branches of one CUDA
//     graph (classes are independent, so their kernels overlap on the
//     device), captured once and replayed; job tables and work items live in
//     device memory and are refreshed with one copy when the caller's
//     pointers change.
#include <algorithm>
#include <map>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <tuple>
#include <unordered_map>

#include "../../include/cumodp.h"
#include "product.cuh"

namespace cmb {

// ------------------------------------------------------------ autotuner ----
// Per size class of a batch the autotuner chooses, by timing on a synthetic
// class of the same shape (`jobs` products of two length-n/2 operands):
//   * kind 0: the row length 2^l2 of the three-pass split (every legal split);
//   * kind 1: for transforms of 2^13 and 2^14 words, one CTA per product
//     (the fused kernel: 256 / 512 threads, 64 / 128 KiB of shared memory)
//     or the three-pass kernels spread over the whole GPU (at the best split).
// Results are cached per (device model, kind, logn, job bucket) in memory and,
// when CUMODP_TUNE_FILE names a file, appended to it and reloaded at start-up;
// the device model (name, SM count, compute capability) keys the cache, so a
// file written on one GPU model is not used on another.
std::vector<int> legal_row_logs(int logn);

namespace {

struct TuneKey {
    std::string device;
    int kind, logn, bucket;
    bool operator<(const TuneKey& o) const {
        return std::tie(device, kind, logn, bucket) < std::tie(o.device, o.kind, o.logn, o.bucket);
    }
};

std::mutex g_tune_m;
std::map<TuneKey, int> g_tune;
bool g_tune_loaded = false;

int job_bucket(int njobs) {
    int b = 1;
    while (b < njobs && b < 256) b <<= 1;
    return b;
}

// "name/SMs/sm_major.minor" of device dev (cached).
const std::string& device_model(int dev) {
    static std::mutex m;
    static std::map<int, std::string> names;
    std::lock_guard<std::mutex> g(m);
    auto it = names.find(dev);
    if (it != names.end()) return it->second;
    cudaDeviceProp pr;
    std::string key = "unknown";
    if (cudaGetDeviceProperties(&pr, dev) == cudaSuccess) {
        char buf[320];
        snprintf(buf, sizeof(buf), "%s/%d/sm_%d.%d", pr.name, pr.multiProcessorCount, pr.major, pr.minor);
        key = buf;
        for (char& c : key)
            if (c == ' ') c = '_';
    } else {
        cudaGetLastError();
    }
    return names[dev] = key;
}

// File lines: "kind logn bucket value device-model".
void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* f = getenv("CUMODP_TUNE_FILE");
    if (!f) return;
    FILE* fh = fopen(f, "r");
    if (!fh) return;
    int kind, logn, bucket, value;
    char model[320];
    while (fscanf(fh, "%d %d %d %d %319s", &kind, &logn, &bucket, &value, model) == 5)
        g_tune[TuneKey{model, kind, logn, bucket}] = value;
    fclose(fh);
}

bool tune_lookup(const TuneKey& key, int* value) {
    std::lock_guard<std::mutex> g(g_tune_m);
    tune_load_locked();
    auto it = g_tune.find(key);
    if (it == g_tune.end()) return false;
    *value = it->second;
    return true;
}

void tune_store(const TuneKey& key, int value) {
    std::lock_guard<std::mutex> g(g_tune_m);
    g_tune[key] = value;
    if (const char* f = getenv("CUMODP_TUNE_FILE")) {
        if (FILE* fh = fopen(f, "a")) {
            fprintf(fh, "%d %d %d %d %s\n", key.kind, key.logn, key.bucket, value, key.device.c_str());
            fclose(fh);
        }
    }
}

// A synthetic class for timing: `jobs` products of two length-n/2 operands
// (zeros: the work does not depend on the values), as three-pass jobs and as
// single-CTA jobs.
struct TuneBufs {
    u32* buf = nullptr;
    LargeJob* djl = nullptr;
    ProdJob* djs = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool ok = false;
    TuneBufs(int jobs, long long n, cudaStream_t st) {
        if (dev_malloc((void**)&buf, (size_t)jobs * 4 * n * sizeof(u32)) != cudaSuccess ||
            dev_malloc((void**)&djl, jobs * sizeof(LargeJob)) != cudaSuccess ||
            dev_malloc((void**)&djs, jobs * sizeof(ProdJob)) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        cudaMemsetAsync(buf, 0, (size_t)jobs * 4 * n * sizeof(u32), st);
        std::vector<LargeJob> hl(jobs);
        std::vector<ProdJob> hs(jobs);
        for (int j = 0; j < jobs; ++j) {
            u32* base = buf + (size_t)j * 4 * n;
            hl[j] = LargeJob{base, base + n / 2, base + n, (int)(n / 2), (int)(n / 2), (int)(n - 1), 0,
                             base + 2 * n, base + 3 * n};
            hs[j] = ProdJob{base, base + n / 2, base + n, (int)(n / 2), (int)(n / 2), (int)(n - 1), 0};
        }
        cudaMemcpyAsync(djl, hl.data(), jobs * sizeof(LargeJob), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(djs, hs.data(), jobs * sizeof(ProdJob), cudaMemcpyHostToDevice, st);
        cudaStreamSynchronize(st);
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        ok = true;
    }
    ~TuneBufs() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (buf) cudaFree(buf);
        if (djl) cudaFree(djl);
        if (djs) cudaFree(djs);
    }
    // mean ms of three launches of `launch` after one warm-up (1e30 on error)
    template <class F>
    float time(F launch, cudaStream_t st) {
        launch();
        cudaEventRecord(e0, st);
        for (int r = 0; r < 3; ++r) launch();
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        return cudaGetLastError() == cudaSuccess ? ms : 1e30f;
    }
};

// Best split for a class of `jobs` products and its time.
int tune_split(const PrimeCtx& pc, int logn, int jobs, int dev, cudaStream_t st, TuneBufs& T, float* best_ms) {
    int best = default_row_log(logn);
    *best_ms = 1e30f;
    const u32 root = canonical_root(pc, logn);
    for (int l2 : legal_row_logs(logn)) {
        LargeArgs A;
        if (large_args(pc, root, logn, l2, dev, &A) != OK) continue;
        A.jobs = T.djl;
        A.njobs = jobs;
        const float ms = T.time([&] { launch_large(A, jobs, st); }, st);
        if (ms < *best_ms) {
            *best_ms = ms;
            best = l2;
        }
    }
    return best;
}

}  // namespace

std::vector<int> legal_row_logs(int logn) {
    std::vector<int> v;
    for (int l2 = kMinRowLog; l2 <= kMaxRowLog; ++l2) {
        const int l1 = logn - l2;
        if (l1 >= 1 && l1 <= kMaxColLog) v.push_back(l2);
    }
    return v;
}

int tune_row_log(const PrimeCtx& pc, int logn, int njobs, int dev, cudaStream_t st, bool allow_tuning) {
    const char* off = getenv("CUMODP_AUTOTUNE");
    if (off && off[0] == '0') return default_row_log(logn);
    const TuneKey key{device_model(dev), 0, logn, job_bucket(njobs)};
    int v;
    if (tune_lookup(key, &v)) return v;
    if (!allow_tuning) return default_row_log(logn);
    const std::vector<int> cands = legal_row_logs(logn);
    if (cands.size() <= 1) return cands.empty() ? default_row_log(logn) : cands[0];
    // timed at the class's own size (its bucket), up to 2^25 operand words: a split that wins for a few
    // products (many small CTAs) can lose for hundreds
    const int jobs = std::min(key.bucket, std::max(1, (int)((1ll << 25) >> logn)));
    TuneBufs T(jobs, 1ll << logn, st);
    if (!T.ok) return default_row_log(logn);
    float ms;
    const int best = tune_split(pc, logn, jobs, dev, st, T, &ms);
    tune_store(key, best);
    return best;
}

bool tune_single_cta(const PrimeCtx& pc, int logn, int njobs, int dev, cudaStream_t st, bool allow_tuning) {
    // the rule measured before tuning: a few products spread over the GPU, many on one CTA each
    const bool rule = njobs > 16;
    if (logn < single_large_min_log() || logn > kMaxSmallLog) return logn <= kMaxSmallLog;
    const char* off = getenv("CUMODP_AUTOTUNE");
    if (off && off[0] == '0') return rule;
    const TuneKey key{device_model(dev), 1, logn, job_bucket(njobs)};
    int v;
    if (tune_lookup(key, &v)) return v != 0;
    if (!allow_tuning) return rule;
    const int jobs = key.bucket;  // the class's own size (up to 256 products: 64 MiB at 2^14)
    TuneBufs T(jobs, 1ll << logn, st);
    if (!T.ok) return rule;
    float large_ms;
    tune_split(pc, logn, jobs, dev, st, T, &large_ms);
    SmallArgs A;
    if (small_args(pc, canonical_root(pc, logn), logn, dev, &A) != OK) return rule;
    A.jobs = T.djs;
    A.njobs = jobs;
    ensure_kernel_attrs();
    const float small_ms = T.time([&] { launch_small(logn, A, jobs, st); }, st);
    const bool single = small_ms <= large_ms;
    tune_store(key, single ? 1 : 0);
    return single;
}

// --------------------------------------------------------------- plans ----
namespace {

struct ClassPlan {
    int logn = 0;
    bool large = false;
    bool queued = false;       // runs in the batch's single work-queue launch (k_small_queue)
    int l2 = 0;
    std::vector<int> members;  // job indices of the batch
    size_t job_off = 0;        // byte offset of this class's job table
    size_t ws_off = 0;         // word offset of this class's workspace (large)
};

struct BatchPlan {
    u32 p = 0;
    int dev = 0;
    std::vector<long long> la, lb;
    std::vector<ClassPlan> classes;
    int nitems = 0;            // work items of the queued classes (0: no queue launch)
    size_t items_off = 0;      // byte offsets in djobs of the items and of the queue counter
    size_t counter_off = 0;
    void* djobs = nullptr;     // device job tables
    size_t jobs_bytes = 0;
    std::vector<unsigned char> hjobs;  // host copy of what djobs holds
    u32* ws = nullptr;
    size_t ws_words = 0;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaStream_t> side;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    size_t bytes = 0;

    ~BatchPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        for (auto s : side) cudaStreamDestroy(s);
        if (fork) cudaEventDestroy(fork);
        for (auto e : joins) cudaEventDestroy(e);
        if (djobs) cudaFree(djobs);
        if (ws) cudaFree(ws);
        account_bytes(-(long long)bytes);
    }
};

struct PlanCache {
    std::mutex m;
    std::unordered_map<size_t, std::unique_ptr<BatchPlan>> plans;
};
PlanCache& plan_cache() {
    static PlanCache* c = new PlanCache();
    return *c;
}

size_t shape_hash(u32 p, int dev, const std::vector<long long>& la, const std::vector<long long>& lb) {
    size_t h = 1469598103934665603ull ^ p ^ ((size_t)dev << 40);
    for (size_t i = 0; i < la.size(); ++i) {
        h = (h ^ (size_t)la[i]) * 1099511628211ull;
        h = (h ^ (size_t)lb[i]) * 1099511628211ull;
    }
    return h;
}

int build_plan(BatchPlan& P, const PrimeCtx& pc, cudaStream_t st) {
    std::map<int, ClassPlan> by;
    for (size_t i = 0; i < P.la.size(); ++i) {
        const int logn = product_logn(P.la[i], P.lb[i]);
        if (logn > pc.info.two_adic || logn > kMaxLog) return FFT_SIZE_TOO_LARGE;
        ClassPlan& c = by[logn];
        c.logn = logn;
        c.members.push_back((int)i);
    }
    size_t jb = 0, ws = 0;
    for (auto& kv : by) {
        ClassPlan c = kv.second;
        // a few products of a length one CTA could hold still run faster
        // spread over many CTAs (the three-pass kernels)
        c.large = !tune_single_cta(pc, c.logn, (int)c.members.size(), P.dev, st, true);
        c.queued = !c.large && c.logn >= kQueueMinLog && c.logn <= kQueueMaxLog;
        if (c.queued) P.nitems += (int)((c.members.size() + small_ppc(c.logn) - 1) / small_ppc(c.logn));
        c.job_off = jb;
        jb += c.members.size() * (c.large ? sizeof(LargeJob) : sizeof(ProdJob));
        jb = (jb + 255) & ~(size_t)255;
        if (c.large) {
            c.l2 = tune_row_log(pc, c.logn, (int)c.members.size(), P.dev, st, true);
            c.ws_off = ws;
            ws += c.members.size() * (2ull << c.logn);
        }
        P.classes.push_back(c);
    }
    P.items_off = jb;
    jb += (size_t)P.nitems * sizeof(SmallItem);
    jb = (jb + 255) & ~(size_t)255;
    P.counter_off = jb;
    jb += 256;
    P.jobs_bytes = std::max<size_t>(jb, 256);
    if (dev_malloc(&P.djobs, P.jobs_bytes) != cudaSuccess) {
        cudaGetLastError();
        return OUT_OF_MEMORY;
    }
    P.bytes += P.jobs_bytes;
    P.hjobs.assign(P.jobs_bytes, 0);
    P.ws_words = ws;
    if (ws) {
        if (dev_malloc((void**)&P.ws, ws * sizeof(u32)) != cudaSuccess) {
            cudaGetLastError();
            return OUT_OF_MEMORY;
        }
        P.bytes += ws * sizeof(u32);
    }
    account_bytes((long long)P.bytes);
    return OK;
}

// Everything graph capture must not do itself: branch streams and events,
// twiddle tables (they are allocated and uploaded on first use).
int prepare_capture(BatchPlan& P, const PrimeCtx& pc) {
    if (!P.fork) {
        cudaEventCreateWithFlags(&P.fork, cudaEventDisableTiming);
        for (size_t i = 0; i < P.classes.size(); ++i) {
            cudaStream_t s;
            cudaEvent_t e;
            cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
            cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            P.side.push_back(s);
            P.joins.push_back(e);
        }
    }
    for (const ClassPlan& c : P.classes) {
        const u32 root = canonical_root(pc, c.logn);
        int err = OK;
        if (!c.large) {
            SmallArgs A;
            err = small_args(pc, root, c.logn, P.dev, &A);
        } else {
            LargeArgs A;
            err = large_args(pc, root, c.logn, c.l2, P.dev, &A);
        }
        if (err != OK) return err;
    }
    return OK;
}

// Enqueue every class on its own branch (fork/join through events).
int enqueue_classes(BatchPlan& P, const PrimeCtx& pc, cudaStream_t st) {
    int err = OK;
    cudaEventRecord(P.fork, st);
    bool queue_done = false;
    for (size_t ci = 0; ci < P.classes.size(); ++ci) {
        const ClassPlan& c = P.classes[ci];
        if (c.queued && queue_done) continue;
        cudaStream_t s = P.side[ci];
        cudaStreamWaitEvent(s, P.fork, 0);
        const u32 root = canonical_root(pc, c.logn);
        if (c.queued) {
            // every queued class in one persistent launch on this branch
            SmallQueueArgs Q;
            memset(&Q, 0, sizeof(Q));
            Q.pk = pc.pk;
            for (const ClassPlan& d : P.classes) {
                if (!d.queued) continue;
                SmallArgs A;
                if ((err = small_args(pc, canonical_root(pc, d.logn), d.logn, P.dev, &A)) != OK) return err;
                Q.tw[d.logn] = A.tw;
                Q.tw_inv_off[d.logn] = A.tw_inv_off;
                Q.scale[d.logn] = A.scale;
            }
            Q.items = (const SmallItem*)((char*)P.djobs + P.items_off);
            Q.nitems = P.nitems;
            Q.counter = (int*)((char*)P.djobs + P.counter_off);
            cudaMemsetAsync(Q.counter, 0, sizeof(int), s);
            const int grid = std::min(P.nitems, sm_count(P.dev) * kQueueCtas);
            k_small_queue<kQueueMaxLog><<<grid, kQueueThreads, kQueueSmemWords * sizeof(u32), s>>>(Q);
            queue_done = true;
        } else if (!c.large) {
            SmallArgs A;
            if ((err = small_args(pc, root, c.logn, P.dev, &A)) != OK) return err;
            A.jobs = (const ProdJob*)((char*)P.djobs + c.job_off);
            A.njobs = (int)c.members.size();
            launch_small(c.logn, A, A.njobs, s);
        } else {
            LargeArgs A;
            if ((err = large_args(pc, root, c.logn, c.l2, P.dev, &A)) != OK) return err;
            A.jobs = (const LargeJob*)((char*)P.djobs + c.job_off);
            A.njobs = (int)c.members.size();
            launch_large(A, A.njobs, s);
        }
        cudaEventRecord(P.joins[ci], s);
        cudaStreamWaitEvent(st, P.joins[ci], 0);
    }
    return cuda_err(cudaGetLastError());
}

// Host job tables for the current pointers.
void fill_jobs(BatchPlan& P, const u32* F, const int64_t* f_off, const u32* G, const int64_t* g_off, u32* H,
               const int64_t* h_off, std::vector<unsigned char>& out) {
    out.assign(P.jobs_bytes, 0);
    // the queue's items, largest class first (pointers into this plan's job tables)
    {
        int it = 0;
        for (auto c = P.classes.rbegin(); c != P.classes.rend(); ++c) {
            if (!c->queued) continue;
            const int ppc = small_ppc(c->logn), n = (int)c->members.size();
            for (int k = 0; k < n; k += ppc) {
                SmallItem I{(const ProdJob*)((char*)P.djobs + c->job_off + (size_t)k * sizeof(ProdJob)), c->logn,
                            std::min(ppc, n - k)};
                memcpy(out.data() + P.items_off + (size_t)it++ * sizeof(SmallItem), &I, sizeof(I));
            }
        }
    }
    for (const ClassPlan& c : P.classes) {
        for (size_t k = 0; k < c.members.size(); ++k) {
            const int i = c.members[k];
            const int la = (int)P.la[i], lb = (int)P.lb[i], lh = la + lb - 1;
            if (!c.large) {
                ProdJob j{F + f_off[i], G + g_off[i], H + h_off[i], la, lb, lh, 0};
                memcpy(out.data() + c.job_off + k * sizeof(ProdJob), &j, sizeof(j));
            } else {
                const size_t n = (size_t)1 << c.logn;
                u32* w = P.ws + c.ws_off + k * 2 * n;
                LargeJob j{F + f_off[i], G + g_off[i], H + h_off[i], la, lb, lh, 0, w, w + n};
                memcpy(out.data() + c.job_off + k * sizeof(LargeJob), &j, sizeof(j));
            }
        }
    }
}

}  // namespace

int batch_mul_dev(int count, const sfixn* df, const int64_t* f_off, const u32* F, const sfixn* dg,
                  const int64_t* g_off, const u32* G, const int64_t* h_off, u32* H, u32 p, cudaStream_t st) {
    if (count < 0) return ASSUMPTION_ERROR;
    if (count == 0) return OK;
    if (!df || !dg || !f_off || !g_off || !h_off || !F || !G || !H) return ASSUMPTION_ERROR;
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    std::vector<long long> la(count), lb(count);
    for (int i = 0; i < count; ++i) {
        if (df[i] < 0 || dg[i] < 0) return ASSUMPTION_ERROR;
        la[i] = (long long)df[i] + 1;
        lb[i] = (long long)dg[i] + 1;
    }
    const int dev = current_device();
    PlanCache& PC = plan_cache();
    std::lock_guard<std::mutex> g(PC.m);
    const size_t key = shape_hash(p, dev, la, lb);
    auto it = PC.plans.find(key);
    BatchPlan* P = nullptr;
    if (it != PC.plans.end() && it->second->p == p && it->second->dev == dev && it->second->la == la &&
        it->second->lb == lb) {
        P = it->second.get();
    } else {
        if (PC.plans.size() >= 64) PC.plans.clear();  // bounded cache of batch shapes
        std::unique_ptr<BatchPlan> np(new BatchPlan());
        np->p = p;
        np->dev = dev;
        np->la = la;
        np->lb = lb;
        if ((err = build_plan(*np, *pc, st)) != OK) return err;
        P = np.get();
        PC.plans[key] = std::move(np);
    }
    std::vector<unsigned char> hj;
    fill_jobs(*P, F, f_off, G, g_off, H, h_off, hj);
    if (hj != P->hjobs) {
        P->hjobs.swap(hj);
        // pageable source: the call returns once the bytes are staged
        cudaError_t ce = cudaMemcpyAsync(P->djobs, P->hjobs.data(), P->jobs_bytes, cudaMemcpyHostToDevice, st);
        if (ce != cudaSuccess) return cuda_err(ce);
    }
    if (!P->exec) {
        ensure_kernel_attrs();
        if ((err = prepare_capture(*P, *pc)) != OK) return err;
        cudaStream_t cap;
        cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        cudaGraph_t graph;
        cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        err = enqueue_classes(*P, *pc, cap);
        cudaError_t ce = cudaStreamEndCapture(cap, &graph);
        cudaStreamDestroy(cap);
        if (err != OK) return err;
        if (ce != cudaSuccess) return cuda_err(ce);
        ce = cudaGraphInstantiate(&P->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) {
            P->exec = nullptr;
            return cuda_err(ce);
        }
    }
    return cuda_err(cudaGraphLaunch(P->exec, st));
}

// ------------------------------------------------------- direct batches ----
// Products on caller-owned buffers with direct launches (no plan cache, no
// graph): used where several batches run concurrently on different streams
// (the serving loop, the exact-product path).  Buffers:
//   ws     workspace words: direct_ws_words()
//   djobs  device job-table bytes: direct_job_bytes(); hjobs a pinned host
//          buffer of the same size that must stay untouched until the stream
//          has passed this call's work.
size_t direct_ws_words(int count, const long long* la, const long long* lb) {
    size_t w = 0;
    for (int i = 0; i < count; ++i) {
        const int logn = product_logn(la[i], lb[i]);
        if (logn > kMaxSmallLog) w += 2ull << logn;
    }
    return w;
}

size_t direct_job_bytes(int count) {
    return (size_t)count * std::max(sizeof(LargeJob), sizeof(ProdJob)) + 64 * 256;
}

int direct_batch(int count, const u32* const* a, const long long* la, const u32* const* b, const long long* lb,
                 u32* const* h, const long long* lh, u32 p, u32* ws, void* djobs, void* hjobs,
                 cudaStream_t st, bool allow_tuning) {
    int err = OK;
    const PrimeCtx* pc = prime_ctx(p, &err);
    if (!pc) return err;
    const int dev = current_device();
    ensure_kernel_attrs();
    std::map<int, std::vector<int>> cls;
    for (int i = 0; i < count; ++i) {
        const int logn = product_logn(la[i], lb[i]);
        if (logn > pc->info.two_adic || logn > kMaxLog) return FFT_SIZE_TOO_LARGE;
        cls[logn].push_back(i);
    }
    size_t off = 0, wsoff = 0;
    unsigned char* hj = (unsigned char*)hjobs;
    struct Launch { int logn; size_t off; int n; int l2; };
    std::vector<Launch> launches;
    for (auto& kv : cls) {
        const int logn = kv.first;
        const std::vector<int>& mem = kv.second;
        const bool large = logn > kMaxSmallLog;
        for (size_t k = 0; k < mem.size(); ++k) {
            const int i = mem[k];
            const long long outl = std::min<long long>(lh[i], 1ll << logn);
            if (!large) {
                ProdJob j{a[i], b[i], h[i], (int)la[i], (int)lb[i], (int)outl, 0};
                memcpy(hj + off + k * sizeof(ProdJob), &j, sizeof(j));
            } else {
                const size_t n = (size_t)1 << logn;
                u32* w = ws + wsoff;
                wsoff += 2 * n;
                LargeJob j{a[i], b[i], h[i], (int)la[i], (int)lb[i], (int)outl, 0, w, w + n};
                memcpy(hj + off + k * sizeof(LargeJob), &j, sizeof(j));
            }
            if (lh[i] > (1ll << logn)) {
                cudaError_t e = cudaMemsetAsync(h[i] + (1ll << logn), 0, (size_t)(lh[i] - (1ll << logn)) * 4, st);
                if (e != cudaSuccess) return cuda_err(e);
            }
        }
        launches.push_back(Launch{logn, off, (int)mem.size(),
                                  large ? tune_row_log(*pc, logn, (int)mem.size(), dev, st, allow_tuning) : 0});
        off += mem.size() * (large ? sizeof(LargeJob) : sizeof(ProdJob));
        off = (off + 255) & ~(size_t)255;
    }
    cudaError_t ce = cudaMemcpyAsync(djobs, hjobs, off ? off : 256, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return cuda_err(ce);
    for (const Launch& L : launches) {
        const u32 root = canonical_root(*pc, L.logn);
        if (L.logn <= kMaxSmallLog) {
            SmallArgs A;
            if ((err = small_args(*pc, root, L.logn, dev, &A)) != OK) return err;
            A.jobs = (const ProdJob*)((char*)djobs + L.off);
            A.njobs = L.n;
            launch_small(L.logn, A, L.n, st);
        } else {
            LargeArgs A;
            if ((err = large_args(*pc, root, L.logn, L.l2, dev, &A)) != OK) return err;
            A.jobs = (const LargeJob*)((char*)djobs + L.off);
            A.njobs = L.n;
            launch_large(A, L.n, st);
        }
    }
    return cuda_err(cudaGetLastError());
}

// Kernel launches one batch issues (for reporting).
int batch_launch_count(int count, const sfixn* df, const sfixn* dg) {
    std::map<int, int> cls;
    for (int i = 0; i < count; ++i) cls[product_logn((long long)df[i] + 1, (long long)dg[i] + 1)]++;
    int n = 0;
    bool queue = false;
    for (auto& kv : cls) {
        if (kv.first >= kQueueMinLog && kv.first <= kQueueMaxLog) {
            n += queue ? 0 : 1;  // the queued classes share one launch
            queue = true;
        } else {
            n += kv.first > kMaxSmallLog ? 3 : 1;
        }
    }
    return n;
}

// out[j][l + t] += a_j[t] + b_j[t] (t < l - 1), out[j][2l - 1] = a_j[l - 1] + b_j[l - 1]:
// the x^l (a + b) term of (x^l + a)(x^l + b) = x^2l + x^l (a + b) + a b.
__global__ void k_monic_level_fixup(const u32* __restrict__ in, u32* __restrict__ out, long long l, long long npairs,
                                    u32 p) {
    const long long total = npairs * l;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long j = i / l, t = i % l;
        const u32 a = in[2 * j * l + t] % p, b = in[(2 * j + 1) * l + t] % p;
        u32 s = a + b;
        s = s >= p ? s - p : s;
        u32* o = out + 2 * j * l + l + t;
        if (t < l - 1) {
            u32 v = *o + s;
            *o = v >= p ? v - p : v;
        } else {
            *o = s;
        }
    }
}

// One level of a subproduct tree of monic polynomials stored without their
// leading coefficient: out[j] = in[2j] * in[2j+1] (degree l each, l words;
// the product has degree 2l, 2l words).  The products a b run as one batch
// of equal-size pairs (the graph-captured batch path), then one kernel adds
// the x^l (a + b) term.
int subproduct_level_dev(long long l, long long npairs, const u32* in, u32* out, u32 p, cudaStream_t st) {
    if (l <= 0 || npairs < 0 || npairs > INT32_MAX || l > (1ll << 23)) return ASSUMPTION_ERROR;
    if (npairs == 0) return OK;
    if (!in || !out) return ASSUMPTION_ERROR;
    if (out < in + 2 * npairs * l && in < out + 2 * npairs * l) return ASSUMPTION_ERROR;  // no aliasing
    const int cnt = (int)npairs;
    std::vector<sfixn> d(cnt, (sfixn)(l - 1));
    std::vector<int64_t> fo(cnt), go(cnt), ho(cnt);
    for (int j = 0; j < cnt; ++j) {
        fo[j] = 2 * (int64_t)j * l;
        go[j] = (2 * (int64_t)j + 1) * l;
        ho[j] = 2 * (int64_t)j * l;
    }
    int err = batch_mul_dev(cnt, d.data(), fo.data(), in, d.data(), go.data(), in, ho.data(), out, p, st);
    if (err != OK) return err;
    const long long total = npairs * l;
    const int grid = (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148 * 16));
    k_monic_level_fixup<<<grid, 256, 0, st>>>(in, out, l, npairs, p);
    return cuda_err(cudaGetLastError());
}

// Host-buffer batch of large products, pipelined: product i's operands are
// copied in on one stream, its kernels run on the library stream, its result
// is copied out on a third stream, so the copies of products i+1 and i-1
// (both directions of the host link at once) overlap the kernels of product
// i.  Three device slots (operands and result) rotate; a slot is refilled
// only after the result copy that last used it has finished.
int pipelined_host_batch(int count, const sfixn* df, const int64_t* f_off, const u32* F, const sfixn* dg,
                         const int64_t* g_off, const u32* G, const int64_t* h_off, u32* H, u32 p, cudaStream_t st) {
    constexpr int kSlots = 3;
    const int dev = current_device();
    long long maxa = 0, maxb = 0, maxh = 0;
    for (int i = 0; i < count; ++i) {
        maxa = std::max<long long>(maxa, (long long)df[i] + 1);
        maxb = std::max<long long>(maxb, (long long)dg[i] + 1);
        maxh = std::max<long long>(maxh, (long long)df[i] + dg[i] + 1);
    }
    const size_t slot_words = (size_t)(maxa + maxb + maxh);
    int err = OK;
    u32* d = (u32*)workspace(dev, kWsBatch, kSlots * slot_words * sizeof(u32), &err);
    if (!d) return err;
    struct Streams {
        cudaStream_t in, out;
        cudaEvent_t in_done[kSlots], comp_done[kSlots], out_done[kSlots];
    };
    static std::map<int, Streams*> per_dev;  // guarded by lib_mutex
    Streams*& S = per_dev[dev];
    if (!S) {
        S = new Streams();
        cudaStreamCreateWithFlags(&S->in, cudaStreamNonBlocking);
        cudaStreamCreateWithFlags(&S->out, cudaStreamNonBlocking);
        for (int k = 0; k < kSlots; ++k) {
            cudaEventCreateWithFlags(&S->in_done[k], cudaEventDisableTiming);
            cudaEventCreateWithFlags(&S->comp_done[k], cudaEventDisableTiming);
            cudaEventCreateWithFlags(&S->out_done[k], cudaEventDisableTiming);
        }
    }
    // nothing of an earlier call may still use the slots
    cudaEventRecord(S->out_done[0], st);
    cudaStreamWaitEvent(S->in, S->out_done[0], 0);
    cudaStreamWaitEvent(S->out, S->out_done[0], 0);
    for (int i = 0; i < count && err == OK; ++i) {
        const int k = i % kSlots;
        u32* a = d + (size_t)k * slot_words;
        u32* b = a + maxa;
        u32* h = b + maxb;
        const long long la = (long long)df[i] + 1, lb = (long long)dg[i] + 1, lh = la + lb - 1;
        if (i >= kSlots) cudaStreamWaitEvent(S->in, S->out_done[k], 0);
        cudaError_t ce = cudaMemcpyAsync(a, F + f_off[i], la * 4, cudaMemcpyHostToDevice, S->in);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(b, G + g_off[i], lb * 4, cudaMemcpyHostToDevice, S->in);
        if (ce != cudaSuccess) {
            err = cuda_err(ce);
            break;
        }
        cudaEventRecord(S->in_done[k], S->in);
        cudaStreamWaitEvent(st, S->in_done[k], 0);
        if ((err = mul_dev(a, la, b, lb, h, lh, p, st)) != OK) break;
        cudaEventRecord(S->comp_done[k], st);
        cudaStreamWaitEvent(S->out, S->comp_done[k], 0);
        ce = cudaMemcpyAsync(H + h_off[i], h, lh * 4, cudaMemcpyDeviceToHost, S->out);
        if (ce != cudaSuccess) {
            err = cuda_err(ce);
            break;
        }
        cudaEventRecord(S->out_done[k], S->out);
    }
    cudaStreamSynchronize(S->in);
    cudaStreamSynchronize(st);
    cudaStreamSynchronize(S->out);
    return err;
}

}  // namespace cmb

using namespace cmb;

extern "C" {

cumodp_err cumodp_subproduct_level_dev(sfixn l, sfixn npairs, const sfixn* M_in, sfixn* M_out, sfixn p,
                                       void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = subproduct_level_dev(l, npairs, (const u32*)M_in, (u32*)M_out, (u32)p, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

cumodp_err cumodp_fftmul_batch_dev(int count, const sfixn* df, const int64_t* f_off, const sfixn* F,
                                   const sfixn* dg, const int64_t* g_off, const sfixn* G, const int64_t* h_off,
                                   sfixn* H, sfixn p, void* stream) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    std::lock_guard<std::mutex> g(lib_mutex());
    cudaStream_t st = stream ? (cudaStream_t)stream : lib_stream(current_device());
    int e = batch_mul_dev(count, df, f_off, (const u32*)F, dg, g_off, (const u32*)G, h_off, (u32*)H, (u32)p, st);
    if (e == OK && !stream) e = cuda_err(cudaStreamSynchronize(st));
    return (cumodp_err)e;
}

cumodp_err cumodp_fftmul_batch(int count, const sfixn* df, const int64_t* f_off, const sfixn* F,
                               const sfixn* dg, const int64_t* g_off, const sfixn* G, const int64_t* h_off,
                               sfixn* H, sfixn p) {
    int cnt = 0;
    if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
        cudaGetLastError();
        return CUMODP_NO_CUDA_DEVICE;
    }
    if (count < 0 || (count > 0 && (!df || !dg || !f_off || !g_off || !h_off || !F || !G || !H)))
        return CUMODP_ASSUMPTION_ERROR;
    if (count == 0) return CUMODP_SUCCESS;
    std::lock_guard<std::mutex> g(lib_mutex());
    const int dev = current_device();
    cudaStream_t st = lib_stream(dev);
    // extents of the three host arrays
    size_t nf = 0, ng = 0, nh = 0, total = 0;
    for (int i = 0; i < count; ++i) {
        if (df[i] < 0 || dg[i] < 0 || f_off[i] < 0 || g_off[i] < 0 || h_off[i] < 0) return CUMODP_ASSUMPTION_ERROR;
        nf = std::max(nf, (size_t)f_off[i] + df[i] + 1);
        ng = std::max(ng, (size_t)g_off[i] + dg[i] + 1);
        nh = std::max(nh, (size_t)h_off[i] + df[i] + dg[i] + 1);
        total += (size_t)df[i] + dg[i] + 2;
    }
    // several large products: pipeline the host copies against the kernels
    if (count > 1 && total / count >= (1u << 20)) {
        const int err = pipelined_host_batch(count, df, f_off, (const u32*)F, dg, g_off, (const u32*)G, h_off,
                                             (u32*)H, (u32)p, st);
        return (cumodp_err)err;
    }
    int err = OK;
    u32* d = (u32*)workspace(dev, kWsBatch, (nf + ng + nh) * sizeof(u32), &err);
    if (!d) return (cumodp_err)err;
    u32 *dF = d, *dG = d + nf, *dH = d + nf + ng;
    cudaError_t ce = cudaMemcpyAsync(dF, F, nf * 4, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(dG, G, ng * 4, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return (cumodp_err)cuda_err(ce);
    err = batch_mul_dev(count, df, f_off, dF, dg, g_off, dG, h_off, dH, (u32)p, st);
    if (err != OK) {
        cudaStreamSynchronize(st);
        return (cumodp_err)err;
    }
    ce = cudaMemcpyAsync(H, dH, nh * 4, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    return (cumodp_err)cuda_err(ce);
}

}  // extern "C"
