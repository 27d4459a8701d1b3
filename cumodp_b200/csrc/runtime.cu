// Host runtime: primes, resident twiddle tables, workspace, streams.
//
// The reference rebuilds its root-power table on every call
// (get_powers_binary, src/fft_aux.cu:87-132: 1024 powers on the host, then
// log-doubling kernels) and cudaMallocs/cudaFrees all buffers per call
// (src/stockham.cu:579-610).  Here tables are built once per (device, prime,
// root, size) on the host with exact arithmetic, uploaded, and kept resident;
// scratch buffers grow once and are reused.
#include "runtime.cuh"

#include <atomic>
#include <cstdio>
#include <map>
#include <cstring>

namespace cmb {

namespace {

bool is_prime_u32(u32 n) {
    if (n < 2) return false;
    for (u32 q : {2u, 3u, 5u, 7u, 11u, 13u, 17u, 19u, 23u, 29u, 31u, 37u}) {
        if (n == q) return true;
        if (n % q == 0) return false;
    }
    u32 d = n - 1;
    int s = 0;
    while (!(d & 1)) { d >>= 1; ++s; }
    // deterministic Miller-Rabin for 32-bit n
    for (u32 a : {2u, 3u, 5u, 7u}) {
        u32 x = powmod_exact(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int r = 1; r < s; ++r) {
            x = mulmod_exact(x, x, n);
            if (x == n - 1) { comp = false; break; }
        }
        if (comp) return false;
    }
    return true;
}

u32 bitrev(u32 x, int bits) {
    u32 r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

struct Caches {
    std::mutex m;
    long long bytes = 0;
    std::map<u32, PrimeCtx*> primes;
    std::map<std::tuple<int, u32, u32, int, int>, Tw*> tables;  // dev, p, root, logl, kind
    std::map<std::tuple<int, u32, u32, int>, u32*> seeds;
    std::map<std::pair<int, int>, std::pair<void*, size_t>> ws;
    std::map<int, std::pair<void*, size_t>> pinned;
    std::map<int, cudaStream_t> streams;
};

Caches& caches() {
    static Caches* c = new Caches();  // never destroyed: device memory lives to process exit
    return *c;
}

std::vector<Tw> build_level_tables(const LevelPlan& pl, int logl, u32 root, u32 p) {
    const int nf = plan_tw_entries(pl, logl);
    std::vector<Tw> t((size_t)2 * nf + 2);
    const u32 rinv = powmod_exact(root, (1ull << logl) - 1, p);  // root^-1
    int off = 0, lb = logl;
    for (int i = 0; i + 1 < pl.nlev; ++i) {
        const int r = pl.logr[i], R = 1 << r, TB = (1 << lb) / R;
        const u32 wb = powmod_exact(root, 1ull << (logl - lb), p);   // w_B
        const u32 wbi = powmod_exact(rinv, 1ull << (logl - lb), p);  // w_B^-1
        for (int o = 0; o < TB; ++o)
            for (int j = 0; j < R; ++j) {
                u64 e = (u64)o * bitrev((u32)j, r);
                t[off + o * R + j] = tw_of(powmod_exact(wb, e, p), p);
                t[nf + off + o * R + j] = tw_of(powmod_exact(wbi, e, p), p);
            }
        off += 1 << lb;
        lb -= r;
    }
    return t;
}

}  // namespace

Tw tw_of(u32 w, u32 p) { return Tw{w, shoup_quot(w, p)}; }

size_t level_tables_entries(int kind, int logl) {
    const LevelPlan pl = kind == 0 ? row_plan(logl) : col_plan(logl);
    return (size_t)2 * plan_tw_entries(pl, logl) + 2;
}

int level_tables_into(int kind, u32 p, u32 root, int logl, Tw* out, size_t cap) {
    const LevelPlan pl = kind == 0 ? row_plan(logl) : col_plan(logl);
    if (pl.nlev == 0 || level_tables_entries(kind, logl) > cap) return ASSUMPTION_ERROR;
    const int nf = plan_tw_entries(pl, logl);
    const u32 rinv = powmod_exact(root, (1ull << logl) - 1, p);
    int off = 0, lb = logl;
    for (int i = 0; i + 1 < pl.nlev; ++i) {
        const int r = pl.logr[i], R = 1 << r, TB = (1 << lb) / R;
        const u32 wb = powmod_exact(root, 1ull << (logl - lb), p);
        const u32 wbi = powmod_exact(rinv, 1ull << (logl - lb), p);
        for (int o = 0; o < TB; ++o)
            for (int j = 0; j < R; ++j) {
                u64 e = (u64)o * bitrev((u32)j, r);
                out[off + o * R + j] = tw_of(powmod_exact(wb, e, p), p);
                out[nf + off + o * R + j] = tw_of(powmod_exact(wbi, e, p), p);
            }
        off += 1 << lb;
        lb -= r;
    }
    return OK;
}

size_t seed_words(int logn) {
    const u64 n = 1ull << logn;
    return 2 * (size_t)(std::min<u64>(n, 4096) + std::max<u64>(1, n / 4096));
}

int seeds_into(u32 p, u32 root, int logn, u32* s, size_t cap) {
    if (seed_words(logn) > cap) return ASSUMPTION_ERROR;
    const u64 n = 1ull << logn;
    const u32 nlo = (u32)std::min<u64>(n, 4096), nhi = (u32)std::max<u64>(1, n / 4096);
    const u32 r1 = (u32)((1ull << 32) % p);
    const u32 rinv = powmod_exact(root, n - 1, p);
    u32 w = 1, wi = 1;
    for (u32 t = 0; t < nlo; ++t) {
        s[t] = mulmod_exact(w, r1, p);
        s[nlo + nhi + t] = mulmod_exact(wi, r1, p);
        w = mulmod_exact(w, root, p);
        wi = mulmod_exact(wi, rinv, p);
    }
    const u32 step = powmod_exact(root, 4096, p), stepi = powmod_exact(rinv, 4096, p);
    w = 1;
    wi = 1;
    for (u32 t = 0; t < nhi; ++t) {
        s[nlo + t] = mulmod_exact(w, r1, p);
        s[2 * nlo + nhi + t] = mulmod_exact(wi, r1, p);
        w = mulmod_exact(w, step, p);
        wi = mulmod_exact(wi, stepi, p);
    }
    return OK;
}

PrimeK make_prime_k(const PrimeInfo& pi, u32 w32) {
    PrimeK k;
    k.p = pi.p;
    k.p2 = pi.p2;
    k.pinv_neg = pi.pinv_neg;
    k.one_q = shoup_quot(1, pi.p);
    const u32 w32i = powmod_exact(w32, 31, pi.p);
    for (int j = 0; j < 16; ++j) {
        k.rc.f[j] = tw_of(powmod_exact(w32, j, pi.p), pi.p);
        k.rc.i[j] = tw_of(powmod_exact(w32i, j, pi.p), pi.p);
    }
    return k;
}

PrimeK make_prime_k_for(const PrimeInfo& pi, u32 root, int logl) {
    if (logl >= 5) return make_prime_k(pi, powmod_exact(root, 1ull << (logl - 5), pi.p));
    PrimeK k = make_prime_k(pi, 1);
    const u32 L = 1u << logl, rinv = powmod_exact(root, L - 1, pi.p);
    for (int e = 0; e < 16; ++e) {
        if ((e * (int)L) % 32) continue;  // w_32^e is a power of w_L only when L*e/32 is integral
        const u32 t = (u32)(e * L / 32);
        k.rc.f[e] = tw_of(powmod_exact(root, t, pi.p), pi.p);
        k.rc.i[e] = tw_of(powmod_exact(rinv, t, pi.p), pi.p);
    }
    return k;
}

const PrimeCtx* prime_ctx(u32 p, int* err) {
    Caches& C = caches();
    std::lock_guard<std::mutex> g(C.m);
    auto it = C.primes.find(p);
    if (it != C.primes.end()) return it->second;
    if (p < 3 || p >= (1u << 30) || !is_prime_u32(p)) { *err = ASSUMPTION_ERROR; return nullptr; }
    PrimeInfo pi;
    pi.p = p;
    pi.p2 = 2 * p;
    u32 inv = 1;  // p^-1 mod 2^32 by Newton iteration
    for (int i = 0; i < 5; ++i) inv *= 2 - p * inv;
    pi.pinv_neg = (u32)(0u - inv);
    pi.r1 = (u32)((1ull << 32) % p);
    pi.r2 = mulmod_exact(pi.r1, pi.r1, p);
    int e = 0;
    while (!(((p - 1) >> e) & 1)) ++e;
    pi.two_adic = e;
    if (e < 5) { *err = FOURIER_DEGREE_TOO_SMALL; return nullptr; }
    // canonical root: g^((p-1)/2^e) for the least g that is a 2^e-th
    // non-residue, i.e. whose power has order exactly 2^e
    u32 root = 0;
    for (u32 g = 2; g < p; ++g) {
        u32 w = powmod_exact(g, (p - 1) >> e, p);
        if (powmod_exact(w, 1ull << (e - 1), p) == p - 1) { root = w; break; }
    }
    PrimeCtx* pc = new PrimeCtx();
    pc->info = pi;
    pc->root_max = root;
    pc->pk = make_prime_k(pi, powmod_exact(root, 1ull << (e - 5), p));
    C.primes[p] = pc;
    return pc;
}

u32 canonical_root(const PrimeCtx& pc, int logn) {
    return powmod_exact(pc.root_max, 1ull << (pc.info.two_adic - logn), pc.info.p);
}

// Host-side fault injection (cumodp_inject_alloc_failures): the next n
// device allocations of the library fail as if the device were full.
static std::atomic<int> g_alloc_failures{0};

void inject_alloc_failures(int n) { g_alloc_failures.store(n < 0 ? 0 : n); }

cudaError_t dev_malloc(void** p, size_t bytes) {
    int left = g_alloc_failures.load();
    while (left > 0) {
        if (g_alloc_failures.compare_exchange_weak(left, left - 1)) {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
    }
    return cudaMalloc(p, bytes);
}

cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t st) {
    int left = g_alloc_failures.load();
    while (left > 0) {
        if (g_alloc_failures.compare_exchange_weak(left, left - 1)) {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
    }
    return cudaMallocAsync(p, bytes, st);
}

// Host-to-device upload of a cached table that has landed when it returns.
// cudaMemcpy from pageable memory may return once the words are staged,
// before the DMA lands, and the kernels that read the table run on
// non-blocking streams, which do not wait for it.
static cudaError_t upload_now(void* d, const void* h, size_t bytes) {
    static std::mutex m;
    static std::map<int, cudaStream_t> streams;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaStream_t s;
    {
        std::lock_guard<std::mutex> g(m);
        auto it = streams.find(dev);
        if (it == streams.end()) {
            cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
            streams[dev] = s;
        } else {
            s = it->second;
        }
    }
    cudaError_t e = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

static const Tw* level_tables(int dev, u32 p, u32 root, int logl, int kind, int* err) {
    Caches& C = caches();
    std::lock_guard<std::mutex> g(C.m);
    auto key = std::make_tuple(dev, p, root, logl, kind);
    auto it = C.tables.find(key);
    if (it != C.tables.end()) return it->second;
    const LevelPlan pl = kind == 0 ? row_plan(logl) : col_plan(logl);
    std::vector<Tw> t = build_level_tables(pl, logl, root, p);
    Tw* d = nullptr;
    if (dev_malloc((void**)&d, t.size() * sizeof(Tw)) != cudaSuccess) {
        cudaGetLastError();
        *err = OUT_OF_MEMORY;
        return nullptr;
    }
    if (upload_now(d, t.data(), t.size() * sizeof(Tw)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d);
        *err = FFT_ERROR;
        return nullptr;
    }
    C.bytes += (long long)(t.size() * sizeof(Tw));
    C.tables[key] = d;
    return d;
}

const Tw* row_tables(int dev, u32 p, u32 root, int logl, int* err) {
    return level_tables(dev, p, root, logl, 0, err);
}
const Tw* col_tables(int dev, u32 p, u32 root, int logl, int* err) {
    return level_tables(dev, p, root, logl, 1, err);
}

const u32* seed_tables(int dev, u32 p, u32 root, int logn, int* err) {
    Caches& C = caches();
    std::lock_guard<std::mutex> g(C.m);
    auto key = std::make_tuple(dev, p, root, logn);
    auto it = C.seeds.find(key);
    if (it != C.seeds.end()) return it->second;
    const u64 n = 1ull << logn;
    const u32 nlo = (u32)std::min<u64>(n, 4096), nhi = (u32)std::max<u64>(1, n / 4096);
    const u32 r1 = (u32)((1ull << 32) % p);
    const u32 rinv = powmod_exact(root, n - 1, p);
    // layout: lo_f[nlo], hi_f[nhi], lo_i[nlo], hi_i[nhi]
    std::vector<u32> s(2 * (size_t)(nlo + nhi));
    u32 w = 1, wi = 1;
    for (u32 t = 0; t < nlo; ++t) {
        s[t] = mulmod_exact(w, r1, p);
        s[nlo + nhi + t] = mulmod_exact(wi, r1, p);
        w = mulmod_exact(w, root, p);
        wi = mulmod_exact(wi, rinv, p);
    }
    const u32 step = powmod_exact(root, 4096, p), stepi = powmod_exact(rinv, 4096, p);
    w = 1; wi = 1;
    for (u32 t = 0; t < nhi; ++t) {
        s[nlo + t] = mulmod_exact(w, r1, p);
        s[2 * nlo + nhi + t] = mulmod_exact(wi, r1, p);
        w = mulmod_exact(w, step, p);
        wi = mulmod_exact(wi, stepi, p);
    }
    u32* d = nullptr;
    if (dev_malloc((void**)&d, s.size() * sizeof(u32)) != cudaSuccess) {
        cudaGetLastError();
        *err = OUT_OF_MEMORY;
        return nullptr;
    }
    if (upload_now(d, s.data(), s.size() * sizeof(u32)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d);
        *err = FFT_ERROR;
        return nullptr;
    }
    C.bytes += (long long)(s.size() * sizeof(u32));
    C.seeds[key] = d;
    return d;
}

void* workspace(int dev, int slot, size_t bytes, int* err) {
    Caches& C = caches();
    std::lock_guard<std::mutex> g(C.m);
    auto& e = C.ws[std::make_pair(dev, slot)];
    if (e.second >= bytes && e.first) return e.first;
    if (e.first) {
        cudaFree(e.first);
        C.bytes -= (long long)e.second;
    }
    e.first = nullptr;
    e.second = 0;
    size_t sz = bytes < 4096 ? 4096 : bytes;
    if (dev_malloc(&e.first, sz) != cudaSuccess) {
        cudaGetLastError();
        *err = OUT_OF_MEMORY;
        e.first = nullptr;
        return nullptr;
    }
    e.second = sz;
    C.bytes += (long long)sz;
    return e.first;
}

void* pinned_workspace(int slot, size_t bytes, int* err) {
    Caches& C = caches();
    std::lock_guard<std::mutex> g(C.m);
    auto& e = C.pinned[slot];
    if (e.second >= bytes && e.first) return e.first;
    if (e.first) cudaFreeHost(e.first);  // synchronises with the device: no copy from it is in flight
    e.first = nullptr;
    e.second = 0;
    const size_t sz = std::max<size_t>(bytes + bytes / 4, 1 << 16);
    if (cudaHostAlloc(&e.first, sz, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        *err = OUT_OF_MEMORY;
        e.first = nullptr;
        return nullptr;
    }
    e.second = sz;
    return e.first;
}

cudaStream_t lib_stream(int dev) {
    Caches& C = caches();
    std::lock_guard<std::mutex> g(C.m);
    auto it = C.streams.find(dev);
    if (it != C.streams.end()) return it->second;
    cudaStream_t s;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    C.streams[dev] = s;
    return s;
}

namespace {
struct AuxSet {
    cudaStream_t s[kAuxStreams];
    cudaEvent_t fork, join[kAuxStreams];
};
}  // namespace

// Side streams for independent work inside one call (fork/join by events).
static AuxSet& aux_set(int dev) {
    static std::mutex m;
    static std::map<int, AuxSet*> sets;
    std::lock_guard<std::mutex> g(m);
    auto it = sets.find(dev);
    if (it != sets.end()) return *it->second;
    AuxSet* a = new AuxSet();
    for (int i = 0; i < kAuxStreams; ++i) {
        cudaStreamCreateWithFlags(&a->s[i], cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&a->join[i], cudaEventDisableTiming);
    }
    cudaEventCreateWithFlags(&a->fork, cudaEventDisableTiming);
    sets[dev] = a;
    return *a;
}

cudaStream_t aux_fork(int dev, cudaStream_t st, int n) {
    AuxSet& a = aux_set(dev);
    cudaEventRecord(a.fork, st);
    for (int i = 0; i < n && i < kAuxStreams; ++i) cudaStreamWaitEvent(a.s[i], a.fork, 0);
    return a.s[0];
}

cudaStream_t aux_stream(int dev, int i) { return aux_set(dev).s[i]; }

void aux_join(int dev, cudaStream_t st, int n) {
    AuxSet& a = aux_set(dev);
    for (int i = 0; i < n && i < kAuxStreams; ++i) {
        cudaEventRecord(a.join[i], a.s[i]);
        cudaStreamWaitEvent(st, a.join[i], 0);
    }
}

std::mutex& lib_mutex() {
    static std::mutex* m = new std::mutex();
    return *m;
}

int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

size_t bytes_in_use() {
    Caches& C = caches();
    std::lock_guard<std::mutex> g(C.m);
    return (size_t)(C.bytes < 0 ? 0 : C.bytes);
}

void account_bytes(long long delta) {
    Caches& C = caches();
    std::lock_guard<std::mutex> g(C.m);
    C.bytes += delta;
}

namespace {
struct PassTiming {
    std::mutex m;
    bool on = false;
    std::vector<cudaEvent_t> pool;
    struct Pending { std::string name; cudaEvent_t e0, e1; };
    std::vector<Pending> pending;
    std::map<std::string, std::pair<long long, double>> totals;
};
PassTiming& pt() {
    static PassTiming* t = new PassTiming();
    return *t;
}
cudaEvent_t pt_get_locked(PassTiming& T) {
    if (!T.pool.empty()) {
        cudaEvent_t e = T.pool.back();
        T.pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}
void pt_drain_locked(PassTiming& T) {
    for (auto& p : T.pending) {
        cudaEventSynchronize(p.e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, p.e0, p.e1);
        auto& t = T.totals[p.name];
        t.first += 1;
        t.second += ms;
        T.pool.push_back(p.e0);
        T.pool.push_back(p.e1);
    }
    T.pending.clear();
}
}  // namespace

bool pass_timing_on() { return pt().on; }

void pass_timing_enable(bool on) {
    PassTiming& T = pt();
    std::lock_guard<std::mutex> g(T.m);
    T.on = on;
}

bool pass_timing_begin(cudaStream_t st, cudaEvent_t* e0) {
    PassTiming& T = pt();
    if (!T.on) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
    std::lock_guard<std::mutex> g(T.m);
    if (T.pending.size() > 100000) pt_drain_locked(T);
    *e0 = pt_get_locked(T);
    cudaEventRecord(*e0, st);
    return true;
}

void pass_timing_end(cudaStream_t st, const char* name, cudaEvent_t e0) {
    PassTiming& T = pt();
    std::lock_guard<std::mutex> g(T.m);
    cudaEvent_t e1 = pt_get_locked(T);
    cudaEventRecord(e1, st);
    T.pending.push_back(PassTiming::Pending{name, e0, e1});
}

std::string pass_timing_report(bool reset) {
    PassTiming& T = pt();
    std::lock_guard<std::mutex> g(T.m);
    pt_drain_locked(T);
    std::string out;
    char line[256];
    for (auto& kv : T.totals) {
        snprintf(line, sizeof(line), "%s %lld %.6f\n", kv.first.c_str(), kv.second.first, kv.second.second);
        out += line;
    }
    if (reset) T.totals.clear();
    return out;
}

int cuda_err(cudaError_t e) {
    if (e == cudaSuccess) return OK;
    if (e == cudaErrorMemoryAllocation) return OUT_OF_MEMORY;
    return FFT_ERROR;
}

}  // namespace cmb
