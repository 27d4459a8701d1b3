// Serving loop: continuous batching of multiplication requests.
//
// The reference has no server; its entry points are synchronous, one
// product per call, device 0, with per-call allocation
// (src/stockham.cu:562-611).  This server keeps a request queue and a few
// device "lanes" (stream + grow-only device/pinned buffers).  A batcher
// thread admits requests in arrival order while the device-memory budget
// allows, groups the admitted ones by (kind, prime) and dispatches each
// group to a free lane as one batch: asynchronous host->device copies of
// the operands (each request's operands were copied once, by the submitting
// thread, into a pinned slab), the batched product kernels (or the
// exact-product pipeline), asynchronous device->host copies into each
// request's pinned result slab, an event.  The waiting thread copies its
// result out of the slab.  Requests that arrive while earlier batches
// are on the GPU are admitted into the next batch at once, so batches from
// different lanes overlap on the device.  A completion thread waits on lane
// events, scatters results into the callers' buffers, releases the memory
// budget and records arrival-to-result latency.
//
// Failures are contained per batch: a request that fails validation is
// completed with its error code; a CUDA error in a batch completes that
// batch's requests with CUMODP_FFT_ERROR and the lane is re-created.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/cumodp.h"
#include "exact.cuh"

namespace cmb {

namespace {

double now_us() {
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Pinned host slabs: a buddy allocator over pinned chunks of 256 MiB (less
// under a smaller limit).  Pinning memory (cudaHostAlloc) is slow and serialises with the
// device, so chunks are pinned up front (reserve) or, past that, at most a
// few times, and never returned before the server ends; slabs are carved
// from them in power-of-two sizes and coalesce with their buddies when freed,
// so a shift in request sizes reuses the same memory.  `limit` bounds the
// pinned bytes: beyond it get() fails (the server sheds the request).
// Chunks are mapped into the device's address space, so kernels can read
// and write slabs directly (dev_of).
struct PinnedPool {
    static constexpr int kMinOrder = 12, kMaxChunkOrder = 28;
    int kChunkOrder = kMaxChunkOrder;  // chunk size: 256 MiB, or less under a smaller limit
    std::mutex m;
    std::vector<char*> chunks;
    std::vector<char*> dchunks;  // each chunk's device address (null: not mapped)
    std::vector<std::unordered_set<uintptr_t>> free_blocks =
        std::vector<std::unordered_set<uintptr_t>>(kMaxChunkOrder + 1);
    size_t in_use = 0;          // bytes of slabs handed out and not yet returned
    size_t limit = ~(size_t)0;  // pinned bytes at most
    static int order(size_t bytes) {
        int c = kMinOrder;
        while (((size_t)1 << c) < bytes) ++c;
        return c;
    }
    bool add_chunk() {  // with m held
        if ((chunks.size() + 1) << kChunkOrder > limit) return false;
        void* p = nullptr;
        if (cudaHostAlloc(&p, (size_t)1 << kChunkOrder, cudaHostAllocPortable | cudaHostAllocMapped) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        void* d = nullptr;
        if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess) {
            cudaGetLastError();
            d = nullptr;
        }
        chunks.push_back((char*)p);
        dchunks.push_back((char*)d);
        free_blocks[kChunkOrder].insert((uintptr_t)p);
        return true;
    }
    void set_limit(size_t bytes) {
        limit = bytes;
        while (kChunkOrder > kMinOrder && ((size_t)1 << kChunkOrder) > limit) --kChunkOrder;
    }
    // Pins chunks for up to `bytes` (within the limit) ahead of serving.
    void reserve(size_t bytes) {
        std::lock_guard<std::mutex> g(m);
        while (chunks.size() << kChunkOrder < bytes && add_chunk()) {
        }
    }
    void* get(size_t bytes) {
        const int c = order(bytes);
        if (c > kChunkOrder) return nullptr;
        std::lock_guard<std::mutex> g(m);
        int o = c;
        while (o <= kChunkOrder && free_blocks[o].empty()) ++o;
        if (o > kChunkOrder) {
            if (!add_chunk()) return nullptr;
            o = kChunkOrder;
        }
        uintptr_t blk = *free_blocks[o].begin();
        free_blocks[o].erase(free_blocks[o].begin());
        while (o > c) {  // split, keeping the lower half
            --o;
            free_blocks[o].insert(blk + ((uintptr_t)1 << o));
        }
        in_use += (size_t)1 << c;
        return (void*)blk;
    }
    void put(void* p, size_t bytes) {
        if (!p) return;
        int o = order(bytes);
        std::lock_guard<std::mutex> g(m);
        in_use -= (size_t)1 << o;
        uintptr_t blk = (uintptr_t)p, base = 0;
        for (char* ch : chunks)
            if (blk >= (uintptr_t)ch && blk < (uintptr_t)ch + ((uintptr_t)1 << kChunkOrder)) base = (uintptr_t)ch;
        while (o < kChunkOrder) {  // coalesce with free buddies
            const uintptr_t buddy = base + ((blk - base) ^ ((uintptr_t)1 << o));
            auto it = free_blocks[o].find(buddy);
            if (it == free_blocks[o].end()) break;
            free_blocks[o].erase(it);
            blk = std::min(blk, buddy);
            ++o;
        }
        free_blocks[o].insert(blk);
    }
    size_t used() {
        std::lock_guard<std::mutex> g(m);
        return in_use;
    }
    // Device address of host address h inside a chunk, or null.
    void* dev_of(const void* h) {
        std::lock_guard<std::mutex> g(m);
        const uintptr_t a = (uintptr_t)h;
        for (size_t i = 0; i < chunks.size(); ++i)
            if (a >= (uintptr_t)chunks[i] && a < (uintptr_t)chunks[i] + ((uintptr_t)1 << kChunkOrder))
                return dchunks[i] ? dchunks[i] + (a - (uintptr_t)chunks[i]) : nullptr;
        return nullptr;
    }
    ~PinnedPool() {
        for (char* ch : chunks) cudaFreeHost(ch);
    }
};

struct Req {
    long long id;
    int kind;  // 0: modular product, 1: exact int64 product
    u32 p;
    long long la, lb;
    void* in = nullptr;   // pinned: operands (kind 0: u32 A then B; kind 1: int64 A then B)
    void* res = nullptr;  // pinned: result (kind 0: la+lb-1 u32; kind 1: 2(la+lb-1) int64)
    size_t in_bytes = 0, res_bytes = 0;
    // operands in memory registered with the server: copied to the device
    // from there (in stays null); res_direct: the result goes straight into out
    const void* a_src = nullptr;
    const void* b_src = nullptr;
    bool res_direct = false;
    size_t direct_bytes = 0;  // bytes of this request counted in Server::direct_inflight
    int bw = 1;
    TwoConvPlan plan{0, 0, 0, 0};  // exact products: the plan (sizes the lane buffers)
    bool long_path = false;         // exact products on the big-coefficient path (exact_i64_prefers_long)
    // exact products with a one-limb plan over three primes: batched together
    // (exact_i64_long_batch) whatever the single-product path
    bool one_limb = false;
    u32 primes[3] = {0, 0, 0};
    void* out;
    size_t bytes;
    double t_submit = 0, t_done = 0;
    int status = -1;
    bool done = false;
};

// Lane buffers grow geometrically (at least 1.5x), so that a stream of
// growing batches reallocates a logarithmic number of times.
size_t grow_to(size_t have, size_t want) { return std::max<size_t>({want, have + have / 2, 1024}); }

template <class T>
// A lane's device buffer, allocated and freed in the order of the lane's
// stream (cudaMallocAsync / cudaFreeAsync): growing it neither waits for the
// device nor stalls the other lanes.
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    int ensure(size_t want, cudaStream_t st) {
        if (want <= n) return OK;
        if (p) cudaFreeAsync(p, st);  // after the stream's earlier work, which used it
        p = nullptr;
        const size_t cap = grow_to(n, want);
        n = 0;
        if (dev_malloc_async((void**)&p, cap * sizeof(T), st) != cudaSuccess) {
            cudaGetLastError();
            return OUT_OF_MEMORY;
        }
        n = cap;
        return OK;
    }
    void release(cudaStream_t st) {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        n = 0;
    }
};

template <class T>
struct PinBuf {
    T* p = nullptr;
    size_t n = 0;
    int ensure(size_t want) {
        if (want <= n) return OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        const size_t cap = grow_to(n, want);
        n = 0;
        if (cudaHostAlloc((void**)&p, cap * sizeof(T), cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return OUT_OF_MEMORY;
        }
        n = cap;
        return OK;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
};

// Host <-> device copies of a batch.  A cudaMemcpyAsync costs the copy
// engine about 4 us on top of its bytes (B200, PCIe host link: 1.1 GB/s for
// 4 KiB copies, 31 GB/s for 256 KiB, 46-53 GB/s from 1 MiB), so a batch's
// many small operands and results move instead through one kernel each way
// that reads or writes the mapped host memory directly (41-43 GB/s at any
// size).  Copies of kDmaMinBytes and more keep the copy engines, which
// pass the kernel from about 1 MiB on; a copy kernel also holds SM slots
// while it waits on the link.  With log-uniform request sizes those copies
// are a fifth of the copies and most of the bytes (serving capacity: 4-5 %
// more requests/s at 512 KiB than at 128 KiB).
constexpr size_t kDmaMinBytes = 512 << 10;
constexpr u32 kCopyChunkWords = 8192;  // 32 KiB per table entry

struct CopyChunk {
    const u32* src;
    u32* dst;
    u32 words;
    u32 pad;
};

// Copies every table entry (4-byte words; source or destination may be
// mapped host memory), a block per entry and step, eight words in flight per
// thread.  One 256-thread block per SM at most (kCopyBlocks): the blocks
// spend their time waiting on the host link, and more of them would hold
// SM slots that other lanes' product kernels need, for no more bandwidth.
constexpr int kCopyBlocks = 148, kCopyInflight = 8;
__global__ void __launch_bounds__(256) k_copy_chunks(const CopyChunk* __restrict__ t, int n) {
    for (int c = blockIdx.x; c < n; c += gridDim.x) {
        const CopyChunk ch = t[c];
        for (u32 i = threadIdx.x; i < ch.words; i += kCopyInflight * blockDim.x) {
            u32 v[kCopyInflight];
#pragma unroll
            for (int k = 0; k < kCopyInflight; ++k) {
                const u32 j = i + k * blockDim.x;
                if (j < ch.words) v[k] = ch.src[j];
            }
#pragma unroll
            for (int k = 0; k < kCopyInflight; ++k) {
                const u32 j = i + k * blockDim.x;
                if (j < ch.words) ch.dst[j] = v[k];
            }
        }
    }
}

void add_copy(std::vector<CopyChunk>& t, const void* src, void* dst, size_t bytes) {
    const u32* s = (const u32*)src;
    u32* d = (u32*)dst;
    const size_t w = bytes / 4;
    for (size_t i = 0; i < w; i += kCopyChunkWords)
        t.push_back(CopyChunk{s + i, d + i, (u32)std::min<size_t>(kCopyChunkWords, w - i), 0});
}

struct Lane {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    DevBuf<u32> din, dout, ws;
    DevBuf<unsigned char> djobs;
    PinBuf<unsigned char> hjobs;
    // the batch's copy tables (operands in, then results out)
    PinBuf<CopyChunk> hcopy;
    DevBuf<CopyChunk> dcopy;
    std::vector<Req*> reqs;
    int status = OK;
    bool busy = false;
    long long seq = 0;
    double t_start = 0, t_launched = 0;  // batch timing for the trace log
    double t_alloc = 0, t_copies = 0;    // after the buffer checks, after the operand copies
    // trace only: device timestamps of the batch's start, operands in, kernels done, results out
    cudaEvent_t tev[4] = {nullptr, nullptr, nullptr, nullptr};
};

}  // namespace

struct Server {
    cumodp_server_config cfg;
    int dev;
    std::mutex m;
    std::condition_variable cv_work, cv_done, cv_free;
    std::deque<Req*> pending;
    std::unordered_map<long long, Req*> reqs;
    std::vector<Lane> lanes;
    PinnedPool pool;
    // host ranges registered by the caller (cumodp_server_register): start ->
    // bytes and the range's device address (mapped registration)
    struct RegRange {
        size_t n;
        uintptr_t dev;
    };
    std::mutex reg_m;
    std::map<uintptr_t, RegRange> regs;
    std::atomic<size_t> direct_inflight{0};  // operand and result bytes of unfinished direct requests
    std::deque<int> dispatched;  // lane indices in dispatch order
    size_t inflight = 0;
    long long next_id = 1, lane_seq = 0;
    bool stop = false;
    std::thread batcher, completer;
    FILE* trace = nullptr;  // CUMODP_SERVER_TRACE: per-batch timing log
    cudaEvent_t t_origin = nullptr;  // trace: device time origin of the lanes' timestamps
    // statistics
    std::vector<double> lat;
    long long completed = 0, failed = 0, batches = 0;
    double t_first = 0, t_last = 0;

    explicit Server(const cumodp_server_config& c) : cfg(c), dev(c.device) {}
};

namespace {

constexpr size_t kBatchBytes = 1ull << 30;

// Lane buffers an exact product takes on its own path, or (one-limb plans)
// the larger of that and its share of a batched group (words, words, bytes).
void exact_sizes(const Req& r, size_t* eval_words, size_t* ws_words, size_t* job_bytes) {
    if (r.long_path) exact_i64_long_sizes(r.la, r.lb, r.bw, eval_words, ws_words, job_bytes);
    else twoconv_buffer_sizes_plan(r.la, r.lb, r.plan, eval_words, ws_words, job_bytes);
    if (r.one_limb) {
        const long long la[1] = {r.la}, lb[1] = {r.lb};
        size_t e, w, j;
        exact_i64_batch_sizes(1, la, lb, &e, &w, &j);
        *eval_words = std::max(*eval_words, e);
        *ws_words = std::max(*ws_words, w);
        *job_bytes = std::max(*job_bytes, j);
    }
}

size_t req_bytes(const Req& r) {
    const long long lc = r.la + r.lb - 1;
    if (r.kind == 0) {
        const int logn = product_logn(r.la, r.lb);
        const size_t ws = logn > kMaxSmallLog ? (2ull << logn) : 0;
        return (size_t)(r.la + r.lb + lc + ws) * 4 + 256;
    }
    size_t ev, ws, jb;
    exact_sizes(r, &ev, &ws, &jb);
    return (r.la + r.lb + 2 * lc) * 8 + (ev + ws) * 4 + jb;
}

// Whether [p, p + n) lies in one range registered with the server; if so
// and dev is given, *dev = its device address (null when not mapped).
bool registered(Server& S, const void* p, size_t n, void** dev = nullptr) {
    const uintptr_t a = (uintptr_t)p;
    std::lock_guard<std::mutex> g(S.reg_m);
    auto it = S.regs.upper_bound(a);
    if (it == S.regs.begin()) return false;
    --it;
    if (!(a >= it->first && a + n <= it->first + it->second.n)) return false;
    if (dev) *dev = it->second.dev ? (void*)(it->second.dev + (a - it->first)) : nullptr;
    return true;
}

// Records [p, p + n) (already page-locked; device address dev) as
// registered; false if it overlaps a recorded range.
bool register_range(Server& S, const void* p, size_t n, const void* dev) {
    const uintptr_t a = (uintptr_t)p;
    std::lock_guard<std::mutex> g(S.reg_m);
    auto it = S.regs.lower_bound(a);
    if (it != S.regs.end() && it->first < a + n) return false;
    if (it != S.regs.begin()) {
        auto pr = std::prev(it);
        if (pr->first + pr->second.n > a) return false;
    }
    S.regs[a] = Server::RegRange{n, (uintptr_t)dev};
    return true;
}

// Device address of host memory [p, p + n) that a kernel may read or write:
// inside a registered range or a pinned slab; null otherwise.
void* dev_view(Server& S, const void* p, size_t n) {
    void* d = nullptr;
    if (registered(S, p, n, &d)) return d;
    return S.pool.dev_of(p);
}

// Moves the batch's copy tables to the device (one copy) and launches the
// copies of entries [0, nin); the entries after them are the results'.
int stage_copies(Lane& L, const std::vector<CopyChunk>& t, int nin) {
    if (t.empty()) return OK;
    int err = OK;
    if ((err = L.hcopy.ensure(t.size())) || (err = L.dcopy.ensure(t.size(), L.st))) return err;
    std::memcpy(L.hcopy.p, t.data(), t.size() * sizeof(CopyChunk));
    cudaError_t ce = cudaMemcpyAsync(L.dcopy.p, L.hcopy.p, t.size() * sizeof(CopyChunk), cudaMemcpyHostToDevice, L.st);
    if (ce != cudaSuccess) return cuda_err(ce);
    if (nin > 0) k_copy_chunks<<<std::min(nin, kCopyBlocks), 256, 0, L.st>>>(L.dcopy.p, nin);
    return cuda_err(cudaGetLastError());
}

int launch_result_copies(Lane& L, int first, int count) {
    if (count <= 0) return OK;
    k_copy_chunks<<<std::min(count, kCopyBlocks), 256, 0, L.st>>>(L.dcopy.p + first, count);
    return cuda_err(cudaGetLastError());
}

// Places a request's operands and result: straight from and into the
// caller's memory where it lies in registered ranges (no copy on the host),
// else in pinned slabs (the operands copied there now).  Unfinished requests
// may hold at most the host budget -- slab bytes plus the bytes of direct
// requests -- beyond which the request is shed (CUMODP_OUT_OF_MEMORY).
void stage_request(Server& S, Req* r, const void* a, size_t abytes, const void* b, size_t bbytes) {
    const bool in_reg = registered(S, a, abytes) && registered(S, b, bbytes);
    const bool out_reg = registered(S, r->out, r->res_bytes);
    const size_t direct = (in_reg ? abytes + bbytes : 0) + (out_reg ? r->res_bytes : 0);
    const size_t slab = (in_reg ? 0 : r->in_bytes) + (out_reg ? 0 : r->res_bytes);
    if (S.pool.used() + S.direct_inflight.load() + direct + slab > S.pool.limit) {
        r->status = OUT_OF_MEMORY;  // shed: the backlog already holds the whole budget
        return;
    }
    if (in_reg) {
        r->a_src = a;
        r->b_src = b;
    } else if (!(r->in = S.pool.get(r->in_bytes))) {
        r->status = OUT_OF_MEMORY;
        return;
    }
    if (out_reg) {
        r->res_direct = true;
    } else if (!(r->res = S.pool.get(r->res_bytes))) {
        S.pool.put(r->in, r->in_bytes);
        r->in = nullptr;
        r->status = OUT_OF_MEMORY;
        return;
    }
    if (r->in) {
        memcpy(r->in, a, abytes);
        memcpy((char*)r->in + abytes, b, bbytes);
    }
    r->direct_bytes = direct;
    S.direct_inflight += direct;
}

void finish(Server& S, Req* r, int status) {
    r->status = status;
    r->t_done = now_us();
    r->done = true;
    if (status == OK) {
        S.completed++;
        S.lat.push_back(r->t_done - r->t_submit);
    } else {
        S.failed++;
    }
    if (!S.t_first) S.t_first = r->t_submit;
    S.t_last = r->t_done;
}

// Runs one batch on a lane (lane.reqs share kind and prime).  Called without
// the server lock; only touches the lane and the requests it owns.
int run_batch(Server& S, Lane& L) {
    cudaSetDevice(S.dev);
    if (S.cfg.inject_fault_batch > 0 && S.batches == S.cfg.inject_fault_batch)
        return OUT_OF_MEMORY;  // host-side fault injection for tests: nothing is launched
    const int kind = L.reqs[0]->kind;
    const u32 p = L.reqs[0]->p;
    const int cnt = (int)L.reqs.size();
    int err = OK;
    auto mark = [&](int i) {
        if (L.tev[i]) cudaEventRecord(L.tev[i], L.st);
    };
    // an operand copy: a table entry of the copy kernel when small and
    // mapped, else the copy engines now
    auto copy_in = [&](std::vector<CopyChunk>& t, const void* h, void* d, size_t bytes) -> cudaError_t {
        void* v = bytes < kDmaMinBytes ? dev_view(S, h, bytes) : nullptr;
        if (v) {
            add_copy(t, v, d, bytes);
            return cudaSuccess;
        }
        return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, L.st);
    };
    // a result copy as a table entry; false: it goes by the copy engines
    auto copy_out_table = [&](std::vector<CopyChunk>& t, const void* d, void* h, size_t bytes) {
        void* v = bytes < kDmaMinBytes ? dev_view(S, h, bytes) : nullptr;
        if (v) add_copy(t, d, v, bytes);
        return v != nullptr;
    };
    mark(0);
    if (kind == 0) {
        std::vector<long long> la(cnt), lb(cnt), lh(cnt);
        size_t nin = 0, nout = 0;
        for (int i = 0; i < cnt; ++i) {
            la[i] = L.reqs[i]->la;
            lb[i] = L.reqs[i]->lb;
            lh[i] = la[i] + lb[i] - 1;
            nin += la[i] + lb[i];
            nout += lh[i];
        }
        if ((err = L.din.ensure(nin, L.st)) || (err = L.dout.ensure(nout, L.st))) return err;
        const size_t wsw = direct_ws_words(cnt, la.data(), lb.data());
        const size_t jb = direct_job_bytes(cnt);
        if ((err = L.ws.ensure(wsw + 1, L.st)) || (err = L.djobs.ensure(jb, L.st)) || (err = L.hjobs.ensure(jb)))
            return err;
        L.t_alloc = now_us();
        std::vector<const u32*> pa(cnt), pb(cnt);
        std::vector<u32*> ph(cnt);
        std::vector<CopyChunk> tab, tout;
        std::vector<int> dma_out;  // requests whose results go by the copy engines
        size_t o = 0, q = 0;
        for (int i = 0; i < cnt; ++i) {
            Req* r = L.reqs[i];
            cudaError_t ce;
            if (r->a_src) {  // straight from the caller's registered memory
                ce = copy_in(tab, r->a_src, L.din.p + o, r->la * 4);
                if (ce == cudaSuccess) ce = copy_in(tab, r->b_src, L.din.p + o + r->la, r->lb * 4);
            } else {
                ce = copy_in(tab, r->in, L.din.p + o, (r->la + r->lb) * 4);
            }
            if (ce != cudaSuccess) return cuda_err(ce);
            pa[i] = L.din.p + o;
            pb[i] = L.din.p + o + r->la;
            o += r->la + r->lb;
            ph[i] = L.dout.p + q;
            q += lh[i];
            if (!copy_out_table(tout, ph[i], r->res_direct ? r->out : r->res, lh[i] * 4)) dma_out.push_back(i);
        }
        const int nt_in = (int)tab.size();
        tab.insert(tab.end(), tout.begin(), tout.end());
        if ((err = stage_copies(L, tab, nt_in)) != OK) return err;
        L.t_copies = now_us();
        mark(1);
        // no autotuning on the serving path: cached or default splits only
        err = direct_batch(cnt, pa.data(), la.data(), pb.data(), lb.data(), ph.data(), lh.data(), p, L.ws.p,
                           L.djobs.p, L.hjobs.p, L.st, false);
        if (err != OK) return err;
        mark(2);
        if ((err = launch_result_copies(L, nt_in, (int)tout.size())) != OK) return err;
        for (int i : dma_out) {
            Req* r = L.reqs[i];
            cudaError_t ce = cudaMemcpyAsync(r->res_direct ? r->out : r->res, ph[i], lh[i] * 4,
                                             cudaMemcpyDeviceToHost, L.st);
            if (ce != cudaSuccess) return cuda_err(ce);
        }
    } else {
        // exact products: those with a one-limb plan over the batch's first
        // such prime triple run together (exact_i64_long_batch: their operands
        // first in the buffers, one residue kernel, one batched product per
        // prime, one CRT kernel); the others one after another
        std::vector<Req*> grp, rest;
        u32 gp[3] = {0, 0, 0};
        for (Req* r : L.reqs) {
            const u32* pp = r->primes;
            if (r->one_limb && (grp.empty() || (pp[0] == gp[0] && pp[1] == gp[1] && pp[2] == gp[2]))) {
                if (grp.empty()) std::copy(pp, pp + 3, gp);
                grp.push_back(r);
            } else {
                rest.push_back(r);
            }
        }
        const int ng = (int)grp.size();
        std::vector<long long> gla(ng), glb(ng);
        for (int i = 0; i < ng; ++i) {
            gla[i] = grp[i]->la;
            glb[i] = grp[i]->lb;
        }
        size_t nin = 0, nout = 0, evw = 0, wsw = 0, jbb = 0;  // eval and workspace: the largest of the steps
        if (ng) exact_i64_batch_sizes(ng, gla.data(), glb.data(), &evw, &wsw, &jbb);
        const size_t jb_grp = jbb;
        for (Req* r : L.reqs) {
            nin += r->la + r->lb;
            nout += 2 * (r->la + r->lb - 1);
        }
        for (Req* r : rest) {
            size_t e, w, j;
            exact_sizes(*r, &e, &w, &j);
            evw = std::max(evw, e);
            wsw = std::max(wsw, w);
            jbb += j;
        }
        // int64 data travels through the u32 buffers (two words per value)
        if ((err = L.din.ensure(2 * nin, L.st)) || (err = L.dout.ensure(2 * nout + evw, L.st)) ||
            (err = L.ws.ensure(wsw + 1, L.st)) || (err = L.djobs.ensure(jbb, L.st)) || (err = L.hjobs.ensure(jbb)))
            return err;
        L.t_alloc = now_us();
        size_t o = 0, q = 0, jo = 0;
        u32* eval = L.dout.p + 2 * nout;
        long long* din64 = (long long*)L.din.p;
        long long* dout64 = (long long*)L.dout.p;
        auto copy_in_dma = [&](Req* r, size_t at) {
            cudaError_t ce;
            if (r->a_src) {
                ce = cudaMemcpyAsync(din64 + at, r->a_src, r->la * 8, cudaMemcpyHostToDevice, L.st);
                if (ce == cudaSuccess)
                    ce = cudaMemcpyAsync(din64 + at + r->la, r->b_src, r->lb * 8, cudaMemcpyHostToDevice, L.st);
            } else {
                ce = cudaMemcpyAsync(din64 + at, r->in, (r->la + r->lb) * 8, cudaMemcpyHostToDevice, L.st);
            }
            return ce;
        };
        auto copy_out = [&](Req* r, size_t at) {
            return cudaMemcpyAsync(r->res_direct ? r->out : r->res, dout64 + 2 * at, (r->la + r->lb - 1) * 16,
                                   cudaMemcpyDeviceToHost, L.st);
        };
        if (ng) {
            std::vector<CopyChunk> tab, tout;
            std::vector<std::pair<Req*, size_t>> dma_out;  // results that go by the copy engines
            for (Req* r : grp) {
                cudaError_t ce;
                if (r->a_src) {
                    ce = copy_in(tab, r->a_src, din64 + o, r->la * 8);
                    if (ce == cudaSuccess) ce = copy_in(tab, r->b_src, din64 + o + r->la, r->lb * 8);
                } else {
                    ce = copy_in(tab, r->in, din64 + o, (r->la + r->lb) * 8);
                }
                if (ce != cudaSuccess) return cuda_err(ce);
                if (!copy_out_table(tout, dout64 + 2 * q, r->res_direct ? r->out : r->res, (r->la + r->lb - 1) * 16))
                    dma_out.emplace_back(r, q);
                o += r->la + r->lb;
                q += r->la + r->lb - 1;
            }
            const int nt_in = (int)tab.size();
            tab.insert(tab.end(), tout.begin(), tout.end());
            if ((err = stage_copies(L, tab, nt_in)) != OK) return err;
            mark(1);
            TwoConvBufs B{eval, L.ws.p, L.djobs.p, L.hjobs.p};
            err = exact_i64_long_batch(ng, din64, gla.data(), glb.data(), dout64, gp, L.st, B);
            if (err != OK) return err;
            mark(2);
            if ((err = launch_result_copies(L, nt_in, (int)tout.size())) != OK) return err;
            for (auto& rq : dma_out) {
                cudaError_t ce = copy_out(rq.first, rq.second);
                if (ce != cudaSuccess) return cuda_err(ce);
            }
            jo = jb_grp;
        } else {
            mark(1);
            mark(2);
        }
        for (Req* r : rest) {
            cudaError_t ce = copy_in_dma(r, o);
            if (ce != cudaSuccess) return cuda_err(ce);
            TwoConvBufs B{eval, L.ws.p, L.djobs.p + jo, L.hjobs.p + jo};
            size_t e, w, j;
            exact_sizes(*r, &e, &w, &j);
            err = r->long_path
                      ? exact_i64_long_dev_bufs(din64 + o, r->la, din64 + o + r->la, r->lb, dout64 + 2 * q, r->bw, L.st,
                                                &B)
                      : twoconv_mul_dev(din64 + o, r->la, din64 + o + r->la, r->lb, dout64 + 2 * q, r->bw, r->bw,
                                        false, L.st, nullptr, &B);
            if (err != OK) return err;
            ce = copy_out(r, q);
            if (ce != cudaSuccess) return cuda_err(ce);
            o += r->la + r->lb;
            q += r->la + r->lb - 1;
            jo += j;
        }
        L.t_copies = now_us();  // the group's phases are marked; the others run in the last one
    }
    mark(3);
    return cuda_err(cudaEventRecord(L.ev, L.st));
}

void recreate_lane(Lane& L) {
    if (L.st) cudaStreamDestroy(L.st);
    if (L.ev) cudaEventDestroy(L.ev);
    cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&L.ev, cudaEventDisableTiming);
}

void batcher_loop(Server* Sp) {
    Server& S = *Sp;
    cudaSetDevice(S.dev);
    std::unique_lock<std::mutex> lk(S.m);
    for (;;) {
        S.cv_work.wait(lk, [&] { return S.stop || !S.pending.empty(); });
        if (S.stop) return;
        // batching window: let a few more requests arrive (continuous
        // batching: lanes already running are not waited for)
        if ((int)S.pending.size() < S.cfg.max_batch && S.cfg.batch_window_us > 0) {
            S.cv_work.wait_for(lk, std::chrono::microseconds(S.cfg.batch_window_us),
                               [&] { return S.stop || (int)S.pending.size() >= S.cfg.max_batch; });
            if (S.stop) return;
        }
        int li = -1;
        S.cv_free.wait(lk, [&] {
            if (S.stop) return true;
            for (size_t i = 0; i < S.lanes.size(); ++i)
                if (!S.lanes[i].busy) { li = (int)i; return true; }
            return false;
        });
        if (S.stop) return;
        // admit in arrival order, same (kind, prime) as the head, within the budget
        Lane& L = S.lanes[li];
        L.reqs.clear();
        Req* head = S.pending.front();
        const int kind = head->kind;
        const u32 p = head->p;
        size_t add = 0;
        for (auto it = S.pending.begin(); it != S.pending.end() && (int)L.reqs.size() < S.cfg.max_batch;) {
            Req* r = *it;
            if (r->kind == kind && r->p == p) {
                if (S.inflight + add + r->bytes > S.cfg.memory_budget && !(L.reqs.empty() && S.inflight == 0)) break;
                // a batch holds at most kBatchBytes of device memory (or one request): lane buffers stay
                // within the memory pool backed at creation, and no batch delays the others for long
                if (!L.reqs.empty() && add + r->bytes > kBatchBytes) break;
                L.reqs.push_back(r);
                add += r->bytes;
                it = S.pending.erase(it);
            } else {
                ++it;
            }
        }
        if (L.reqs.empty()) {  // head does not fit yet: wait for a completion
            S.cv_done.wait(lk);
            continue;
        }
        S.inflight += add;
        L.busy = true;
        L.seq = ++S.lane_seq;
        S.batches++;
        lk.unlock();
        L.t_start = now_us();
        L.t_alloc = L.t_copies = 0;
        L.status = run_batch(S, L);
        L.t_launched = now_us();
        if (L.status != OK) cudaEventRecord(L.ev, L.st);  // completer still waits on the lane
        lk.lock();
        S.dispatched.push_back(li);
        S.cv_done.notify_all();
    }
}

void completer_loop(Server* Sp) {
    Server& S = *Sp;
    cudaSetDevice(S.dev);
    std::unique_lock<std::mutex> lk(S.m);
    for (;;) {
        S.cv_done.wait(lk, [&] { return S.stop || !S.dispatched.empty(); });
        if (S.dispatched.empty() && S.stop) return;
        if (S.dispatched.empty()) continue;
        // the first lane whose batch has finished: batches of different lanes
        // finish in any order, and a lane whose batch is done must not wait
        // behind an older, longer batch to be freed
        size_t pos = 0;
        while (S.dispatched.size() > 1) {
            bool found = false;
            for (size_t k = 0; k < S.dispatched.size() && !found; ++k) {
                if (cudaEventQuery(S.lanes[S.dispatched[k]].ev) != cudaErrorNotReady) {
                    pos = k;
                    found = true;
                }
            }
            cudaGetLastError();  // a not-ready query leaves its status as the thread's last error
            if (found) break;
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(10));
            lk.lock();
        }
        if (S.dispatched.empty()) continue;
        const int li = S.dispatched[pos];
        S.dispatched.erase(S.dispatched.begin() + pos);
        Lane& L = S.lanes[li];
        lk.unlock();
        cudaError_t ce = cudaEventSynchronize(L.ev);  // done (several lanes) or the only one in flight
        int st = L.status != OK ? L.status : cuda_err(ce);
        if (st == OK) st = cuda_err(cudaGetLastError());
        if (st != OK) {
            // contain the failure: drain and re-create the lane
            cudaStreamSynchronize(L.st);
            cudaGetLastError();
            recreate_lane(L);
        }
        if (S.trace) {
            // one line per batch: start, host launch time, completion seen,
            // kind, prime, requests, operand words, status, host time to the
            // buffer checks and to the operand copies issued (us)
            long long words = 0;
            for (Req* r : L.reqs) words += r->la + r->lb;
            // then the device side: start after the origin, operands in, kernels, results out (us)
            float d[4] = {-1.f, -1.f, -1.f, -1.f};
            if (st == OK && L.tev[0] && S.t_origin) {
                cudaEventElapsedTime(&d[0], S.t_origin, L.tev[0]);
                for (int i = 1; i < 4; ++i) cudaEventElapsedTime(&d[i], L.tev[i - 1], L.tev[i]);
                cudaGetLastError();
            }
            std::fprintf(S.trace, "%.1f %.1f %.1f %d %u %zu %lld %d %.1f %.1f %.1f %.1f %.1f %.1f\n", L.t_start,
                         L.t_launched - L.t_start, now_us() - L.t_start, L.reqs.empty() ? -1 : L.reqs[0]->kind,
                         L.reqs.empty() ? 0u : L.reqs[0]->p, L.reqs.size(), words, st,
                         L.t_alloc ? L.t_alloc - L.t_start : -1.0, L.t_copies ? L.t_copies - L.t_start : -1.0,
                         d[0] * 1e3, d[1] * 1e3, d[2] * 1e3, d[3] * 1e3);
        }
        lk.lock();
        size_t freed = 0;
        for (Req* r : L.reqs) {
            freed += r->bytes;
            finish(S, r, st == FFT_SIZE_TOO_LARGE || st == OK || st == ASSUMPTION_ERROR ||
                                 st == OUT_OF_MEMORY ? st : FFT_ERROR);
            S.pool.put(r->in, r->in_bytes);  // the operands' copy has completed
            r->in = nullptr;
            S.direct_inflight -= r->direct_bytes;  // operands read, result in the caller's buffer
            r->direct_bytes = 0;
        }
        S.inflight -= std::min(S.inflight, freed);
        L.reqs.clear();
        L.busy = false;
        S.cv_free.notify_all();
        S.cv_done.notify_all();
        S.cv_work.notify_all();
    }
}

long long submit(Server& S, Req* r) {
    std::lock_guard<std::mutex> g(S.m);
    if (S.stop) {
        delete r;
        return -1;
    }
    r->id = S.next_id++;
    r->t_submit = now_us();
    r->bytes = req_bytes(*r);
    S.reqs[r->id] = r;
    if (r->status != -1) {  // rejected at submission
        finish(S, r, r->status);
        S.cv_done.notify_all();
        return r->id;
    }
    S.pending.push_back(r);
    S.cv_work.notify_one();
    return r->id;
}

// Waits for request `id`, copies its result into the caller's buffer and
// releases it.  *t_ready (optional) receives the time at which the result
// reached the caller's buffer, as if a thread had been waiting for exactly
// this request: completion time plus the copy's duration.
int wait_request(Server* S, long long id, long long timeout_us, double* t_ready) {
    if (!S) return -1;
    std::unique_lock<std::mutex> lk(S->m);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return -1;
    Req* r = it->second;
    auto pred = [&] { return r->done; };
    if (timeout_us < 0) S->cv_done.wait(lk, pred);
    else if (!S->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), pred)) return -2;
    const int st = r->status;
    const double t_done = r->t_done;
    S->reqs.erase(it);
    lk.unlock();
    const double c0 = now_us();
    if (st == OK && !r->res_direct && r->out) memcpy(r->out, r->res, r->res_bytes);
    if (t_ready) *t_ready = t_done + (now_us() - c0);
    S->pool.put(r->in, r->in_bytes);
    S->pool.put(r->res, r->res_bytes);
    S->direct_inflight -= r->direct_bytes;
    delete r;
    return st;
}

// Replay of a timed trace (cumodp_server_replay): `threads` submitters, each
// with a collector thread that waits for its requests in submission order.
struct Replay {
    Server* S;
    long long count;
    const double* arrival;
    const int* kind;
    const sfixn* p;
    const long long *la, *lb;
    const void* const* a;
    const void* const* b;
    void* const* h;
    double* lat;
    int* status;
    double t0;
};

// Request submission; H / c may be null (replayed requests: the result is dropped).
long long submit_mod_req(Server& Sr, sfixn p, sfixn df, const sfixn* F, sfixn dg, const sfixn* G, sfixn* H) {
    Server* S = &Sr;
    if (!F || !G || df < 0 || dg < 0) return -1;
    Req* r = new Req();
    r->kind = 0;
    r->p = (u32)p;
    r->la = (long long)df + 1;
    r->lb = (long long)dg + 1;
    r->out = H;
    int err = OK;
    const PrimeCtx* pc = prime_ctx((u32)p, &err);
    if (!pc) r->status = err;
    else if (product_logn(r->la, r->lb) > std::min(pc->info.two_adic, kMaxLog)) r->status = FFT_SIZE_TOO_LARGE;
    else {
        r->in_bytes = (size_t)(r->la + r->lb) * 4;
        r->res_bytes = (size_t)(r->la + r->lb - 1) * 4;
        stage_request(*S, r, F, (size_t)r->la * 4, G, (size_t)r->lb * 4);
    }
    return submit(*S, r);
}

long long submit_i64_req(Server& Sr, long long na, const int64_t* a, long long nb, const int64_t* b, int64_t* c) {
    Server* S = &Sr;
    if (!a || !b || na <= 0 || nb <= 0) return -1;
    Req* r = new Req();
    r->kind = 1;
    r->p = 0;
    r->la = na;
    r->lb = nb;
    r->out = c;
    unsigned long long m = 0;
    for (long long i = 0; i < na; ++i) m |= a[i] < 0 ? 0ull - (unsigned long long)a[i] : (unsigned long long)a[i];
    for (long long i = 0; i < nb; ++i) m |= b[i] < 0 ? 0ull - (unsigned long long)b[i] : (unsigned long long)b[i];
    r->bw = m ? 64 - __builtin_clzll(m) : 1;
    // the two-convolution plan, or the big-coefficient path where it is the
    // only or the cheaper one (up to 2^22 coefficients here)
    int e = na + nb - 1 > (1ll << 22) ? FFT_SIZE_TOO_LARGE : OK;
    if (e == OK) {
        r->long_path = exact_i64_prefers_long(r->bw, r->bw, na, nb);
        if (!r->long_path) e = twoconv_plan(r->bw, r->bw, na, nb, false, &r->plan);
        r->one_limb = e == OK && exact_i64_long_one_limb(r->bw, na, nb, r->primes);
    }
    if (e != OK) r->status = e;
    else {
        r->in_bytes = (size_t)(na + nb) * 8;
        r->res_bytes = (size_t)(na + nb - 1) * 16;
        stage_request(*S, r, a, (size_t)na * 8, b, (size_t)nb * 8);
    }
    return submit(*S, r);
}

void replay_thread(const Replay& R, int t, int threads) {
    struct Item {
        long long i, id;
    };
    std::mutex qm;
    std::condition_variable qcv;
    std::deque<Item> q;
    bool done = false;
    std::thread collector([&] {
        for (;;) {
            Item it;
            {
                std::unique_lock<std::mutex> lk(qm);
                qcv.wait(lk, [&] { return done || !q.empty(); });
                if (q.empty()) return;
                it = q.front();
                q.pop_front();
            }
            if (it.id < 0) {
                R.status[it.i] = -1;
                R.lat[it.i] = 0;
            } else {
                double t_ready = 0;
                R.status[it.i] = wait_request(R.S, it.id, -1, &t_ready);
                R.lat[it.i] = t_ready - (R.t0 + R.arrival[it.i]);
            }
        }
    });
    for (long long i = t; i < R.count; i += threads) {
        const double target = R.t0 + R.arrival[i];
        for (;;) {
            const double d = target - now_us();
            if (d <= 0) break;
            if (d > 200) std::this_thread::sleep_for(std::chrono::microseconds((long long)(d - 100)));
            else std::this_thread::yield();
        }
        // without an output buffer the result stays in the server's pinned slab (dropped when collected)
        void* out = R.h ? R.h[i] : nullptr;
        long long id;
        if (R.kind[i] == 0)
            id = submit_mod_req(*R.S, R.p[i], (sfixn)(R.la[i] - 1), (const sfixn*)R.a[i], (sfixn)(R.lb[i] - 1),
                                (const sfixn*)R.b[i], (sfixn*)out);
        else
            id = submit_i64_req(*R.S, R.la[i], (const int64_t*)R.a[i], R.lb[i], (const int64_t*)R.b[i],
                                (int64_t*)out);
        {
            std::lock_guard<std::mutex> g(qm);
            q.push_back(Item{i, id});
        }
        qcv.notify_one();
    }
    {
        std::lock_guard<std::mutex> g(qm);
        done = true;
    }
    qcv.notify_one();
    collector.join();
}

}  // namespace

}  // namespace cmb

using namespace cmb;

extern "C" {

void cumodp_server_default_config(cumodp_server_config* c) {
    if (!c) return;
    c->device = 0;
    c->memory_budget = 0;
    c->max_batch = 512;
    c->batch_window_us = 50;
    c->lanes = 4;
    c->inject_fault_batch = 0;
    c->host_budget = 0;
}

cumodp_server* cumodp_server_create(const cumodp_server_config* cfg) {
    cumodp_server_config c;
    cumodp_server_default_config(&c);
    if (cfg) c = *cfg;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || c.device < 0 || c.device >= n) {
        cudaGetLastError();
        return nullptr;
    }
    cudaSetDevice(c.device);
    if (c.memory_budget == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        c.memory_budget = fr / 4;
    }
    if (c.max_batch <= 0) c.max_batch = 512;
    if (c.lanes <= 0) c.lanes = 4;
    Server* S = new Server(c);
    S->lanes.resize(c.lanes);
    for (Lane& L : S->lanes) recreate_lane(L);
    // lane buffers come from the device's default memory pool (stream-ordered
    // allocation); keep what they free cached in this process instead of
    // returning it at every synchronisation
    cudaMemPool_t mp;
    if (cudaDeviceGetDefaultMemPool(&mp, c.device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep);
        // back the pool with physical memory now (growing it later maps new
        // memory inside a batch's launch, which took up to a second)
        const size_t reserve = std::min<size_t>(c.memory_budget, 16ull << 30);
        void* tmp = nullptr;
        cudaStream_t s0 = S->lanes[0].st;
        if (cudaMallocAsync(&tmp, reserve, s0) == cudaSuccess) cudaFreeAsync(tmp, s0);
        cudaStreamSynchronize(s0);
    }
    cudaGetLastError();
    // lane buffers for a full batch, allocated now so that serving does not
    // grow them: job tables (pinned memory is not reallocated while serving,
    // cudaFreeHost waits for the device) for max_batch modular products or
    // max_batch exact ones (up to 3 primes x 8 evaluation points each), and
    // device operand, result and workspace buffers of kBatchBytes each (a
    // batch holds at most kBatchBytes; only a single larger request grows them)
    const size_t jobs = std::max(direct_job_bytes(c.max_batch), (size_t)c.max_batch * 3 * direct_job_bytes(8));
    const size_t words = std::min<size_t>(kBatchBytes, c.memory_budget / (3 * (size_t)c.lanes)) / 4;
    // copy tables: up to three copies per request below kDmaMinBytes, 16 entries each
    const size_t copy_entries = 3 * (size_t)c.max_batch * (kDmaMinBytes / (4 * kCopyChunkWords));
    for (Lane& L : S->lanes) {
        L.hjobs.ensure(jobs);
        L.djobs.ensure(jobs, L.st);
        L.hcopy.ensure(copy_entries);
        L.dcopy.ensure(copy_entries, L.st);
        L.din.ensure(words, L.st);
        L.dout.ensure(words, L.st);
        L.ws.ensure(words, L.st);
    }
    for (Lane& L : S->lanes) cudaStreamSynchronize(L.st);
    cudaGetLastError();
    // pinned slabs: the whole host budget is pinned now, so that serving never
    // calls cudaHostAlloc (slow, and it stalls other CUDA calls)
    S->pool.set_limit(c.host_budget ? c.host_budget : (2ull << 30));
    S->pool.reserve(S->pool.limit);
    if (const char* tf = getenv("CUMODP_SERVER_TRACE")) S->trace = fopen(tf, "a");
    if (S->trace) {
        cudaEventCreate(&S->t_origin);
        cudaEventRecord(S->t_origin, S->lanes[0].st);
        for (Lane& L : S->lanes)
            for (cudaEvent_t& e : L.tev) cudaEventCreate(&e);
        cudaStreamSynchronize(S->lanes[0].st);
        cudaGetLastError();
    }
    S->batcher = std::thread(batcher_loop, S);
    S->completer = std::thread(completer_loop, S);
    return (cumodp_server*)S;
}

long long cumodp_server_submit_mod(cumodp_server* h, sfixn p, sfixn df, const sfixn* F, sfixn dg, const sfixn* G,
                                   sfixn* H) {
    if (!h || !H) return -1;
    return submit_mod_req(*(Server*)h, p, df, F, dg, G, H);
}

long long cumodp_server_submit_i64(cumodp_server* h, long long na, const int64_t* a, long long nb, const int64_t* b,
                                   int64_t* c) {
    if (!h || !c) return -1;
    return submit_i64_req(*(Server*)h, na, a, nb, b, c);
}

int cumodp_server_poll(cumodp_server* h, long long id) {
    Server* S = (Server*)h;
    if (!S) return -1;
    std::lock_guard<std::mutex> g(S->m);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return -1;
    return it->second->done ? 1 : 0;
}

int cumodp_server_wait(cumodp_server* h, long long id, long long timeout_us) {
    return wait_request((Server*)h, id, timeout_us, nullptr);
}

cumodp_err cumodp_server_replay(cumodp_server* s, long long count, const double* arrival_us, const int* kind,
                                const sfixn* p, const long long* la, const long long* lb, const void* const* a,
                                const void* const* b, void* const* h, int threads, double* lat_us, int* status,
                                double* span_us) {
    Server* S = (Server*)s;
    if (!S || count < 0 || threads <= 0 || (count > 0 && (!arrival_us || !kind || !p || !la || !lb || !a || !b ||
                                                          !lat_us || !status)))
        return CUMODP_ASSUMPTION_ERROR;
    for (long long i = 0; i < count; ++i)
        if (la[i] <= 0 || lb[i] <= 0 || !a[i] || !b[i] || (kind[i] != 0 && kind[i] != 1) ||
            (kind[i] == 0 && (la[i] > INT32_MAX || lb[i] > INT32_MAX)))
            return CUMODP_ASSUMPTION_ERROR;
    Replay R{S, count, arrival_us, kind, p, la, lb, a, b, h, lat_us, status, now_us()};
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t) th.emplace_back(replay_thread, std::cref(R), t, threads);
    for (auto& x : th) x.join();
    double last = R.t0;
    for (long long i = 0; i < count; ++i)
        if (status[i] != -1) last = std::max(last, R.t0 + arrival_us[i] + lat_us[i]);
    if (span_us) *span_us = last - R.t0;
    return CUMODP_SUCCESS;
}

cumodp_err cumodp_server_register(cumodp_server* h, void* ptr, size_t bytes) {
    Server* S = (Server*)h;
    if (!S || !ptr || bytes == 0) return CUMODP_ASSUMPTION_ERROR;
    if (registered(*S, ptr, 1) || registered(*S, (char*)ptr + bytes - 1, 1)) return CUMODP_ASSUMPTION_ERROR;
    cudaSetDevice(S->dev);
    if (cudaHostRegister(ptr, bytes, cudaHostRegisterPortable | cudaHostRegisterMapped) != cudaSuccess) {
        cudaGetLastError();
        return CUMODP_FAILURE;
    }
    void* dev = nullptr;
    if (cudaHostGetDevicePointer(&dev, ptr, 0) != cudaSuccess) {
        cudaGetLastError();
        dev = nullptr;  // copies from this range then go through the copy engines
    }
    if (!register_range(*S, ptr, bytes, dev)) {
        cudaHostUnregister(ptr);
        return CUMODP_ASSUMPTION_ERROR;
    }
    return CUMODP_SUCCESS;
}

cumodp_err cumodp_server_unregister(cumodp_server* h, void* ptr) {
    Server* S = (Server*)h;
    if (!S || !ptr) return CUMODP_ASSUMPTION_ERROR;
    {
        std::lock_guard<std::mutex> g(S->reg_m);
        auto it = S->regs.find((uintptr_t)ptr);
        if (it == S->regs.end()) return CUMODP_ASSUMPTION_ERROR;
        S->regs.erase(it);
    }
    cudaSetDevice(S->dev);
    const cudaError_t e = cudaHostUnregister(ptr);
    cudaGetLastError();
    return e == cudaSuccess ? CUMODP_SUCCESS : CUMODP_FAILURE;
}

void cumodp_server_get_stats(cumodp_server* h, cumodp_server_stats* out) {
    Server* S = (Server*)h;
    if (!S || !out) return;
    std::lock_guard<std::mutex> g(S->m);
    memset(out, 0, sizeof(*out));
    out->completed = S->completed;
    out->failed = S->failed;
    out->batches = S->batches;
    out->pending = (long long)S->pending.size();
    out->inflight_bytes = S->inflight;
    std::vector<double> l = S->lat;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        out->p50_us = l[l.size() / 2];
        out->p99_us = l[std::min(l.size() - 1, (size_t)(0.99 * l.size()))];
        out->max_us = l.back();
    }
    const double span = (S->t_last - S->t_first) * 1e-6;
    out->products_per_s = span > 0 ? S->completed / span : 0;
}

void cumodp_server_reset_stats(cumodp_server* h) {
    Server* S = (Server*)h;
    if (!S) return;
    std::lock_guard<std::mutex> g(S->m);
    S->lat.clear();
    S->completed = S->failed = S->batches = 0;
    S->t_first = S->t_last = 0;
}

void cumodp_server_destroy(cumodp_server* h) {
    Server* S = (Server*)h;
    if (!S) return;
    {
        std::unique_lock<std::mutex> lk(S->m);
        // drain: wait for queued and in-flight work
        S->cv_done.wait(lk, [&] {
            bool busy = false;
            for (auto& L : S->lanes) busy |= L.busy;
            return S->pending.empty() && !busy && S->dispatched.empty();
        });
        S->stop = true;
    }
    S->cv_work.notify_all();
    S->cv_free.notify_all();
    S->cv_done.notify_all();
    S->batcher.join();
    S->completer.join();
    cudaSetDevice(S->dev);
    for (Lane& L : S->lanes) {
        if (L.st) cudaStreamSynchronize(L.st);
        L.din.release(L.st); L.dout.release(L.st); L.ws.release(L.st); L.djobs.release(L.st);
        L.dcopy.release(L.st);
        L.hjobs.release();
        L.hcopy.release();
        if (L.st) cudaStreamDestroy(L.st);
        if (L.ev) cudaEventDestroy(L.ev);
        for (cudaEvent_t e : L.tev)
            if (e) cudaEventDestroy(e);
    }
    if (S->t_origin) cudaEventDestroy(S->t_origin);
    if (S->trace) fclose(S->trace);
    for (auto& kv : S->regs) cudaHostUnregister((void*)kv.first);  // ranges the caller left registered
    cudaGetLastError();
    for (auto& kv : S->reqs) {
        S->pool.put(kv.second->in, kv.second->in_bytes);
        S->pool.put(kv.second->res, kv.second->res_bytes);
        delete kv.second;
    }
    delete S;
}

}  // extern "C"
