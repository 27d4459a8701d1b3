"""Serving loop: continuous batching gives each request the same result alone and in the mix."""
import threading

import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64

PRIMES = [469762049, 754974721, 962592769]
pytestmark = pytest.mark.gpu


def _mix(r, count, max_log=17):
    reqs = []
    kinds = r.uniform01(count)
    degs_a = r.log_uniform_int(count, 32, 1 << max_log)
    degs_b = r.log_uniform_int(count, 32, 1 << max_log)
    pidx = (r.next_u64(count) % np.uint64(3)).astype(int)
    for i in range(count):
        if kinds[i] < 0.2:
            n, m = int(min(degs_a[i], 20000)), int(min(degs_b[i], 20000))
            reqs.append(("i64", r.int64_in(n + 1, 10**10), r.int64_in(m + 1, 10**10)))
        else:
            p = PRIMES[pidx[i]]
            reqs.append(("mod", p, r.residues(int(degs_a[i]) + 1, p), r.residues(int(degs_b[i]) + 1, p)))
    return reqs


def _submit(srv, req):
    if req[0] == "mod":
        return srv.submit_mod(req[2], req[3], req[1])
    return srv.submit_i64(req[1], req[2])


def test_same_result_alone_and_in_the_mix(cm):
    r = SplitMix64(99)
    reqs = _mix(r, 120)
    with cm.Server(max_batch=64, batch_window_us=100) as srv:
        alone = []
        for q in reqs:  # one at a time: each request is its own batch
            rid, out = _submit(srv, q)
            assert srv.wait(rid) == 0
            alone.append(out.copy())
        # the same requests from 4 submitting threads at once, interleaved
        mixed = [None] * len(reqs)

        def worker(k):
            ids = []
            for i in range(k, len(reqs), 4):
                ids.append((i, _submit(srv, reqs[i])))
            for i, (rid, out) in ids:
                assert srv.wait(rid) == 0
                mixed[i] = out.copy()

        th = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        st = srv.stats()
    for a, m in zip(alone, mixed):
        assert np.array_equal(a, m)
    assert st["completed"] >= 2 * len(reqs) and st["failed"] == 0
    assert st["batches"] < 2 * len(reqs)  # the mixed phase was batched
    assert st["p99_us"] >= st["p50_us"] > 0


def test_results_match_single_calls(cm, oracle_mod):
    r = SplitMix64(7)
    reqs = _mix(r, 40, max_log=15)
    with cm.Server() as srv:
        handles = [_submit(srv, q) for q in reqs]
        for q, (rid, out) in zip(reqs, handles):
            assert srv.wait(rid) == 0
            if q[0] == "mod":
                assert np.array_equal(out, oracle_mod.polymul(q[2], q[3], q[1]))
            else:
                assert cm.int128_words_to_ints(out) == oracle_mod.polymul_i128(q[1], q[2])


def test_invalid_request_reports_error_and_server_continues(cm):
    with cm.Server() as srv:
        rid, _ = srv.submit_mod(np.ones(10, np.uint32), np.ones(10, np.uint32), 1000)  # not prime
        assert srv.wait(rid) == cm.ASSUMPTION_ERROR
        big = np.ones(200, np.uint32)
        rid, _ = srv.submit_mod(big, big, 257)  # beyond 257's 2-adic order
        assert srv.wait(rid) == cm.FFT_SIZE_TOO_LARGE
        a = np.arange(1, 100, dtype=np.uint32)
        rid, out = srv.submit_mod(a, a, 469762049)
        assert srv.wait(rid) == 0
        assert np.array_equal(out, cm.fftmul_uni(a, a, 469762049))


def test_injected_batch_failure_is_contained(cm):
    """Host-side fault injection: batch 2 fails before any launch; later batches are exact."""
    r = SplitMix64(5)
    p = 469762049
    with cm.Server(inject_fault_batch=2, batch_window_us=0) as srv:
        results = []
        for i in range(4):
            a, b = r.residues(500 + i, p), r.residues(300, p)
            rid, out = srv.submit_mod(a, b, p)
            results.append((srv.wait(rid), a, b, out.copy()))
        codes = [c for c, *_ in results]
        assert codes.count(cm.OUT_OF_MEMORY) == 1 and codes[1] == cm.OUT_OF_MEMORY
        for c, a, b, out in results:
            if c == 0:
                assert np.array_equal(out, cm.fftmul_uni(a, b, p))
        st = srv.stats()
        assert st["failed"] == 1


def test_tight_memory_budget_still_completes(cm):
    r = SplitMix64(8)
    p = 469762049
    with cm.Server(memory_budget=4 << 20, batch_window_us=0) as srv:  # 4 MiB: about one request at a time
        hs = []
        for _ in range(12):
            a, b = r.residues(100000, p), r.residues(90000, p)
            hs.append((a, b) + srv.submit_mod(a, b, p))
        for a, b, rid, out in hs:
            assert srv.wait(rid) == 0
            assert np.array_equal(out, cm.fftmul_uni(a, b, p))


def test_wait_timeout_and_unknown_id(cm):
    with cm.Server() as srv:
        assert srv.wait(123456, timeout_us=1000) == -1
        assert srv.poll(123456) == -1


def test_replay_trace_results_and_latency(cm, oracle_mod):
    """Native open-loop replay: every result equals the oracle's, latencies are positive."""
    r = SplitMix64(0xC0DA0105)
    reqs = _mix(r, 60, max_log=14)
    arrival = np.cumsum(-np.log(1.0 - r.uniform01(len(reqs))) / 2000.0) * 1e6
    trace, outs = [], []
    for q in reqs:
        if q[0] == "mod":
            trace.append((q[2], q[3], q[1]))
            outs.append(np.zeros(len(q[2]) + len(q[3]) - 1, np.uint32))
        else:
            trace.append((q[1], q[2], None))
            outs.append(np.zeros(2 * (len(q[1]) + len(q[2]) - 1), np.int64))
    with cm.Server(max_batch=32) as srv:
        st, lat, span = srv.replay(arrival, trace, threads=3, outputs=outs)
    assert (st == 0).all()
    assert (lat > 0).all() and span >= arrival[-1]
    for q, o in zip(reqs, outs):
        if q[0] == "mod":
            assert np.array_equal(o, oracle_mod.polymul(q[2], q[3], q[1]))
        else:
            assert cm.int128_words_to_ints(o) == oracle_mod.polymul_i128(q[1], q[2])


def test_host_budget_sheds_and_server_continues(cm, oracle_mod):
    """Beyond the pinned host budget a submission completes at once with OUT_OF_MEMORY."""
    p = PRIMES[0]
    r = SplitMix64(0xC0DA0106)
    big = [r.residues(1 << 17, p) for _ in range(2)]
    with cm.Server(host_budget=3 << 20, batch_window_us=20000) as srv:
        # each request holds a 1 MiB operand slab and a 1 MiB result slab
        h1 = srv.submit_mod(big[0], big[1], p)
        h2 = srv.submit_mod(big[0], big[1], p)
        assert srv.wait(h2[0]) == cm.OUT_OF_MEMORY
        assert srv.wait(h1[0]) == 0
        assert np.array_equal(h1[1], oracle_mod.polymul(big[0], big[1], p))
        h3 = srv.submit_mod(big[0], big[1], p)  # slabs returned: admitted again
        assert srv.wait(h3[0]) == 0


def test_registered_memory_gives_the_same_results(cm):
    """Operands and outputs in memory registered with the server (no staging copies) give the same
    words as the copied path, for modular and exact requests, alone and in a concurrent mix."""
    r = SplitMix64(2031)
    reqs = _mix(r, 60, max_log=16)
    # every operand and output placed in one registered arena
    sizes = []
    for q in reqs:
        if q[0] == "mod":
            sizes += [len(q[2]) * 4, len(q[3]) * 4, (len(q[2]) + len(q[3]) - 1) * 4]
        else:
            sizes += [len(q[1]) * 8, len(q[2]) * 8, (len(q[1]) + len(q[2]) - 1) * 16]
    total = sum((s + 63) // 64 * 64 for s in sizes)
    raw = np.zeros(total + 8192, np.uint8)
    base = (-raw.ctypes.data) % 4096
    arena = raw[base:base + total + 4096]
    cursor = [0]

    def place(nbytes, dtype, values=None):
        a = arena[cursor[0]:cursor[0] + nbytes].view(dtype)
        cursor[0] += (nbytes + 63) // 64 * 64
        if values is not None:
            a[:] = values
        return a

    with cm.Server(max_batch=32, batch_window_us=100) as srv:
        srv.register(arena)
        L = cm.lib()
        want, got, ids = [], [], []
        for q in reqs:
            rid, out = _submit(srv, q)  # copied path (unregistered host arrays)
            assert srv.wait(rid) == 0
            want.append(out.copy())
        for q in reqs:
            if q[0] == "mod":
                a = place(len(q[2]) * 4, np.uint32, q[2])
                b = place(len(q[3]) * 4, np.uint32, q[3])
                o = place((len(a) + len(b) - 1) * 4, np.uint32)
                rid = L.cumodp_server_submit_mod(srv._h, q[1], len(a) - 1, a.ctypes.data, len(b) - 1, b.ctypes.data,
                                                 o.ctypes.data)
            else:
                a = place(len(q[1]) * 8, np.int64, q[1])
                b = place(len(q[2]) * 8, np.int64, q[2])
                o = place((len(a) + len(b) - 1) * 16, np.int64)
                rid = L.cumodp_server_submit_i64(srv._h, len(a), a.ctypes.data, len(b), b.ctypes.data, o.ctypes.data)
            assert rid > 0
            ids.append(rid)
            got.append(o)
        for rid in ids:
            assert L.cumodp_server_wait(srv._h, rid, -1) == 0
        for w, g in zip(want, got):
            assert np.array_equal(w.view(g.dtype), g)
        srv.unregister(arena)
        with pytest.raises(cm.CumodpError):
            srv.unregister(arena)  # already gone


def test_long_exact_requests_match_the_host_entry(cm):
    """Exact requests on both paths (two-convolution and, for 2^21-point products, the big-coefficient one)
    return the same words as cumodp_twoconv_mul_i64, alone and together in one batch."""
    r = SplitMix64(2032)
    shapes = [((1 << 20) - 3, (1 << 20) - 7), ((1 << 19) + 5, 1000), (300000, 600000), (70, 90)]
    ops = [(r.int64_in(na, 10**10), r.int64_in(nb, 10**10)) for na, nb in shapes]
    want = [cm.twoconv_mul(a, b, raw=True) for a, b in ops]
    with cm.Server(max_batch=8, batch_window_us=2000) as srv:
        for (a, b), w in zip(ops, want):  # alone
            rid, out = srv.submit_i64(a, b)
            assert srv.wait(rid) == 0
            assert np.array_equal(out, w)
        subs = [srv.submit_i64(a, b) for a, b in ops]  # together
        for (rid, out), w in zip(subs, want):
            assert srv.wait(rid) == 0
            assert np.array_equal(out, w)


def test_exact_batch_mixes_plans(cm):
    """One batch of exact requests on three plans: one-limb big-coefficient products (run together as one
    batched product per prime), two-limb ones (|c| ~ 2^50) and small coefficients on the two-convolution
    path (both one after another); every result equals cumodp_twoconv_mul_i64's, in any order of arrival."""
    r = SplitMix64(2033)
    ops = []
    for i in range(18):
        bound = (10**10, 1 << 50, 100)[i % 3]
        na, nb = [(3000, 5000), (1, 70000), (40000, 9), (65536, 65536), (17, 33), (123457, 1000)][i % 6]
        ops.append((r.int64_in(na, bound), r.int64_in(nb, bound)))
    want = [cm.twoconv_mul(a, b, raw=True) for a, b in ops]
    with cm.Server(max_batch=64, batch_window_us=20000) as srv:
        subs = [srv.submit_i64(a, b) for a, b in ops]
        for (rid, out), w in zip(subs, want):
            assert srv.wait(rid) == 0
            assert np.array_equal(out, w)
        st = srv.stats()
    assert st["batches"] <= 3  # the burst shared batches
