"""Batched products of uneven degree (one graph launch per batch) vs the oracle."""
import numpy as np
import pytest

from cumodp_b200.workloads import SplitMix64, seed_for

P0 = 469762049
pytestmark = pytest.mark.gpu


def make_pairs(r, degs, p):
    return [(r.residues(int(a) + 1, p), r.residues(int(b) + 1, p)) for a, b in degs]


def test_mixed_batch_all_classes(cm, oracle_mod):
    """Every size class from 2^5 to 2^20 in one batch, each checked."""
    r = SplitMix64(11)
    degs = [(0, 0), (3, 9), (31, 32), (40, 100), (300, 200), (1000, 1023), (2000, 2047), (4095, 4096),
            (8191, 8000), (9000, 9000), (16383, 16384), (30000, 40000), (65535, 65535), (200000, 100000),
            (5, 7), (511, 511), (1, 70000)]
    pairs = make_pairs(r, degs, P0)
    outs = cm.fftmul_batch(pairs, P0)
    for (a, b), h in zip(pairs, outs):
        assert np.array_equal(h, oracle_mod.polymul(a, b, P0))


def test_batch_repeat_uses_cached_plan_and_new_data(cm, oracle_mod):
    r = SplitMix64(12)
    degs = [(100, 200), (5000, 5000), (20000, 3)] * 3
    for rep in range(3):
        pairs = make_pairs(r, degs, P0)
        outs = cm.fftmul_batch(pairs, P0)
        for (a, b), h in zip(pairs, outs):
            assert np.array_equal(h, oracle_mod.polymul(a, b, P0))


def test_c4_shape_sample(cm, oracle_mod):
    """A 256-pair slice of the C4 workload (degrees log-uniform in [32, 65536])."""
    r = SplitMix64(seed_for(3))
    da = r.log_uniform_int(256, 32, 65536)
    db = r.log_uniform_int(256, 32, 65536)
    pairs = make_pairs(r, list(zip(da, db)), P0)
    outs = cm.fftmul_batch(pairs, P0)
    for (a, b), h in zip(pairs, outs):
        assert np.array_equal(h, oracle_mod.polymul(a, b, P0))


def test_batch_same_result_as_single_calls(cm):
    r = SplitMix64(13)
    degs = [(17, 4000), (777, 778), (12000, 30000)]
    pairs = make_pairs(r, degs, 962592769)
    outs = cm.fftmul_batch(pairs, 962592769)
    for (a, b), h in zip(pairs, outs):
        assert np.array_equal(h, cm.fftmul_uni(a, b, 962592769))


def test_empty_batch(cm):
    assert cm.fftmul_batch([], P0) == []


def test_batch_rejects_oversize(cm):
    a = np.ones(200, np.uint32)
    with pytest.raises(cm.CumodpError) as e:
        cm.fftmul_batch([(a, a)], 257)
    assert e.value.code == cm.FFT_SIZE_TOO_LARGE


def test_large_host_batch_is_pipelined_and_exact(cm, oracle_mod):
    """Host-buffer batch of large products (the pipelined copy path): every product
    equals the single-call path, one checked against the oracle; more products
    than device slots, mixed sizes, one shared operand."""
    r = SplitMix64(0xC0DA0501)
    shared = r.residues((1 << 19) + 7, P0)
    pairs = [(r.residues((1 << 19), P0), r.residues((1 << 19), P0)),
             (r.residues(700001, P0), r.residues(400000, P0)),
             (shared, r.residues((1 << 20) - 5, P0)),
             (r.residues(1 << 20, P0), shared),
             (r.residues(600000, P0), r.residues(600000, P0))]
    outs = cm.fftmul_batch(pairs, P0)
    for (a, b), h in zip(pairs, outs):
        assert np.array_equal(h, cm.fftmul_uni(a, b, P0))
    assert np.array_equal(outs[1], oracle_mod.polymul(pairs[1][0], pairs[1][1], P0))


def test_device_batch_of_large_classes(cm):
    """Device-resident batch with several products per large size class
    (2^20-2^22 transforms: one launch of each pass kernel per class covers
    every job, including operands longer than half the transform and
    operands starting off a 16-byte boundary); each product equals its
    single call."""
    import torch
    r = SplitMix64(0xC0DA0502)
    degs = [(2**19 - 1, 2**19 - 1), (2**19 - 1, 2**19 - 1), (600000, 100), (100, 600000), (2**19 - 1, 3),
            (2**20 - 1, 2**20 - 1), (2**20 - 1, 2**20 - 2), (2**21 - 1, 2**21 - 1), (2**21 - 1, 2**21 - 7)]
    df = np.array([a for a, _ in degs], np.int32)
    dg = np.array([b for _, b in degs], np.int32)
    # odd gaps between operands: most of them start off a 16-byte boundary
    f_off = np.zeros(len(degs), np.int64)
    g_off = np.zeros(len(degs), np.int64)
    h_off = np.zeros(len(degs), np.int64)
    f_off[1:] = np.cumsum(df.astype(np.int64) + 2)[:-1]
    g_off[1:] = np.cumsum(dg.astype(np.int64) + 3)[:-1]
    h_off[1:] = np.cumsum(df.astype(np.int64) + dg + 1)[:-1]
    F = r.residues(int(f_off[-1] + df[-1] + 1), P0)
    G = r.residues(int(g_off[-1] + dg[-1] + 1), P0)
    tF = torch.from_numpy(F.view(np.int32)).cuda()
    tG = torch.from_numpy(G.view(np.int32)).cuda()
    tH = torch.zeros(int(h_off[-1] + df[-1] + dg[-1] + 1), dtype=torch.int32, device="cuda")
    cm.fftmul_batch_dev(df, f_off, tF.data_ptr(), dg, g_off, tG.data_ptr(), h_off, tH.data_ptr(), P0)
    torch.cuda.synchronize()
    H = tH.cpu().numpy().view(np.uint32)
    for i, (a, b) in enumerate(degs):
        fa = F[f_off[i]:f_off[i] + a + 1]
        gb = G[g_off[i]:g_off[i] + b + 1]
        assert np.array_equal(H[h_off[i]:h_off[i] + a + b + 1], cm.fftmul_uni(fa, gb, P0)), i


def test_queued_small_classes_many_items(cm, oracle_mod):
    """Every product of transform length 2^5 .. 2^12 runs in the batch's one work-queue launch: thousands
    of items of all eight classes, partial last items (counts not multiples of a class's products per
    CTA), with large classes beside them; every product checked against the oracle's schoolbook."""
    r = SplitMix64(14)
    degs = []
    for logn, count in [(5, 300), (6, 129), (7, 65), (8, 33), (9, 300), (10, 17), (11, 9), (12, 41)]:
        hi = (1 << logn) - 1  # da + db + 1 <= 2^logn, > 2^(logn-1)
        for _ in range(count):
            da = int(r.next_u64(1)[0] % np.uint64(hi))
            db = max(0, hi - 1 - da - int(r.next_u64(1)[0] % np.uint64(max(1, hi // 4))))
            degs.append((da, db))
    degs += [(20000, 30000), (8191, 8191)]
    pairs = make_pairs(r, degs, P0)
    for rep in range(2):  # the graph replayed: the queue counter is reset every launch
        outs = cm.fftmul_batch(pairs, P0)
        for (a, b), h in zip(pairs, outs):
            want = oracle_mod.polymul_school(a, b, P0) if len(a) * len(b) < 1 << 22 else oracle_mod.polymul(a, b, P0)
            assert np.array_equal(h, want)
