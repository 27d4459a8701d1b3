"""Benchmark of the FFT-based polynomial product on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the configuration the headline metric is quoted on, one GPU): the
product of two dense degree-(2^23 - 1) polynomials mod p = 469762049
(7 * 2^26 + 1), transform length n = 2^24, coefficients uniform in [0, p)
from a fixed splitmix64 seed.  One step = one product.  Inputs are resident
in HBM and rotate over 4 input sets (4 x 64 MiB > the 126 MB L2) so no step
reads an operand the previous step left in L2.

Printed JSON line (rank 0):
  value        products/s over the K timed steps (device time, CUDA events,
               max over ranks; N ranks run independent replicas)
  e2e          the same metric through the host C entry point
               cumodp_fftmul_uni with pinned host buffers: every step copies
               both operands in and the product out
  roofline     the dominant kernel: algorithmic bytes per launch / its mean
               launch time (events around every launch), against the measured
               HBM copy bandwidth
  cpu_baseline modpn's own FFT multiply (the reference CPU path) on the host
  extras       2^24-point forward+inverse transform GB/s; the batched
               mixed-degree workload (4096 pairs) against one call per pair;
               the list transform, the 2-D transform, the bivariate product
               and a subproduct-tree level, each with its own check

--impl reference runs the reference's CPU implementation of the same path
(modpn EX_Mont_FFTMul, compiled from the reference sources into
oracle/_ref) on all usable host threads.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P = 469762049
LOGN = 24
DEG = (1 << 23) - 1
METRIC = "products/s & NTT HBM GB/s (% of peak), batched vs plain GPU, bit-exact"
UNIT = "products/s"
WORKLOAD = "poly_product_deg(2^23-1)x(2^23-1)_mod_469762049_n2^24"


def peaks():
    f = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(f):
        d = json.load(open(f))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ helpers ----
def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank timing over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as td
    if not (td.is_available() and td.is_initialized()) or td.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, units_per_rank: int, seconds_max: float) -> float:
    """Whole-job units/s for independent replicas: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / seconds_max


def gen_operands(seed: int, sets: int):
    from cumodp_b200.workloads import SplitMix64
    r = SplitMix64(seed)
    return [(r.residues(DEG + 1, P), r.residues(DEG + 1, P)) for _ in range(sets)]


def powers_mod(x0: int, n: int) -> np.ndarray:
    pw = np.ones(n, dtype=np.uint64)
    m = 1
    step = x0 % P
    while m < n:
        k = min(m, n - m)
        pw[m:m + k] = (pw[:k] * np.uint64(step)) % np.uint64(P)
        step = step * step % P
        m *= 2
    return pw


def eval_mod(c: np.ndarray, pw: np.ndarray) -> int:
    acc = 0
    for i in range(0, len(c), 1 << 20):
        acc += int(((c[i:i + (1 << 20)].astype(np.uint64) * pw[i:i + (1 << 20)]) % np.uint64(P)).sum())
    return acc % P


def product_check(a, b, h) -> bool:
    """Size-independent check: H(x0) == A(x0) * B(x0) mod p at a fixed point."""
    x0 = 123456789
    pw = powers_mod(x0, len(h))
    return eval_mod(h, pw) == eval_mod(a, pw[:len(a)]) * eval_mod(b, pw[:len(b)]) % P


def host_link_bound(torch, dev, h2d_bytes: int, d2h_bytes: int, reps: int = 5) -> dict:
    """The host link's ceiling for a step that moves h2d_bytes in and d2h_bytes
    out: one step's copies, both directions at once from pinned buffers on two
    streams, timed with CUDA events (best of reps); e2e can at most reach
    1 / that time per GPU."""
    hi = torch.empty(h2d_bytes // 4, dtype=torch.int32).pin_memory()
    ho = torch.empty(d2h_bytes // 4, dtype=torch.int32).pin_memory()
    di = torch.empty(h2d_bytes // 4, dtype=torch.int32, device=dev)
    do = torch.empty(d2h_bytes // 4, dtype=torch.int32, device=dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    best = None
    for _ in range(reps + 1):
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s_in)
        s_out.wait_event(e0)
        with torch.cuda.stream(s_in):
            di.copy_(hi, non_blocking=True)
        with torch.cuda.stream(s_out):
            ho.copy_(do, non_blocking=True)
        e1.record(s_in)
        e2.record(s_out)
        torch.cuda.synchronize(dev)
        ms = max(e0.elapsed_time(e1), e0.elapsed_time(e2))
        best = ms if best is None else min(best, ms)
    return {"ms_per_step_copies": round(best, 4), "bound_per_s": round(1000.0 / best, 1),
            "gbs_per_direction": round(max(h2d_bytes, d2h_bytes) / (best / 1000.0) / 1e9, 1),
            "how": "one step's H2D and D2H copies at once (pinned, two streams), CUDA events, best of %d" % reps}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def modpn_sample(threads: int, products: int, seed: int):
    """Time `products` modpn products of the workload's size on `threads` host threads."""
    import oracle
    from cumodp_b200.workloads import SplitMix64
    r = SplitMix64(seed)
    a, b = r.residues(DEG + 1, P), r.residues(DEG + 1, P)
    pairs = [(a, b)] * products
    t0 = time.perf_counter()
    oracle.ref_polymul_batch(pairs, P, threads)
    return time.perf_counter() - t0


def ref_threads_bounded() -> int:
    t = host_threads()
    try:
        import psutil
        avail = psutil.virtual_memory().available
        t = min(t, max(1, int(avail * 0.5 // (3 * (1 << LOGN) * 4 + (3 << 24)))))
    except ImportError:
        pass
    return max(1, min(t, 64))


# ------------------------------------------------------- reference arm ----
def run_reference(args, rank: int):
    if rank != 0:
        return
    import oracle
    if not oracle.ref_available():
        try:
            oracle.build(ref=True)
        except Exception:
            pass
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "modpn reference CPU build (oracle/_ref/libmodpn_ref.so) is not present"}))
        return
    threads = ref_threads_bounded()
    per_step = threads  # one product per thread per step
    for _ in range(args.warmup):
        modpn_sample(threads, per_step, 0xC0DA0001)
    times = [modpn_sample(threads, per_step, 0xC0DA0001) for _ in range(args.steps)]
    total = sum(times)
    value = args.steps * per_step / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded splitmix64)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "per_step": f"{per_step} independent products, one per host thread"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{args.steps} steps x {per_step} products of degree 2^23-1 mod 469762049"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- ours ----
def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import cumodp_b200 as cm

    torch.cuda.set_device(local_rank)
    cm.select_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = world > 1
    if dist:
        import torch.distributed as td

    hbm_peak, peak_kind = peaks()
    n = 1 << LOGN
    sets = 4
    ops = gen_operands(0xC0DA0001 + rank, sets)
    dA = [torch.from_numpy(a.view(np.int32)).to(dev) for a, _ in ops]
    dB = [torch.from_numpy(b.view(np.int32)).to(dev) for _, b in ops]
    dH = torch.empty(n - 1, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream

    def step(i):
        s = i % sets
        cm.fftmul_uni_dev(dH.data_ptr(), n - 1, dA[s].data_ptr(), DEG, dB[s].data_ptr(), DEG, P, sp)

    # correctness of the measured path (untimed): evaluation-point identity
    step(0)
    torch.cuda.synchronize()
    ok = product_check(ops[0][0], ops[0][1], dH.cpu().numpy().view(np.uint32))

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if dist:
        td.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        # keep the GPU under this workload until the sampler reports (untimed),
        # so the clock record covers load right up to and through the timed region
        t_load = time.perf_counter()
        i = 0
        while (len(clk.lines) < 5 and time.perf_counter() - t_load < 4.0) or i < 4:
            step(i)
            i += 1
            if i % 16 == 0:
                torch.cuda.synchronize()
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(args.steps):
            step(i)
        e1.record(stream)
        torch.cuda.synchronize()
        # the same K steps again with an event pair around every kernel on the
        # launching stream (per-kernel durations for the roofline; the events
        # serialise the kernels, so this region is not the one `value` uses)
        cm.trace_passes(True)
        cm.trace_report(reset=True)
        for i in range(args.steps):
            step(i)
        torch.cuda.synchronize()
    cm.trace_passes(False)
    passes = cm.trace_report(reset=True)
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    if dist:
        td.barrier()
    value = replica_throughput(world, args.steps, ms / 1000.0)

    # dominant kernel and its roofline
    dom = max(passes.items(), key=lambda kv: kv[1][1])
    dom_name, (dom_cnt, dom_ms) = dom
    # algorithmic bytes per launch: one transform pass over n words moves 8n
    # bytes (read + write); col_fwd runs the first pass of both operands
    # (16n), row_fwd_g the second pass of G's forward transform (8n),
    # row_mul_f the second pass of F's forward transform and the first of the
    # inverse (16n), col_inv the last pass of the inverse (8n); the legacy
    # fused row kernel does both row kernels' passes (24n)
    units = {"col_fwd": 2, "row_fwd_g": 1, "row_mul_f": 2, "row_fused": 3, "col_inv": 1}
    unit_key = dom_name.rsplit("_", 1)[0]
    alg_bytes = units.get(unit_key, 1) * 8 * n
    mean_s = dom_ms / dom_cnt / 1000.0
    achieved = alg_bytes / mean_s / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get(dom_name)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                "frac": round(achieved / hbm_peak, 4), "traffic": traffic, "kernel": dom_name,
                "peak_kind": peak_kind, "alg_bytes_per_launch": alg_bytes,
                "mean_launch_ms": round(mean_s * 1000, 5),
                "window": "a second run of the K timed steps with CUDA events around every kernel",
                "passes_ms_per_step": {k: round(v[1] / v[0], 5) for k, v in passes.items()}}

    # whole-product roofline: pass-aware I/O bound of 3 transforms, 24 n ceil(log2 n / 14) bytes
    prod_alg = 24 * n * 2
    product_gbs = prod_alg / (ms / args.steps / 1000.0) / 1e9 / world

    # e2e through the host C entry point, pinned host buffers
    L = ctypes.CDLL(cm.LIB_PATH)  # own function objects: the binding's prototypes stay untouched
    hA = torch.from_numpy(ops[0][0].view(np.int32)).pin_memory()
    hB = torch.from_numpy(ops[0][1].view(np.int32)).pin_memory()
    hH = torch.empty(n - 1, dtype=torch.int32).pin_memory()
    cm_fn = L.cumodp_fftmul_uni
    cm_fn.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
                      ctypes.c_void_p, ctypes.c_int32]
    e2e_steps = max(3, min(args.steps, 40))
    for _ in range(2):
        cm_fn(n - 2, hH.data_ptr(), DEG, hA.data_ptr(), DEG, hB.data_ptr(), P)
    if dist:
        td.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        rc = cm_fn(n - 2, hH.data_ptr(), DEG, hA.data_ptr(), DEG, hB.data_ptr(), P)
        assert rc == 0, rc
    single_s = max_over_ranks(time.perf_counter() - t0, dev)
    single_ok = product_check(ops[0][0], ops[0][1], hH.numpy().view(np.uint32))
    # the same steps through the batched host entry point cumodp_fftmul_batch
    # (pinned host arrays; the library pipelines each product's copies in and
    # out against the kernels of its neighbours): step i multiplies operand
    # set i % 4 into output region i % 4
    sets = len(ops)
    hF = torch.from_numpy(np.concatenate([o[0] for o in ops]).view(np.int32)).pin_memory()
    hG = torch.from_numpy(np.concatenate([o[1] for o in ops]).view(np.int32)).pin_memory()
    hHb = torch.empty(sets * (n - 1), dtype=torch.int32).pin_memory()
    bfn = L.cumodp_fftmul_batch
    bfn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]
    dfa = np.full(e2e_steps, DEG, np.int32)
    f_off = (np.arange(e2e_steps, dtype=np.int64) % sets) * (DEG + 1)
    h_off = (np.arange(e2e_steps, dtype=np.int64) % sets) * (n - 1)

    def batch_call(k):
        rc = bfn(k, dfa.ctypes.data, f_off.ctypes.data, hF.data_ptr(), dfa.ctypes.data, f_off.ctypes.data,
                 hG.data_ptr(), h_off.ctypes.data, hHb.data_ptr(), P)
        assert rc == 0, rc
    batch_call(min(4, e2e_steps))
    if dist:
        td.barrier()
    t0 = time.perf_counter()
    batch_call(e2e_steps)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dev)
    e2e_ok = all(product_check(ops[k][0], ops[k][1], hHb[k * (n - 1):(k + 1) * (n - 1)].numpy().view(np.uint32))
                 for k in range(min(sets, e2e_steps)))
    e2e = {"value": replica_throughput(world, e2e_steps, e2e_s), "unit": UNIT, "h2d_bytes_per_step": 2 * (DEG + 1) * 4,
           "d2h_bytes_per_step": (n - 1) * 4, "steps": e2e_steps, "eval_point_identity": e2e_ok,
           "api": "cumodp_fftmul_batch (host arrays, pinned)",
           "single_call": {"value": replica_throughput(world, e2e_steps, single_s), "api": "cumodp_fftmul_uni",
                           "eval_point_identity": single_ok},
           "host_link": host_link_bound(torch, dev, 2 * (DEG + 1) * 4, (n - 1) * 4)}

    extras = {}
    if rank == 0 and not args.no_extras:
        extras["ntt_2_24"] = ntt_2_24(cm, torch, dev, stream, hbm_peak)
        extras["batched_c4"] = batched_c4(cm, torch, dev, stream)
        extras["c1_4095x4095"] = c1_latency(cm, torch, dev, stream)
        extras["c3_exact_int64"] = c3_exact(cm, torch, dev, stream)
        extras["big_1024bit_1024terms"] = big_coefficients(cm, torch, dev, stream)
        extras["serving_c5"] = serving_c5(cm)
        extras["list_and_bivariate"] = list_and_bivariate(cm, torch, dev, stream, hbm_peak)
        extras["reference_gpu"] = reference_gpu(cm, torch, dev, stream, extras,
                                                {"product_ms": round(ms / args.steps, 5),
                                                 "host_product_ms": host_product_ms(cm, ops[0][0], ops[0][1])})
    cpu = None
    if rank == 0 and world == 1 and not args.no_extras:
        cpu = cpu_baseline()

    if rank == 0:
        launches = args.steps * len(passes)  # one launch per traced pass per product
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic (seeded splitmix64, uniform residues)",
                "config": {"workload": WORKLOAD, "prime": P, "transform_log2": LOGN,
                           "l2_policy": "inputs rotate over 4 sets of 64 MiB (> 126 MB L2)",
                           "parallelism": f"replicas x{world}"},
                "check": {"eval_point_identity": ok},
                "product_alg_gbs": round(product_gbs, 1),
                "roofline": roofline, "e2e": e2e, "gpu_launches": launches,
                "clocks": dict(clk.summary(), window="sampled from 1 s of untimed load through the timed region"),
                "cpu_baseline": cpu}
        line.update(extras)
        print(json.dumps(line))


def ntt_2_24(cm, torch, dev, stream, hbm_peak):
    """Forward + inverse natural-order 2^24 transform (device pointers): GB/s on 8n*ceil(24/14) per transform."""
    from cumodp_b200.workloads import SplitMix64
    n = 1 << LOGN
    x = SplitMix64(0xC0DA0001).residues(n, P)
    w = pow(3, (P - 1) >> LOGN, P)  # 3 generates the multiplicative group of 469762049
    dx = torch.from_numpy(x.view(np.int32)).to(dev)
    sp = stream.cuda_stream
    for _ in range(2):
        cm.fft_uni_dev(dx.data_ptr(), LOGN, w, P, False, sp)
        cm.fft_uni_dev(dx.data_ptr(), LOGN, w, P, True, sp)
    torch.cuda.synchronize()
    reps = 10
    # the transforms alone (no events between their kernels)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        cm.fft_uni_dev(dx.data_ptr(), LOGN, w, P, False, sp)
        cm.fft_uni_dev(dx.data_ptr(), LOGN, w, P, True, sp)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / (2 * reps)
    # the same again with an event pair around every kernel: per-pass times
    cm.trace_passes(True)
    cm.trace_report(reset=True)
    for _ in range(reps):
        cm.fft_uni_dev(dx.data_ptr(), LOGN, w, P, False, sp)
        cm.fft_uni_dev(dx.data_ptr(), LOGN, w, P, True, sp)
    torch.cuda.synchronize()
    cm.trace_passes(False)
    passes = cm.trace_report(reset=True)
    round_trip_ok = bool(np.array_equal(dx.cpu().numpy().view(np.uint32), x))
    bio = 8 * n * 2
    per_pass = {k: {"ms": round(v[1] / v[0], 5), "gbs": round(8 * n / (v[1] / v[0] / 1000) / 1e9, 1),
                    "frac": round(8 * n / (v[1] / v[0] / 1000) / 1e9 / hbm_peak, 4)} for k, v in passes.items()}
    return {"ms_per_transform": round(ms, 5), "gbs_bio": round(bio / (ms / 1000) / 1e9, 1),
            "frac_bio": round(bio / (ms / 1000) / 1e9 / hbm_peak, 4),
            "gbs_strict_8n": round(8 * n / (ms / 1000) / 1e9, 1), "per_pass": per_pass,
            "round_trip_bit_exact": round_trip_ok}


def _timed(torch, stream, fn, reps: int = 10, warm: int = 2) -> float:
    """Mean ms of fn() over reps calls on stream (CUDA events), after warm calls."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def list_and_bivariate(cm, torch, dev, stream, hbm_peak):
    """The list transform, the 2-D transform, the bivariate product and a subproduct-tree level on
    resident operands larger than L2, each with a bit-exact check.  GB/s are on the algorithmic
    bytes: one HBM round trip (8 bytes a word) per pass the kernels need."""
    from cumodp_b200.workloads import SplitMix64
    r = SplitMix64(0xC0DA0F00)
    sp = stream.cuda_stream
    out = {}

    def rate(nbytes, ms):
        gbs = nbytes / (ms / 1000) / 1e9
        return round(gbs, 1), round(gbs / hbm_peak, 4)

    # list transform: 2^13 rows of 2^12 words (128 MiB), one CTA per row -> one pass
    m, k = 1 << 13, 12
    x = r.residues(m << k, P)
    dx = torch.from_numpy(x.view(np.int32)).to(dev)
    w = pow(3, (P - 1) >> k, P)

    def lst():
        cm.list_fft_dev(dx.data_ptr(), m, k, w, P, False, sp)
        cm.list_fft_dev(dx.data_ptr(), m, k, w, P, True, sp)
    ms = _timed(torch, stream, lst) / 2
    gbs, frac = rate(8 * (m << k), ms)
    out["list_fft_2^13x2^12"] = {"ms_per_transform": round(ms, 5), "gbs": gbs, "frac": frac,
                                 "round_trip_bit_exact": bool(np.array_equal(dx.cpu().numpy().view(np.uint32), x))}
    del dx
    # 2-D transform: 2^11 x 2^14 (128 MiB): column pass + row pass
    em, en = 11, 14
    x = r.residues(1 << (em + en), P)
    dx = torch.from_numpy(x.view(np.int32)).to(dev)
    wm, wn = pow(3, (P - 1) >> em, P), pow(3, (P - 1) >> en, P)

    def biv():
        cm.fft_bivariate_dev(dx.data_ptr(), em, wm, en, wn, P, False, sp)
        cm.fft_bivariate_dev(dx.data_ptr(), em, wm, en, wn, P, True, sp)
    ms = _timed(torch, stream, biv) / 2
    gbs, frac = rate(16 << (em + en), ms)
    out["bivariate_fft_2^11x2^14"] = {"ms_per_transform": round(ms, 5), "gbs_bio": gbs, "frac_bio": frac,
                                      "round_trip_bit_exact": bool(np.array_equal(dx.cpu().numpy().view(np.uint32), x))}
    del dx
    # bivariate product on a 2^12 x 2^12 grid: operands of 2^11 x 2^11 coefficients, zero padded
    em = en = 12
    half = 1 << (em - 1)
    fa = np.zeros((1 << em, 1 << en), dtype=np.uint32)
    ga = np.zeros_like(fa)
    fa[:half, :half] = r.residues(half * half, P).reshape(half, half)
    ga[:half, :half] = r.residues(half * half, P).reshape(half, half)
    dF = torch.from_numpy(fa.view(np.int32)).to(dev)
    dG = torch.from_numpy(ga.view(np.int32)).to(dev)
    tF, tG = torch.empty_like(dF), torch.empty_like(dG)

    def bmul():
        tF.copy_(dF)
        tG.copy_(dG)
        cm.bivariate_mul_dev(em, en, tF.data_ptr(), tG.data_ptr(), P, sp)
    with torch.cuda.stream(stream):
        ms = _timed(torch, stream, bmul)
    h = tF.cpu().numpy().view(np.uint32)
    x0, y0 = 987654321 % P, 192837465 % P
    px, py = powers_mod(x0, 1 << en), powers_mod(y0, 1 << em)

    def ev(a):
        rows = [eval_mod(a[j], px) for j in range(a.shape[0])]
        return eval_mod(np.array(rows, dtype=np.uint64), py[:len(rows)])
    ok = ev(h) == ev(fa) * ev(ga) % P
    n2 = 1 << (em + en)
    out["bivariate_mul_2^12x2^12"] = {"ms_per_product_incl_operand_copies": round(ms, 5),
                                      "products_per_s": round(1000 / ms, 1),
                                      "gbs_strict_12N": rate(12 * n2, ms)[0], "eval_point_identity": bool(ok)}
    del dF, dG, tF, tG
    # subproduct-tree level: 2^16 monic polynomials of degree 512 -> 2^15 products of degree 1024
    l, npairs = 512, 1 << 15
    mi = r.residues(2 * npairs * l, P)
    dI = torch.from_numpy(mi.view(np.int32)).to(dev)
    dO = torch.empty(2 * npairs * l, dtype=torch.int32, device=dev)
    ms = _timed(torch, stream, lambda: cm.subproduct_level_dev(l, npairs, dI.data_ptr(), dO.data_ptr(), P, sp))
    mo = dO.cpu().numpy().view(np.uint32)
    ok = True
    for j in (0, npairs - 1):
        a = np.append(mi[2 * j * l:(2 * j + 1) * l], 1).astype(np.uint32)
        b = np.append(mi[(2 * j + 1) * l:(2 * j + 2) * l], 1).astype(np.uint32)
        ok = ok and np.array_equal(cm.fftmul_uni(a, b, P)[:2 * l], mo[2 * j * l:2 * (j + 1) * l])
    gbs, frac = rate(16 * npairs * l, ms)
    out["subproduct_level_l512_x32768"] = {"ms": round(ms, 5), "pairs_per_s": round(npairs / (ms / 1000), 1),
                                          "gbs_strict": gbs, "frac_strict": frac,
                                          "equals_single_products": bool(ok)}
    del dI, dO
    return out


def batched_c4(cm, torch, dev, stream):
    """4096 pairs, degrees log-uniform in [32, 65536]: one batched call vs one call per pair."""
    from cumodp_b200.workloads import SplitMix64, seed_for
    r = SplitMix64(seed_for(3))
    cnt = 4096
    da = r.log_uniform_int(cnt, 32, 65536).astype(np.int32)
    db = r.log_uniform_int(cnt, 32, 65536).astype(np.int32)
    f_off = np.zeros(cnt, np.int64)
    g_off = np.zeros(cnt, np.int64)
    h_off = np.zeros(cnt, np.int64)
    f_off[1:] = np.cumsum(da.astype(np.int64) + 1)[:-1]
    g_off[1:] = np.cumsum(db.astype(np.int64) + 1)[:-1]
    h_off[1:] = np.cumsum(da.astype(np.int64) + db + 1)[:-1]
    nf, ng, nh = int((da + 1).sum()), int((db + 1).sum()), int((da.astype(np.int64) + db + 1).sum())
    F = torch.from_numpy(r.residues(nf, P).view(np.int32)).to(dev)
    G = torch.from_numpy(r.residues(ng, P).view(np.int32)).to(dev)
    H = torch.zeros(nh, dtype=torch.int32, device=dev)
    H1 = torch.zeros(nh, dtype=torch.int32, device=dev)
    sp = stream.cuda_stream
    for _ in range(2):
        cm.fftmul_batch_dev(da, f_off, F.data_ptr(), db, g_off, G.data_ptr(), h_off, H.data_ptr(), P, sp)
    torch.cuda.synchronize()
    reps = 5
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        cm.fftmul_batch_dev(da, f_off, F.data_ptr(), db, g_off, G.data_ptr(), h_off, H.data_ptr(), P, sp)
    e1.record(stream)
    torch.cuda.synchronize()
    t_batch = e0.elapsed_time(e1) / reps
    # one call per pair (the plain path), same stream, device pointers
    fp, gp, hp = F.data_ptr(), G.data_ptr(), H1.data_ptr()
    for i in range(cnt):  # warm
        cm.fftmul_uni_dev(hp + 4 * int(h_off[i]), int(da[i] + db[i] + 1), fp + 4 * int(f_off[i]), int(da[i]),
                          gp + 4 * int(g_off[i]), int(db[i]), P, sp)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    for i in range(cnt):
        cm.fftmul_uni_dev(hp + 4 * int(h_off[i]), int(da[i] + db[i] + 1), fp + 4 * int(f_off[i]), int(da[i]),
                          gp + 4 * int(g_off[i]), int(db[i]), P, sp)
    e1.record(stream)
    torch.cuda.synchronize()
    t_single_wall = (time.perf_counter() - t0) * 1000
    t_single = e0.elapsed_time(e1)
    same = bool(torch.equal(H, H1))
    # the same one-call-per-pair path from a compiled C loop (no interpreter between the calls)
    import ctypes as C
    pc = C.CDLL(os.path.join(ROOT, "cumodp_b200", "libcumodp_percall.so"))
    pc.percall_fftmul.restype = C.c_int
    pc.percall_fftmul.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    H1.zero_()

    def c_loop():
        rc = pc.percall_fftmul(cnt, da.ctypes.data, f_off.ctypes.data, fp, db.ctypes.data, g_off.ctypes.data, gp,
                               h_off.ctypes.data, hp, P, C.c_void_p(sp))
        assert rc == 0, rc
    c_loop()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    c_loop()
    e1.record(stream)
    torch.cuda.synchronize()
    t_c_wall = (time.perf_counter() - t0) * 1000
    t_c = e0.elapsed_time(e1)
    same_c = bool(torch.equal(H, H1))
    # algorithmic bytes of the batch: per pair, its operands and result for a transform of n <= 2^14
    # (one pass), else the pass-aware 24 n ceil(log2 n / 14) of three transforms
    alg = 0
    for a, b in zip(da.tolist(), db.tolist()):
        logn = max(0, int(a + b).bit_length())  # n = 2^ceil(log2(a + b + 1))
        alg += 4 * (a + 1) + 4 * (b + 1) + 4 * (a + b + 1) if logn <= 14 else 24 * (1 << logn) * -(-logn // 14)
    peak, kind = peaks()
    gbs = alg / (t_batch * 1e-3) / 1e9
    return {"pairs": cnt, "ms_batched": round(t_batch, 4), "products_per_s_batched": round(cnt / (t_batch / 1000), 1),
            "roofline": {"bound": "hbm", "alg_bytes": alg, "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / peak, 4), "peak_kind": kind,
                         "how": "per pair 4(da+1)+4(db+1)+4(da+db+1) bytes when n <= 2^14, else "
                                "24 n ceil(log2 n / 14), over the batched call's CUDA-event time"},
            "ms_one_call_per_pair": round(t_single, 4), "ms_one_call_per_pair_wall": round(t_single_wall, 4),
            "speedup_vs_one_call": round(t_single / t_batch, 2), "batched_equals_single": same,
            "one_call_per_pair_c_loop": {"ms": round(t_c, 4), "ms_wall": round(t_c_wall, 4),
                                         "us_per_call": round(1000 * t_c / cnt, 2),
                                         "speedup_batched_vs_c_loop": round(t_c / t_batch, 2),
                                         "equals_batched": same_c,
                                         "how": "cumodp_fftmul_uni_dev once per pair from a compiled C loop "
                                                "(cumodp_b200/bench/percall.c), device pointers, one stream, "
                                                "CUDA events"}}


def c3_exact(cm, torch, dev, stream):
    """Config 3: exact products of int64 polynomials, |c| <= 10^10, degrees 8191 and 16383.

    Device latency through cumodp_twoconv_mul_i64_dev (device buffers) and
    through the host entry cumodp_twoconv_mul_i64; checked by the identity
    c(1) = a(1) b(1) on Python ints (size-independent).
    """
    import ctypes as C
    from cumodp_b200.workloads import SplitMix64, seed_for
    r = SplitMix64(seed_for(2))
    out = {}
    for d in (8191, 16383):
        a, b = r.int64_in(d + 1, 10**10), r.int64_in(d + 1, 10**10)
        bw = cm.twoconv_bit_width(a, b)
        dA = torch.from_numpy(a).to(dev)
        dB = torch.from_numpy(b).to(dev)
        dC = torch.empty(2 * (2 * d + 1), dtype=torch.int64, device=dev)
        sp = stream.cuda_stream
        f = cm.lib().cumodp_twoconv_mul_i64_dev

        def run():
            rc = f(d + 1, dA.data_ptr(), d + 1, dB.data_ptr(), dC.data_ptr(), bw, 0, C.c_void_p(sp))
            assert rc == 0, rc
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record(stream)
        for _ in range(reps):
            run()
        e1.record(stream)
        torch.cuda.synchronize()
        dev_ms = e0.elapsed_time(e1) / reps
        # the C host entry alone (raw 128-bit words: no Python int per coefficient)
        for _ in range(3):
            cm.twoconv_mul(a, b, raw=True)
        t0 = time.perf_counter()
        for _ in range(20):
            cw = cm.twoconv_mul(a, b, raw=True)
        host_ms = (time.perf_counter() - t0) * 1000 / 20
        t0 = time.perf_counter()
        c = cm.int128_words_to_ints(cw)
        conv_ms = (time.perf_counter() - t0) * 1000
        ok = sum(c) == sum(int(x) for x in a) * sum(int(x) for x in b)
        K, M, npr = cm.twoconv_plan(bw, bw, d + 1, d + 1)
        out[f"deg_{d}"] = {"device_ms": round(dev_ms, 4), "host_entry_ms": round(host_ms, 3),
                           "host_entry_api": "cumodp_twoconv_mul_i64 (host int64 arrays in, 128-bit words out, "
                                             "pinned staging inside)",
                           "python_int_conversion_ms": round(conv_ms, 3),
                           "products_per_s_device": round(1000 / dev_ms, 1), "plan": {"K": K, "M": M, "primes": npr},
                           "sum_identity": bool(ok)}
    return out


def big_coefficients(cm, torch, dev, stream):
    """Big-coefficient exact product at the shape of the reference's benchmark/n1024.test:
    1024 x 1024 coefficients of 1024 bits (signed here), device latency and host entry."""
    import ctypes as C
    from cumodp_b200.workloads import SplitMix64, seed_for
    r = SplitMix64(seed_for(5))
    n, bits, words = 1024, 1024, 17

    def ints(k):
        raw = r.next_u64(k * 16).reshape(k, 16)
        vals = []
        for row in raw:
            v = 0
            for w in row[::-1]:
                v = (v << 64) | int(w)
            vals.append(-v if int(row[0]) & 1 else v)
        return vals
    a, b = ints(n), ints(n)
    wa, wb = cm.ints_to_words(a, words), cm.ints_to_words(b, words)
    bw = bits
    ow = int(cm.lib().cumodp_twoconv_big_out_words(n, n, bw))
    dA = torch.from_numpy(wa.view(np.int64)).to(dev)
    dB = torch.from_numpy(wb.view(np.int64)).to(dev)
    dC = torch.empty((2 * n - 1) * ow, dtype=torch.int64, device=dev)
    f = cm.lib().cumodp_twoconv_mul_big_dev
    sp = stream.cuda_stream

    def run():
        rc = f(n, dA.data_ptr(), n, dB.data_ptr(), words, dC.data_ptr(), ow, bw, C.c_void_p(sp))
        assert rc == 0, rc
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 20
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    torch.cuda.synchronize()
    dev_ms = e0.elapsed_time(e1) / reps
    t0 = time.perf_counter()
    c = cm.twoconv_mul_big(a, b, in_words=words)
    host_ms = (time.perf_counter() - t0) * 1000
    ok = sum(c) == sum(a) * sum(b)
    K, M, npr, lg = cm.twoconv_big_plan(bw, n, n)
    return {"device_ms": round(dev_ms, 4), "host_entry_ms_incl_python_conversion": round(host_ms, 2),
            "plan": {"K": K, "M": M, "primes": npr, "log2_transform": lg}, "sum_identity": bool(ok)}


def c1_latency(cm, torch, dev, stream):
    """Config 1: one 4095 x 4095 product mod 469762049 (transform 8192): latency and batched copies."""
    from cumodp_b200.workloads import SplitMix64, seed_for
    r = SplitMix64(seed_for(0))
    a, b = r.residues(4096, P), r.residues(4096, P)
    dA = torch.from_numpy(a.view(np.int32)).to(dev)
    dB = torch.from_numpy(b.view(np.int32)).to(dev)
    dH = torch.empty(8191, dtype=torch.int32, device=dev)
    sp = stream.cuda_stream
    for _ in range(5):
        cm.fftmul_uni_dev(dH.data_ptr(), 8191, dA.data_ptr(), 4095, dB.data_ptr(), 4095, P, sp)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 200
    e0.record(stream)
    for _ in range(reps):
        cm.fftmul_uni_dev(dH.data_ptr(), 8191, dA.data_ptr(), 4095, dB.data_ptr(), 4095, P, sp)
    e1.record(stream)
    torch.cuda.synchronize()
    dev_us = e0.elapsed_time(e1) * 1000 / reps
    # host entry point, pageable numpy buffers, one product per call
    for _ in range(5):
        cm.fftmul_uni(a, b, P)
    t0 = time.perf_counter()
    for _ in range(reps):
        h = cm.fftmul_uni(a, b, P)
    host_us = (time.perf_counter() - t0) * 1e6 / reps
    ok = product_check(a, b, h)
    # R = 4096 independent copies in one batched call (device buffers)
    R = 4096
    F = dA.repeat(R)
    G = dB.repeat(R)
    H = torch.empty(R * 8191, dtype=torch.int32, device=dev)
    df = np.full(R, 4095, np.int32)
    offs = np.arange(R, dtype=np.int64) * 4096
    hoff = np.arange(R, dtype=np.int64) * 8191
    for _ in range(3):
        cm.fftmul_batch_dev(df, offs, F.data_ptr(), df, offs, G.data_ptr(), hoff, H.data_ptr(), P, sp)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(5):
        cm.fftmul_batch_dev(df, offs, F.data_ptr(), df, offs, G.data_ptr(), hoff, H.data_ptr(), P, sp)
    e1.record(stream)
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1) / 5
    same = bool(torch.equal(H[:8191], dH))
    return {"device_us_per_call": round(dev_us, 2), "host_us_per_call": round(host_us, 2),
            "eval_point_identity": ok, "batched_copies": R, "batched_ms": round(batch_ms, 4),
            "batched_products_per_s": round(R / (batch_ms / 1000), 1),
            "batched_mulmods_per_s": round(R * 167936 / (batch_ms / 1000), 1), "batched_equals_single": same}


def _page_aligned(values: np.ndarray) -> np.ndarray:
    """A copy of `values` in page-aligned memory (what page-locking registers)."""
    buf = np.empty(values.nbytes + 4096, np.uint8)
    off = (-buf.ctypes.data) % 4096
    out = buf[off:off + values.nbytes].view(values.dtype)
    out[:] = values
    return out


def serving_c5(cm, rates=(1000, 3000, 10000, 30000, 100000), max_requests=100000, max_seconds=10.0, threads=4):
    """Config 5: Poisson arrivals of mixed requests into the continuous-batching server.

    Degrees log-uniform in [2^5, 2^20]; prime uniform over {469762049,
    754974721, 962592769}; 20% exact int64 products (|c| <= 10^10, degrees
    log-uniform in [2^5, 2^20] too).  The trace is replayed open-loop by the
    library's native replay threads (cumodp_server_replay): request i is
    submitted at its arrival time whatever happened before, and its latency
    runs from the scheduled arrival to the result in a host buffer.  Each
    rate replays min(max_requests, rate * max_seconds) requests.  The operand
    pools are registered with the server (cumodp_server_register), so
    operands go to the device straight from them, and each result lands in
    the server's pinned slab (the replay gives no output buffer): operands
    and results cross the host link with no host copy.  Requests whose
    product exceeds the prime's 2-adic order (962592769 supports 2^21 points)
    are answered with CUMODP_FFT_SIZE_TOO_LARGE and counted as rejected;
    requests shed by the server's host budget (4 GiB of unfinished operand
    and result bytes) are counted as shed.  `link_ceiling_per_s` is the rate
    the measured host link allows for the trace's mean request (its operand
    bytes at the measured host-to-device bandwidth, its result bytes at the
    device-to-host one, both directions busy at once).
    """
    import torch
    from cumodp_b200.workloads import SplitMix64, seed_for
    primes = (469762049, 754974721, 962592769)
    r = SplitMix64(seed_for(4))
    pool_u = _page_aligned(r.residues((1 << 21) + 2, 469762049))  # operand slices come from these pools
    pool_i = _page_aligned(r.int64_in((1 << 21) + 2, 10**10))
    link = host_link_bound(torch, torch.device("cuda", torch.cuda.current_device()), 64 << 20, 64 << 20)
    link_bps = link["gbs_per_direction"] * 1e9
    out = {}
    with cm.Server(max_batch=256, batch_window_us=50, lanes=8, host_budget=4 << 30) as srv:
        srv.register(pool_u)
        srv.register(pool_i)
        # warm-up: tables for every prime and size class, lane buffers
        warm = [(pool_u[:(1 << k) + 1], pool_u[:(1 << k) + 1], p) for p in primes for k in range(4, 21)]
        warm += [(pool_i[:(1 << k) + 1], pool_i[:(1 << k) + 1], None) for k in range(4, 21)]
        srv.replay(np.zeros(len(warm)), warm, threads=threads)
        for rate in rates:
            n = int(min(max_requests, rate * max_seconds))
            arrival = np.cumsum(-np.log(1.0 - r.uniform01(n)) / rate) * 1e6
            da = r.log_uniform_int(n, 32, 1 << 20)
            db = r.log_uniform_int(n, 32, 1 << 20)
            kind = r.uniform01(n)
            pidx = (r.next_u64(n) % np.uint64(3)).astype(int)
            offs = (r.next_u64(2 * n) % np.uint64(1 << 20)).astype(np.int64)
            reqs = []
            for i in range(n):
                if kind[i] < 0.2:
                    reqs.append((pool_i[offs[i]:offs[i] + int(da[i]) + 1],
                                 pool_i[offs[n + i]:offs[n + i] + int(db[i]) + 1], None))
                else:
                    reqs.append((pool_u[offs[i]:offs[i] + int(da[i]) + 1],
                                 pool_u[offs[n + i]:offs[n + i] + int(db[i]) + 1], primes[pidx[i]]))
            srv.reset_stats()
            st, lat, span_us = srv.replay(arrival, reqs, threads=threads)
            ok = st == 0
            lat_ok = np.sort(lat[ok]) / 1000.0
            pct = (lambda q: round(float(lat_ok[min(len(lat_ok) - 1, int(q * len(lat_ok)))]), 3)) \
                if len(lat_ok) else (lambda q: None)
            in_bytes = sum(a.nbytes + b.nbytes for a, b, _ in reqs)
            res_bytes = sum((len(a) + len(b) - 1) * (16 if p is None else 4) for a, b, p in reqs)
            ceiling = n / max(in_bytes / link_bps, res_bytes / link_bps)
            done_in = sum(reqs[i][0].nbytes + reqs[i][1].nbytes for i in np.flatnonzero(ok))
            done_res = sum((len(reqs[i][0]) + len(reqs[i][1]) - 1) * (16 if reqs[i][2] is None else 4)
                           for i in np.flatnonzero(ok))
            out[str(rate)] = {"requests": n, "completed": int(ok.sum()),
                              "rejected_size": int((st == cm.FFT_SIZE_TOO_LARGE).sum()),
                              "shed": int((st == cm.OUT_OF_MEMORY).sum()),
                              "failed_other": int((~ok & (st != cm.FFT_SIZE_TOO_LARGE) &
                                                   (st != cm.OUT_OF_MEMORY)).sum()),
                              "p50_ms": pct(0.5), "p99_ms": pct(0.99), "max_ms": pct(1.0),
                              "products_per_s": round(ok.sum() / (span_us * 1e-6), 1),
                              "offered_per_s": round(n / (arrival[-1] * 1e-6), 1),
                              "operand_gb_per_s": round(done_in / (span_us * 1e3), 2),
                              "result_gb_per_s": round(done_res / (span_us * 1e3), 2),
                              "link_gbs_per_direction": link["gbs_per_direction"],
                              "link_ceiling_per_s": round(ceiling, 1),
                              "batches": srv.stats()["batches"], "replay_threads": threads,
                              "copies": "registered operand pools, results in pinned slabs: no host copy"}
    return out


def reference_gpu(cm, torch, dev, stream, extras, ours):
    """The reference's own GPU path on the same GPU in the same run (src/stockham.cu and src/fft_aux.cu,
    compiled from the reference sources for sm_100a by oracle/Makefile into oracle/_ref/libcumodp_refgpu.so and
    run as shipped: radix-2 Stockham, one launch and one device sync per step, per-call allocation).

    C1 and C2 products device-resident (stockham_poly_mul_dev, CUDA events on the default stream it uses) and
    host to host (stockham_poly_mul_host, the body of cumodp_fftmul_uni; both sides on pageable numpy arrays);
    the 2^24 transform device-resident
    (stockham_dev) and host to host (stockham_host, the body of cumodp_fft_uni); C4 as a loop of host-to-host
    products, pairs whose transform is below 256 (refused by the reference) counted apart.  Each figure sits
    beside this library's figure for the same work and their ratio (reference time / ours)."""
    import oracle
    from cumodp_b200.workloads import SplitMix64, seed_for
    if not oracle.ref_gpu_available():
        return {"unavailable": "reference GPU build absent (make -C oracle ref_gpu needs the reference sources)"}
    out = {}
    sp = stream.cuda_stream

    def host_ms(fn, reps):
        with oracle.quiet_stdout():
            fn()
            t0 = time.perf_counter()
            for _ in range(reps):
                fn()
            return (time.perf_counter() - t0) * 1000 / reps

    # C1: 4095 x 4095, transform 8192
    r = SplitMix64(seed_for(0))
    a, b = r.residues(4096, P), r.residues(4096, P)
    F = torch.zeros(8192, dtype=torch.int32, device=dev)
    G = torch.zeros(8192, dtype=torch.int32, device=dev)
    F[:4096] = torch.from_numpy(a.view(np.int32)).to(dev)
    G[:4096] = torch.from_numpy(b.view(np.int32)).to(dev)
    torch.cuda.synchronize()
    ref_dev = oracle.ref_gpu_time_polymul_dev(F.data_ptr(), G.data_ptr(), 13, P, 50)
    ref_host = host_ms(lambda: oracle.ref_gpu_polymul(a, b, P), 20)
    c1 = extras.get("c1_4095x4095") or {}
    ours_dev = c1.get("device_us_per_call", float("nan")) / 1000
    ours_host = c1.get("host_us_per_call", float("nan")) / 1000
    out["c1_product_4095x4095"] = {"reference_device_ms": round(ref_dev, 4), "ours_device_ms": round(ours_dev, 4),
                                   "ratio_device": round(ref_dev / ours_dev, 1),
                                   "reference_host_ms": round(ref_host, 4), "ours_host_ms": round(ours_host, 4),
                                   "ratio_host": round(ref_host / ours_host, 1)}
    # C2: the 2^24 product and transform
    n = 1 << LOGN
    r = SplitMix64(0xC0DA0001)
    a, b = r.residues(DEG + 1, P), r.residues(DEG + 1, P)
    F = torch.zeros(n, dtype=torch.int32, device=dev)
    G = torch.zeros(n, dtype=torch.int32, device=dev)
    F[:DEG + 1] = torch.from_numpy(a.view(np.int32)).to(dev)
    G[:DEG + 1] = torch.from_numpy(b.view(np.int32)).to(dev)
    torch.cuda.synchronize()
    ref_dev = oracle.ref_gpu_time_polymul_dev(F.data_ptr(), G.data_ptr(), LOGN, P, 3)
    ref_host = host_ms(lambda: oracle.ref_gpu_polymul(a, b, P), 2)
    out["c2_product_2^24"] = {"reference_device_ms": round(ref_dev, 3), "ours_device_ms": ours["product_ms"],
                              "ratio_device": round(ref_dev / ours["product_ms"], 1),
                              "reference_host_ms": round(ref_host, 2), "ours_host_ms": ours["host_product_ms"],
                              "ratio_host": round(ref_host / ours["host_product_ms"], 1)}
    w = oracle.primitive_root(LOGN, P)
    ref_dev = oracle.ref_gpu_time_fft_dev(F.data_ptr(), LOGN, w, P, 3)  # F: any 2^24 device words
    x = SplitMix64(0xC0DA0002).residues(n, P)
    ref_host = host_ms(lambda: oracle.ref_gpu_fft(x, w, P), 2)
    cm.fft_uni(x, w, P)
    t0 = time.perf_counter()
    for _ in range(2):
        cm.fft_uni(x, w, P)
    our_host = (time.perf_counter() - t0) * 1000 / 2
    ntt = extras.get("ntt_2_24") or {}
    our_dev = ntt.get("ms_per_transform", float("nan"))
    out["c2_transform_2^24"] = {"reference_device_ms": round(ref_dev, 3), "ours_device_ms": our_dev,
                                "ratio_device": round(ref_dev / our_dev, 1),
                                "reference_host_ms": round(ref_host, 2), "ours_host_ms": round(our_host, 2),
                                "ratio_host": round(ref_host / our_host, 1)}
    # C4: 4096 pairs (the batched leg's seed), one host-to-host reference call per pair
    r = SplitMix64(seed_for(3))
    cnt = 4096
    da = r.log_uniform_int(cnt, 32, 65536)
    db = r.log_uniform_int(cnt, 32, 65536)
    fa = r.residues(int((da + 1).sum()), P)
    gb = r.residues(int((db + 1).sum()), P)
    fo = np.concatenate([[0], np.cumsum(da + 1)])
    go = np.concatenate([[0], np.cumsum(db + 1)])
    pairs = [(fa[fo[i]:fo[i + 1]], gb[go[i]:go[i + 1]]) for i in range(cnt)]
    small = [i for i in range(cnt) if (1 << int(da[i] + db[i]).bit_length()) < 256]
    big = [i for i in range(cnt) if i not in set(small)]
    with oracle.quiet_stdout():
        oracle.ref_gpu_polymul(*pairs[big[0]], P)
        t0 = time.perf_counter()
        for i in big:
            oracle.ref_gpu_polymul(*pairs[i], P)
        ref_loop = (time.perf_counter() - t0) * 1000
    cm.fftmul_batch(pairs, P)
    t0 = time.perf_counter()
    cm.fftmul_batch(pairs, P)
    our_batch_host = (time.perf_counter() - t0) * 1000
    c4 = extras.get("batched_c4") or {}
    out["c4_4096_pairs"] = {"reference_loop_ms_host_to_host": round(ref_loop, 1),
                            "reference_pairs_timed": len(big), "pairs_refused_by_reference_transform_below_256": len(small),
                            "ours_batched_host_to_host_ms": round(our_batch_host, 2),
                            "ratio_host": round(ref_loop / our_batch_host, 1),
                            "ours_batched_device_ms": c4.get("ms_batched"),
                            "ours_c_loop_device_ms": (c4.get("one_call_per_pair_c_loop") or {}).get("ms"),
                            "note": "ours host-to-host covers all 4096 pairs (the refused ones included)"}
    return out


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline():
    """modpn's own CPU product (the reference's CPU path) on this host: one product on one thread, and one
    product per thread on every usable thread (capped by memory and at 64)."""
    import oracle
    if not oracle.ref_available():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "unavailable"}
    one = modpn_sample(1, 1, 0xC0DA0001)
    threads = ref_threads_bounded()
    secs = modpn_sample(threads, threads, 0xC0DA0001)
    return {"value": round(threads / secs, 4), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{threads} products of degree 2^23-1 mod 469762049, one per host thread "
                      f"({secs:.1f} s wall)",
            "single_thread": {"value": round(1 / one, 4), "unit": UNIT, "cores": 1,
                              "sample": f"1 product of degree 2^23-1 on one thread ({one:.2f} s)"},
            "host_threads": host_threads(), "nproc": os.cpu_count(), "cpu_model": cpu_model()}


def run_leg(name: str) -> None:
    import torch
    import cumodp_b200 as cm
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    hbm_peak, _ = peaks()
    with torch.cuda.stream(stream):
        fn = {"ntt": lambda: ntt_2_24(cm, torch, dev, stream, hbm_peak),
              "c1": lambda: c1_latency(cm, torch, dev, stream),
              "c3": lambda: c3_exact(cm, torch, dev, stream),
              "c4": lambda: batched_c4(cm, torch, dev, stream),
              "big": lambda: big_coefficients(cm, torch, dev, stream),
              "serving": lambda: serving_c5(cm),
              "refgpu": lambda: refgpu_leg(cm, torch, dev, stream, hbm_peak)}[name]
        print(json.dumps({"leg": name, "result": fn()}))


def refgpu_leg(cm, torch, dev, stream, hbm_peak):
    """reference_gpu on its own: the legs it compares with, then the reference's GPU path."""
    extras = {"ntt_2_24": ntt_2_24(cm, torch, dev, stream, hbm_peak), "c1_4095x4095": c1_latency(cm, torch, dev, stream),
              "batched_c4": batched_c4(cm, torch, dev, stream)}
    ops = gen_operands(0xC0DA0001, 1)
    a, b = ops[0]
    dA = torch.from_numpy(a.view(np.int32)).to(dev)
    dB = torch.from_numpy(b.view(np.int32)).to(dev)
    n = 1 << LOGN
    dH = torch.empty(n - 1, dtype=torch.int32, device=dev)
    prod = lambda: cm.fftmul_uni_dev(dH.data_ptr(), n - 1, dA.data_ptr(), DEG, dB.data_ptr(), DEG, P,
                                     stream.cuda_stream)
    dev_ms = _timed(torch, stream, prod, reps=10, warm=3)
    return reference_gpu(cm, torch, dev, stream, extras, {"product_ms": round(dev_ms, 5),
                                                          "host_product_ms": host_product_ms(cm, a, b)})


def host_product_ms(cm, a, b, reps: int = 3) -> float:
    """cumodp_fftmul_uni on pageable numpy operands (the reference's host entry gets the same kind of arrays)."""
    cm.fftmul_uni(a, b, P)
    t0 = time.perf_counter()
    for _ in range(reps):
        cm.fftmul_uni(a, b, P)
    return round((time.perf_counter() - t0) * 1000 / reps, 3)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only (no e2e extras, transform, batch or CPU legs); for profiling")
    ap.add_argument("--leg", choices=["ntt", "c1", "c3", "c4", "big", "serving", "refgpu"],
                    help="run only this extra leg and print its result (for profiling it alone)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.leg:
        run_leg(args.leg)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                              device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as td
            td.destroy_process_group()


if __name__ == "__main__":
    main()
