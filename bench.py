"""Benchmark of the modular-squaring engine (one JSON line on rank 0).

Workload (default): a batch of 64 Fermat PRP tests of b^(2^16) + 1, b even,
seeded uniform in [10^6, 10^8] (seed 1002), run as Gerbicz-Li blocks of 1000
squarings; one step = one block (1000 squarings of every test + the d(t)
update), replayed from a CUDA graph.  Metric: digit-squarings per second
(sum over tests of 2^n x squarings / time; the Gerbicz-Li products are timed
but not counted).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the reference's own CPU transforms (oracle/_ref, the
reference sources compiled here) on the host cores for the same workload.
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

N_LOG = 16
COUNT = 64
BLOCK = 1000
SEED = 1002
B_LO, B_HI = 10**6, 10**8
METRIC = "digit-squarings/s"
WORKLOAD = "batch of 64 Fermat PRP tests b^(2^16)+1, b even uniform [1e6,1e8] seed 1002, Gerbicz-Li block of 1000 squarings"


def bases(seed: int = SEED, count: int = COUNT):
    rng = np.random.default_rng(seed)
    return (rng.integers(B_LO // 2, B_HI // 2 + 1, size=count) * 2).astype(np.int64).tolist()


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_info():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


# ------------------------------------------------------------------ reference CPU path

def cpu_reference(n: int, test_bases, seconds: float, impl: str = ""):
    """The reference's CPU transform (transform::create_cpu, src/transform.h:122-193,
    built from the reference sources into oracle/_ref) on the host cores.  One test
    per worker thread, several threads per test when there are more cores than
    tests; every worker runs squareDup on its own test for ~`seconds`.
    Returns (digit-squarings/s, cores, sample description, transform type)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gf_oracle as G
    if not G.ref_available():
        raise RuntimeError("oracle/_ref/libgfref.so not built")
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    workers = max(1, min(cores, len(test_bases)))
    tpt = 1 if impl == "i32" else max(1, cores // workers)
    rng = np.random.default_rng(7)
    trs = []
    for i in range(workers):
        b = int(test_bases[i])
        t = G.RefTransform(b, n, num_regs=3, impl=impl, threads=tpt)
        t.setInt(rng.integers(-(b // 2), b // 2 + 1, size=1 << n).astype(np.int32))
        trs.append(t)
    # calibrate the per-worker squaring count on one worker alone
    t0 = time.perf_counter()
    trs[0].run_squarings(np.ones(4, np.uint8))
    per = max((time.perf_counter() - t0) / 4, 1e-6)
    sq = max(4, int(seconds / per))
    bits = (np.arange(sq) % 2).astype(np.uint8)
    th = [threading.Thread(target=t.run_squarings, args=(bits,)) for t in trs]
    t0 = time.perf_counter()
    for x in th:
        x.start()
    for x in th:
        x.join()
    dt = time.perf_counter() - t0
    value = workers * (1 << n) * sq / dt
    sample = f"{workers} tests x {sq} squarings at n={n} ({tpt} thread(s) each), {dt:.1f} s"
    return value, workers * tpt, sample, trs[0].ttype


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    bs = bases()
    per_step = 3.0
    vals = []
    for k in range(args.warmup + args.steps):
        v, cores, sample, ttype = cpu_reference(N_LOG, bs, per_step)
        if k >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    ms = COUNT * (1 << N_LOG) * BLOCK / value * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if ttype != "i32" else "u32",
            "data": "synthetic", "config": {"workload": WORKLOAD, "n": N_LOG, "tests": COUNT, "block": BLOCK,
                                            "seed": SEED, "reference_transform": ttype},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm

def plan_geometry(n: int, plan: int):
    """(log2 of the transform length, log2 of the column length) of a plan:
    packed plans (200 + lr, 300 + lr2) transform N/2 points; six-step plans
    (100 + lr2, 300 + lr2) have columns of 2^(4 + lr2)."""
    if plan > 300:
        return n - 1, 4 + plan - 300
    if plan > 200:
        return n - 1, plan - 200
    if plan > 100:
        return n, 4 + plan - 100
    return n, plan


def algorithmic(kind: int, widths: np.ndarray, n: int, lr: int):
    """Algorithmic DRAM bytes and radix-2 butterflies of one launch of kernel
    kind `kind` (see Batch.time_kernels) over all tests of the batch.  n and
    lr are those of the transform (n - 1 for packed digits, whose N/2
    coefficients each carry two digits)."""
    N = 1 << n
    W = widths.astype(np.float64)
    lc = n - lr
    dig = 4 * N * (2 if int(W[0]) == 4 else 1)      # digit bytes: two digits per packed coefficient
    if kind == 1:   # column forward: read digits, write W planes; lr stages
        return float(np.sum(dig + 4 * W * N)), float(np.sum(W * (N / 2) * lr))
    if kind == 2:   # rows: read + write W planes; 2 lc stages + pointwise
        return float(np.sum(8 * W * N)), float(np.sum(W * (N / 2) * 2 * lc + W * N))
    if kind == 3:   # column inverse + CRT + carry: read W planes, write digits and carries
        return float(np.sum(4 * W * N + dig + 8 * (dig // 4) / 16)), float(np.sum(W * (N / 2) * lr))
    if kind == 4:   # carry fix-up: read carries
        return float(np.sum(8 * N / 16 + 0 * W)), 0.0
    # single-CTA squaring: digits in and out; the whole transform in shared memory
    return float(np.sum(8 * N + 0 * W)), float(np.sum(W * (N / 2) * 2 * n + W * N))


def run_ours(args):
    import torch
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from genefer22_b200 import Batch, Transform, _lib
    from genefer22_b200 import genefer as gf

    L = _lib.lib()
    from genefer22_b200.autotune import Autotuner
    bs = bases(SEED + rank)
    bt = Batch(bs, N_LOG, num_regs=3, device=local)
    tuned = Autotuner(squarings=16, replays=3).tune(bt)      # plan per size class, as production batches run
    widths = bt.widths()
    runner = gf.BatchPRP(bt, B=BLOCK)
    runner.load()
    first = runner.schedule()[0]
    bt.square_exp(first)          # align to the Gerbicz-Li block boundary
    bt.gl_step()
    g = runner.block_graph()
    stream = torch.cuda.ExternalStream(bt.stream, device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(args.warmup):
        g.launch()
    bt.sync()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = L.gfc_launch_count()
    with Clocks(local) as ck:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()     # L2 flush between timed steps (outside the events)
            ev[k][0].record(stream)
            g.launch()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    launches = int(L.gfc_launch_count() - l0)
    if dist is not None:
        dist.barrier()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)
    if dist is not None:
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    digits_per_step = world * COUNT * (1 << N_LOG) * BLOCK
    value = digits_per_step * args.steps / (total_ms * 1e-3)

    # end to end through the public API: host digits in (pinned), one block, host digits out
    pin0 = torch.empty((COUNT, 1 << N_LOG), dtype=torch.int32, pin_memory=True).numpy()
    pin1 = torch.empty((COUNT, 1 << N_LOG), dtype=torch.int32, pin_memory=True).numpy()
    bt.get_all(0, out=pin0)
    bt.get_all(1, out=pin1)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        bt.put_all(pin0, 0)
        bt.put_all(pin1, 1)
        g.launch()
        bt.get_all(0, out=pin0)
        bt.get_all(1, out=pin1)
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = digits_per_step * args.steps / e2e_s
    io_bytes = 2 * COUNT * (1 << N_LOG) * 4

    if rank != 0:
        if dist is not None:
            del g
            dist.destroy_process_group()
        return

    # per-kernel durations (CUDA events on the batch's stream) -> roofline of the dominant kernel
    lr = bt.plan()
    n_t, lr_t = plan_geometry(N_LOG, lr)
    bt.time_kernels(2)                 # first launches of each kernel kind load it
    kms = bt.time_kernels(5)
    dom = int(np.argmax(kms[:4]))      # the stand-alone fix-up is not part of a graph step
    names = ["k_small", "k_col_fwd", "k_row", "k_col_inv", "k_fixup"]
    abytes, abfly = algorithmic(dom, widths, n_t, lr_t)
    hbm, hbm_kind = peaks()
    achieved = abytes / (kms[dom] * 1e-3) / 1e9
    probe = (ctypes.c_double * 4)()
    L.gfc_probe_int_throughput(local, probe)
    frac_w3 = float(np.mean(widths >= 3))       # 31-bit primes (3 or 4 of them) vs 32-bit (2)
    bfly_peak = frac_w3 * probe[3] + (1 - frac_w3) * probe[2]
    traffic = None
    tj = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tj):
        with open(tj) as f:
            traffic = json.load(f).get(f"{names[dom]}_lr{lr}_n{N_LOG}_x{COUNT}")

    # plain path: one test, one squareDup call per squaring from the host
    tr = Transform(int(bs[0]), N_LOG)
    tr.set(3)
    for _ in range(20):
        tr.squareDup(False)
    tr.sync()
    kp = 300
    t0 = time.perf_counter()
    for i in range(kp):
        tr.squareDup(i % 2 == 1)
    tr.sync()
    plain = (1 << N_LOG) * kp / (time.perf_counter() - t0)

    extras = north_star(args, bs) if (world == 1 and not args.no_extras) else None

    cpu = None
    if world == 1 and not args.no_cpu:
        try:
            v, cores, sample, ttype = cpu_reference(N_LOG, bs, args.cpu_seconds)
            cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": "reference",
                   "sample": f"reference {ttype} transform: {sample}"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": METRIC, "cores": None, "kind": "reference", "sample": f"unavailable: {e}"}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": N_LOG, "tests_per_gpu": COUNT, "block": BLOCK, "seed": SEED,
                   "plan": lr, "plan_us_per_squaring": {str(k): round(v, 1) for k, v in tuned.us.items()},
                   "rns_widths": {str(w): int(np.sum(widths == w)) for w in sorted(set(widths.tolist()))},
                   "l2": "256 MB buffer written between timed steps", "graph": "one CUDA graph per block"},
        "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": hbm_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": abytes, "launch_ms": float(kms[dom]),
                     "int_pipe": {"achieved_bfly_per_s": abfly / (kms[dom] * 1e-3), "peak_bfly_per_s": bfly_peak,
                                  "frac": abfly / (kms[dom] * 1e-3) / bfly_peak,
                                  "peak_kind": "measured (gfc_probe_int_throughput)"},
                     "kernel_ms": {nm: float(x) for nm, x in zip(names, kms)}},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
        "gpu_launches": launches,
        "clocks": ck.summary(),
        "plain": {"value": plain, "unit": METRIC, "what": "one test, one gfc_square_dup call per squaring"},
        "batched_over_plain": value / world / plain,
    }
    if extras is not None:
        line["north_star"] = extras
    print(json.dumps(line), flush=True)
    if dist is not None:
        del g
        dist.destroy_process_group()


# ------------------------------------------------------------------ other workloads (not the default line)

def _device_time(streams, launch_all, torch):
    """Device milliseconds of launch_all() whose work spans several streams:
    every stream waits for a start event on a common stream, which then
    waits for every stream before the end event."""
    s0 = torch.cuda.current_stream()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(s0)
    for s in streams:
        s.wait_event(start)
    launch_all()
    for s in streams:
        e = torch.cuda.Event()
        e.record(s)
        s0.wait_event(e)
    end.record(s0)
    end.synchronize()
    return start.elapsed_time(end)


def _plain_rate(b: int, n: int, squarings: int) -> float:
    """One test, one gfc_square_dup call per squaring (digit-squarings/s)."""
    from genefer22_b200 import Transform
    tr = Transform(int(b), n)
    tr.set(3)
    for _ in range(5):
        tr.squareDup(False)
    tr.sync()
    t0 = time.perf_counter()
    for i in range(squarings):
        tr.squareDup(i % 2 == 1)
    tr.sync()
    return (1 << n) * squarings / (time.perf_counter() - t0)


def run_uneven(args):
    """256 tests, n from {12:40%,...,18:2%}, b log-uniform [1024, 2e9) clipped
    to the per-n limits (seed 1004), each running `steps` Gerbicz-Li blocks of
    1000 squarings, all submitted at once to the native loop: one pool per size
    class with a slot per test, the classes' graphs in flight together."""
    import torch
    from genefer22_b200.autotune import Autotuner
    from genefer22_b200.genefer import Job
    from genefer22_b200.mixed import MixedBatch, uneven_tests
    torch.cuda.set_device(0)
    tests = uneven_tests(256, seed=1004)
    jobs = [Job.prefix(b, n, args.steps * BLOCK) for b, n in tests]
    mb = MixedBatch(jobs, B=BLOCK, tuner=Autotuner())
    with Clocks(0) as ck:
        res = mb.run(validate=True, warmup=True)       # a first wave opens the pools
    st = mb.stats
    per_class = {}
    plain_s = 0.0
    for n, c in sorted(st.per_class.items()):
        b0 = next(b for b, m in tests if m == n)
        pr = _plain_rate(b0, n, 200 if n <= 16 else 60)
        plain_s += c["digit_squarings"] / pr
        per_class[n] = {"tests": c["tests"], "plan": c["plan"], "plain_digit_sq_per_s": pr}
    plain = st.digit_squarings / plain_s
    line = {"metric": METRIC, "value": st.rate, "unit": METRIC, "n_gpus": 1, "steps": args.steps, "warmup": 1,
            "ms_per_step": st.seconds / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "uneven batch of 256 tests, n 12..18 (40/20/15/10/8/5/2 %), b log-uniform "
                                   "[1024,2e9) clipped per n, seed 1004, Gerbicz-Li block of 1000 squarings, "
                                   "native loop (one pool per size class)",
                       "classes": per_class,
                       "timing": "host clock, submission of the second wave (pools opened by a first wave of one "
                                 "block per test) to the last residue read back"},
            "gl_failures": sum(1 for r in res if not r.gl_ok),
            "plain": {"value": plain, "what": "each test alone, one gfc_square_dup call per squaring"},
            "mixed_over_plain": st.rate / plain, "clocks": ck.summary()}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Poisson arrivals of tests with n uniform in 15..22 and b even uniform up
    to the per-n limit, plus one n=23 test with b near 2.5e7 (seed 1005), an
    80 GB device-memory budget, Gerbicz-Li block B = 1000.  Each request runs
    the first 2..4 blocks of its test's exponent.  A first pass with every
    request arriving at once measures the service rate; the arrival rate is
    then 80 % of it.  Each pass starts on warm pools: a wave of one
    single-block request per pool shape runs before its clock starts."""
    from genefer22_b200.serve import Server, serve_requests, warmup_requests
    count = args.serve_requests
    sat = serve_requests(count, rate=1e9, blocks=[2, 3, 4], B=BLOCK, seed=1005)
    srv = Server(B=BLOCK, budget_bytes=80 * 10**9)
    with Clocks(0) as ck0:
        srv.run(sat, timeout_s=1800, warmup=warmup_requests(sat, BLOCK))
    cap = srv.stats
    rate = 0.8 * cap.completed / cap.seconds
    reqs = serve_requests(count, rate=rate, blocks=[2, 3, 4], B=BLOCK, seed=1005)
    srv = Server(B=BLOCK, budget_bytes=80 * 10**9)
    with Clocks(0) as ck:
        comps = srv.run(reqs, timeout_s=1800, warmup=warmup_requests(reqs, BLOCK))
    st = srv.stats
    line = {"metric": METRIC, "value": st.rate, "unit": METRIC, "n_gpus": 1, "higher_is_better": True,
            "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"serving: {count} Poisson requests n~U{{15..22}} + one n=23 b~2.5e7, "
                                   "b even uniform up to the per-n limit, seed 1005, 80 GB budget, B=1000, "
                                   "2..4 blocks per request; a warm-up wave of one single-block request per pool "
                                   "shape opens the pools and checkers first (its opens are in open_s_*)",
                       "arrival_rate_per_s": rate, "service_rate_per_s": cap.completed / cap.seconds},
            "p50_time_to_residue_s": st.p50, "p99_time_to_residue_s": st.p99,
            "p50_time_to_validated_s": st.p50_validated, "p99_time_to_validated_s": st.p99_validated,
            "mean_queue_wait_s": st.mean_wait, "completed": st.completed, "gl_failures": st.gl_failures,
            "pools_created": st.pools_created, "blocks_run": st.blocks_run, "peak_budget_bytes": st.peak_bytes,
            "open_s_sum": st.open_s_sum, "open_s_max": st.open_s_max, "dispatcher_step_s_max": st.step_s_max,
            "dispatcher_phase_s_max": dict(zip(("continuations", "pools", "placing", "checks", "closing",
                                                "pool_query", "pool_read", "pool_admit", "pool_launch"),
                                               st.phase_s_max)),
            "saturated_open_s": {"sum": cap.open_s_sum, "max": cap.open_s_max, "step_max": cap.step_s_max,
                                 "phase_max": list(cap.phase_s_max)},
            "saturated": {"value": cap.rate, "seconds": cap.seconds, "p50_s": cap.p50, "p99_s": cap.p99},
            "per_n": {str(k): v for k, v in st.per_n.items()},
            "clocks": ck.summary()}
    print(json.dumps(line), flush=True)


def run_verify(args):
    """One test at n = 20 (b even, seeded uniform in [1e6, 5e7], seed 1003) with a
    Gerbicz-Li check every 2000 squarings (B = 200, spans of 10 blocks) and one
    seeded single-bit fault (seed 1013) that the check detects and rolls back;
    the first `steps` spans of the exponent, timed against the same spans
    without checks (plain blocks of squarings)."""
    import torch
    from genefer22_b200.verify import VerifiedPRP, flip_bit
    torch.cuda.set_device(0)
    rng = np.random.default_rng(1003)
    b = int(rng.integers(5 * 10**5, 25 * 10**6)) * 2
    spans = max(2, args.steps)
    at = int(np.random.default_rng(1013).integers(2000, 4000))
    warm = VerifiedPRP(b, 20, B=200, span=10)
    warm.run(max_spans=1)
    v = VerifiedPRP(b, 20, B=200, span=10)
    t0 = time.perf_counter()
    v.run(fault=flip_bit(1013), fault_at=at, max_spans=spans)
    dt = time.perf_counter() - t0
    useful = spans * 2000 * (1 << 20)
    # the same squarings without checks
    bt = v.batch
    bt.set(3)
    bt.sync()
    t1 = time.perf_counter()
    bt.square(False, spans * 2000)
    bt.sync()
    plain_s = time.perf_counter() - t1
    st = v.stats
    line = {"metric": METRIC, "value": useful / dt, "unit": METRIC, "n_gpus": 1, "higher_is_better": True,
            "dtype": "u32", "data": "synthetic",
            "config": {"workload": "one test n=20, b even uniform [1e6,5e7] seed 1003, Gerbicz-Li check every "
                                   "2000 squarings (B=200, span 10), one seeded single-bit fault (seed 1013)",
                       "b": b, "spans": spans, "fault_at_squaring": at, "plan": bt.plan()},
            "checks": st.checks, "failures": st.failures, "rollbacks": st.rollbacks,
            "squarings_done": st.squarings, "check_squarings": st.check_squarings,
            "unchecked_value": useful / plain_s,
            "overhead_vs_unchecked": dt / plain_s - 1.0}
    print(json.dumps(line), flush=True)


SIZE_TESTS = {12: 256, 13: 128, 14: 64, 15: 64, 16: 64, 17: 16, 18: 8, 19: 4, 20: 2, 21: 2, 22: 1, 23: 1}


def w_min(b: int, n: int) -> int:
    """RNS width the reference GPU transform picks (src/transform_ocl.cpp:35-50,
    32-bit primes 125*2^25+1, 243*2^24+1): the W of the 16 W N roofline unit."""
    return 2 if b * b < ((125 * 2**25 + 1) * (243 * 2**24 + 1) // 2) // (1 << n) else 3


def size_rates(ns, tuner, rng, hbm):
    """Per size n: a batch of SIZE_TESTS[n] tests (as in serving pools, plan
    chosen by the autotuner) run as graph-replayed Gerbicz-Li blocks, against
    the plain path (one test, one gfc_square_dup call per squaring); both as
    digit-squarings/s, with the plain path's fraction of HBM roofline in the
    16 W N bytes-per-squaring unit."""
    import torch
    from genefer22_b200 import Batch
    from genefer22_b200 import genefer as gf
    from genefer22_b200.mixed import b_limit
    out = {}
    for n in ns:
        count = SIZE_TESTS[n]
        lim = min(b_limit(n), 100_000_000 if n >= 16 else 2_000_000_000)
        bs = [int(x) & ~1 for x in rng.integers(1_000_000, lim, size=count)]
        bt = Batch(bs, n, num_regs=3)
        tr = tuner.tune(bt)
        blk = 200 if n <= 18 else 50
        runner = gf.BatchPRP(bt, B=blk, exps=[gf.Job.prefix(b, n, 8 * blk).words_nbits() for b in bs])
        runner.load()
        bt.square_exp(runner.schedule()[0])
        bt.gl_step()
        g = runner.block_graph()
        g.launch()
        s = torch.cuda.ExternalStream(bt.stream)
        ms = min(_device_time([s], g.launch, torch) for _ in range(3))
        batched = count * (1 << n) * blk / (ms * 1e-3)
        plain = _plain_rate(bs[0], n, 100 if n <= 18 else 30)
        W = bt.widths()
        sq_ms = ms / blk
        n_t, _ = plan_geometry(n, tr.lr)                  # packed plans: W = 4 planes of N/2
        alg_bytes = float(np.sum(16 * W * (1 << n_t)))
        plain_us = (1 << n) / plain * 1e6
        out[n] = {"tests": count, "plan_lr": tr.lr, "widths": sorted(set(int(w) for w in W)),
                  "batched": batched, "plain": plain, "batched_over_plain": batched / plain,
                  "us_per_batch_squaring": sq_ms * 1e3, "plain_us_per_squaring": plain_us,
                  "hbm_frac_16WN": alg_bytes / (sq_ms * 1e-3) / 1e9 / hbm,
                  "plain_hbm_frac_16WminN": 16 * w_min(bs[0], n) * (1 << n) / (plain_us * 1e-6) / 1e9 / hbm,
                  "plain_b": bs[0]}
        g.close()
        bt.close()
    return out


def run_sizes(args):
    """Per size n = 12..23: a batch (tests per launch as in serving pools) run as
    graph-replayed blocks vs the plain path (one test, one call per squaring)."""
    import torch
    from genefer22_b200.autotune import Autotuner
    torch.cuda.set_device(0)
    hbm, hbm_kind = peaks()
    out = size_rates(range(12, 24), Autotuner(squarings=4, replays=2), np.random.default_rng(11), hbm)
    print(json.dumps({"metric": METRIC, "unit": METRIC, "workload": "sizes", "hbm_peak_gbs": hbm,
                      "hbm_peak_kind": hbm_kind, "sizes": out}), flush=True)


def north_star(args, bs):
    """The north-star figures beside the default line, a few minutes in all:
    the plain one-test path at n = 20 and 22 against the HBM roofline,
    batched / plain for n = 16..22, a short serving pass (p50 / p99 time to
    residue), and the reference's i32 transform (the same arithmetic, one
    test per host core)."""
    from genefer22_b200.autotune import Autotuner
    from genefer22_b200.serve import Server, serve_requests
    hbm, _ = peaks()
    sz = size_rates(range(16, 23), Autotuner(squarings=4, replays=2), np.random.default_rng(11), hbm)
    out = {"plain": {str(n): {"value": sz[n]["plain"], "us_per_squaring": sz[n]["plain_us_per_squaring"],
                              "hbm_frac_16WminN": sz[n]["plain_hbm_frac_16WminN"], "b": sz[n]["plain_b"]}
                     for n in (20, 22)},
           "batched_over_plain": {str(n): sz[n]["batched_over_plain"] for n in sz},
           "sizes": {str(n): {k: sz[n][k] for k in ("tests", "plan_lr", "batched", "plain", "us_per_batch_squaring")}
                     for n in sz}}
    reqs = serve_requests(args.serve_requests, rate=1e9, blocks=[2], B=BLOCK, seed=1005, ns=tuple(range(15, 21)),
                          big=None)
    srv = Server(B=BLOCK, budget_bytes=80 * 10**9)
    srv.run(reqs, timeout_s=600)
    st = srv.stats
    out["serving"] = {"requests": st.completed, "arrivals": "all at t=0", "p50_time_to_residue_s": st.p50,
                      "p99_time_to_residue_s": st.p99, "p99_time_to_validated_s": st.p99_validated,
                      "value": st.rate, "gl_failures": st.gl_failures,
                      "what": "native loop, n uniform 15..20, b even uniform up to the per-n limit, "
                              "2 blocks of 1000 squarings each, seed 1005"}
    try:
        v, cores, sample, ttype = cpu_reference(N_LOG, bs, min(args.cpu_seconds, 8.0), impl="i32")
        out["cpu_baseline_i32"] = {"value": v, "unit": METRIC, "cores": cores, "kind": "reference",
                                   "sample": f"reference {ttype} transform (same integer arithmetic): {sample}"}
    except Exception as e:          # reported, not fatal
        out["cpu_baseline_i32"] = {"value": None, "sample": f"unavailable: {e}"}
    return out


def spawn_ranks(n: int) -> int:
    """`python bench.py --gpus N` outside torchrun: the same command as N ranks,
    one process per GPU (torch.distributed.run on 127.0.0.1, a free port),
    so that the line reports N GPUs; returns the launcher's exit code."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="batch", choices=["batch", "uneven", "serve", "sizes", "verify"],
                    help="batch: the default line; the others print their own line")
    ap.add_argument("--serve-requests", type=int, default=40)
    ap.add_argument("--no-extras", action="store_true", help="skip the north-star block of the default line")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if (args.gpus > 1) and ("WORLD_SIZE" not in os.environ):
        sys.exit(spawn_ranks(args.gpus))
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "uneven":
        run_uneven(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "sizes":
        run_sizes(args)
    elif args.workload == "verify":
        run_verify(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
