"""Serving: continuous batching on one GPU, run by the native request loop.

The loop is libgfcuda.so's ``gfc_server_*`` (genefer22_b200/csrc/gf_server.cpp):
a dispatcher thread keeps one pool of slots per size n, each pool a batch
whose Gerbicz-Li block (the d(t) update of src/genefer.h:529-535, then B
squarings with each slot's own exponent bits) is one CUDA graph replay.
Between two blocks of a pool, finished tests are read back and waiting tests
of that size enter free slots without any allocation or synchronisation, so
requests that arrive while others run are admitted as slots and memory free
up and the pools' blocks overlap on the device.  Pools open while the
device-memory budget allows and close when idle.  Finished tests get
genefer's Gerbicz-Li check (src/genefer.h:557-615), several of one size at
once, on a checker batch of their own.

This module is the thin Python driver: it submits each request at its
arrival time, collects the completions and summarises them (time to residue
p50 / p99, digit-squarings per second).  Every test's arithmetic reads only
its own slot, base and exponent bits, so a residue is the same whether the
test ran alone or among others; tests check this against ``mixed.run_alone``.

The reference has no counterpart: genefer runs one test per process
(src/genefer.h:1360-1480).
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from ._lib import GFC_OK, SERVER_SIGNATURES, CompletionC, GfcError, ServerConfig, ServerStatsC, lib
from .autotune import packed_ok
from .genefer import Job

NUM_REGS = 3
MAX_N = 23


vp = ctypes.c_void_p


def bind(L):
    """Sets the gfc_server_* signatures on a loaded library (libgfcuda.so, or
    the CPU build of the same loop the host-logic tests use)."""
    for name, (res, args) in {**SERVER_SIGNATURES, "gfc_last_error": (ctypes.c_char_p, [])}.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


_bound = None


def _default_lib():
    global _bound
    if _bound is None:
        _bound = bind(lib())
    return _bound


def slot_bytes(n: int, max_bits: int = 0) -> int:
    """Device bytes of one pool slot of size n (registers, transform planes,
    multiplicand, segment carries, descriptor) plus an exponent of max_bits."""
    return int(_default_lib().gfc_server_slot_bytes(int(n), int(max_bits)))


def pool_slot_bytes(n: int, B: int) -> int:
    """Device bytes of one slot of a serving pool of size n and block length B:
    the slot holds room for the longest exponent of its size (b < 2^31, so
    b^(2^n) has fewer than 31 2^n bits), padded to whole blocks."""
    return slot_bytes(n, (31 << int(n)) + int(B))


def table_bytes(n: int) -> int:
    """Root tables of size n, counted once per size while a pool of it is open."""
    return int(_default_lib().gfc_server_table_bytes(int(n)))


def default_capacity(n: int) -> int:
    """Slots per pool: enough tests per launch to fill the GPU at small n,
    few at large n where one test already fills it."""
    return int(_default_lib().gfc_server_default_capacity(int(n)))


# From this size a pool opened for a base in the packed-digit range takes only
# such bases (the native loop's rule, gfs::Devices::packed_pool_min_n).
PACKED_POOL_MIN_N = 19


def _packed_pool(b: int, n: int) -> bool:
    return (int(n) >= PACKED_POOL_MIN_N) and packed_ok(b, n)


@dataclass
class Request:
    id: int
    job: Job
    arrival: float                  # seconds after the start of the run


@dataclass
class Completion:
    id: int
    b: int
    n: int
    nbits: int
    arrival: float                  # seconds after the start of the run (all times below too)
    admitted: float = 0.0
    residue_at: float = 0.0
    validated_at: Optional[float] = None
    is_prp: bool = False
    res64: int = 0
    old64: int = 0
    gl_ok: Optional[bool] = None
    pool: int = -1
    slot: int = -1
    plan: int = -1
    digits: Optional[np.ndarray] = None

    @property
    def latency(self) -> float:
        """Time to residue: arrival to the residue read back."""
        return self.residue_at - self.arrival


@dataclass
class ServeStats:
    requests: int = 0
    completed: int = 0
    seconds: float = 0.0
    digit_squarings: float = 0.0
    p50: float = 0.0
    p99: float = 0.0
    p50_validated: float = 0.0
    p99_validated: float = 0.0
    mean_wait: float = 0.0
    pools_created: int = 0
    blocks_run: int = 0
    peak_bytes: int = 0
    budget_bytes: int = 0
    gl_failures: int = 0
    open_s_sum: float = 0.0          # seconds the helper threads spent opening pools and checkers
    open_s_max: float = 0.0
    step_s_max: float = 0.0          # longest pass of the native dispatcher over its pools
    phase_s_max: tuple = ()          # its longest continuations / pools / placing / checks / closing parts
    per_n: Dict[int, dict] = field(default_factory=dict)

    @property
    def rate(self) -> float:
        return self.digit_squarings / self.seconds if self.seconds > 0 else 0.0


class Server:
    """Driver of the native continuous-batching loop on one device.

    B: Gerbicz-Li block length shared by every pool; capacity(n): slots per
    pool; budget_bytes: device memory that pools and checkers may hold;
    tune: autotune each pool shape's plan (before the clock starts);
    validate_group: finished tests checked together (validate=False: none);
    lib: a library exporting the gfc_server_* ABI (default libgfcuda.so).
    """

    def __init__(self, B: int = 1000, budget_bytes: int = 80 * 10**9,
                 capacity: Optional[Callable[[int], int]] = None, tune: bool = True, validate: bool = True,
                 validate_group: int = 4, keep_digits: bool = False, device: int = 0, idle_close_s: float = 10.0,
                 lib=None):
        self.B = int(B)
        self.budget_bytes = int(budget_bytes)
        self.capacity = capacity
        self.tune = bool(tune)
        self.validate = bool(validate)
        self.validate_group = int(validate_group) if validate else 0
        self.keep_digits = bool(keep_digits)
        self.device = int(device)
        self.idle_close_s = float(idle_close_s)
        self.L = bind(lib) if lib is not None else _default_lib()
        self.stats = ServeStats()

    def _check(self, rc: int):
        if rc != GFC_OK:
            raise GfcError(rc, self.L.gfc_last_error().decode(errors="replace"))

    def _config(self) -> ServerConfig:
        cfg = ServerConfig()
        self.L.gfc_server_default_config(ctypes.byref(cfg))
        cfg.block = self.B
        cfg.validate_group = self.validate_group
        cfg.budget_bytes = self.budget_bytes
        for n in range(24):
            cfg.capacity[n] = max(1, int(self.capacity(n))) if self.capacity is not None else 0
        cfg.device = self.device
        cfg.tune = 1 if self.tune else 0
        cfg.keep_digits = 1 if self.keep_digits else 0
        cfg.idle_close_s = self.idle_close_s
        return cfg

    def run(self, requests: Sequence[Request], timeout_s: float = 3600.0,
            warmup: Sequence[Request] = ()) -> List[Completion]:
        """Serves ``requests`` (arrival times in seconds from the start of the
        run) and returns their completions in request order.  ``warmup``
        requests (ids distinct from the others) are served first, all at once,
        and left out of the results and statistics: they open the pools, so
        that the run measures the pools' steady state."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.id))
        L = self.L
        h = vp()
        cfg = self._config()
        self._check(L.gfc_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        comps: Dict[int, Completion] = {}
        try:
            if self.tune:                       # plans chosen before the clock starts
                for n in sorted({int(r.job.n) for r in reqs}):
                    reps = {1024} | {int(r.job.b) for r in reqs if int(r.job.n) == n and _packed_pool(r.job.b, n)}
                    for rep in sorted(reps)[:2]:
                        self._check(L.gfc_server_pretune(h, n, rep))
            buf = (CompletionC * 64)()
            got = ctypes.c_size_t(0)
            if warmup:
                for r in warmup:
                    w = np.ascontiguousarray(r.job.words, dtype=np.uint32)
                    self._check(L.gfc_server_submit(h, r.id, int(r.job.b), int(r.job.n),
                                                    w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), int(r.job.nbits)))
                left = len(warmup)
                while left > 0:
                    self._check(L.gfc_server_poll(h, buf, 64, ctypes.byref(got), 20))
                    left -= got.value
                    for i in range(got.value):
                        if self.keep_digits:       # release the kept residue
                            d = np.empty(1 << int(buf[i].n), dtype=np.int32)
                            L.gfc_server_digits(h, buf[i].id, d.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), d.size)
            t0 = L.gfc_server_clock(h)
            k = 0
            deadline = t0 + timeout_s
            while len(comps) < len(reqs):
                now = L.gfc_server_clock(h)
                while k < len(reqs) and t0 + reqs[k].arrival <= now:
                    j = reqs[k].job
                    w = np.ascontiguousarray(j.words, dtype=np.uint32)
                    self._check(L.gfc_server_submit(h, reqs[k].id, int(j.b), int(j.n),
                                                    w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), int(j.nbits)))
                    k += 1
                if now > deadline:
                    raise TimeoutError("serving run exceeded its time limit")
                wait_ms = 5 if k == len(reqs) else int(max(0.0, min(0.005, t0 + reqs[k].arrival - now)) * 1000)
                self._check(L.gfc_server_poll(h, buf, 64, ctypes.byref(got), wait_ms))
                for i in range(got.value):
                    c = buf[i]
                    comp = Completion(int(c.id), int(c.b), int(c.n), int(c.nbits), c.arrival - t0, c.admitted - t0,
                                      c.residue_at - t0, (c.validated_at - t0) if c.validated_at >= 0 else None,
                                      bool(c.is_prp), int(c.res64), int(c.old64),
                                      None if c.gl_ok < 0 else bool(c.gl_ok), int(c.pool), int(c.slot),
                                      int(c.plan))
                    if self.keep_digits:
                        d = np.empty(1 << comp.n, dtype=np.int32)
                        self._check(L.gfc_server_digits(h, comp.id, d.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                        d.size))
                        comp.digits = d
                    comps[comp.id] = comp
            st = ServerStatsC()
            self._check(L.gfc_server_get_stats(h, ctypes.byref(st)))
        finally:
            L.gfc_server_destroy(h)
        self._summarise(reqs, list(comps.values()), st)
        return [comps[r.id] for r in requests]

    def _summarise(self, reqs, cs: List[Completion], st: ServerStatsC):
        s = ServeStats(requests=len(reqs), completed=len(cs), pools_created=int(st.pools_created),
                       blocks_run=int(st.blocks_run), peak_bytes=int(st.peak_bytes), budget_bytes=int(st.budget_bytes),
                       gl_failures=int(st.gl_failures), open_s_sum=float(st.open_s_sum),
                       open_s_max=float(st.open_s_max), step_s_max=float(st.step_s_max),
                       phase_s_max=tuple(float(x) for x in st.phase_s_max))
        self.stats = s
        if not cs:
            return
        s.seconds = max(c.residue_at for c in cs) - min(c.arrival for c in cs)
        s.digit_squarings = float(sum((1 << c.n) * c.nbits for c in cs))
        lat = np.array([c.latency for c in cs])
        s.p50, s.p99 = float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
        vl = np.array([c.validated_at - c.arrival for c in cs if c.validated_at is not None])
        if vl.size:
            s.p50_validated, s.p99_validated = float(np.percentile(vl, 50)), float(np.percentile(vl, 99))
        s.mean_wait = float(np.mean([c.admitted - c.arrival for c in cs]))
        for n in sorted({c.n for c in cs}):
            sub = [c for c in cs if c.n == n]
            s.per_n[n] = {"tests": len(sub), "p50_s": float(np.median([c.latency for c in sub])),
                          "digit_squarings": float(sum((1 << n) * c.nbits for c in sub))}


# ------------------------------------------------------------------ the serving workload


def warmup_requests(requests: Sequence[Request], B: int, first_id: int = 10**9) -> List[Request]:
    """One single-block request per pool shape that ``requests`` open (size,
    and packed-digit range from 2^19 on), arriving at once: served before a
    run, they open the pools and checkers the run then finds warm."""
    out: List[Request] = []
    seen = set()
    for r in requests:
        key = (int(r.job.n), _packed_pool(r.job.b, r.job.n))
        if key in seen:
            continue
        seen.add(key)
        out.append(Request(first_id + len(out), Job.prefix(int(r.job.b), int(r.job.n), int(B)), 0.0))
    return out


SERVE_LIMITS = {15: 2_000_000_000, 16: 1_500_000_000, 17: 1_000_000_000, 18: 1_000_000_000,
                19: 70_000_000, 20: 55_000_000, 21: 45_000_000, 22: 35_000_000, 23: 25_000_000}


def serve_requests(count: int, rate: float, blocks: Sequence[int], B: int, seed: int = 1005,
                   ns: Sequence[int] = tuple(range(15, 23)), big: Optional[int] = 23,
                   big_b: int = 25_000_000) -> List[Request]:
    """Poisson arrivals at ``rate`` per second of tests with n uniform over
    ``ns`` and b even, uniform in [1024, limit(n)]; each runs the first
    blocks * B exponent bits of its test, blocks drawn uniformly from
    ``blocks``.  With ``big``, one test of that size and base near big_b
    arrives with the first request."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out: List[Request] = []
    for i in range(count):
        n = int(rng.choice(np.asarray(ns)))
        b = int(rng.integers(1024, SERVE_LIMITS[n])) & ~1
        if b & (b - 1) == 0:
            b += 2
        nb = int(rng.choice(np.asarray(blocks))) * B
        out.append(Request(i, Job.prefix(b, n, nb), t))
        t += float(rng.exponential(1.0 / rate))
    if big is not None:
        b = big_b + 2 * int(rng.integers(-50, 50))
        nb = int(max(blocks)) * B
        out.append(Request(count, Job.prefix(b, big, nb), 0.0))
    return out
