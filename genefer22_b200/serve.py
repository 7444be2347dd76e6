"""Serving: a request loop with continuous batching on one GPU.

Requests (a PRP test, or the first k squarings of one: ``Job``) arrive over
time.  Tests of one size n share a *pool*: a ``Batch`` of ``capacity`` slots
with its own CUDA stream and host thread, whose CUDA graph runs one
Gerbicz-Li block for every slot:

    d <- d * x   (the d(t) update of src/genefer.h:529-535)
    B squarings of x, exponent bits taken per slot from its own position

A slot that holds no test, or whose test has run out of exponent bits, sits
out the squarings (its position is below 0).  A new test enters a free slot
between two blocks with x = d = 1, so the d update that opens its first block
leaves d = 1, as genefer starts (src/genefer.h:492-497); its exponent is
padded with leading zero bits to a whole number of blocks.  When a test's
last block ends, its x and d(t) are read back, the residue is reported
(``residue_at``), the slot is freed, and x and d(t) go to the validator
thread of that size, which runs genefer's Gerbicz-Li check
(src/genefer.h:557-615) for several finished tests at once on a batch of its
own (``validated_at``).

Pools are created while the device-memory budget allows (per slot:
registers, transform planes, multiplicand, carries and room for the longest
exponent of its size; per size: the root tables) and closed after a short idle time, which returns their memory
to the budget.  Requests wait in a per-size queue until a slot is free.

Every test's arithmetic reads only its own slot, base and exponent bits, so a
residue is the same whether the test ran alone or among others; tests check
this against ``mixed.run_alone``.

The reference has no counterpart: genefer runs one test per process
(src/genefer.h:1360-1480).
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field
from typing import Deque, Dict, List, Optional, Sequence

import numpy as np

from . import gint
from .autotune import Autotuner, packed_ok
from .exponent import chunk_sum
from .genefer import Job, gl_validate
from .transform import Batch

NUM_REGS = 3


def slot_bytes(n: int, num_regs: int = NUM_REGS) -> int:
    """Device bytes of one batch slot of size n: registers, 3 transform planes,
    3 multiplicand planes, segment carries, descriptor and position."""
    N = 1 << int(n)
    return num_regs * 4 * N + 12 * N + 12 * N + (N // 16) * 8 + 256


def table_bytes(n: int) -> int:
    """Root tables of size n, shared by every batch of that size on a device:
    the two 32-bit primes at one word per root, the three 31-bit primes at two
    (root and Shoup quotient), forward and inverse (16 N words), and the four
    primes of packed digits on N/2 points at two words per root (8 N words)."""
    return 24 * 4 * (1 << int(n))


def exponent_bytes(nbits: int) -> int:
    return 4 * ((int(nbits) + 31) // 32) + 256


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
    arrival: float
    admitted: float = 0.0
    residue_at: float = 0.0
    validated_at: Optional[float] = None
    is_prp: bool = False
    res64: int = 0
    old64: int = 0
    gl_ok: Optional[bool] = None
    pool: int = -1
    slot: int = -1
    digits: Optional[np.ndarray] = None

    @property
    def latency(self) -> float:
        """Time to residue: arrival to the residue read back."""
        return self.residue_at - self.arrival


@dataclass
class _Active:
    req: Request
    comp: Completion
    blocks_left: int


def default_capacity(n: int) -> int:
    """Slots per pool: enough tests per launch to fill the GPU at small n,
    few at large n where one test already fills it."""
    return {15: 32, 16: 32, 17: 16, 18: 8, 19: 4, 20: 2, 21: 2, 22: 1, 23: 1}.get(int(n), 32 if n < 15 else 1)


class _Budget:
    def __init__(self, limit: int):
        self.limit = int(limit)
        self.used = 0
        self.peak = 0
        self.tables: Dict[int, int] = {}       # n -> pools holding the tables

    def need(self, n: int, nbytes: int) -> int:
        return nbytes + (0 if self.tables.get(n, 0) > 0 else table_bytes(n))

    def take(self, n: int, nbytes: int) -> bool:
        total = self.need(n, nbytes)
        if self.used + total > self.limit:
            return False
        self.used += total
        self.peak = max(self.peak, self.used)
        self.tables[n] = self.tables.get(n, 0) + 1
        return True

    def give(self, n: int, nbytes: int):
        self.tables[n] -= 1
        self.used -= nbytes + (table_bytes(n) if self.tables[n] == 0 else 0)


# From this size, packed digits are faster even for pools of one or two tests
# (measured); smaller sizes keep one kind of pool, so that requests are not
# split between two half-full pools.
PACKED_POOL_MIN_N = 19


def _packed_pool(b: int, n: int) -> bool:
    return (int(n) >= PACKED_POOL_MIN_N) and packed_ok(b, n)


class _Pool:
    """Slots of one size.  A pool opened (at n >= PACKED_POOL_MIN_N) for a base
    in the packed range tunes with that base, so that packed plans are
    candidates, and takes only such bases; any other pool takes every base."""

    def __init__(self, server: "Server", pid: int, n: int, capacity: int, nbytes: int, rep_b: int = 1024):
        self.server, self.pid, self.n, self.capacity, self.nbytes = server, pid, n, capacity, nbytes
        self.rep_b = int(rep_b)
        self.packed_only = _packed_pool(rep_b, n)
        self.slots: List[Optional[_Active]] = [None] * capacity
        self.reserved = 0                       # admitted by the dispatcher, not yet loaded
        self.batch: Optional[Batch] = None
        self.graph = None
        self.plan = -1
        self.blocks_run = 0
        self.thread = threading.Thread(target=self._main, name=f"pool{pid}-n{n}", daemon=True)

    def free_slots(self) -> int:
        return self.capacity - sum(s is not None for s in self.slots) - self.reserved

    # -- runs on the pool's thread
    def _setup(self):
        srv = self.server
        self.batch = Batch([self.rep_b] * self.capacity, self.n, num_regs=NUM_REGS, device=srv.device)
        if srv.tuner is not None:
            self.plan = srv.tuner.tune(self.batch).lr
        else:
            self.plan = self.batch.plan()
        bt, B = self.batch, srv.B
        self.graph = bt.capture(lambda: (bt.gl_step(), bt.square_exp(B)))
        self.one = np.zeros(1 << self.n, dtype=np.int32)
        self.one[0] = 1

    def _load(self, slot: int, act: _Active):
        bt, B = self.batch, self.server.B
        job = act.req.job
        nb_pad = ((job.nbits + B - 1) // B) * B
        words = np.zeros((nb_pad + 31) // 32, dtype=np.uint32)
        words[: job.words.size] = job.words
        bt.assign(slot, job.b)
        bt.put(slot, self.one, 0)
        bt.put(slot, self.one, 1)
        bt.set_exponent(slot, words, nb_pad)
        act.blocks_left = nb_pad // B

    def _retire(self, slot: int, act: _Active):
        bt = self.batch
        x = bt.get(slot, 0)
        d = bt.get(slot, 1)
        c = act.comp
        canon = gint.unbalance(x, c.b)
        c.is_prp, c.res64, c.old64 = gint.is_one(canon, c.b)
        c.residue_at = self.server.clock()
        if self.server.keep_digits:
            c.digits = canon
        self.server._finished(self, slot, act, x, d)

    def _main(self):
        srv = self.server
        try:
            self._setup()
            idle_since = srv.clock()
            while True:
                with srv.cv:
                    new = srv._take_for(self)
                for slot, act in new:
                    self._load(slot, act)
                    with srv.cv:
                        self.slots[slot] = act
                        self.reserved -= 1
                if not any(s is not None for s in self.slots):
                    with srv.cv:
                        if srv._pool_should_close(self, idle_since):
                            srv._close_pool(self)
                            break
                        srv.cv.wait(0.002)
                    continue
                self.graph.launch()
                self.batch.sync()
                self.blocks_run += 1
                for slot, act in enumerate(self.slots):
                    if act is None:
                        continue
                    act.blocks_left -= 1
                    if act.blocks_left == 0:
                        self._retire(slot, act)
                idle_since = srv.clock()
        except BaseException as e:            # surfaced by Server.run
            with srv.cv:
                srv.errors.append(e)
                srv._close_pool(self)
        finally:
            self.graph = None
            if self.batch is not None:
                self.batch.close()
                self.batch = None


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
    peak_bytes: int = 0
    budget_bytes: int = 0
    gl_failures: int = 0
    per_n: Dict[int, dict] = field(default_factory=dict)

    @property
    def rate(self) -> float:
        return self.digit_squarings / self.seconds if self.seconds > 0 else 0.0


class Server:
    """Continuous-batching request loop on one device.

    B: Gerbicz-Li block length shared by every pool; capacity(n): slots per
    pool; budget_bytes: device memory that pools and validators may hold.
    """

    def __init__(self, B: int = 1000, budget_bytes: int = 80 * 10**9, capacity=default_capacity,
                 tuner: Optional[Autotuner] = None, validate: bool = True, validate_group: int = 4,
                 keep_digits: bool = False, device: int = 0, idle_close_s: float = 0.25):
        self.B = int(B)
        self.budget = _Budget(budget_bytes)
        self.capacity = capacity
        self.tuner = tuner
        self.validate = validate
        self.validate_group = int(validate_group)
        self.keep_digits = keep_digits
        self.device = device
        self.idle_close_s = idle_close_s
        self.cv = threading.Condition()
        self.errors: List[BaseException] = []

    # ---------------------------------------------------------------- clock
    def clock(self) -> float:
        return time.perf_counter() - self._t0

    # ------------------------------------------------------ called under cv
    def _take_for(self, pool: _Pool):
        """Moves waiting requests of the pool's size into its free slots."""
        q = self.waiting[pool.n]
        out = []
        for slot in range(pool.capacity):
            if pool.slots[slot] is not None:
                continue
            req = next((r for r in q if not pool.packed_only or _packed_pool(r.job.b, pool.n)), None)
            if req is None:
                break
            q.remove(req)
            pool.reserved += 1
            c = Completion(req.id, req.job.b, req.job.n, req.job.nbits, req.arrival, admitted=self.clock(),
                           pool=pool.pid, slot=slot)
            out.append((slot, _Active(req, c, 0)))
        return out

    def _pool_should_close(self, pool: _Pool, idle_since: float) -> bool:
        if self.waiting[pool.n]:
            return False
        if self._dispatch_done and not any(self.waiting.values()):
            return True
        return (self.clock() - idle_since) > self.idle_close_s

    def _close_pool(self, pool: _Pool):
        if pool in self.pools:
            self.pools.remove(pool)
            self.budget.give(pool.n, pool.nbytes)
            self.cv.notify_all()

    def _place(self):
        """Opens pools for waiting requests while the budget allows."""
        for n, q in self.waiting.items():
            if not q:
                continue
            anyb = [r for r in q if not _packed_pool(r.job.b, n)]   # need a pool that takes every base
            packb = [r for r in q if _packed_pool(r.job.b, n)]
            free_any = sum(p.free_slots() for p in self.pools if p.n == n and not p.packed_only)
            free_pk = sum(p.free_slots() for p in self.pools if p.n == n and p.packed_only)
            while True:
                if free_any < len(anyb):
                    rep, is_pk = 1024, False
                elif free_pk + (free_any - len(anyb)) < len(packb):
                    rep, is_pk = packb[0].job.b, True
                else:
                    break
                cap = max(1, int(self.capacity(n)))
                nb = cap * (slot_bytes(n) + self._exp_bytes[n])
                if not self.budget.take(n, nb):
                    break
                p = _Pool(self, self._next_pid, n, cap, nb, rep_b=rep)
                self._next_pid += 1
                self.pools.append(p)
                self.stats.pools_created += 1
                p.thread.start()
                if is_pk:
                    free_pk += cap
                else:
                    free_any += cap

    # -------------------------------------------------- from pool threads
    def _finished(self, pool: _Pool, slot: int, act: _Active, x: np.ndarray, d: np.ndarray):
        with self.cv:
            pool.slots[slot] = None
            job = act.req.job
            self.completions.append(act.comp)
            if self.validate:
                self.vqueue[pool.n].append((act.comp, job, x, d))
            self.cv.notify_all()

    # -------------------------------------------------------- validators
    def _validator(self, n: int):
        """Gerbicz-Li checks of finished tests of size n, up to validate_group
        at once, on a batch and stream of its own."""
        bt: Optional[Batch] = None
        q = self.vqueue[n]
        try:
            while True:
                with self.cv:
                    while not q and not self._stop_validator:
                        self.cv.wait(0.01)
                    if not q:
                        break
                    group = [q.popleft() for _ in range(min(len(q), self.validate_group))]
                if bt is None:
                    bt = Batch([1024] * self.validate_group, n, num_regs=NUM_REGS, device=self.device)
                zero = np.zeros(1 << n, dtype=np.int32)
                res = []
                for i in range(self.validate_group):
                    if i < len(group):
                        c, job, x, d = group[i]
                        bt.assign(i, c.b)
                        bt.put(i, x, 0)
                        bt.put(i, d, 1)
                        res.append(chunk_sum(job.words, job.nbits, self.B))
                    else:
                        bt.put(i, zero, 0)
                        bt.put(i, zero, 1)
                        res.append(0)
                ok = gl_validate(bt, self.B, res)
                now = self.clock()
                with self.cv:
                    for i, (c, _, _, _) in enumerate(group):
                        c.gl_ok = bool(ok[i])
                        c.validated_at = now
                    self.cv.notify_all()
        except BaseException as e:
            with self.cv:
                self.errors.append(e)
                self.cv.notify_all()
        finally:
            if bt is not None:
                bt.close()

    def _validator_bytes(self, ns: Sequence[int]) -> int:
        return sum(self.validate_group * slot_bytes(n) for n in set(ns))

    # ------------------------------------------------------------- run
    def run(self, requests: Sequence[Request], timeout_s: float = 3600.0) -> List[Completion]:
        """Serves ``requests`` (arrival times in seconds from now) and returns
        their completions in request order."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.id))
        ns = sorted({int(r.job.n) for r in reqs})
        self.waiting: Dict[int, Deque[Request]] = {n: collections.deque() for n in ns}
        self.vqueue: Dict[int, Deque] = {n: collections.deque() for n in ns}
        self.pools: List[_Pool] = []
        self.completions: List[Completion] = []
        self.errors = []
        self.stats = ServeStats(requests=len(reqs), budget_bytes=self.budget.limit)
        # every slot of a pool may hold the longest exponent of its size
        self._exp_bytes = {n: max(exponent_bytes(((r.job.nbits + self.B - 1) // self.B) * self.B)
                                  for r in reqs if int(r.job.n) == n) for n in ns}
        self._next_pid = 0
        self._dispatch_done = False
        self._stop_validator = False
        vbytes = 0
        if self.validate:
            vbytes = self._validator_bytes(ns)
            if vbytes > self.budget.limit:
                raise ValueError("budget smaller than the validators' memory")
            self.budget.limit -= vbytes
        if self.tuner is not None:               # plans chosen before the clock starts
            for n in ns:
                reps = [1024] + [next((int(r.job.b) for r in reqs if int(r.job.n) == n and _packed_pool(r.job.b, n)), 1024)]
                for rep in sorted(set(reps)):
                    with Batch([rep] * max(1, int(self.capacity(n))), n, num_regs=NUM_REGS, device=self.device) as bt:
                        self.tuner.tune(bt)
        self._t0 = time.perf_counter()
        vths = [threading.Thread(target=self._validator, args=(n,), name=f"validator-n{n}", daemon=True)
                for n in ns] if self.validate else []
        for v in vths:
            v.start()
        k = 0
        deadline = timeout_s
        try:
            with self.cv:
                while True:
                    now = self.clock()
                    while k < len(reqs) and reqs[k].arrival <= now:
                        self.waiting[int(reqs[k].job.n)].append(reqs[k])
                        k += 1
                    self._place()
                    self.cv.notify_all()
                    if self.errors:
                        raise self.errors[0]
                    if k == len(reqs):
                        self._dispatch_done = True
                        if len(self.completions) == len(reqs):
                            break
                    if now > deadline:
                        raise TimeoutError("serving run exceeded its time limit")
                    wait = 0.01 if k == len(reqs) else max(0.0, min(0.01, reqs[k].arrival - now))
                    self.cv.wait(wait)
                while any(p.thread.is_alive() for p in list(self.pools)):
                    self.cv.notify_all()
                    self.cv.wait(0.01)
                    if self.errors:
                        raise self.errors[0]
                self._stop_validator = True
                self.cv.notify_all()
        finally:
            self._dispatch_done = True
            self._stop_validator = True
            with self.cv:
                self.cv.notify_all()
        for v in vths:
            v.join(timeout=max(1.0, deadline - self.clock() + 60))
        for p in list(self.pools):
            p.thread.join(timeout=5)
        self.budget.limit += vbytes
        if self.errors:
            raise self.errors[0]
        self._summarise()
        order = {r.id: i for i, r in enumerate(requests)}
        return sorted(self.completions, key=lambda c: order[c.id])

    def _summarise(self):
        st = self.stats
        cs = self.completions
        st.completed = len(cs)
        if not cs:
            return
        t_first = min(c.arrival for c in cs)
        t_last = max(c.residue_at for c in cs)
        st.seconds = t_last - t_first
        st.digit_squarings = float(sum((1 << c.n) * c.nbits for c in cs))
        lat = np.array([c.latency for c in cs])
        st.p50, st.p99 = float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
        vl = np.array([c.validated_at - c.arrival for c in cs if c.validated_at is not None])
        if vl.size:
            st.p50_validated, st.p99_validated = float(np.percentile(vl, 50)), float(np.percentile(vl, 99))
        st.mean_wait = float(np.mean([c.admitted - c.arrival for c in cs]))
        st.peak_bytes = self.budget.peak
        st.gl_failures = sum(1 for c in cs if c.gl_ok is False)
        for n in sorted({c.n for c in cs}):
            sub = [c for c in cs if c.n == n]
            st.per_n[n] = {"tests": len(sub), "p50_s": float(np.median([c.latency for c in sub])),
                           "digit_squarings": float(sum((1 << n) * c.nbits for c in sub))}


# ------------------------------------------------------------------ the serving workload

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
