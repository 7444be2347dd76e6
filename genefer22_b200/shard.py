"""Distributing PRP tests over GPUs (one process per GPU).

Tests are independent, so the data path has no collective: each rank takes a
queue of tests, balanced by predicted cost, runs them on its own GPU and the
results are gathered on the host.  A single test never spans GPUs (splitting
one transform would need an all-to-all of the state every squaring).
"""
from __future__ import annotations

import heapq
import math
from typing import Callable, Dict, List, Sequence, Tuple

Test = Tuple[int, int]          # (b, n)


def predicted_cost(b: int, n: int) -> float:
    """Work of one test: |E| = 2^n log2 b squarings of cost ~ N log2 N each."""
    N = 1 << n
    return N * math.log2(b) * N * n


def shard_tests(tests: Sequence[Test], world: int) -> List[List[int]]:
    """Indices of the tests for each rank: longest-processing-time-first
    assignment to the least-loaded rank (deterministic for equal costs)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(tests)), key=lambda i: (-predicted_cost(*tests[i]), i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + predicted_cost(*tests[i]), r))
    for lst in out:
        lst.sort()
    return out


def run_sharded(tests: Sequence[Test], run: Callable[[List[Test]], List[object]], rank: int, world: int,
                gather: Callable[[object], List[object]]) -> Dict[int, object]:
    """Runs this rank's share of `tests` with `run` (a list of (b, n) in, one
    result per test out) and gathers every rank's results with `gather` (e.g.
    torch.distributed.all_gather_object).  Returns {test index: result} on
    every rank."""
    mine = shard_tests(tests, world)[rank]
    results = run([tests[i] for i in mine])
    if len(results) != len(mine):
        raise RuntimeError("runner returned a wrong number of results")
    parts = gather(list(zip(mine, results)))
    merged: Dict[int, object] = {}
    for part in parts:
        for i, r in part:
            merged[i] = r
    return merged


def torch_gather(obj: object) -> List[object]:
    """all_gather_object over the default process group."""
    import torch.distributed as dist
    out: List[object] = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
