"""Multi-GPU host logic on CPU: cost-balanced test queues per rank and the
host-side gather, run as two gloo ranks (the per-test work is the CPU oracle,
standing in for a GPU)."""
import os
import socket

import torch.multiprocessing as mp

from genefer22_b200.shard import predicted_cost, run_sharded, shard_tests

TESTS = [(10**9, 6), (1024, 5), (123456, 7), (2 * 10**9 - 2, 6), (65538, 5), (999998, 7), (30, 5)]


def test_shard_balanced_and_complete():
    for world in (1, 2, 3, 8):
        parts = shard_tests(TESTS, world)
        assert sorted(i for p in parts for i in p) == list(range(len(TESTS)))
        loads = [sum(predicted_cost(*TESTS[i]) for i in p) for p in parts]
        if world <= len(TESTS):
            assert max(loads) <= sum(loads) / world + max(predicted_cost(*t) for t in TESTS)


def _oracle_run(tests):
    import gf_oracle as G
    out = []
    for b, n in tests:
        _, res64, _, ok = G.quick(G.OracleTransform(b, n), b, n)
        out.append((res64, ok))
    return out


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    sys.path.insert(0, os.path.dirname(here))
    import torch.distributed as dist
    from genefer22_b200.shard import torch_gather
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        merged = run_sharded(TESTS, _oracle_run, rank, world, torch_gather)
        q.put((rank, merged))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_matches_single():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    single = dict(enumerate(_oracle_run(TESTS)))
    for rank, merged in got:
        assert merged == single
