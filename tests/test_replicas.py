"""Multi-GPU replica plumbing on CPU: two gloo ranks shard requests, prove their share (with the
oracle standing in for the device), take the max of their timings and gather the proofs."""
import os
import socket
import sys

import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "stwo-zig_b200", "stwo_b200"))
import replicas  # noqa: E402  (the module alone: no CUDA library needed)


def _requests():
    shapes = [(3, 4), (4, 8), (2, 3), (5, 8), (3, 16), (4, 4), (1, 2), (5, 4), (2, 8), (3, 3)]
    return [dict(log_n=a, W=b, seed=100 + i) for i, (a, b) in enumerate(shapes)]


def _cost(r):
    return replicas.request_cost(r["log_n"], r["W"])


def test_assignment_is_a_partition_and_balanced():
    costs = [replicas.request_cost(n, w) for n in range(10, 21) for w in (16, 32, 100)]
    for world in (1, 2, 3, 8):
        owner = replicas.assign(costs, world)
        assert sorted(set(owner)) == list(range(min(world, len(costs))))
        loads = [sum(c for c, o in zip(costs, owner) if o == r) for r in range(world)]
        assert max(loads) - min(loads) <= max(costs)  # LPT bound
        assert replicas.assign(costs, world) == owner  # deterministic


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = replicas.shard(_requests(), rank, world, cost=_cost)
        cfg = oracle.config("smoke")
        local = {i: oracle.prove_wide_fib(r["log_n"], r["W"], cfg, trace_kind=1, trace_seed=r["seed"],
                                          n_threads=1) for i, r in mine}
        t = replicas.max_over_ranks(float(rank + 1))
        merged = replicas.gather_proofs(local)
        if rank == 0:
            q.put((t, merged))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharding():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert t == 2.0
    reqs = _requests()
    assert sorted(merged) == list(range(len(reqs)))
    cfg = oracle.config("smoke")
    for i, r in enumerate(reqs):
        assert merged[i] == oracle.prove_wide_fib(r["log_n"], r["W"], cfg, trace_kind=1, trace_seed=r["seed"])
