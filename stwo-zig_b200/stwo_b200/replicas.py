"""Proof-level sharding over GPUs, one process per GPU.

Proofs are independent, so N GPUs run N replicas: a host router assigns each
request to one rank, every rank proves its share with its own context (and
serving loop), and nothing crosses NVLink on the data path. The only
collectives are host plumbing: the max over ranks of a timed region, and an
optional all-gather of the proof bytes to one rank. They work on any
torch.distributed backend (nccl on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq


def request_cost(log_n_rows: int, sequence_len: int) -> int:
    """Accounted device bytes of a wide-Fibonacci request: 16 per committed cell, the measure of
    the reference's resource admission (src/prover/native/resource_admission.zig:5-10)."""
    return 16 * (sequence_len << log_n_rows)


def assign(costs: list[int], world: int) -> list[int]:
    """Rank of every request: longest-processing-time-first greedy over the costs, ties broken by
    request index and rank number, so every rank computes the same assignment."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world)]
    out = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(heap)
        out[i] = r
        heapq.heappush(heap, (load + costs[i], r))
    return out


def shard(requests: list, rank: int, world: int, cost=None) -> list[tuple[int, object]]:
    """(index, request) pairs this rank proves. `cost` maps a request to its cost (default: the
    accounted bytes of r["statement"])."""
    if cost is None:
        def cost(r):
            st = r["statement"]
            return request_cost(st.log_n_rows, st.sequence_len)
    owner = assign([cost(r) for r in requests], world)
    return [(i, r) for i, r in enumerate(requests) if owner[i] == rank]


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank number (a timed region) over all ranks; the value itself without a process
    group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_proofs(local: dict[int, bytes], dst: int = 0) -> dict[int, bytes] | None:
    """All ranks' {index: proof bytes} merged on rank `dst` (None elsewhere)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(local, parts, dst=dst)
    if dist.get_rank() != dst:
        return None
    merged: dict[int, bytes] = {}
    for p in parts:
        merged.update(p)
    return merged
