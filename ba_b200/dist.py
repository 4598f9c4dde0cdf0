"""Host-side helpers for running the path on several GPUs, one process per
GPU (torch.distributed; NCCL on GPUs, gloo in the CPU tests).

The batched and served workloads are sets of independent solves, so their
ranks never exchange solver data: each rank owns its share of the systems (its
own seeded batch or request stream, a cost-balanced part of one batch from
partition_by_cost, or its share of one request stream routed by route_jsq)
and only one scalar -- the step time -- is reduced, as the maximum over
ranks.  The reference's multi-rank path, one system partitioned
by rows with a ghost halo (CoupledVector/CoupledMatrix,
linear_algebra/coupled_vector.cc:890-973), lives in ba_b200/coupled.py.
"""
from __future__ import annotations

import heapq

SEED_STRIDE = 7919  # a prime: per-rank seeds never collide with the per-system offsets (+1 .. +count)


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s own batch or request stream."""
    return int(base) + SEED_STRIDE * int(rank)


def partition_by_cost(costs, world: int) -> list[list[int]]:
    """Split items (e.g. systems weighted by nnz) over `world` ranks: longest
    first, each to the least-loaded rank (ties to the lower rank), so every
    rank gets a deterministic share within the largest item of the mean.
    Returns the item indices of each rank in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def route_jsq(times, costs, world: int, drain_rate: float) -> list[int]:
    """Route one request stream over `world` ranks, join the shortest queue
    by outstanding work: request i arrives at times[i] (seconds, ascending)
    with work costs[i] (e.g. its matrix nonzeros); every rank is a server
    that works its backlog off at `drain_rate` cost units per second (0:
    never, so the rule becomes least assigned work); the request goes to the
    rank with the least backlog at its arrival; ties (idle ranks, at light
    load) to the least work assigned so far, then to the lower rank.
    Depends only on the stream, so every rank computes the same routing
    without a message; a front end would run the same rule online with the
    servers' reported backlogs.  Returns each request's rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if len(times) != len(costs):
        raise ValueError("times and costs differ in length")
    backlog = [0.0] * world
    assigned = [0.0] * world
    last = None
    out = []
    for t, c in zip(times, costs):
        if last is not None:
            if t < last:
                raise ValueError("arrival times must be ascending")
            done = float(drain_rate) * (t - last)
            backlog = [max(0.0, b - done) for b in backlog]
        last = t
        r = min(range(world), key=lambda k: (backlog[k], assigned[k], k))
        backlog[r] += float(c)
        assigned[r] += float(c)
        out.append(r)
    return out


def stream_share(reqs, world: int, rank: int, drain_rate: float, cost) -> list:
    """This rank's part of one request stream routed by route_jsq: reqs are
    dicts with an arrival time "t" (0 when absent: all at once), cost(req)
    their work.  Every rank gets a disjoint part; together they are the
    stream, each part in arrival order."""
    route = route_jsq([rq.get("t", 0.0) for rq in reqs], [cost(rq) for rq in reqs], world, drain_rate)
    return [rq for rq, r in zip(reqs, route) if r == rank]


def _reduce(value: float, op: str, device: str) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(value: float, device: str = "cuda") -> float:
    """The maximum of `value` over all ranks (the value itself on one rank)."""
    return _reduce(value, "max", device)


def sum_over_ranks(value: float, device: str = "cuda") -> float:
    return _reduce(value, "sum", device)


def aggregate_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput: every rank processed `units_per_rank` units and
    the job took the slowest rank's time."""
    return world * units_per_rank / (max_ms / 1e3)
