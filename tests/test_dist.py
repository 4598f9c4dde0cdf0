"""Multi-rank host logic on CPU: two gloo ranks, as bench.py runs one
process per GPU.  Checks per-rank seeds, the cost-balanced partition, the
max-over-ranks step time and the whole-job rate."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp

from ba_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from ba_b200 import dist as D
    from ba_b200 import problems as P
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        seed = D.rank_seed(P.SEED_BATCH, rank)
        sizes = P.batch_sizes(64, seed=seed)
        costs = [(int(n) + 1) ** 2 for n in sizes]
        parts = D.partition_by_cost(costs, world)
        my_ms = 100.0 + 25.0 * rank           # this rank's step time
        mx = D.max_over_ranks(my_ms, device="cpu")
        total = D.sum_over_ranks(len(sizes), device="cpu")
        rate = D.aggregate_rate(len(sizes), world, mx)
        # one served stream, routed alike on every rank: this rank's share
        stream = P.serve_stream(300, rate=40.0, hi_dofs=2e5, seed=P.SEED_SERVE)
        share = D.stream_share(stream, world, rank, 5e6, lambda rq: rq["dofs"] * (9 if rq["dim"] == 2 else 27))
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"seed": seed, "sizes": [int(x) for x in sizes], "parts": parts, "max": mx,
                       "total": total, "rate": rate, "share": [rq["seed"] for rq in share]}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(world)]
    # each rank has its own seeded batch
    assert r[0]["seed"] != r[1]["seed"] and r[0]["sizes"] != r[1]["sizes"]
    # the step time is the slowest rank's, on every rank
    assert r[0]["max"] == r[1]["max"] == 125.0
    assert r[0]["total"] == r[1]["total"] == 128
    assert r[0]["rate"] == pytest.approx(2 * 64 / 0.125)
    # the routed stream: disjoint shares that together are the whole stream
    a, b = set(r[0]["share"]), set(r[1]["share"])
    assert a and b and not (a & b) and len(a) + len(b) == 300


def test_partition_by_cost_is_balanced_and_complete():
    costs = [97, 5, 40, 40, 3, 61, 8, 22, 22, 1]
    for world in (1, 2, 3, 4):
        parts = D.partition_by_cost(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert D.partition_by_cost(costs, 2) == D.partition_by_cost(costs, 2)
    with pytest.raises(ValueError):
        D.partition_by_cost(costs, 0)


def test_single_process_reductions_are_identity():
    assert D.max_over_ranks(3.5, device="cpu") == 3.5
    assert D.sum_over_ranks(2.0, device="cpu") == 2.0
    assert D.rank_seed(10, 0) == 10 and D.rank_seed(10, 3) == 10 + 3 * D.SEED_STRIDE


def test_route_jsq_balances_outstanding_work():
    # all at once: least assigned work, in arrival order, ties to the lower rank
    assert D.route_jsq([0.0] * 5, [5, 3, 3, 1, 1], 2, 1.0) == [0, 1, 1, 0, 0]
    # backlogs drain: at t = 5 rank 0 still holds 3 units, rank 1 none
    assert D.route_jsq([0.0, 0.0, 5.0], [8, 2, 1], 2, 1.0) == [0, 1, 1]
    # both idle again at t = 20: the one assigned less work so far
    assert D.route_jsq([0.0, 0.0, 20.0], [2, 8, 1], 2, 1.0) == [0, 1, 0]
    # a served stream: every request is routed, the split is deterministic,
    # and the ranks' total work stays within one large request of each other
    import numpy as np
    rng = np.random.default_rng(5)
    times = np.cumsum(rng.exponential(0.02, 400))
    costs = np.exp(rng.uniform(np.log(1e3), np.log(2e6), 400))
    for world in (1, 2, 4):
        r = D.route_jsq(times, costs, world, 0.5 * world * costs.sum() / times[-1])
        assert len(r) == 400 and set(r) <= set(range(world))
        assert r == D.route_jsq(times, costs, world, 0.5 * world * costs.sum() / times[-1])
        loads = [costs[np.array(r) == k].sum() for k in range(world)]
        assert max(loads) - min(loads) <= 2 * costs.max()
    with pytest.raises(ValueError):
        D.route_jsq([1.0, 0.5], [1, 1], 2, 1.0)
    with pytest.raises(ValueError):
        D.route_jsq([0.0], [1], 0, 1.0)

