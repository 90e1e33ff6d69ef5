"""Sharding batched instances over ranks (CPU: gloo ranks, host-side runner).

The multi-GPU batch has no data-path collective: each rank runs its share of
the instances as one batch and the results are gathered on the host.  These
tests cover the partition (every instance exactly once, balanced, the same on
every rank), the cost model, and the gather through a real 2-rank gloo group
with a runner that records which rank ran what.
"""
import multiprocessing as mp
import os
import socket

import pytest

from polyswift_plusplus_b200 import workloads as W
from polyswift_plusplus_b200.sharding import instance_cost, partition, run_sharded


def _items(count=7):
    sizes = (8, 16, 12, 16, 8, 24, 16)
    out = []
    for i in range(count):
        cfg = W.blend(sizes[i % len(sizes)], 15.0 + i, 0.3, 0.1 if i % 2 else 0.0, seed=i)
        out.append((cfg, None))
    return out


def test_instance_cost_counts_sweeps():
    cfg, _ = W.diblock32(n=16)
    assert instance_cost(cfg) == 16 ** 3 * 2 * (30 + 70)       # two distinct sweeps
    blend = W.blend(16, 15.0, 0.3, 0.1)
    assert instance_cost(blend) == 16 ** 3 * (2 * 100 + 50)     # homopolymer: one aliased sweep
    diblock_only = W.blend(16, 15.0, 0.3, 0.0)
    assert instance_cost(diblock_only) == 16 ** 3 * 200


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_and_balances(world):
    costs = [instance_cost(c) for c, _ in W.blend_instances(count=64)] if world == 8 else \
        [float(x) for x in (5, 3, 3, 2, 9, 1, 7, 7, 4)]
    shares = partition(costs, world)
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(costs)))
    assert shares == partition(costs, world)  # deterministic
    loads = [sum(costs[i] for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(costs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _host_runner(items, iters, device):
    import torch.distributed as dist
    return [{"seed": c.seed, "n": c.n[0], "iters": iters, "rank": dist.get_rank()} for c, _ in items]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = run_sharded(_items(), iters=3, runner=_host_runner)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_run_sharded_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    items = _items()
    shares = partition([instance_cost(c) for c, _ in items], 2)
    for rank in (0, 1):
        res = got[rank]
        assert [r["seed"] for r in res] == [c.seed for c, _ in items]  # item order on every rank
        assert all(r["iters"] == 3 for r in res)
        for r_, share in enumerate(shares):
            assert {res[i]["rank"] for i in share} <= {r_}
    assert got[0] == got[1]
    assert all(shares)  # both ranks had work
