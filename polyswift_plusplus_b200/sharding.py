"""Batched instances over several GPUs: one process per GPU, instances sharded.

SCFT instances are independent, so a batch shards by instance with no
collective on the data path: rank r builds one ``ScftBatch`` from its share of
the instances on its own GPU, iterates it, and only the per-instance results
(scalars, optionally fields) are gathered on the host at the end.  Shares are
balanced by work: an instance costs its grid points times the propagator
steps of one iteration (every executed sweep of every polymer), the product
that sets its sweep time.

    from polyswift_plusplus_b200.sharding import run_sharded
    results = run_sharded(instances, iters=300)   # under torchrun, every rank

``run_sharded`` takes a ``runner`` so the partition and gather logic can run
without a GPU (tests use gloo ranks with a host-side runner).
"""
from __future__ import annotations

import math
import os
from typing import Callable, Sequence

from .config import ScftConfig


def _block_steps(alpha: float, lengthfrac: float, ds: float) -> int:
    return max(4, int(math.floor(alpha * lengthfrac / ds + 0.5)))


def instance_cost(cfg: ScftConfig) -> float:
    """Grid points x propagator steps of one iteration (mirror-symmetric chains
    run one sweep, others two)."""
    scale = float(cfg.polymers[0].length)
    steps = 0
    for p in cfg.polymers:
        alpha = p.length / scale
        seq = [(b.scfield, _block_steps(alpha, b.lengthfrac, b.ds), b.ds) for b in p.blocks]
        sweeps = 1 if seq == seq[::-1] else 2
        steps += sweeps * sum(s for _, s, _ in seq)
    return float(cfg.n_total) * steps


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time split of instance indices over `world` ranks.

    Deterministic: instances are taken in decreasing cost (ties by index) and
    each goes to the currently lightest rank (ties by rank).  Every index lands
    on exactly one rank; each rank's list is in increasing index order.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        shares[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shares]


def gpu_runner(items, iters: int, device: int) -> list[dict]:
    """Run (cfg, w) items as one batch on `device`; per-instance scalars."""
    import dataclasses

    from .scft import ScftBatch
    if not items:
        return []
    cfgs = [dataclasses.replace(c, device=device) for c, _ in items]
    with ScftBatch(cfgs) as b:
        for i, (_, w) in enumerate(items):
            b.instance(i).restore(w)
        b.update(iters)
        return b.scalars()


def run_sharded(items, iters: int, runner: Callable | None = None, group=None) -> list[dict]:
    """Run every (cfg, w) item for `iters` iterations across the ranks of the
    default process group (or `group`); returns all results, in item order, on
    every rank.  Without an initialised process group it runs everything locally."""
    import torch.distributed as dist
    runner = runner or gpu_runner
    if not (dist.is_available() and dist.is_initialized()):
        return runner(list(items), iters, int(os.environ.get("LOCAL_RANK", 0)))
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    shares = partition([instance_cost(c) for c, _ in items], world)
    mine = shares[rank]
    local = runner([items[i] for i in mine], iters, int(os.environ.get("LOCAL_RANK", rank)))
    if len(local) != len(mine):
        raise RuntimeError("runner returned the wrong number of results")
    gathered: list = [None] * world
    dist.all_gather_object(gathered, list(zip(mine, local)), group=group)
    out: list = [None] * len(items)
    for part in gathered:
        for i, res in part:
            out[i] = res
    if any(r is None for r in out):
        raise RuntimeError("an instance was not run by any rank")
    return out
