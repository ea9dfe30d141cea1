"""Sharding a batch of independent domains over ranks (one process per GPU).

The domains of a batch never exchange data during a step, so a multi-GPU run
splits the domain list across ranks and each rank steps its share as one batch;
the only communication is one gather of per-domain results at the end.  The
split is longest-processing-time-first bin packing on cells x nonlinear
iterations, which keeps the slowest rank within one domain of the mean.
"""
from __future__ import annotations

from typing import Sequence


def domain_cost(shape: Sequence[int], nonlinear_iters: int = 1) -> int:
    """Work of one domain per step: box cells times nonlinear (global) iterations."""
    n = 1
    for x in shape:
        n *= int(x)
    return n * int(nonlinear_iters)


def lpt_partition(costs: Sequence[float], n_parts: int) -> list[list[int]]:
    """Assigns items to n_parts bins: items in descending cost order (ties by
    index), each to the currently least-loaded bin (ties by bin index).  Returns
    the item indices of every bin in ascending order.  Deterministic, so every rank
    computes the same split without communicating."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * n_parts
    parts: list[list[int]] = [[] for _ in range(n_parts)]
    for i in order:
        b = min(range(n_parts), key=lambda p: (load[p], p))
        parts[b].append(i)
        load[b] += float(costs[i])
    return [sorted(p) for p in parts]


def part_loads(costs: Sequence[float], parts: Sequence[Sequence[int]]) -> list[float]:
    return [float(sum(costs[i] for i in p)) for p in parts]


def gather_per_domain(local: dict[int, object], world_size: int) -> dict[int, object]:
    """Merges every rank's {domain index: result} through torch.distributed (any
    backend; one all_gather_object).  With world_size 1 it returns a copy."""
    if world_size == 1:
        return dict(local)
    import torch.distributed as dist
    got: list[dict] = [None] * world_size  # type: ignore[list-item]
    dist.all_gather_object(got, local)
    out: dict[int, object] = {}
    for g in got:
        out.update(g)
    return out
