"""Replica data parallelism over GPUs (one process per GPU).

Micrographs and tilt series are independent (a series is refined package by
package, so it never splits), and GCtfFind has no collective.  A run over
several GPUs is therefore N replicas: each rank takes a share of the
series / micrographs, processes it on its own GPU through its own Context,
and the result rows are gathered on the host.  The only communication is
that gather (``torch.distributed`` object collective on the process group
the caller set up: gloo or NCCL); no device memory is shared and nothing
crosses NVLink on the data path.
"""
from __future__ import annotations

from typing import Callable, Sequence


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the items each rank processes: longest-processing-time
    greedy on `costs` (e.g. pixels x micrographs of a series), ties broken by
    index, so every rank computes the same split without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shares[r].append(i)
        load[r] += float(costs[i])
    for s in shares:
        s.sort()
    return shares


def run_replicas(items: Sequence, costs: Sequence[float], process: Callable, rank: int = 0,
                 world: int = 1, group=None) -> list:
    """Runs `process(item)` for this rank's share and returns every item's
    result, in item order, on every rank (one all_gather of the rows)."""
    shares = partition(costs, world)
    mine = {i: process(items[i]) for i in shares[rank]}
    if world == 1:
        return [mine[i] for i in range(len(items))]
    import torch.distributed as dist
    gathered: list = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    out: list = [None] * len(items)
    for part in gathered:
        for i, v in part.items():
            out[i] = v
    missing = [i for i, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError(f"items without a result after the gather: {missing}")
    return out


def series_rows(ctx, series: Sequence, optics, is_tomo: bool = True):
    """`process` for run_replicas over tilt series on a Context: one
    gcf_run_series per series (item = (images, tilts)); returns the rows
    (df_min, df_max, azimuth, ext_phase, score) in image order."""
    from .api import series_order
    images, tilts = series
    order = series_order(tilts).order if is_tomo else list(range(len(images)))
    res = ctx.run_series(images, optics, order, is_tomo=is_tomo)
    return [(r.df_min, r.df_max, r.azimuth, r.ext_phase, r.score) for r in res]
