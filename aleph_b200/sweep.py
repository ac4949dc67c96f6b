"""Parameter sweeps over several GPUs: the batched QAOA sweep's sets split
across ranks (one process per GPU), each rank running its share as one
persistent launch on its own device, and the <C> values gathered.

The units are independent circuits, so there is no data-path exchange: the
only collective is the gather of one double per set (4096 sets = 32 KB) once
the ranks have run their shares. The reference runs the same sweep one set at
a time through ``qaoa_energy`` (crates/aleph-py/src/energy.rs:58-90).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def partition_by_work(sizes: Sequence[int], world: int) -> list[tuple[int, int]]:
    """Contiguous ranges [a, b) of the sets, one per rank, balanced by the
    work sum(2^n): range r ends at the first set where the running work
    reaches (r + 1) / world of the total. Every set lands in exactly one range;
    ranges may be empty when there are fewer sets than ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = np.asarray([float(1 << int(n)) for n in sizes], dtype=np.float64)
    cum = np.cumsum(w)
    total = float(cum[-1]) if len(w) else 0.0
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        # first index whose inclusive prefix reaches the target, not before the last cut
        k = int(np.searchsorted(cum, target, side="left")) + 1 if len(w) else 0
        cuts.append(min(max(k, cuts[-1]), len(w)))
    cuts.append(len(w))
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def sharded_sweep(graphs, gammas, betas, evaluate: Callable, rank: int = 0, world: int = 1,
                  gather: Callable | None = None) -> np.ndarray:
    """<C> for every set: this rank evaluates its range of the partition with
    ``evaluate(graphs, gammas, betas) -> array`` (one persistent launch on its
    GPU), and ``gather(local_values, rank_range)`` assembles the full vector
    (a torch.distributed all-gather when world > 1). Returns the full vector
    on every rank."""
    gam = np.atleast_2d(np.asarray(gammas, dtype=np.float64))
    bet = np.atleast_2d(np.asarray(betas, dtype=np.float64))
    parts = partition_by_work([n for n, _ in graphs], world)
    a, b = parts[rank]
    local = np.asarray(evaluate(graphs[a:b], gam[a:b], bet[a:b]) if b > a else np.zeros(0), dtype=np.float64)
    if world == 1:
        return local
    if gather is None:
        gather = torch_gather
    pieces = gather(local, parts)
    return np.concatenate([np.asarray(p, dtype=np.float64) for p in pieces])


def torch_gather(local: np.ndarray, parts: list[tuple[int, int]]) -> list[np.ndarray]:
    """All-gather of every rank's values over the default process group (NCCL
    between GPUs, gloo on CPU): each rank's piece is padded to the longest
    range, so the collective has one fixed shape on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size()
    longest = max(b - a for a, b in parts)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    buf = torch.zeros(longest, dtype=torch.float64, device=dev)
    if local.size:
        buf[: local.size] = torch.from_numpy(local).to(dev)
    out = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(out, buf)
    return [out[r][: b - a].cpu().numpy() for r, (a, b) in enumerate(parts)]
