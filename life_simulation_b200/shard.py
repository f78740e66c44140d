"""Many independent worlds over several GPUs, one process per GPU.

The worlds of a sweep do not interact, so an N-GPU job gives every rank a
share of them and runs each share as its own batch: nothing crosses between
GPUs on the data path, and only the small per-world result records come
back (a host-side gather). The reference runs its variants one at a time on
one GPU (Apps/LifePresetLab/main.cpp:718-795); the shares here balance an
estimate of each world's cost by greedy largest-first assignment to the
least-loaded rank (list scheduling in the LPT order, whose makespan is
within 4/3 of the optimum).
"""
from __future__ import annotations

import heapq
import math
from typing import List, Sequence

# Per-pixel cost model of one substep, in seconds, from the kernels'
# measured rates on one B200: the direct path sustains ~25 TFLOP/s of its
# 2 * taps + 12 FLOP per pixel (taps ~ pi R^2 for a disc of radius R); a
# single-kernel spectral step costs ~10 ps per pixel at the sweep's sizes.
DIRECT_FLOP_PER_S = 25e12
SPECTRAL_S_PER_PX = 10e-12


def world_cost(width: int, height: int, radius: float) -> float:
    """Estimated device seconds of one substep of a single-kernel world: the
    cheaper of the direct and the spectral path, as the batch's own autotuner
    would pick."""
    px = float(width) * float(height)
    taps = math.pi * float(radius) ** 2
    direct = px * (2.0 * taps + 12.0) / DIRECT_FLOP_PER_S
    spectral = px * SPECTRAL_S_PER_PX
    return min(direct, spectral)


def partition(costs: Sequence[float], world_size: int) -> List[List[int]]:
    """World indices per rank: largest cost first, each to the rank with the
    least total so far (ties to the lower rank); each share in ascending
    index order. Deterministic, so every rank computes the same split."""
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world_size)]
    shares: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shares]


def loads(costs: Sequence[float], shares: Sequence[Sequence[int]]) -> List[float]:
    """Total estimated cost per rank."""
    return [sum(float(costs[i]) for i in s) for s in shares]


def gather_records(records: Sequence[dict], group=None) -> List[dict]:
    """Every rank's per-world result records (each with an integer "world"
    key), merged in world order on every rank: one all_gather_object of host
    data, after the ranks' device work is done."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return sorted(records, key=lambda r: r["world"])
    parts: List[List[dict]] = [None] * dist.get_world_size(group)  # type: ignore[list-item]
    dist.all_gather_object(parts, list(records), group=group)
    return sorted((r for p in parts for r in p), key=lambda r: r["world"])
