"""Multi-GPU by release sharding (replicas): releases share nothing but met, so a
batch of releases splits across ranks with no collective on the data path. Each
rank runs its own releases on its own GPU against its own copy of the met; the
only collectives are bookkeeping (max-over-ranks timing, summed counters).
"""

from __future__ import annotations

import numpy as np


def balance_releases(counts, world: int) -> list[np.ndarray]:
    """Partition release indices over ``world`` ranks so particle counts balance:
    longest-processing-time first (largest release to the least-loaded rank).
    Every release lands on exactly one rank; each rank's list is sorted."""
    counts = np.asarray(counts, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    load = np.zeros(world, dtype=np.int64)
    parts: list[list[int]] = [[] for _ in range(world)]
    for r in np.argsort(-counts, kind="stable"):
        k = int(np.argmin(load))
        parts[k].append(int(r))
        load[k] += counts[r]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def rank_particle_mask(release_idx, releases: np.ndarray) -> np.ndarray:
    """Boolean mask of the particles whose release belongs to ``releases``."""
    return np.isin(np.asarray(release_idx), releases)


def local_release_index(release_idx, releases: np.ndarray) -> np.ndarray:
    """Rank-local release numbers (position in ``releases``) of the given particles."""
    lut = np.full(int(max(np.max(releases), np.max(release_idx))) + 1, -1, dtype=np.int64)
    lut[releases] = np.arange(len(releases))
    return lut[np.asarray(release_idx)]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (device timings are reported as the max over ranks)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: int, device=None) -> int:
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return int(value)
    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())
