"""Multi-GPU plumbing for batches of independent grids.

Grids never exchange data, so a batch shards by grid with no collective on the
data path: each rank (one process per GPU, torch.distributed for the plumbing)
advances its own subset, and the only exchange is a final host gather of
per-grid digests.  The reference has no multi-process path (one OpenMP team,
CPUBenchmark.cpp:63-85).
"""
import hashlib


def partition(cells, world):
    """Longest-processing-time greedy split of grid indices over `world` ranks,
    balancing total cells (cells[i] = n_i^2).  Deterministic: ties go to the
    lowest rank and equal grids keep index order."""
    order = sorted(range(len(cells)), key=lambda i: (-cells[i], i))
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += cells[i]
    return [sorted(p) for p in parts]


def digest(grid):
    """SHA-256 of a grid's cells (uint8 0/1, row-major)."""
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(grid, dtype=np.uint8).tobytes()).hexdigest()


def gather_digests(local):
    """All ranks' {grid index: digest} merged on every rank (torch.distributed
    must be initialised; works with the gloo and nccl backends)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return dict(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, dict(local))
    merged = {}
    for d in out:
        merged.update(d)
    return merged
