"""Partition of independent worlds over ranks (one process per GPU).

Worlds of a group never interact (PhysicsWorld::update touches only its own
world's components), so a multi-GPU run gives every rank one contiguous
block of worlds and steps it with no exchange during the steps.  The only
collectives are end-of-run gathers: the max-over-ranks step time and, where
a caller wants them, the per-world results.

Blocks are balanced by a per-world cost (the body count is the natural one:
broad phase, narrow phase, islands and the solver all grow with it); the
split is a pure function of the cost list and the rank count, so every rank
computes the same blocks without communicating.
"""
import numpy as np


def block_bounds(costs, world_size):
    """Boundaries [b_0 = 0, b_1, ..., b_W = n] of W contiguous blocks whose
    cost sums are as even as a contiguous split allows: block r ends at the
    first world where the running cost reaches (r + 1) / W of the total.
    Every block is non-empty when there are at least W worlds."""
    c = np.asarray(costs, dtype=np.float64)
    n = len(c)
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    if n == 0:
        return [0] * (world_size + 1)
    if np.any(c < 0):
        raise ValueError("costs must be non-negative")
    prefix = np.cumsum(c)
    total = prefix[-1]
    bounds = [0]
    for r in range(1, world_size):
        if total > 0:
            b = int(np.searchsorted(prefix, total * r / world_size, side="left")) + 1
        else:
            b = (n * r) // world_size
        # keep at least one world per remaining block when there are enough
        lo = bounds[-1] + (1 if n - bounds[-1] >= world_size - r + 1 else 0)
        hi = n - (world_size - r) if n >= world_size else n
        bounds.append(int(min(max(b, lo), max(hi, lo))))
    bounds.append(n)
    return bounds


def rank_block(costs, rank, world_size):
    """(lo, hi): the worlds [lo, hi) that rank `rank` steps."""
    if not 0 <= rank < world_size:
        raise ValueError("rank out of range")
    b = block_bounds(costs, world_size)
    return b[rank], b[rank + 1]


def gather_objects(obj):
    """Every rank's `obj`, in rank order (torch.distributed, any backend);
    [obj] when no process group is initialised."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def max_over_ranks(value):
    """The maximum of a float over all ranks (the slowest rank's time)."""
    return max(float(v) for v in gather_objects(float(value)))
