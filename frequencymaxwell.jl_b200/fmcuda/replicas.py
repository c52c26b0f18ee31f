"""Replicas over right-hand sides for several GPUs (one process per GPU, torch.distributed).

The solve path has no exchange inside the iteration: right-hand sides (illuminations) and requests are
independent given the potential.  So several GPUs run independent replicas: every rank builds the potential
on its own device, solves its share of the right-hand sides and, when asked, the shares are gathered on rank 0.
There is no collective on the data path; the only collectives are the gather of results and the maximum of
per-rank timings.  (New; the reference runs on one device.)
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def shard(n: int, world: int, rank: int, costs: Optional[Sequence[float]] = None) -> List[int]:
    """Indices of the items rank ``rank`` of ``world`` handles.

    Without costs: round robin.  With costs: greedy longest-processing-time assignment (items sorted by
    decreasing cost, each to the least-loaded rank; ties to the lowest rank), which every rank computes the same
    way, so no communication is needed."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    if costs is None:
        return list(range(rank, n, world))
    if len(costs) != n:
        raise ValueError("one cost per item")
    load = [0.0] * world
    owner = [0] * n
    for i in sorted(range(n), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(n) if owner[i] == rank]


def max_over_ranks(value: float) -> float:
    """Maximum of ``value`` over all ranks of the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def solve_batch_sharded(solve_batch: Callable, solver, sources_list: Sequence, medium,
                        gather: bool = True, group=None) -> Tuple[List[int], list, Optional[list]]:
    """Solve this rank's share of ``sources_list`` with ``solve_batch(solver, share, medium)`` (a list of
    ElectromagneticField in share order).

    Returns (indices of this rank's share, its fields, and on rank 0 with ``gather`` the fields of all right-hand
    sides in their original order; None elsewhere).  The gather moves the E and H arrays as complex128 CPU tensors
    over a gloo group (``group``, or one created here by every rank) with one tensor gather per rank block; nothing
    is pickled.  Every rank must call this with the same ``sources_list`` length and grid."""
    import torch
    import torch.distributed as dist
    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size() if dist_on else 1
    rank = dist.get_rank() if dist_on else 0
    n = len(sources_list)
    idx = shard(n, world, rank)
    mine = solve_batch(solver, [sources_list[i] for i in idx], medium) if idx else []
    if not gather:
        return idx, mine, None
    if world == 1:
        return idx, mine, list(mine)
    from .fields import ElectromagneticField
    if group is None:
        group = dist.new_group(backend="gloo")
    # the grid shape and the field metadata come from rank 0's first field (rank 0 always has a share when n > 0)
    meta = [None]
    if rank == 0:
        f0 = mine[0]
        meta = [(tuple(f0.E.shape), f0.resolution, f0.wavelength)]
    dist.broadcast_object_list(meta, src=0, group=group)
    shape, resolution, wavelength = meta[0]
    n_max = (n + world - 1) // world  # round robin: the largest share
    # complex values travel as (re, im) FP64 pairs
    buf = torch.zeros((n_max, 2) + shape + (2,), dtype=torch.float64)
    for j, f in enumerate(mine):
        for k, a in enumerate((f.E, f.H)):
            buf[j, k] = torch.view_as_real(torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128)))
    parts = [torch.empty_like(buf) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, parts, dst=0, group=group)
    if rank != 0:
        return idx, mine, None
    out = [None] * n
    for r in range(world):
        blk = torch.view_as_complex(parts[r]).numpy()
        for j, i in enumerate(shard(n, world, r)):
            out[i] = ElectromagneticField(np.asfortranarray(blk[j, 0]), np.asfortranarray(blk[j, 1]), resolution,
                                          wavelength)
    return idx, mine, out
