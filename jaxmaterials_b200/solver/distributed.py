"""Many structures over several GPUs: one process per GPU, independent shards.

Every (structure, load case) solve is independent, so a dataset is split across ranks
with no collective inside the solve: structures are assigned by greedy
longest-processing-time-first packing on their voxel counts (the iteration counts of the
batched workload hardly depend on the grid size, so voxels are the work), every rank
solves its shard with lsb_c_eff_batch, and one all-gather of the small results (6x6
C_eff, iterations and status per structure) assembles the dataset on every rank.
"""

import heapq

import numpy as np


def assign_lpt(work, world):
    """Rank of every item: items in decreasing `work`, each to the least loaded rank
    (ties to the lower rank). Returns an int array of len(work)."""
    work = np.asarray(work, dtype=np.float64)
    owner = np.zeros(len(work), dtype=np.int64)
    heap = [(0.0, r) for r in range(world)]
    for i in sorted(range(len(work)), key=lambda i: (-work[i], i)):
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + work[i], r))
    return owner


def c_eff_batch_sharded(lmbdas, mus, grid_specs, group=None, solve=None, **kwargs):
    """C_eff of the whole dataset on every rank of `group` (torch.distributed; the
    default group if None). Each rank solves the structures assign_lpt gives it with
    `solve` (default solver.c_eff_batch, keyword arguments passed on) and the results
    are all-gathered. Returns (C [n, 6, 6], iters [n, 6], status [n, 6], owner [n])."""
    import torch.distributed as dist

    if solve is None:
        from .batch import c_eff_batch as solve
    n = len(lmbdas)
    if not isinstance(grid_specs, (list, tuple)):
        grid_specs = [grid_specs] * n
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    owner = assign_lpt([g.nx * g.ny * g.nz for g in grid_specs], world)
    mine = np.flatnonzero(owner == rank)
    if len(mine):
        c, it, st = solve([lmbdas[i] for i in mine], [mus[i] for i in mine],
                          [grid_specs[i] for i in mine], **kwargs)
    else:
        c = np.zeros((0, 6, 6))
        it = np.zeros((0, 6), dtype=np.int32)
        st = np.zeros((0, 6), dtype=np.int32)
    parts = [None] * world
    dist.all_gather_object(parts, (mine, np.asarray(c), np.asarray(it), np.asarray(st)),
                           group=group)
    C = np.zeros((n, 6, 6))
    iters = np.zeros((n, 6), dtype=np.int32)
    status = np.zeros((n, 6), dtype=np.int32)
    seen = np.zeros(n, dtype=np.int64)
    for idx, c, it, st in parts:
        C[idx], iters[idx], status[idx] = c, it, st
        seen[idx] += 1
    if not (seen == 1).all():
        raise RuntimeError("a structure was solved by no rank or by several")
    return C, iters, status, owner
