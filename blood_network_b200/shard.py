"""Sharding of the batched workloads over ranks (one process per GPU).

Both batched workloads split into independent units, so the ranks share no
data while they solve; the host gathers the results afterwards (no device
collective):

* many networks: bin-packed by nonzeros onto the ranks (largest first, each
  to the least loaded rank), every rank packing its share block-diagonally
  into one segmented PCG;
* many right-hand sides of one network: contiguous column blocks, every rank
  holding its own hierarchy of the same matrix.

The gather uses torch.distributed's object collectives, so it runs on any
backend (gloo for the CPU tests, nccl on the GPUs).
"""
from typing import Callable, List, Sequence

import numpy as np


def partition_networks(nnz: Sequence[int], world_size: int) -> List[List[int]]:
    """Longest-processing-time bin packing: network indices per rank, each
    rank's list in increasing index order.  Ties go to the lower rank."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(nnz)), key=lambda i: (-int(nnz[i]), i))
    load = [0] * world_size
    parts: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += int(nnz[i])
    return [sorted(p) for p in parts]


def partition_columns(k: int, world_size: int) -> List[range]:
    """Contiguous column blocks, sizes differing by at most one."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    base, extra = divmod(k, world_size)
    out, c0 = [], 0
    for r in range(world_size):
        c1 = c0 + base + (1 if r < extra else 0)
        out.append(range(c0, c1))
        c0 = c1
    return out


def _rank_world(group=None):
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def solve_networks_distributed(nets, solve_fn: Callable, group=None):
    """Solve independent networks across the ranks of the process group.

    solve_fn(list_of_networks) -> list of (x, iterations) in the same order;
    every rank calls this with the same `nets` and gets the full result list
    back in the original order."""
    import torch.distributed as dist
    rank, ws = _rank_world(group)
    parts = partition_networks([nt.nnz for nt in nets], ws)
    mine = parts[rank]
    res = solve_fn([nets[i] for i in mine]) if mine else []
    local = list(zip(mine, res))
    if ws == 1:
        gathered = [local]
    else:
        gathered = [None] * ws
        dist.all_gather_object(gathered, local, group=group)
    out = [None] * len(nets)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out


def solve_columns_distributed(B: np.ndarray, solve_fn: Callable, group=None):
    """Solve the columns of B (n x k) across the ranks, each rank a
    contiguous block.  solve_fn(B_block) -> (X_block, iterations_block);
    every rank gets the full (X, iterations)."""
    import torch.distributed as dist
    rank, ws = _rank_world(group)
    cols = partition_columns(B.shape[1], ws)[rank]
    if len(cols):
        X, its = solve_fn(np.asfortranarray(B[:, cols.start:cols.stop]))
        local = (cols.start, np.asarray(X), np.asarray(its))
    else:
        local = (cols.start, np.zeros((B.shape[0], 0)), np.zeros(0, np.int32))
    if ws == 1:
        gathered = [local]
    else:
        gathered = [None] * ws
        dist.all_gather_object(gathered, local, group=group)
    gathered.sort(key=lambda t: t[0])
    X = np.concatenate([g[1] for g in gathered], axis=1)
    its = np.concatenate([g[2] for g in gathered])
    return X, its
