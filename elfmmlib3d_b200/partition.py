"""Work partition across GPUs (one process per GPU, torch.distributed).

The reference runs on one node with OpenMP inside each call
(src/lfmm3drouts.f:204 parallelises over boxes); it has no multi-GPU path.
Here the units that are independent are split across ranks, with no
exchange on the data path:

* many right-hand sides on one geometry (the 64-slip half-space batch):
  every rank holds the geometry, its plans and their stored near fields, and
  evaluates a contiguous block of the right-hand-side columns
  (`rhs_columns`); `all_gather_columns` assembles the full output on every
  rank when the caller wants it there (NCCL over NVLink on GPUs);
* many independent geometries (the uneven batch): problems are assigned by a
  greedy longest-processing-time balance of their cost, n^2 triangle
  evaluations each (`balance_problems`), and every rank evaluates its own.

One problem is never split across GPUs: that would need an exchange of the
locally essential expansions per tree level.
"""
import numpy as np

__all__ = ["rhs_columns", "balance_problems", "all_gather_columns"]


def rhs_columns(nrhs, world, rank):
    """Contiguous block [start, stop) of nrhs right-hand-side columns for
    `rank` of `world`: blocks differ in size by at most one, lower ranks get
    the larger ones."""
    if world < 1 or not 0 <= rank < world or nrhs < 0:
        raise ValueError(f"rhs_columns: nrhs={nrhs} world={world} rank={rank}")
    base, extra = divmod(nrhs, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def balance_problems(costs, world):
    """Greedy longest-processing-time assignment of independent problems to
    `world` ranks: problems in decreasing cost, each to the rank with the
    least total so far (ties to the lower rank).  Returns one list of
    problem indices per rank, each in increasing index order.  The largest
    total is at most 4/3 of the optimum (Graham's bound)."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("balance_problems: world < 1")
    load = np.zeros(world)
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def all_gather_columns(local, nrhs, group=None):
    """Assemble the per-rank blocks of right-hand-side columns (rank r holds
    rows rhs_columns(nrhs, world, r) of a (nrhs, ...) tensor in `local`)
    into the full (nrhs, ...) tensor on every rank.  One all_gather of
    equally sized (padded) blocks; with the NCCL backend the blocks move
    GPU to GPU over NVLink."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    a, b = rhs_columns(nrhs, world, rank)
    if local.shape[0] != b - a:
        raise ValueError(f"all_gather_columns: rank {rank} holds {local.shape[0]} columns, expected {b - a}")
    width = -(-nrhs // world)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: b - a] = local
    blocks = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(blocks, pad, group=group)
    out = []
    for r in range(world):
        s, e = rhs_columns(nrhs, world, r)
        out.append(blocks[r][: e - s])
    return torch.cat(out, dim=0)
