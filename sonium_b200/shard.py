"""Independent work spread over ranks (one process per GPU), with no collective on the data path.

The instances of a frequency sweep (one mesh, wavenumber and right-hand side each) and the groups
of right-hand sides of one operator are independent solves. A run on several GPUs therefore gives
each rank a share and gathers the solutions once at the end; nothing is exchanged while the
ranks assemble and solve. This is the role of the reference's deterministic ownership planners
(the Morton row partition of crates/sonium-bem/src/core/distributed.rs:18-60 and the batch planner
plan_bem_batch, crates/sonium-bem/src/core/scheduling.rs:98), applied here at the granularity
that shards without communication: whole instances and whole right-hand-side groups.

* ``partition_by_cost``: the instances' costs (N^2 for a dense solve: assembly and every product
  scale with the matrix) go to ranks largest first, each to the rank with the least total so far
  (ties to the lower rank); every rank's list is returned in ascending instance order, so the
  partition is deterministic and the same on every rank.
* ``rhs_groups``: right-hand sides in contiguous groups of the tensor-core tile (128), dealt to
  ranks the same way (their costs are equal).
* ``gather_ordered``: each rank's results (one array per local instance) gathered to every rank
  in the global instance order, with torch.distributed (gloo or NCCL; one all_gather_object).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np

RHS_GROUP = 128  # right-hand sides per tensor-core block product tile


def partition_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time partition of items with the given costs over `world` ranks."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def dense_solve_costs(sizes: Sequence[int]) -> list[float]:
    """Cost model of one dense solve of N unknowns: N^2 (matrix entries assembled and streamed)."""
    return [float(n) * float(n) for n in sizes]


def rhs_groups(r: int, world: int, group: int = RHS_GROUP) -> list[list[tuple[int, int]]]:
    """Right-hand sides 0..r-1 in contiguous groups of `group`, groups dealt over the ranks:
    per rank a list of (start, stop) column ranges."""
    spans = [(s, min(r, s + group)) for s in range(0, r, group)]
    parts = partition_by_cost([stop - start for start, stop in spans], world)
    return [[spans[g] for g in p] for p in parts]


def balance(costs: Sequence[float], parts: Sequence[Sequence[int]]) -> float:
    """Largest rank load over the mean load (1.0 = perfect)."""
    loads = [sum(float(costs[i]) for i in p) for p in parts]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0


def gather_ordered(local_ids: Sequence[int], local_results: Sequence[np.ndarray], total: int,
                   dist=None) -> list[np.ndarray]:
    """Results of every instance in global order, on every rank. Without a process group (or with
    one rank) the local results are the whole set."""
    if len(local_ids) != len(local_results):
        raise ValueError("one result per local instance")
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        pairs = list(zip(local_ids, local_results))
    else:
        shards = [None] * dist.get_world_size()
        dist.all_gather_object(shards, [(int(i), np.asarray(x)) for i, x in zip(local_ids, local_results)])
        pairs = [p for s in shards for p in s]
    out: list = [None] * total
    for i, x in pairs:
        if out[i] is not None:
            raise ValueError(f"instance {i} solved by two ranks")
        out[i] = x
    missing = [i for i, x in enumerate(out) if x is None]
    if missing:
        raise ValueError(f"instances {missing[:8]} solved by no rank")
    return out


def sharded_solve(costs: Sequence[float], solve_subset: Callable[[list[int]], list[np.ndarray]], dist=None,
                  rank: int = 0, world: int = 1) -> tuple[list[np.ndarray], list[int]]:
    """Solve this rank's share of the instances with `solve_subset` (instance ids in ascending
    order -> one solution each) and gather all solutions in global order. Returns (solutions,
    this rank's instance ids)."""
    parts = partition_by_cost(costs, world)
    mine = parts[rank]
    local = solve_subset(mine) if mine else []
    return gather_ordered(mine, local, len(costs), dist), mine


def sharded_sweep(meshes, physics, betas, direction, config, dist=None, rank: int = 0, world: int = 1,
                  inner_precision: int | None = None, block_jacobi: int = 0):
    """A batched frequency sweep with its instances spread over ranks: each rank assembles and
    solves its share as one SweepBatch (persistent or two-stream assembly, batched mixed GMRES),
    then the solutions are gathered in instance order. Returns (solutions, this rank's ids)."""
    from . import _lib as L
    from .sweep import SweepBatch

    sizes = [m.num_elements for m in meshes]

    def solve_subset(ids):
        batch = SweepBatch([meshes[i] for i in ids], [physics[i] for i in ids], [betas[i] for i in ids])
        try:
            if inner_precision is not None:
                batch.set_inner_precision(inner_precision)
            if block_jacobi:
                batch.set_inner_preconditioner(L.SB_INNER_PRECOND_BLOCK_JACOBI, block_jacobi)
            batch.assemble()
            batch.set_rhs_plane_wave(direction)
            batch.solve(config)
            return [batch.solution(q) for q in range(len(ids))]
        finally:
            batch.close()

    return sharded_solve(dense_solve_costs(sizes), solve_subset, dist, rank, world)
