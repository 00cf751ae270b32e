"""Multi-GPU host logic: independent systems sharded across ranks.

One pressure system never spans GPUs (the whole theta x z domain stays on
one device), so there is no data-path collective: batches of systems and
serving streams are partitioned across ranks by footprint and estimated
work, each rank solves its share on its own GPU, and only timings and small
per-system results travel, on the host side, through torch.distributed
(NCCL on GPU ranks, gloo for CPU-side checks).

The reference's own parallelism -- MPI domain decomposition with two-layer
halos and scalar allreduces (src/mod_mpi_topology.f90:79-285,291-417) -- is
not used: it would split a single system, which this design never does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass


@dataclass(frozen=True)
class Item:
    """One independent system or run to place."""
    key: int
    cells: int
    footprint: float   # device bytes
    work: float        # estimated cost (any unit, e.g. cell-iterations)


def estimated_work(nr: int, nth: int, nz: int) -> float:
    """Cell-iterations of a solve to 1e-8 on these meshes (iterations grow
    about as 8 sqrt(cells) for the synthetic furnace operators)."""
    n = nr * nth * nz
    return n * 8.0 * math.sqrt(n)


def device_footprint(nr: int, nth: int, nz: int, mixed: bool = False) -> float:
    """Device bytes of one resident system (compact FP64 state, halo-layout
    staging, FP32 shadow when mixed) -- the server's admission figure."""
    n = nr * nth * nz
    nh = (nr + 4) * (nth + 4) * (nz + 4)
    b = n * 8 * 14 + nh * 8 * 9 + 256
    if mixed:
        b += n * 4 * 13
    return float(b)


def partition(items: list[Item], n_ranks: int,
              budget: float | None = None) -> list[list[Item]]:
    """Longest-processing-time assignment: items by decreasing work, each to
    the rank with the least assigned work that still has room in its device
    budget. Deterministic (ties go to the lower rank). Raises if an item
    fits on no rank."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    load = [0.0] * n_ranks
    used = [0.0] * n_ranks
    out: list[list[Item]] = [[] for _ in range(n_ranks)]
    for it in sorted(items, key=lambda i: (-i.work, i.key)):
        order = sorted(range(n_ranks), key=lambda r: (load[r], r))
        for r in order:
            if budget is None or used[r] + it.footprint <= budget:
                out[r].append(it)
                load[r] += it.work
                used[r] += it.footprint
                break
        else:
            raise RuntimeError(f"item {it.key} ({it.footprint:.3g} B) fits on no rank")
    return out


def reduce_timing(elapsed_s: float, units: float, group=None) -> tuple[float, float]:
    """(max elapsed over ranks, total units over ranks): the whole-job time is
    the slowest rank's, the work is everybody's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return elapsed_s, units
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([elapsed_s], dtype=torch.float64, device=dev)
    u = torch.tensor([units], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(u, op=dist.ReduceOp.SUM, group=group)
    return float(t.item()), float(u.item())


def gather_results(local: dict, group=None) -> dict:
    """Per-key results of every rank, merged on every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return dict(local)
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    merged = {}
    for p in parts:
        overlap = set(merged) & set(p)
        if overlap:
            raise RuntimeError(f"keys solved on two ranks: {sorted(overlap)[:5]}")
        merged.update(p)
    return merged


class ShardError(RuntimeError):
    """A rank's share failed; raised on every rank of the collective."""


def gather_outcomes(fn, group=None) -> list:
    """Collective over `group` (or a single process when torch.distributed is
    not initialised): run `fn()` on every rank and return every rank's result,
    in rank order, on every rank. Each rank takes exactly one collective step
    (an object all-gather of its error and result), also when `fn` raised, so
    a failure on one rank cannot leave the others waiting: every rank then
    raises ShardError naming the failed ranks."""
    import torch.distributed as dist
    on = dist.is_available() and dist.is_initialized()
    err, out = None, None
    try:
        out = fn()
    except Exception as exc:  # reported to every rank below
        err = f"{type(exc).__name__}: {exc}"
    if on:
        gathered = [None] * dist.get_world_size(group)
        dist.all_gather_object(gathered, (err, out), group=group)
    else:
        gathered = [(err, out)]
    failed = [(r, e) for r, (e, _) in enumerate(gathered) if e is not None]
    if failed:
        raise ShardError("; ".join(f"rank {r}: {e}" for r, e in failed))
    return [o for _, o in gathered]


def solve_sharded(items: list[Item], solve_share, group=None,
                  budget: float | None = None) -> tuple[float, dict, list[list[Item]]]:
    """Collective over `group`: partition `items` across the ranks
    (`partition`), call `solve_share(my_items) -> (elapsed_s, {key: result})`
    on every rank with its share, and return (the slowest rank's elapsed
    seconds, the results of every rank merged by key, the partition) on every
    rank; failures as in `gather_outcomes`."""
    import torch.distributed as dist
    on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if on else 1
    rank = dist.get_rank(group) if on else 0
    parts = partition(items, world, budget)
    outs = gather_outcomes(lambda: solve_share(parts[rank]), group)
    merged: dict = {}
    for _, p in outs:
        overlap = set(merged) & set(p)
        if overlap:
            raise RuntimeError(f"keys solved on two ranks: {sorted(overlap)[:5]}")
        merged.update(p)
    return max(float(t) for t, _ in outs), merged, parts
