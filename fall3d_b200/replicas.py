"""Multi-GPU plumbing for independent ensemble members (replicas).

FALL3D runs ensemble members in separate MPI communicators that never
exchange data during the time loop (mod_Parallel.F90:188-217), so members
shard across GPUs with no data-path collective.  torch.distributed is used
only for the barrier around timed regions and max/sum reductions of
scalars; NCCL on GPUs, gloo on CPU.
"""
from __future__ import annotations


def partition_members(costs, world_size: int, rank: int):
    """Members owned by `rank`: greedy longest-processing-time assignment of
    the per-member costs (cell*bins) so every rank gets a similar load.
    Deterministic: every rank computes the same partition."""
    order = sorted(range(len(costs)), key=lambda m: (-costs[m], m))
    load = [0.0] * world_size
    owner = [0] * len(costs)
    for m in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        owner[m] = r
        load[r] += costs[m]
    return [m for m in range(len(costs)) if owner[m] == rank], load


def _tensor(x, pg_mod, device):
    import torch
    return torch.tensor([float(x)], dtype=torch.float64, device=device)


def reduce_max(x: float, pg_mod=None, device="cpu") -> float:
    """Max over ranks (device time of the slowest rank)."""
    if pg_mod is None or not pg_mod.is_initialized() or pg_mod.get_world_size() == 1:
        return float(x)
    t = _tensor(x, pg_mod, device)
    pg_mod.all_reduce(t, op=pg_mod.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float, pg_mod=None, device="cpu") -> float:
    if pg_mod is None or not pg_mod.is_initialized() or pg_mod.get_world_size() == 1:
        return float(x)
    t = _tensor(x, pg_mod, device)
    pg_mod.all_reduce(t, op=pg_mod.ReduceOp.SUM)
    return float(t.item())
