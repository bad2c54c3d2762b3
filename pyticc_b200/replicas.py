"""Replica scheduling across GPUs: independent (block, energy batch) units, no exchange.

Every (J, parity) block and every energy is an independent solve, so N GPUs run N
replicas of the single-GPU path over disjoint units (weak scaling).  The only
collectives are the barrier around the timed region and the max-over-ranks reduction of
its duration; the data path has none.
"""

from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Unit:
    """One solve batch: a block index and a half-open range of energy indices."""

    block: int
    start: int
    stop: int


def all_units(n_blocks: int, n_energy: int, batch: int) -> list[Unit]:
    """Every (block, energy batch) unit in a fixed global order."""
    per_block = -(-n_energy // batch)
    return [Unit(b, k * batch, min(n_energy, (k + 1) * batch)) for b in range(n_blocks) for k in range(per_block)]


def rank_units(n_blocks: int, n_energy: int, batch: int, rank: int, world: int, count: int) -> list[Unit]:
    """`count` units for one rank: global units rank, rank + world, ... (cycling), so ranks
    never share a unit within one pass over the workload."""
    units = all_units(n_blocks, n_energy, batch)
    return [units[(rank + world * k) % len(units)] for k in range(count)]


def max_over_ranks(seconds: float, group=None) -> float:
    """The slowest rank's duration (every rank must call this, in the same order)."""
    if group is None:
        return float(seconds)
    import torch

    backend = group.get_backend()
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    group.all_reduce(t, op=group.ReduceOp.MAX)
    return float(t.item())
