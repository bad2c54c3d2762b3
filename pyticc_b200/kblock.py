"""Coupled-states (CS) and nearest-neighbour-K (NNCC) channel blocks.

Mirrors ``src/pyticc/basis/kblock.py:17-158``: a CS system propagates one block per
helicity K; an NNCC system propagates overlapping windows of K values around each
centre and takes the result for each incoming K from exactly one window (its owner).
The blocks only select channels; the block propagation itself is the batched LDMD of
``ticc_ldmd_propagate_blocks``.
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass

from loguru import logger


@dataclass(frozen=True)
class KBlock:
    """One propagation block: the K window it propagates and the K values it owns
    (reference ``basis/kblock.py:17-45``)."""

    index: int
    center_K: float
    K_delta: int
    K_values: tuple[float, ...]
    channel_indices: tuple[int, ...]
    owned_K_values: tuple[float, ...]
    owned_channel_indices: tuple[int, ...]

    def __str__(self) -> str:
        return (
            f"KBlock[{self.index}] center_K={self.center_K} K_delta={self.K_delta} K_values={self.K_values} "
            f"N_channel={len(self.channel_indices)} owned_K_values={self.owned_K_values} N_owned={len(self.owned_channel_indices)}"
        )


def _positions(channels, accept) -> tuple[int, ...]:
    return tuple(position for position, channel in enumerate(channels) if accept(channel.K))


def build_cs_blocks(channels: Sequence) -> tuple[KBlock, ...]:
    """One block per distinct K, owning its own channels (kblock.py:53-81)."""
    blocks = []
    for number, K in enumerate(sorted({channel.K for channel in channels})):
        members = _positions(channels, lambda k, K=K: k == K)
        blocks.append(KBlock(number, K, 0, (K,), members, (K,), members))
    return tuple(blocks)


def build_nncc_blocks(channels: Sequence, K_delta: int = 1) -> tuple[KBlock, ...]:
    """Windows |K - K_c| <= K_delta around the centres K_delta .. K_count-1-K_delta of the
    K ladder (a single middle centre when one window spans the ladder); incoming K is
    owned by the centre nearest to it, clamped to the first and last centre
    (kblock.py:88-158)."""
    if isinstance(K_delta, bool) or not isinstance(K_delta, int) or K_delta < 1:
        message = f"NNCC requires K_delta >= 1, but got K_delta={K_delta}"
        logger.error(message)
        raise ValueError(message)
    if len(channels) == 0:
        return ()
    helicities = [channel.K for channel in channels]
    K_low, K_high = min(helicities), max(helicities)
    on_ladder = 2 * K_low == round(2 * K_low) and all(K >= 0 and K - K_low == round(K - K_low) for K in helicities)
    if not on_ladder:
        raise ValueError("NNCC channels must belong to one nonnegative integer or half-integer K ladder")
    count = int(K_high - K_low) + 1
    ladder = tuple(K_low + step for step in range(count))
    centres = (ladder[(count - 1) // 2],) if 2 * K_delta + 1 >= count else ladder[K_delta : count - K_delta]

    def owner(K: float) -> float:
        return min(max(K, centres[0]), centres[-1])

    blocks = []
    for number, centre in enumerate(centres):
        lo, hi = max(K_low, centre - K_delta), min(K_high, centre + K_delta)
        blocks.append(
            KBlock(
                number,
                centre,
                K_delta,
                tuple(K for K in ladder if lo <= K <= hi),
                _positions(channels, lambda k, lo=lo, hi=hi: lo <= k <= hi),
                tuple(K for K in ladder if owner(K) == centre),
                _positions(channels, lambda k, centre=centre: owner(k) == centre),
            )
        )
    return tuple(blocks)
