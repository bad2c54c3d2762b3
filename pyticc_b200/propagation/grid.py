"""Radial sectors and memory-bounded windows (reference ``src/pyticc/propagation/grid.py``)."""

from __future__ import annotations

from collections.abc import Iterator, Sequence
from dataclasses import dataclass
from math import ceil

import numpy as np
from loguru import logger
from numpy.typing import ArrayLike, NDArray

MAX_SECTORS_PER_WINDOW = 64


@dataclass(frozen=True, slots=True)
class RadialSector:
    """One LDMD sector [radial_start, radial_end]."""

    radial_start: float
    radial_end: float

    @property
    def radial_mid(self) -> float:
        return 0.5 * (self.radial_start + self.radial_end)

    @property
    def radial_half_step(self) -> float:
        return 0.5 * (self.radial_end - self.radial_start)


def build_radial_sectors(radial_boundaries: ArrayLike, radial_half_steps: ArrayLike) -> tuple[RadialSector, ...]:
    """Sectors of width 2h per interval, the last one shortened to end on the boundary;
    a 1e-12 guard keeps round-off from adding a sliver sector (grid.py:193-239)."""
    bounds = np.asarray(radial_boundaries, dtype=np.float64)
    halves = np.asarray(radial_half_steps, dtype=np.float64)
    if bounds.ndim != 1 or halves.ndim != 1 or bounds.size != halves.size + 1:
        message = f"radial_boundaries and radial_half_steps must be one-dimensional with sizes N+1 and N, but got {bounds.shape} and {halves.shape}"
        logger.error(message)
        raise ValueError(message)
    if halves.size == 0:
        message = "At least one radial interval is required"
        logger.error(message)
        raise ValueError(message)
    if not np.all(np.diff(bounds) > 0.0):
        message = "radial_boundaries must be strictly increasing"
        logger.error(message)
        raise ValueError(message)
    sectors: list[RadialSector] = []
    for start, end, h in zip(bounds[:-1].tolist(), bounds[1:].tolist(), halves.tolist(), strict=True):
        width = 2.0 * h
        count = max(1, int(np.ceil((end - start) / width - 1.0e-12)))
        edges = [start + k * width for k in range(count)] + [end]
        sectors.extend(RadialSector(edges[k], edges[k + 1]) for k in range(count))
    return tuple(sectors)


def radial_points_of(sectors: Sequence[RadialSector]) -> NDArray[np.float64]:
    """[start, mid0, end0, mid1, end1, ...] for consecutive sectors."""
    points = np.empty(2 * len(sectors) + 1)
    points[0] = sectors[0].radial_start
    points[1::2] = [s.radial_mid for s in sectors]
    points[2::2] = [s.radial_end for s in sectors]
    return points


def window_size(n_sector: int, *, n_grid: int, n_channel: int, n_energy: int, memory_limit_mb: float, state_matrix_elements: int | None = None) -> int:
    """Sectors per window under the reference's transient-memory model (grid.py:246-309)."""
    largest = n_channel**2
    resident = largest if state_matrix_elements is None else state_matrix_elements
    available = max(0, int(memory_limit_mb * 1024**2) - 32 * n_energy * resident - 8 * (n_grid + 3 * largest))
    return min(n_sector, MAX_SECTORS_PER_WINDOW, max(1, available // max(1, 16 * n_grid + 128 * largest)))


def iter_radial_windows(
    sectors: Sequence[RadialSector], *, n_grid: int, n_channel: int, n_energy: int, memory_limit_mb: float, state_matrix_elements: int | None = None
) -> Iterator[tuple[tuple[RadialSector, ...], NDArray[np.float64]]]:
    """Consecutive windows of sectors and their unique points; neighbours share one point."""
    n_sector = len(sectors)
    if n_sector < 1 or n_grid < 0 or n_channel < 1 or n_energy < 1:
        message = f"Window dimensions must satisfy n_sector >= 1, n_grid >= 0, n_channel >= 1, and n_energy >= 1, but got {(n_sector, n_grid, n_channel, n_energy)}"
        logger.error(message)
        raise ValueError(message)
    size = window_size(n_sector, n_grid=n_grid, n_channel=n_channel, n_energy=n_energy, memory_limit_mb=memory_limit_mb, state_matrix_elements=state_matrix_elements)
    logger.trace(f"Using {ceil(n_sector / size)} radial windows of at most {size} sectors")
    for start in range(0, n_sector, size):
        window = tuple(sectors[start : start + size])
        yield window, radial_points_of(window)
