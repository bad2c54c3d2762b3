"""Interaction PES wrapper and tensor-grid evaluation (reference ``src/pyticc/pes/adiabatic.py``).

PES evaluation is geometry setup: it runs on the host once per PotentialGrid."""

from __future__ import annotations

from collections.abc import Callable
from dataclasses import dataclass

import numpy as np
from loguru import logger


@dataclass(frozen=True)
class PESWrapper:
    """interaction(R, coordinates (n_coord, n_grid)) -> (n_grid,); optional batched
    interaction_many(R (n_R,), coordinates) -> (n_R, n_grid)."""

    interaction: Callable
    monomer_X: Callable | None = None
    monomer_Y: Callable | None = None
    interaction_many: Callable | None = None


def _evaluate(pes: PESWrapper, R, coordinates: np.ndarray, grid_shape: tuple[int, ...]) -> np.ndarray:
    points = np.asarray(R, dtype=np.float64)
    if points.ndim == 0:
        values = np.asarray(pes.interaction(float(points), coordinates), dtype=np.float64)
        expected, out_shape = (coordinates.shape[1],), grid_shape
    elif points.ndim == 1:
        if pes.interaction_many is not None:
            values = np.asarray(pes.interaction_many(points, coordinates), dtype=np.float64)
        else:
            values = np.stack([np.asarray(pes.interaction(float(r), coordinates), dtype=np.float64) for r in points]) if points.size else np.empty((0, coordinates.shape[1]))
        expected, out_shape = (points.size, coordinates.shape[1]), (points.size, *grid_shape)
    else:
        message = f"R must be a scalar or one-dimensional array, but got shape {points.shape}"
        logger.error(message)
        raise ValueError(message)
    if values.shape != expected:
        message = f"Interaction PES returned shape {values.shape}, but expected {expected}"
        logger.error(message)
        raise ValueError(message)
    return values.reshape(out_shape)


def get_Vgrid_atom_diatom(pes: PESWrapper, R, r: np.ndarray, theta: np.ndarray) -> np.ndarray:
    """PES on the (r, theta) tensor grid: coordinates rows (r, theta)."""
    grids = np.meshgrid(r, theta, indexing="ij")
    coordinates = np.asfortranarray(np.stack([g.ravel() for g in grids]))
    return _evaluate(pes, R, coordinates, grids[0].shape)


def get_Vgrid_diatom_diatom(pes: PESWrapper, R, r_X, r_Y, theta_X, theta_Y, phi) -> np.ndarray:
    """PES on the (r_X, r_Y, theta_X, theta_Y, phi) tensor grid."""
    grids = np.meshgrid(r_X, r_Y, theta_X, theta_Y, phi, indexing="ij")
    coordinates = np.asfortranarray(np.stack([g.ravel() for g in grids]))
    return _evaluate(pes, R, coordinates, grids[0].shape)
