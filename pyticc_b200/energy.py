"""Total-energy input validation (reference ``src/pyticc/energy.py:12-55``)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
from loguru import logger


def get_Etot(source) -> np.ndarray:
    """Read-only float64 (n_energy,) array from an array-like or a one-column text file."""
    if isinstance(source, (str, Path)):
        try:
            energies = np.loadtxt(Path(source), dtype=np.float64, comments="#", ndmin=1)
        except (OSError, ValueError) as error:
            message = f"Failed to read total energies from {source}: {error}"
            logger.error(message)
            raise ValueError(message) from error
    else:
        try:
            energies = np.asarray(source.cpu() if hasattr(source, "cpu") else source, dtype=np.float64)
        except (TypeError, ValueError) as error:
            message = f"Failed to convert total energies to an array: {error}"
            logger.error(message)
            raise ValueError(message) from error
    if energies.ndim != 1:
        message = f"Total energies must be one-dimensional, but got shape={energies.shape}"
        logger.error(message)
        raise ValueError(message)
    if energies.size == 0:
        message = "At least one total energy is required"
        logger.error(message)
        raise ValueError(message)
    if not np.all(np.isfinite(energies)):
        message = "Total energies must be finite"
        logger.error(message)
        raise ValueError(message)
    energies = energies.copy()
    energies.setflags(write=False)
    return energies
