"""Solver results (reference ``src/pyticc/result.py:27-86``)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Timing:
    wall_seconds: float
    cpu_seconds: float


@dataclass(frozen=True)
class ScatteringResult:
    """Propagated and asymptotic log-derivatives and one S matrix per energy."""

    basis: object
    Etot: np.ndarray
    Y_propagated: np.ndarray
    asymptotic_transform: np.ndarray
    L: np.ndarray
    Smat: tuple[np.ndarray, ...]
    timing: Timing | None = None

    @property
    def open_channel_indices(self) -> tuple[np.ndarray, ...]:
        E_int = self.basis.E_int
        return tuple(np.flatnonzero(E_int < e) for e in self.Etot)

    def unitarity_defect(self) -> np.ndarray:
        """max |S^dagger S - I| per energy."""
        return np.asarray([np.abs(s.conj().T @ s - np.eye(s.shape[0])).max() if s.size else 0.0 for s in self.Smat])
