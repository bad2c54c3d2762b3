"""Partial state-to-state cross sections of one (J, parity) block from its S matrices.

The reference stops at S (``src/pyticc/match/smatrix.py:139-223``, ``result.py:39-86``).  The
level-to-level integral cross section of distinguishable collision partners is the
Arthurs–Dalgarno sum; one (J, parity) block contributes

    sigma_{i->f}(E) = pi (2J + 1) / (g_i k_i^2) * sum_{a in i, b in f} |delta_ab - S_ab|^2,

with k_i^2 = 2 mu (E - E_i), g_i = (2 j_X + 1)(2 j_Y + 1) the degeneracy of the initial level
(j = 0 for an atom) and a, b the space-fixed channels (any j12, L) of levels i and f.  Summing
the blocks of every J and both parities gives the integral cross section.  Molecule-exchange
symmetrisation of identical partners is not applied (such channels are not built here).
Units: bohr^2.
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass

import numpy as np
from loguru import logger


@dataclass(frozen=True)
class PartialCrossSections:
    """sigma[e, i, f]: level i -> level f at energy Etot[e] (bohr^2), levels in threshold
    order; rows and columns of levels closed at that energy are zero."""

    Jtot: int
    levels: tuple[tuple[object, object], ...]
    thresholds: np.ndarray
    degeneracy: np.ndarray
    Etot: np.ndarray
    sigma: np.ndarray

    def open_levels(self, e: int) -> np.ndarray:
        return np.flatnonzero(self.thresholds < self.Etot[e])


def _level_labels(basis) -> tuple[list[tuple[object, object]], np.ndarray]:
    levels: dict[tuple[object, object], int] = {}
    index = np.empty(basis.n_channel, dtype=np.int64)
    for c, channel in enumerate(basis):
        key = (channel.mis_X, channel.mis_Y)
        index[c] = levels.setdefault(key, len(levels))
    return list(levels), index


def partial_cross_sections(basis, Etot, Smat: Sequence[np.ndarray], reduced_mass: float) -> PartialCrossSections:
    """Level-to-level partial cross sections from one S matrix per energy, each over the
    channels open at that energy (E_int < E, in channel order), as ``solve`` returns them."""
    energies = np.atleast_1d(np.asarray(Etot, dtype=np.float64))
    if len(Smat) != energies.size:
        message = f"Smat holds {len(Smat)} matrices, but Etot has {energies.size} energies"
        logger.error(message)
        raise ValueError(message)
    if not reduced_mass > 0.0:
        message = f"reduced_mass must be positive, but got {reduced_mass}"
        logger.error(message)
        raise ValueError(message)
    levels, level_of = _level_labels(basis)
    E_int = basis.E_int
    thresholds = np.empty(len(levels))
    degeneracy = np.empty(len(levels))
    for k, (mis_X, mis_Y) in enumerate(levels):
        thresholds[k] = E_int[np.flatnonzero(level_of == k)[0]]
        degeneracy[k] = (2 * mis_X.j + 1) * (2 * mis_Y.j + 1)
    sigma = np.zeros((energies.size, len(levels), len(levels)))
    prefactor = np.pi * (2 * basis.Jtot + 1)
    for e, (energy, S) in enumerate(zip(energies, Smat, strict=True)):
        open_channels = np.flatnonzero(E_int < energy)
        S = np.asarray(S)
        if S.shape != (open_channels.size, open_channels.size):
            message = f"S at energy {e} has shape {S.shape}, but {open_channels.size} channels are open"
            logger.error(message)
            raise ValueError(message)
        if open_channels.size == 0:
            continue
        T2 = np.abs(np.eye(open_channels.size) - S) ** 2
        onehot = np.zeros((open_channels.size, len(levels)))
        onehot[np.arange(open_channels.size), level_of[open_channels]] = 1.0
        summed = onehot.T @ T2 @ onehot
        k2 = 2.0 * reduced_mass * (energy - thresholds)
        with np.errstate(divide="ignore", invalid="ignore"):
            scale = np.where(k2 > 0.0, prefactor / (degeneracy * k2), 0.0)
        sigma[e] = scale[:, None] * summed
    return PartialCrossSections(int(basis.Jtot), tuple(levels), thresholds, degeneracy, energies, sigma)
