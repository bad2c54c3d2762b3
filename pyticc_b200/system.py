"""System description for field-free atom-diatom (A+BC) and diatom-diatom (AB+CD) scattering.

Mirrors the reference's ``build_ScattSystem`` / ``ScattSystem`` / ``ChannelSpec``
(``src/pyticc/system.py:243-299,307-420,466-777``) for the two geometries on this
library's path.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, replace
from enum import Enum

import numpy as np
from loguru import logger


class MonomerType(Enum):
    ATOM = "atom"
    DIATOM = "diatom"


class Approx(Enum):
    EXACT = "exact"
    CS = "cs"
    NNCC = "nncc"


class ScatteringType(Enum):
    ATOM_DIATOM = "A+BC"
    DIATOM_DIATOM = "AB+CD"


@dataclass(frozen=True)
class MolInnerState:
    """One monomer internal state (rotational j, vibrational v or None for an atom)."""

    j: int
    v: int | None = None
    Eint: float = 0.0


@dataclass(frozen=True)
class ChannelSpec:
    """Channel selections: lowest v, rotational exchange parity (-1 odd, 0 all, 1 even j),
    monomer energy cutoffs (hartree) and an optional helicity cutoff."""

    vmin_X: int = 0
    vmin_Y: int = 0
    exchange_parity_X: int = 0
    exchange_parity_Y: int = 0
    E_X_cut: float = math.inf
    E_Y_cut: float = math.inf
    K_cut: int | None = None

    def __post_init__(self) -> None:
        if self.vmin_X < 0 or self.vmin_Y < 0:
            message = f"vmin must be non-negative, but got {self.vmin_X}, {self.vmin_Y}"
            logger.error(message)
            raise ValueError(message)
        if self.exchange_parity_X not in (-1, 0, 1) or self.exchange_parity_Y not in (-1, 0, 1):
            message = "exchange parity must be -1, 0, or 1"
            logger.error(message)
            raise ValueError(message)
        if self.K_cut is not None and self.K_cut < 0:
            message = f"K_cut must be non-negative, but got K_cut={self.K_cut}"
            logger.error(message)
            raise ValueError(message)


@dataclass(frozen=True)
class ScattSystem:
    """A prepared scattering block: monomers, (J, parity), PES, collision reduced mass, channels."""

    monomer_X: object
    monomer_Y: object
    Jtot: int
    system_parity: int
    potential: object = None
    reduced_mass: float | None = None
    channel_spec: ChannelSpec = ChannelSpec()
    approx: Approx = Approx.EXACT
    scattering_type: ScatteringType | None = None
    basis: object = None
    K_delta: int = 1

    def __post_init__(self) -> None:
        if self.system_parity not in (-1, 1):
            message = f"system_parity must be -1 or 1, but got {self.system_parity}"
            logger.error(message)
            raise ValueError(message)
        if self.Jtot < 0:
            message = f"Jtot must be non-negative, but got {self.Jtot}"
            logger.error(message)
            raise ValueError(message)
        if self.K_delta < 1:
            message = f"Invalid K_delta {self.K_delta}. Must be positive."
            logger.error(message)
            raise ValueError(message)

    @property
    def n_channel(self) -> int:
        return 0 if self.basis is None else self.basis.n_channel


def _infer_type(monomer_X, monomer_Y) -> ScatteringType:
    types = (monomer_X.type, monomer_Y.type)
    if types == (MonomerType.ATOM, MonomerType.DIATOM):
        return ScatteringType.ATOM_DIATOM
    if types == (MonomerType.DIATOM, MonomerType.DIATOM):
        return ScatteringType.DIATOM_DIATOM
    message = f"Unsupported monomer pair {types}: this library covers A+BC and AB+CD field-free scattering"
    logger.error(message)
    raise TypeError(message)


def build_ScattSystem(
    monomer_X,
    monomer_Y,
    *,
    Jtot: int,
    system_parity: int,
    channel: ChannelSpec | None = None,
    approx: Approx = Approx.EXACT,
    K_delta: int = 1,
    potential=None,
    reduced_mass: float | None = None,
) -> ScattSystem:
    """Build a system and its channel basis (reference ``system.py:466-777``, field-free branch).

    ``approx`` selects exact coupled channels, coupled states (one block per K) or NNCC
    (overlapping windows of 2 K_delta + 1 helicities)."""
    from .basis import build_ChannelBasis

    if not isinstance(approx, Approx):
        message = f"approx must be an Approx, but got {approx!r}"
        logger.error(message)
        raise TypeError(message)
    if reduced_mass is not None and (not np.isfinite(reduced_mass) or reduced_mass <= 0.0):
        message = f"reduced_mass must be positive, but got {reduced_mass}"
        logger.error(message)
        raise ValueError(message)
    spec = ChannelSpec() if channel is None else channel
    system = ScattSystem(monomer_X, monomer_Y, Jtot, system_parity, potential, reduced_mass, spec, approx, _infer_type(monomer_X, monomer_Y), K_delta=K_delta)
    return replace(system, basis=build_ChannelBasis(monomer_X, monomer_Y, Jtot, system_parity, spec))


def reduced_mass(mass1: float, mass2: float) -> float:
    """mu = m1 m2 / (m1 + m2)."""
    return mass1 * mass2 / (mass1 + mass2)
