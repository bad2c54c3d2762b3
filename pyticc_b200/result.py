"""Solver results (reference ``src/pyticc/result.py:27-238``)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .kblock import KBlock
from .system import Approx


def _transform_logD(Y: np.ndarray, B: np.ndarray) -> np.ndarray:
    """B^T Y B over a batch of log-derivative matrices (result.py:20-23)."""
    return np.einsum("ia,...ij,jb->...ab", B, Y, B, optimize=True)


@dataclass(frozen=True)
class Timing:
    wall_seconds: float
    cpu_seconds: float

    def __str__(self) -> str:
        return f"wall={self.wall_seconds:.3f} s, CPU={self.cpu_seconds:.3f} s"


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
    reduced_mass: float | None = None
    # filled by an audited solve (Propagation(audit=True)): per energy, max|S - S_fp64| against
    # an all-FP64 fixed-step solve of the same block on the same device
    max_dS: np.ndarray | None = None

    @property
    def Y_asymptotic(self) -> np.ndarray:
        return _transform_logD(self.Y_propagated, self.asymptotic_transform)

    def partial_cross_sections(self):
        """Level-to-level cross sections of this (J, parity) block (bohr^2)."""
        from .cross_section import partial_cross_sections

        if self.reduced_mass is None:
            raise ValueError("partial cross sections need the reduced mass of the solve")
        return partial_cross_sections(self.basis, self.Etot, self.Smat, self.reduced_mass)

    @property
    def open_channel_indices(self) -> tuple[np.ndarray, ...]:
        E_int = self.basis.E_int
        return tuple(np.flatnonzero(E_int < e) for e in self.Etot)

    def unitarity_defect(self) -> np.ndarray:
        """max |S^dagger S - I| per energy."""
        return np.asarray([np.abs(s.conj().T @ s - np.eye(s.shape[0])).max() if s.size else 0.0 for s in self.Smat])


@dataclass(frozen=True)
class KBlockResult:
    """Matched result of one CS or NNCC block (result.py:145-205): block log-derivatives
    in the BF basis, the block's BF -> SF transform and L, and one S matrix per energy
    over the block's open channels (global positions in ``open_channel_indices``)."""

    block: KBlock
    open_channel_indices: tuple[np.ndarray, ...]
    Y_BF: np.ndarray
    Bmat: np.ndarray
    L: np.ndarray
    Smat_asymptotic: tuple[np.ndarray, ...]

    @property
    def Y_asymptotic(self) -> np.ndarray:
        return _transform_logD(self.Y_BF, self.Bmat)

    @property
    def Smat_BF(self) -> tuple[np.ndarray, ...]:
        """S_BF(E) = B_open S_asym(E) B_open^T over the open channels, K-labelled."""
        local = {g: i for i, g in enumerate(self.block.channel_indices)}
        out = []
        for open_indices, S in zip(self.open_channel_indices, self.Smat_asymptotic, strict=True):
            rows = np.asarray([local[int(g)] for g in open_indices], dtype=np.int64)
            B_open = self.Bmat[np.ix_(rows, rows)]
            out.append(np.asarray(B_open @ S @ B_open.T, dtype=np.complex128))
        return tuple(out)


@dataclass(frozen=True)
class CoupledStatesResult:
    """CS or NNCC result of one (J, parity) system: independently propagated and matched
    blocks (result.py:207-238)."""

    basis: object
    Etot: np.ndarray
    approx: Approx
    blocks: tuple[KBlockResult, ...]
    timing: Timing | None = None

    @property
    def open_closed(self) -> np.ndarray:
        return self.basis.open_closed(self.Etot)
