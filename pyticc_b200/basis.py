"""Host-side basis construction: angular functions, DVR rovibrational states, channels.

These run once per Hamiltonian (geometry setup, outside the propagation hot path) and
follow PyTICC's conventions exactly, because phases and channel order change the sign
pattern of V and S:
* Gauss–Legendre nodes/weights, optional half rule (``basis/angle.py:13-52``);
* normalised associated Legendre functions with the Condon–Shortley phase and the
  odd-|K| sign for K < 0 (``basis/angle.py:69-97``);
* sine-DVR kinetic matrix and rovibrational states, first significant element of
  every eigenvector positive (``basis/dvr.py:14-303``);
* channel enumeration X-state, Y-state, j12, K with the K=0 parity rule, then a
  stable sort by threshold (``basis/channel.py:428-576``).
"""

from __future__ import annotations

import math
from collections.abc import Iterator, Sequence
from dataclasses import dataclass, field
from fractions import Fraction
from functools import lru_cache

import numpy as np
from loguru import logger
from numpy.typing import NDArray
from scipy.linalg import eigh

from .system import ChannelSpec, MolInnerState, MonomerType

# ----------------------------------------------------------------------------------------
# angular functions


def gauss_legendre_dvr(lower: float, upper: float, n_points: int, symmetry: bool = False) -> tuple[NDArray[np.float64], NDArray[np.float64]]:
    """Gauss–Legendre nodes and weights on [lower, upper]; with ``symmetry`` the lower
    half of a 2n rule with doubled weights (valid for integrands symmetric about the centre)."""
    if n_points < 1:
        message = f"n_points must be positive, but got {n_points}"
        logger.error(message)
        raise ValueError(message)
    if not np.isfinite(lower) or not np.isfinite(upper) or lower >= upper:
        message = f"Quadrature bounds must be finite and increasing, but got lower={lower}, upper={upper}"
        logger.error(message)
        raise ValueError(message)
    total = 2 * n_points if symmetry else n_points
    nodes, weights = np.polynomial.legendre.leggauss(total)
    centre, half = 0.5 * (upper + lower), 0.5 * (upper - lower)
    if symmetry:
        return (centre + half * nodes[:n_points]).copy(), (2.0 * half * weights[:n_points]).copy()
    return centre + half * nodes, half * weights


def norm_YjK(j: int, K: int, x) -> NDArray[np.float64]:
    """sqrt((2j+1)/2 (j-m)!/(j+m)!) P_j^m(x), m = |K|, Condon–Shortley phase, times -1 for
    K < 0 with odd m.  Computed by the stable normalised recurrence in j at fixed m."""
    m = abs(K)
    if m > j:
        message = f"Invalid input: |K|={m} exceeds j={j}"
        logger.error(message)
        raise ValueError(message)
    x = np.asarray(x, dtype=np.float64)
    s = np.sqrt(np.clip(1.0 - x * x, 0.0, None))
    # P̄_m^m = (-1)^m sqrt((2m+1)/2 * prod_{k<=m} (2k-1)/(2k)) s^m
    value = np.full_like(x, math.sqrt(0.5))
    for k in range(1, m + 1):
        value = -value * s * math.sqrt((2.0 * k + 1.0) / (2.0 * k))
    if j > m:
        previous = value
        value = x * math.sqrt(2.0 * m + 3.0) * previous
        for ell in range(m + 2, j + 1):
            a = math.sqrt((4.0 * ell * ell - 1.0) / (ell * ell - m * m))
            b = math.sqrt(((ell - 1.0) ** 2 - m * m) / (4.0 * (ell - 1.0) ** 2 - 1.0))
            previous, value = value, a * (x * value - b * previous)
    if K < 0 and m % 2 == 1:
        value = -value
    return value


def lambda_plus(j: float, K: float) -> float:
    """sqrt(j(j+1) - K(K+1))."""
    return math.sqrt(j * (j + 1) - K * (K + 1))


@lru_cache(maxsize=None)
def clebsch_gordan(j1: int, m1: int, j2: int, m2: int, J: int) -> float:
    """<j1 m1 j2 m2 | J m1+m2> by Racah's closed form in exact rational arithmetic."""
    M = m1 + m2
    if abs(m1) > j1 or abs(m2) > j2 or abs(M) > J or J < abs(j1 - j2) or J > j1 + j2:
        return 0.0
    f = math.factorial
    prefactor = Fraction((2 * J + 1) * f(J + j1 - j2) * f(J - j1 + j2) * f(j1 + j2 - J), f(j1 + j2 + J + 1))
    prefactor *= Fraction(f(J + M) * f(J - M) * f(j1 - m1) * f(j1 + m1) * f(j2 - m2) * f(j2 + m2), 1)
    total = Fraction(0)
    for k in range(0, j1 + j2 - J + 1):
        terms = (k, j1 + j2 - J - k, j1 - m1 - k, j2 + m2 - k, J - j2 + m1 + k, J - j1 - m2 + k)
        if min(terms) < 0:
            continue
        denominator = 1
        for t in terms:
            denominator *= f(t)
        total += Fraction((-1) ** k, denominator)
    return float(math.copysign(math.sqrt(prefactor), 1.0) * total)


# ----------------------------------------------------------------------------------------
# rovibrational states


@dataclass(frozen=True)
class RovibBasis:
    """Diatomic rovibrational states on a radial grid: grids (n_r,), E_vj (n_v, n_j),
    WF_vj (n_r, n_v, n_j)."""

    grids: NDArray[np.float64]
    E_vj: NDArray[np.float64]
    WF_vj: NDArray[np.float64]

    def __post_init__(self) -> None:
        g, e, w = np.asarray(self.grids), np.asarray(self.E_vj), np.asarray(self.WF_vj)
        if g.ndim != 1 or e.ndim != 2 or w.shape != (g.size, *e.shape):
            message = f"RovibBasis shapes must satisfy grids=(n_grid,), E_vj=(n_v,n_j), and WF_vj=(n_grid,n_v,n_j), but got {g.shape}, {e.shape}, and {w.shape}"
            logger.error(message)
            raise ValueError(message)


def _first_significant_positive(vectors: NDArray[np.float64]) -> NDArray[np.float64]:
    """Flip each column so that its first element above 1e-4 in magnitude is positive."""
    out = np.array(vectors, dtype=np.float64, copy=True)
    for column in range(out.shape[1]):
        significant = np.flatnonzero(np.abs(out[:, column]) > 1.0e-4)
        if significant.size == 0:
            message = "All elements are below the threshold."
            logger.error(message)
            raise ValueError(message)
        if out[significant[0], column] < 0.0:
            out[:, column] *= -1.0
    return out


def sine_dvr_kinetic(a: float, b: float, n: int, mass: float) -> NDArray[np.float64]:
    """Sine-DVR kinetic energy on n interior points of [a, b] (analytic matrix elements)."""
    m = n + 1
    index = np.arange(1, n + 1, dtype=np.float64)
    i, j = np.meshgrid(index, index, indexing="ij")
    with np.errstate(divide="ignore", invalid="ignore"):
        off = 1.0 / np.sin(np.pi * (i - j) / (2.0 * m)) ** 2 - 1.0 / np.sin(np.pi * (i + j) / (2.0 * m)) ** 2
    off[~np.isfinite(off)] = 0.0
    np.fill_diagonal(off, 0.0)
    sign = np.where((i - j) % 2 == 0, 1.0, -1.0)
    np.fill_diagonal(sign, 1.0)
    diagonal = (2.0 * m * m + 1.0) / 3.0 - 1.0 / np.sin(np.pi * index / m) ** 2
    T = np.diag(diagonal) + off * sign
    return T * (np.pi**2 / (4.0 * mass * (b - a) ** 2))


@dataclass(frozen=True)
class SineDVR:
    """Primitive sine DVR with its vibrational eigenstates."""

    n_dvr: int
    interval: tuple[float, float]
    grids: NDArray[np.float64]
    weights: float
    eigen_val: NDArray[np.float64]
    eigen_vec: NDArray[np.float64]


def build_SineDVR(a: float, b: float, n_dvr: int, mass: float, pot_func) -> SineDVR:
    """Vibrational states of a 1D potential in a sine DVR on [a, b] (basis/dvr.py:271-303)."""
    if a >= b:
        message = f"Invalid interval: a ({a}) must be less than b ({b})"
        logger.error(message)
        raise ValueError(message)
    grids = a + np.arange(1, n_dvr + 1, dtype=np.float64) * (b - a) / (n_dvr + 1)
    H = sine_dvr_kinetic(a, b, n_dvr, mass)
    H[np.diag_indices(n_dvr)] += np.asarray(pot_func(grids), dtype=np.float64)
    values, vectors = eigh(H)
    return SineDVR(n_dvr, (a, b), grids, (b - a) / (n_dvr + 1), values, _first_significant_positive(vectors))


def build_RovibDVR(dvr: SineDVR, vmax: int, jmax: int, mass: float) -> RovibBasis:
    """Rovibrational states j = 0..jmax, v = 0..vmax on the primitive grid (basis/dvr.py:223-264)."""
    if vmax < 0 or jmax < 0:
        message = f"vmax and jmax must be non-negative, but got vmax={vmax}, jmax={jmax}"
        logger.error(message)
        raise ValueError(message)
    n = dvr.grids.size
    n_v = min(vmax + 1, n)
    energies = np.zeros((vmax + 1, jmax + 1))
    wavefunctions = np.zeros((n, vmax + 1, jmax + 1))
    H0 = (dvr.eigen_vec * dvr.eigen_val[None, :]) @ dvr.eigen_vec.T
    for j in range(jmax + 1):
        H = H0.copy()
        H[np.diag_indices(n)] += j * (j + 1) / (2.0 * mass * dvr.grids**2)
        values, vectors = eigh(H, subset_by_index=(0, n_v - 1))
        energies[:n_v, j] = values
        wavefunctions[:, :n_v, j] = _first_significant_positive(vectors)
    return RovibBasis(grids=dvr.grids, E_vj=energies, WF_vj=wavefunctions)


# ----------------------------------------------------------------------------------------
# monomers


class AtomSpec:
    """Structureless atom: one internal state j = 0 at zero energy."""

    type = MonomerType.ATOM

    def mis_iter(self, E_cut: float) -> Iterator[MolInnerState]:
        yield MolInnerState(j=0, Eint=0.0)

    def energy(self, mis: MolInnerState, K: int) -> float:
        return 0.0


@dataclass(frozen=True)
class DiatomSpec:
    """Diatomic state table Eint[v, j] without wavefunctions (channel counting only)."""

    Eint: NDArray[np.float64]
    type = MonomerType.DIATOM

    def mis_iter(self, E_cut: float) -> Iterator[MolInnerState]:
        table = np.asarray(self.Eint)
        for v in range(table.shape[0]):
            for j in range(table.shape[1]):
                e = float(table[v, j])
                if np.isfinite(e) and e <= E_cut:
                    yield MolInnerState(j=j, v=v, Eint=e)

    def energy(self, mis: MolInnerState, K: int) -> float:
        return float(np.asarray(self.Eint)[mis.v, mis.j])


@dataclass(frozen=True)
class DiatomBasis:
    """Adiabatic diatom: rovibrational states and the energy zero of its thresholds."""

    rovib: RovibBasis
    energy_zero: float
    type = MonomerType.DIATOM

    @property
    def Eint(self) -> NDArray[np.float64]:
        return np.asarray(self.rovib.E_vj - self.energy_zero)

    def mis_iter(self, E_cut: float) -> Iterator[MolInnerState]:
        table = self.Eint
        for v in range(table.shape[0]):
            for j in range(table.shape[1]):
                e = float(table[v, j])
                if np.isfinite(e) and e <= E_cut:
                    yield MolInnerState(j=j, v=v, Eint=e)

    def energy(self, mis: MolInnerState, K: int) -> float:
        return float(self.rovib.E_vj[mis.v, mis.j] - self.energy_zero)


# ----------------------------------------------------------------------------------------
# channels


@dataclass(frozen=True)
class Channel:
    """One body-fixed channel (mis_X, mis_Y, j12, K) with threshold E_int."""

    mis_X: MolInnerState
    mis_Y: MolInnerState
    j_couple: int
    K: int
    E_int: float


@dataclass(frozen=True)
class ChannelBasis(Sequence[Channel]):
    """Channels of one (J, parity) block, ordered by threshold."""

    channels: tuple[Channel, ...]
    Jtot: int
    system_parity: int
    channel_spec: ChannelSpec = field(default_factory=ChannelSpec)

    @property
    def n_channel(self) -> int:
        return len(self.channels)

    @property
    def E_int(self) -> NDArray[np.float64]:
        return np.asarray([c.E_int for c in self.channels], dtype=np.float64)

    def __len__(self) -> int:
        return len(self.channels)

    def __getitem__(self, index):
        return self.channels[index]

    def open_closed(self, total_energies) -> NDArray[np.bool_]:
        """Open-channel mask (n_energy, n_channel): E_int < E (basis/channel.py:173-187)."""
        energies = np.asarray(total_energies, dtype=np.float64)
        return self.E_int[None, :] < energies[:, None]


def _selected_states(monomer, E_cut: float, vmin: int, exchange_parity: int) -> list[MolInnerState]:
    states = list(monomer.mis_iter(E_cut))
    if monomer.type is not MonomerType.DIATOM:
        return states
    return [s for s in states if s.v >= vmin and (exchange_parity == 0 or (-1) ** s.j == exchange_parity)]


def build_ChannelBasis(monomer_X, monomer_Y, Jtot: int, system_parity: int, spec: ChannelSpec | None = None) -> ChannelBasis:
    """All (X state, Y state, j12, K) channels of one (J, parity) block (basis/channel.py:491-576).

    K runs over 0..min(j12, J, K_cut); K = 0 is kept only when
    parity * (-1)^(jX + jY + j12 + J) = 1; the list is stable-sorted by threshold."""
    spec = ChannelSpec() if spec is None else spec
    states_X = _selected_states(monomer_X, spec.E_X_cut, spec.vmin_X, spec.exchange_parity_X)
    states_Y = _selected_states(monomer_Y, spec.E_Y_cut, spec.vmin_Y, spec.exchange_parity_Y)
    channels: list[Channel] = []
    for mx in states_X:
        for my in states_Y:
            for j12 in range(abs(mx.j - my.j), mx.j + my.j + 1):
                K_max = min(j12, Jtot) if spec.K_cut is None else min(j12, Jtot, spec.K_cut)
                for K in range(K_max + 1):
                    if K == 0 and system_parity * (-1) ** (mx.j + my.j + j12 + Jtot) != 1:
                        continue
                    channels.append(Channel(mx, my, j12, K, float(monomer_X.energy(mx, K) + monomer_Y.energy(my, K))))
    channels.sort(key=lambda c: c.E_int)
    return ChannelBasis(tuple(channels), Jtot, system_parity, spec)


def get_Umat_BF(basis: ChannelBasis, channel_indices: Sequence[int] | None = None) -> NDArray[np.float64]:
    """Dimensionless BF centrifugal matrix (matrix/centrifugal.py:27-85):
    U_ii = J(J+1) + j12(j12+1) - 2K^2, U_{K,K+1} = -sqrt(2)^{delta_K0} lambda+(J,K) lambda+(j12,K)
    within each (mis_X, mis_Y, j12) ladder."""
    indices = tuple(range(basis.n_channel)) if channel_indices is None else tuple(channel_indices)
    channels = [basis[i] for i in indices]
    J = basis.Jtot
    U = np.zeros((len(channels), len(channels)))
    ladders: dict[tuple, dict[int, int]] = {}
    for local, c in enumerate(channels):
        ladders.setdefault((c.mis_X, c.mis_Y, c.j_couple), {})[c.K] = local
        U[local, local] = J * (J + 1) + c.j_couple * (c.j_couple + 1) - 2 * c.K**2
    for (_, _, j12), by_K in ladders.items():
        for K, local in by_K.items():
            other = by_K.get(K + 1)
            if other is None:
                continue
            coupling = -(math.sqrt(2.0) if K == 0 else 1.0) * lambda_plus(J, K) * lambda_plus(j12, K)
            U[local, other] = U[other, local] = coupling
    return U
