"""Delves hyperspherical reactive propagation on the GPU (reference ``src/pyticc/propagation/delves.py:54-286``).

A reactive calculation propagates the log-derivative matrix in a hyperradius-dependent
adiabatic surface basis.  Per sector s (midpoint rho_s, width w_s) the surface provider gives
surface energies eps_s and, between consecutive sectors, the overlap T_(s-1,s); then

    Y_s^L = T^T Y_(s-1)^R T            (ticc_transform_bf_to_sf, batched over energies)
    Y_s^R = LDMD(Y_s^L; W = 2 mu diag(eps_s), half-step w_s / 2)   (ticc_ldmd_propagate)

and the first sector starts from the exact hard-wall log-derivative (inelastic) or the
incoming-wave one (capture).  Y stays on the device for the whole traversal.

The surface provider is the reference's ``DelvesHamiltonian`` or anything with the same
surface: ``basis.rho_min``, ``basis.mass`` (the three masses), ``surface(rho)`` (an object with
``rho``, ``energies`` and ``coefficients``) and ``transform(surface_a, surface_b)`` (the
directed overlap, n_a x n_b).  The surface solves themselves (the Delves basis machinery) run on
the host, as in the reference.
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass
from time import perf_counter

import numpy as np
import torch
from loguru import logger
from numpy.typing import NDArray

from .. import _native as nat
from ..energy import get_Etot
from ..match.asymptotic import transform_device
from .config import Propagation, resolve_device
from .grid import RadialSector
from .logd import initialize_logD_capture, propagate_device


@dataclass(frozen=True)
class DelvesPropagationResult:
    """Final state of a Delves propagation (the reference's fields)."""

    Y_final: torch.Tensor
    rho_final: float
    surface_rho: float
    surface_energies: NDArray[np.float64]
    surface_coefficients: NDArray[np.float64]
    radial_points: NDArray[np.float64]


def delves_reduced_mass(mass) -> float:
    """mu = sqrt(m_A m_B m_C / (m_A + m_B + m_C)) (matrix/delves/geometry.py:14-50)."""
    m = np.asarray(mass, dtype=np.float64)
    if m.shape != (3,) or np.any(~np.isfinite(m)) or np.any(m <= 0.0):
        message = f"Delves masses must be three finite positive values, but got {mass!r}"
        logger.error(message)
        raise ValueError(message)
    return float(np.sqrt(m[0] * m[1] * m[2] / m.sum()))


def hard_wall_logD(energies: NDArray[np.float64], reduced_mass: float, surface_energies: NDArray[np.float64], width: float) -> NDArray[np.float64]:
    """The exact constant-sector log-derivative for F(rho_left) = 0 (delves.py:197-236):
    p coth(p w) where p^2 = 2 mu (eps - E) > 0, q cot(q w) where it is -q^2, the series
    1/w + p^2 w / 3 - p^4 w^3 / 45 where |p| w < 1e-6; diagonal, batched over energies."""
    radial = 2.0 * reduced_mass * (surface_energies[None, :] - energies[:, None])
    magnitude = np.sqrt(np.abs(radial))
    argument = magnitude * width
    small = argument < 1.0e-6
    safe = np.where(small, 1.0, argument)
    positive = magnitude / np.tanh(safe)
    negative = magnitude / np.tan(safe)
    series = 1.0 / width + radial * width / 3.0 - radial**2 * width**3 / 45.0
    diagonal = np.where(small, series, np.where(radial >= 0.0, positive, negative))
    return diagonal[:, :, None] * np.eye(surface_energies.size)[None, :, :]


def _congruence(Y: torch.Tensor, T: NDArray[np.float64], dev) -> torch.Tensor:
    """T^T Y T for every energy; a rectangular T (the surface count changed) is padded to a
    square one with zeros, whose leading block is the product."""
    n_a, n_b = T.shape
    if Y.shape[-1] != n_a:
        message = f"transform has {n_a} rows, but the log-derivative has {Y.shape[-1]} surfaces"
        logger.error(message)
        raise ValueError(message)
    n = max(n_a, n_b)
    if n_a == n_b:
        return transform_device(Y.contiguous(), torch.as_tensor(np.ascontiguousarray(T, dtype=np.float64), device=dev))
    Tp = np.zeros((n, n))
    Tp[:n_a, :n_b] = T
    Yp = torch.zeros((Y.shape[0], n, n), dtype=Y.dtype, device=dev)
    Yp[:, :n_a, :n_a] = Y
    out = transform_device(Yp, torch.as_tensor(Tp, device=dev))
    return out[:, :n_b, :n_b].contiguous()


def _constant_sector(Y: torch.Tensor, energies_dev: torch.Tensor, reduced_mass: float, surface_energies: NDArray[np.float64], width: float, dev) -> torch.Tensor:
    """One LDMD sector with the constant diagonal W = 2 mu diag(eps) (delves.py:255-286)."""
    W = torch.as_tensor(np.diag(2.0 * reduced_mass * np.asarray(surface_energies, dtype=np.float64))[None, :, :], device=dev)
    half = torch.as_tensor(np.asarray([0.5 * width]), device=dev)
    return propagate_device(Y.contiguous(), energies_dev, reduced_mass, half, W, W, W)


def propagate_delves(hamiltonian, Etot, radial_sectors: Sequence[RadialSector], config: Propagation) -> DelvesPropagationResult:
    """Propagate reactive Delves surface channels through the radial sectors (delves.py:54-182)."""
    for name in ("surface", "transform", "basis"):
        if not hasattr(hamiltonian, name):
            message = "Delves propagation requires a DelvesHamiltonian"
            logger.error(message)
            raise TypeError(message)
    basis = hamiltonian.basis
    energies = get_Etot(Etot)
    if not radial_sectors:
        message = "Delves propagation produced no sectors"
        logger.error(message)
        raise RuntimeError(message)
    if not np.isclose(radial_sectors[0].radial_start, basis.rho_min, rtol=0.0, atol=1.0e-12):
        message = f"Delves propagation must start at the basis hard wall rho_min={basis.rho_min}, but got {radial_sectors[0].radial_start}"
        logger.error(message)
        raise ValueError(message)
    dev = nat.require_cuda(resolve_device(config.device))
    reduced_mass = delves_reduced_mass(basis.mass)
    energies_dev = torch.as_tensor(np.array(energies, dtype=np.float64), device=dev)
    started = perf_counter()
    if config.print_verbose:
        logger.info(f"Delves propagation started: sectors={len(radial_sectors)}, energies={energies.size}")
    surface_current = None
    Y = None
    for sector in radial_sectors:
        surface_next = hamiltonian.surface(sector.radial_mid)
        eps = np.asarray(surface_next.energies, dtype=np.float64)
        width = sector.radial_end - sector.radial_start
        if Y is None:
            if config.mode == "capture":
                W0 = 2.0 * reduced_mass * (eps[None, :] - energies[:, None])
                Y0 = initialize_logD_capture(torch.as_tensor(W0[:, :, None] * np.eye(eps.size)[None], device=dev), dev)
                Y = _constant_sector(Y0, energies_dev, reduced_mass, eps, width, dev)
            else:
                Y = torch.as_tensor(hard_wall_logD(energies, reduced_mass, eps, width), device=dev)
        else:
            T = np.asarray(hamiltonian.transform(surface_current, surface_next), dtype=np.float64)
            Y = _constant_sector(_congruence(Y, T, dev), energies_dev, reduced_mass, eps, width, dev)
        surface_current = surface_next
    if config.print_verbose:
        torch.cuda.synchronize(dev)
        logger.info(f"Delves propagation complete: rho={radial_sectors[-1].radial_end:.6f} bohr, surfaces={surface_current.energies.size}, wall={perf_counter() - started:.3f} s")
    radial_points = np.asarray([radial_sectors[0].radial_start, *(s.radial_end for s in radial_sectors)], dtype=np.float64)
    return DelvesPropagationResult(
        Y_final=Y,
        rho_final=radial_sectors[-1].radial_end,
        surface_rho=float(surface_current.rho),
        surface_energies=np.asarray(surface_current.energies),
        surface_coefficients=np.asarray(surface_current.coefficients),
        radial_points=radial_points,
    )
