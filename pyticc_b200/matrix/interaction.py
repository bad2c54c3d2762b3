"""Weighted contraction rows and the V(R) contraction on the GPU.

``VBasisBF`` and the ``prepare_*`` row builders mirror
``src/pyticc/matrix/interaction/common.py:19-28``, ``atom_diatom.py:351-386`` and
``diatom_diatom.py:16-137``; ``contract_device`` is the drop-in for
``common.py:153-211`` and runs ``ticc_contract`` (optionally fusing the W_base assembly
of ``propagation/runner.py:265-271``).
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass, field
from math import prod

import numpy as np
import torch
from loguru import logger
from numpy.typing import NDArray

from .. import _native as nat
from ..basis import clebsch_gordan, norm_YjK


@dataclass(frozen=True)
class VBasisBF:
    """PES-independent weighted rows grouped by K (B_real[K], B_imag[K]: (n_K, n_grid))."""

    n_channel: int
    grid_shape: tuple[int, ...]
    channel_indices: dict[int, tuple[int, ...]]
    B_real: dict[int, NDArray[np.float64]]
    B_imag: dict[int, NDArray[np.float64]] | None
    normalization: float = 1.0


@dataclass
class DeviceRows:
    """One channel block's rows on a device, grouped by K, with their output positions."""

    rows_real: torch.Tensor
    rows_imag: torch.Tensor | None
    group_offsets: np.ndarray
    row_out: torch.Tensor
    n_grid: int
    normalization: float
    n_channel: int


@dataclass
class DeviceBasisCache:
    """Device copies of a VBasisBF per (device, channel block)."""

    entries: dict = field(default_factory=dict)


def prepare_atom_diatom(basis, rovib, cos_theta: NDArray[np.float64], theta_weights: NDArray[np.float64]) -> VBasisBF:
    """B_K[c, (r, theta)] = WF_vj(r) sqrt(w_theta) Ytilde_jK(cos theta) (atom_diatom.py:351-386)."""
    grid_shape = (rovib.grids.size, cos_theta.size)
    sqrt_w = np.sqrt(theta_weights)
    angular: dict[tuple[int, int], NDArray[np.float64]] = {}
    groups: dict[int, tuple[int, ...]] = {}
    rows: dict[int, NDArray[np.float64]] = {}
    for K in sorted({c.K for c in basis}):
        members = tuple(i for i, c in enumerate(basis) if c.K == K)
        block = np.empty((len(members), prod(grid_shape)))
        for row, index in enumerate(members):
            c = basis[index]
            state = c.mis_X if c.mis_X.v is not None else c.mis_Y
            key = (state.j, K)
            if key not in angular:
                angular[key] = sqrt_w * norm_YjK(state.j, K, cos_theta)
            block[row] = np.outer(rovib.WF_vj[:, state.v, state.j], angular[key]).ravel()
        groups[K] = members
        rows[K] = block
    return VBasisBF(basis.n_channel, grid_shape, groups, rows, None)


def _pair_angular(jX, jY, j12, K, cX, wX, cY, wY, phi, wphi):
    shape = (cX.size, cY.size, phi.size)
    real, imag = np.zeros(shape), np.zeros(shape)
    sX, sY, sP = np.sqrt(wX), np.sqrt(wY), np.sqrt(wphi)
    for omega in range(-jX, jX + 1):
        other = K - omega
        if abs(other) > jY:
            continue
        amp = clebsch_gordan(jX, omega, jY, other, j12) * (sX * norm_YjK(jX, omega, cX))[:, None, None] * (sY * norm_YjK(jY, other, cY))[None, :, None]
        real += amp * (sP * np.cos(omega * phi))[None, None, :]
        imag += amp * (sP * np.sin(omega * phi))[None, None, :]
    return real, imag


def prepare_diatom_diatom(basis, rovib_X, rovib_Y, cX, wX, cY, wY, phi, wphi) -> VBasisBF:
    """Coupled bispherical rows with cos/sin(omega phi) parts and normalisation 1/pi
    (diatom_diatom.py:16-137, without molecule-exchange adaptation)."""
    grid_shape = (rovib_X.grids.size, rovib_Y.grids.size, cX.size, cY.size, phi.size)
    angular: dict[tuple[int, int, int, int], tuple] = {}
    groups, real_rows, imag_rows = {}, {}, {}
    for K in sorted({c.K for c in basis}):
        members = tuple(i for i, c in enumerate(basis) if c.K == K)
        re = np.empty((len(members), prod(grid_shape)))
        im = np.empty_like(re)
        for row, index in enumerate(members):
            c = basis[index]
            key = (c.mis_X.j, c.mis_Y.j, c.j_couple, K)
            if key not in angular:
                angular[key] = _pair_angular(c.mis_X.j, c.mis_Y.j, c.j_couple, K, cX, wX, cY, wY, phi, wphi)
            a_re, a_im = angular[key]
            radial = np.multiply.outer(rovib_X.WF_vj[:, c.mis_X.v, c.mis_X.j], rovib_Y.WF_vj[:, c.mis_Y.v, c.mis_Y.j])
            re[row] = (radial[:, :, None, None, None] * a_re[None, None]).ravel()
            im[row] = (radial[:, :, None, None, None] * a_im[None, None]).ravel()
        groups[K] = members
        real_rows[K] = re
        imag_rows[K] = im
    return VBasisBF(basis.n_channel, grid_shape, groups, real_rows, imag_rows, 1.0 / np.pi)


def device_rows(basis: VBasisBF, device: torch.device, channel_indices: Sequence[int] | None = None) -> DeviceRows:
    """Gather the rows of one channel block (in block order within each K group) to the device."""
    indices = tuple(range(basis.n_channel)) if channel_indices is None else tuple(channel_indices)
    if len(set(indices)) != len(indices) or any(i < 0 or i >= basis.n_channel for i in indices):
        message = "channel_indices must be unique complete-basis positions"
        logger.error(message)
        raise ValueError(message)
    local = {g: i for i, g in enumerate(indices)}
    real, imag, out, offsets = [], [], [], [0]
    for K, members in basis.channel_indices.items():
        picked = [(row, local[g]) for row, g in enumerate(members) if g in local]
        if not picked:
            continue
        rows = np.asarray([p[0] for p in picked])
        real.append(basis.B_real[K][rows])
        if basis.B_imag is not None:
            imag.append(basis.B_imag[K][rows])
        out.extend(p[1] for p in picked)
        offsets.append(offsets[-1] + len(picked))
    n_grid = prod(basis.grid_shape)
    rr = np.concatenate(real) if real else np.zeros((0, n_grid))
    ri = np.concatenate(imag) if imag else None
    return DeviceRows(
        torch.as_tensor(np.ascontiguousarray(rr), device=device),
        None if ri is None else torch.as_tensor(np.ascontiguousarray(ri), device=device),
        np.asarray(offsets, dtype=np.int32),
        torch.as_tensor(np.asarray(out, dtype=np.int32), device=device),
        n_grid,
        float(basis.normalization),
        len(indices),
    )


def contract_rows(rows: DeviceRows, potential: torch.Tensor, *, radial_points: torch.Tensor | None = None, U: torch.Tensor | None = None, E_int: torch.Tensor | None = None, reduced_mass: float = 0.0, out: torch.Tensor | None = None) -> torch.Tensor:
    """V(R) (or W_base(R) when U is given) for every row of ``potential`` (n_R, n_grid)."""
    lib = nat.load_library()
    dev = rows.row_out.device
    potential = potential.reshape(potential.shape[0], -1)
    if potential.stride(-1) != 1:
        potential = potential.contiguous()
    n_R = potential.shape[0]
    n = rows.n_channel
    if out is None:
        out = torch.empty((n_R, n, n), dtype=torch.float64, device=dev)
    offsets = rows.group_offsets
    c_offsets = (nat._I * offsets.size)(*offsets.tolist())
    with torch.cuda.device(dev):
        nat.check(
            lib.ticc_contract(
                nat.ptr(rows.rows_real), nat.ptr(rows.rows_imag), c_offsets, offsets.size - 1, nat.ptr(rows.row_out), rows.n_grid,
                rows.normalization, nat.ptr(potential), potential.stride(0), n_R, n, nat.ptr(radial_points), nat.ptr(U), nat.ptr(E_int),
                float(reduced_mass), nat.ptr(out), nat.stream_handle(dev),
            ),
            "ticc_contract",
        )
    return out


def _potential_batches(basis: VBasisBF, potential):
    n_grid = prod(basis.grid_shape)
    shape = tuple(potential.shape)
    if shape == basis.grid_shape or shape == (n_grid,):
        return potential.reshape(1, n_grid), False
    if len(shape) == len(basis.grid_shape) + 1 and shape[1:] == basis.grid_shape:
        return potential.reshape(shape[0], n_grid), True
    if len(shape) == 2 and shape[1] == n_grid:
        return potential, True
    message = f"Potential grid has shape {shape}, but V basis requires {basis.grid_shape} with an optional leading R axis"
    logger.error(message)
    raise ValueError(message)


def contract_device(basis: VBasisBF, basis_device, potential, device=None, channel_indices: Sequence[int] | None = None) -> torch.Tensor:
    """Symmetric V(R) for one channel block on the GPU (common.py:153-211).

    ``basis_device`` is a DeviceBasisCache (or None); ``potential`` is host or device,
    shaped like the PES grid with an optional leading R axis."""
    dev = nat.require_cuda(device)
    key = (dev.index, None if channel_indices is None else tuple(channel_indices))
    cache = basis_device if isinstance(basis_device, DeviceBasisCache) else DeviceBasisCache()
    rows = cache.entries.get(key)
    if rows is None:
        rows = device_rows(basis, dev, channel_indices)
        cache.entries[key] = rows
    values = potential if isinstance(potential, torch.Tensor) else np.asarray(potential, dtype=np.float64)
    batches, batched = _potential_batches(basis, values)
    V = contract_rows(rows, nat.as_device(batches, dev, torch.float64))
    return V if batched else V[0]


def device_basis(basis: VBasisBF, device=None) -> DeviceBasisCache:
    """Device cache holder for ``contract_device`` (common.py:77-90)."""
    return DeviceBasisCache()
