"""Further contraction families on the GPU: electric-field space-fixed and diabatic atom-diatom.

Both are the weighted-row contraction of the exact-CC path with another axis:

* electric-field SF (reference ``src/pyticc/matrix/interaction/atom_diatom.py:26-80, 271-345``):
  ``V = sym(B_cos diag(v) B_cos^T + B_sin diag(v) B_sin^T)``, one group of rows, so it runs on
  ``ticc_contract`` exactly like a K group of the BF contraction;
* diabatic (``diabatic_atom_diatom.py:30-60, 262-287, 325-520``): per electronic state and K a
  symmetric block ``B diag(v_state) B^T`` on the state's own grid, and per pair of states and K
  a coupling block ``B_a diag(v_ab) B_b^T`` placed at (a, b) and mirrored to (b, a); every block
  is one ``ticc_contract_block`` launch into a zeroed output.

The functions take the reference's basis objects as they are (attributes are read by name), so
they are drop-ins for the reference's ``contract_electric_sf_device`` and the diabatic
``contract_device``; the dataclasses below mirror the reference's for callers without it.
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass
from math import prod

import numpy as np
import torch
from loguru import logger
from numpy.typing import NDArray

from .. import _native as nat
from .interaction import DeviceRows, contract_rows


def _error(message: str, kind=ValueError):
    logger.error(message)
    return kind(message)


def _selection(n_channel: int, channel_indices) -> tuple[int, ...]:
    indices = tuple(range(n_channel)) if channel_indices is None else tuple(int(i) for i in channel_indices)
    if len(set(indices)) != len(indices) or any(i < 0 or i >= n_channel for i in indices):
        raise _error("channel_indices must be unique complete-basis positions")
    return indices


# ---- electric-field space-fixed atom-diatom ----------------------------------------------------------
@dataclass(frozen=True)
class AtomDiatomVBasisElectricSF:
    """Weighted SF rows B_cos, B_sin (n_channel, prod(grid_shape)) of an electric-field basis."""

    n_channel: int
    grid_shape: tuple[int, ...]
    r: NDArray[np.float64]
    gamma: NDArray[np.float64]
    B_cos: NDArray[np.float64]
    B_sin: NDArray[np.float64]


@dataclass(frozen=True)
class AtomDiatomVBasisElectricSFDevice:
    B_cos: torch.Tensor
    B_sin: torch.Tensor


def device_basis_electric_sf(V_basis, device) -> AtomDiatomVBasisElectricSFDevice:
    """The basis rows on one device (atom_diatom.py:280-294)."""
    dev = nat.require_cuda(device)
    return AtomDiatomVBasisElectricSFDevice(
        torch.as_tensor(np.ascontiguousarray(V_basis.B_cos, dtype=np.float64), device=dev), torch.as_tensor(np.ascontiguousarray(V_basis.B_sin, dtype=np.float64), device=dev)
    )


def contract_electric_sf_device(V_basis, basis_device, potential, device, channel_indices: Sequence[int] | None = None) -> torch.Tensor:
    """V(R) = sum_g dV(R, g) [B_cos B_cos + B_sin B_sin] (atom_diatom.py:297-345): symmetric
    (n, n) matrices, preceded by R when ``potential`` has a leading radial axis."""
    dev = nat.require_cuda(device)
    grid_shape = tuple(V_basis.grid_shape)
    n_grid = prod(grid_shape)
    values = potential if isinstance(potential, torch.Tensor) else np.asarray(potential, dtype=np.float64)
    shape = tuple(values.shape)
    if shape == grid_shape:
        batches, batched = values.reshape(1, n_grid), False
    elif len(shape) == len(grid_shape) + 1 and shape[1:] == grid_shape:
        batches, batched = values.reshape(shape[0], n_grid), True
    else:
        raise _error(f"Potential grid has shape {shape}, but SF basis requires {grid_shape} with an optional leading R axis")
    indices = _selection(V_basis.n_channel, channel_indices)
    if basis_device is None:
        basis_device = device_basis_electric_sf(V_basis, dev)
    pos = torch.as_tensor(np.asarray(indices, dtype=np.int64), device=dev)
    n = len(indices)
    rows = DeviceRows(
        basis_device.B_cos.index_select(0, pos).contiguous(),
        basis_device.B_sin.index_select(0, pos).contiguous(),
        np.asarray([0, n], dtype=np.int32),
        torch.arange(n, dtype=torch.int32, device=dev),
        n_grid,
        1.0,
        n,
    )
    V = contract_rows(rows, nat.as_device(batches, dev, torch.float64))
    return V if batched else V[0]


# ---- diabatic atom-diatom ----------------------------------------------------------------------------
@dataclass(frozen=True)
class DiabaticVBasisBF:
    """State-aware bases (diabatic_atom_diatom.py:30-40): rows per (electronic state, K) on the
    state's diagonal grid (B_diagonal) and on the shared coupling grid (B_coupling)."""

    n_channel: int
    n_state: int
    theta: NDArray[np.float64]
    diagonal_grids: tuple[NDArray[np.float64], ...]
    coupling_grid: NDArray[np.float64]
    channel_indices: dict
    B_diagonal: dict
    B_coupling: dict


@dataclass(frozen=True)
class DiabaticVGridBF:
    diagonal: tuple
    coupling: object


@dataclass(frozen=True)
class DiabaticVBasisDevice:
    B_diagonal: dict
    B_coupling: dict


def device_basis_diabatic(V_basis, device) -> DiabaticVBasisDevice:
    """The state bases on one device (diabatic_atom_diatom.py:290-304)."""
    dev = nat.require_cuda(device)
    put = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
    return DiabaticVBasisDevice({k: put(v) for k, v in V_basis.B_diagonal.items()}, {k: put(v) for k, v in V_basis.B_coupling.items()})


def _grid_batch(values, grid_shape: tuple[int, ...], tail: tuple[int, ...], label: str, dev) -> tuple[torch.Tensor, bool]:
    """(n_batch, *grid_shape, *tail) on the device, and whether a radial axis led."""
    t = values if isinstance(values, torch.Tensor) else torch.as_tensor(np.asarray(values, dtype=np.float64))
    shape = tuple(t.shape)
    full = (*grid_shape, *tail)
    if shape == full:
        return t.reshape(1, *full).to(dev, torch.float64), False
    if len(shape) == len(full) + 1 and shape[1:] == full:
        return t.to(dev, torch.float64), True
    raise _error(f"{label} has shape {shape}, but expected {full} with an optional leading R axis")


def contract_diabatic_device(V_basis, basis_device, potential, device, channel_indices: Sequence[int] | None = None) -> torch.Tensor:
    """V[c_i, c'_j] = delta_KK' sum_g B[c_i, g] V[i, j, g] B[c'_j, g] on the GPU
    (diabatic_atom_diatom.py:325-520): symmetric (n, n) matrices, preceded by R when the
    grids have a leading radial axis."""
    dev = nat.require_cuda(device)
    if len(potential.diagonal) != V_basis.n_state:
        raise _error(f"Expected {V_basis.n_state} diagonal potential grids, but got {len(potential.diagonal)}")
    n_theta = int(np.asarray(V_basis.theta).size)
    diagonal, flags = [], []
    for state, (values, grid) in enumerate(zip(potential.diagonal, V_basis.diagonal_grids, strict=True)):
        batch, batched = _grid_batch(values, (int(np.asarray(grid).size), n_theta), (), f"State {state} diagonal potential", dev)
        diagonal.append(batch.reshape(batch.shape[0], -1).contiguous())
        flags.append(batched)
    coupling, cb = _grid_batch(potential.coupling, (int(np.asarray(V_basis.coupling_grid).size), n_theta), (V_basis.n_state, V_basis.n_state), "Diabatic coupling potential", dev)
    flags.append(cb)
    sizes = {b.shape[0] for b in (*diagonal, coupling)}
    if len(set(flags)) != 1 or len(sizes) != 1:
        raise _error("Diagonal and coupling potential grids must use the same scalar or radial-batch shape")
    if not torch.allclose(coupling, coupling.transpose(-2, -1), rtol=1.0e-12, atol=1.0e-12):
        raise _error("Diabatic coupling potential must be symmetric")
    indices = _selection(V_basis.n_channel, channel_indices)
    local = {g: i for i, g in enumerate(indices)}
    n, n_batch = len(indices), next(iter(sizes))
    coupling_flat = coupling.reshape(n_batch, -1, V_basis.n_state, V_basis.n_state)
    if basis_device is None:
        basis_device = device_basis_diabatic(V_basis, dev)
    out = torch.zeros((n_batch, n, n), dtype=torch.float64, device=dev)
    lib = nat.load_library()
    stream = nat.stream_handle(dev)

    def picked(key):
        members = V_basis.channel_indices[key]
        sel = [(row, local[g]) for row, g in enumerate(members) if g in local]
        rows = torch.as_tensor(np.asarray([s[0] for s in sel], dtype=np.int64), device=dev)
        pos = torch.as_tensor(np.asarray([s[1] for s in sel], dtype=np.int32), device=dev)
        return rows, pos

    def launch(A, B, weights, pos_a, pos_b, symmetric, mirror):
        nat.check(
            lib.ticc_contract_block(nat.ptr(A), A.shape[0], nat.ptr(B), B.shape[0], A.shape[1], nat.ptr(weights), weights.stride(0), n_batch, nat.ptr(pos_a), nat.ptr(pos_b),
                                    int(symmetric), int(mirror), n, nat.ptr(out), stream),
            "ticc_contract_block",
        )

    with torch.cuda.device(dev):
        for key in V_basis.channel_indices:
            state, _ = key
            rows, pos = picked(key)
            if rows.numel() == 0:
                continue
            B = basis_device.B_diagonal[key].index_select(0, rows).contiguous()
            launch(B, B, diagonal[state], pos, pos, True, False)
        for K in sorted({K for _, K in V_basis.channel_indices}):
            for a in range(V_basis.n_state):
                if (a, K) not in V_basis.channel_indices:
                    continue
                rows_a, pos_a = picked((a, K))
                if rows_a.numel() == 0:
                    continue
                for b in range(a + 1, V_basis.n_state):
                    if (b, K) not in V_basis.channel_indices:
                        continue
                    rows_b, pos_b = picked((b, K))
                    if rows_b.numel() == 0:
                        continue
                    A = basis_device.B_coupling[(a, K)].index_select(0, rows_a).contiguous()
                    Bb = basis_device.B_coupling[(b, K)].index_select(0, rows_b).contiguous()
                    launch(A, Bb, coupling_flat[:, :, a, b].contiguous(), pos_a, pos_b, False, True)
    return out if flags[0] else out[0]
