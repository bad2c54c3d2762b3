"""Further contraction families on the GPU: electric-field space-fixed and diabatic atom-diatom,
and the fine-structure diatom-diatom families (scalar and spin-resolved).

The first two are the weighted-row contraction of the exact-CC path with another axis:

* electric-field SF (reference ``src/pyticc/matrix/interaction/atom_diatom.py:26-80, 271-345``):
  ``V = sym(B_cos diag(v) B_cos^T + B_sin diag(v) B_sin^T)``, one group of rows, so it runs on
  ``ticc_contract`` exactly like a K group of the BF contraction;
* diabatic (``diabatic_atom_diatom.py:30-60, 262-287, 325-520``): per electronic state and K a
  symmetric block ``B diag(v_state) B^T`` on the state's own grid, and per pair of states and K
  a coupling block ``B_a diag(v_ab) B_b^T`` placed at (a, b) and mirrored to (b, a); every block
  is one ``ticc_contract_block`` launch into a zeroed output.

The fine-structure families contract with a packed kernel over lower-triangle channel pairs
(a cuBLAS GEMM) and scatter the pairs into symmetric or Hermitian matrices (``ticc_pairs_to_matrix``).

The functions take the reference's basis objects as they are (attributes are read by name), so
they are drop-ins for the reference's ``contract_electric_sf_device``, the diabatic and the
fine-structure ``contract_device``; the dataclasses below mirror the reference's for callers
without it.
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


# ---- fine-structure diatom-diatom (scalar and spin-resolved) -----------------------------------------
# Both contract the PES grid with a packed kernel over lower-triangle channel pairs,
#   contracted(R, p) = sum_k potential(R, k) kernel(k, packed(p)),
# a plain GEMM (cuBLAS through torch), then scatter the pairs into matrices (ticc_pairs_to_matrix):
# symmetric for the scalar family (fs_diatom_diatom.py:356-470), Hermitian with conjugation of
# reversed pairs for the spin-resolved one (fs_diatom_diatom_spin.py:459-550).
_KERNEL_CHUNK_BYTES = 256 * 1024**2


def packed_positions(n_channel: int, indices: tuple[int, ...]):
    """Selected lower-triangle pairs and their positions in the complete packed order
    (the reference's packing, fs_diatom_diatom.py:336-349)."""
    indices = _selection(n_channel, indices)
    pair_rows, pair_columns = np.tril_indices(len(indices))
    selected = np.asarray(indices, dtype=np.int64)
    rows, cols = selected[pair_rows], selected[pair_columns]
    hi, lo = np.maximum(rows, cols), np.minimum(rows, cols)
    return pair_rows.astype(np.int64), pair_columns.astype(np.int64), (hi * (hi + 1) // 2 + lo).astype(np.int64), selected


@dataclass(frozen=True)
class FSKernelDevice:
    """The packed kernel (n_k, n_packed) on the device, or None to stream it from the host."""

    kernel: NDArray
    resident: torch.Tensor | None


def device_basis_fs(V_basis, device) -> FSKernelDevice:
    """Keep kernels up to 256 MiB resident on the device; stream larger ones by pair chunks."""
    dev = nat.require_cuda(device)
    k = np.asarray(V_basis.kernel)
    return FSKernelDevice(k, torch.as_tensor(k.reshape(-1, k.shape[-1]), device=dev) if k.nbytes <= _KERNEL_CHUNK_BYTES else None)


def _contract_packed(batches: torch.Tensor, basis_device: FSKernelDevice, n_channel: int, channel_indices, hermitian: bool, dev) -> torch.Tensor:
    indices = tuple(range(n_channel)) if channel_indices is None else tuple(channel_indices)
    pair_rows, pair_cols, packed, selected = packed_positions(n_channel, indices)
    host_kernel = basis_device.kernel.reshape(-1, basis_device.kernel.shape[-1])
    dtype = torch.complex128 if (hermitian and (torch.is_complex(batches) or np.iscomplexobj(host_kernel))) else torch.float64
    lhs = batches.to(dev, dtype)
    n_k = lhs.shape[1]
    itemsize = 16 if dtype == torch.complex128 else 8
    per_chunk = max(1, _KERNEL_CHUNK_BYTES // (n_k * itemsize))
    contracted = torch.empty((lhs.shape[0], packed.size), dtype=dtype, device=dev)
    for start in range(0, packed.size, per_chunk):
        chunk = packed[start : start + per_chunk]
        if basis_device.resident is not None:
            kern = basis_device.resident.index_select(1, torch.as_tensor(chunk, device=dev)).to(dtype)
        else:
            kern = torch.as_tensor(np.ascontiguousarray(host_kernel[:, chunk]), device=dev).to(dtype)
        contracted[:, start : start + chunk.size] = lhs @ kern
    n = len(indices)
    is_complex = dtype == torch.complex128
    out = torch.zeros((lhs.shape[0], n, n), dtype=dtype, device=dev)
    src = torch.view_as_real(contracted).reshape(lhs.shape[0], -1) if is_complex else contracted
    reversed_pairs = None
    if is_complex:
        reversed_pairs = torch.as_tensor((selected[pair_rows] < selected[pair_cols]).astype(np.uint8), device=dev)
    pr = torch.as_tensor(pair_rows.astype(np.int32), device=dev)
    pc = torch.as_tensor(pair_cols.astype(np.int32), device=dev)
    lib = nat.load_library()
    with torch.cuda.device(dev):
        nat.check(
            lib.ticc_pairs_to_matrix(nat.ptr(src), int(is_complex), src.stride(0), int(packed.size), nat.ptr(pr), nat.ptr(pc), nat.ptr(reversed_pairs), n, lhs.shape[0],
                                     nat.ptr(torch.view_as_real(out) if is_complex else out), nat.stream_handle(dev)),
            "ticc_pairs_to_matrix",
        )
    return out


def contract_fs_device(V_basis, basis_device, potential, device, channel_indices: Sequence[int] | None = None) -> torch.Tensor:
    """Scalar PES into two-fine-structure-diatom channel matrices (fs_diatom_diatom.py:417-470)."""
    dev = nat.require_cuda(device)
    grid_shape = tuple(V_basis.grid_shape)
    n_grid = prod(grid_shape)
    values = potential if isinstance(potential, torch.Tensor) else torch.as_tensor(np.asarray(potential, dtype=np.float64))
    shape = tuple(values.shape)
    if shape == grid_shape:
        batches, batched = values.reshape(1, n_grid), False
    elif len(shape) == len(grid_shape) + 1 and shape[1:] == grid_shape:
        batches, batched = values.reshape(shape[0], n_grid), True
    elif len(shape) == 2 and shape[1] == n_grid:
        batches, batched = values, True
    else:
        raise _error(f"Scalar FS diatom-diatom PES grid has shape {shape}, expected {grid_shape} with optional leading R axis")
    if basis_device is None:
        basis_device = device_basis_fs(V_basis, dev)
    V = _contract_packed(batches, basis_device, V_basis.n_channel, channel_indices, False, dev)
    return V if batched else V[0]


def contract_fs_spin_device(V_basis, basis_device, potential, device, channel_indices: Sequence[int] | None = None) -> torch.Tensor:
    """Spin-resolved orbital PES grids into Hermitian channel matrices (fs_diatom_diatom_spin.py:504-550)."""
    dev = nat.require_cuda(device)
    grid_shape = tuple(V_basis.grid_shape)
    electronic = (len(V_basis.two_total_spins), len(V_basis.orbital_states), len(V_basis.orbital_states))
    n_grid, n_el = prod(grid_shape), prod(electronic)
    values = potential if isinstance(potential, torch.Tensor) else torch.as_tensor(np.asarray(potential))
    shape = tuple(values.shape)
    expected = (*grid_shape, *electronic)
    if shape == expected:
        batches, batched = values.reshape(1, n_grid * n_el), False
    elif len(shape) == len(expected) + 1 and shape[1:] == expected:
        batches, batched = values.reshape(shape[0], n_grid * n_el), True
    elif len(shape) == 3 and shape[1:] == (n_grid, n_el):
        batches, batched = values.reshape(shape[0], n_grid * n_el), True
    else:
        raise _error(f"Spin-resolved FS diatom-diatom PES grid has shape {shape}, expected {expected} with optional leading R axis")
    if basis_device is None:
        basis_device = device_basis_fs(V_basis, dev)
    V = _contract_packed(batches, basis_device, V_basis.n_channel, channel_indices, True, dev)
    return V if batched else V[0]
