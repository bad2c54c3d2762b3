"""LDMD log-derivative propagation on the GPU — drop-in for ``pyticc.propagation.logd``.

``propagate_logD`` keeps the reference signature (``src/pyticc/propagation/logd.py:340-398``)
and returns a CUDA ``torch.Tensor`` where the reference returns a device ``jax.Array``.
The sector recurrence runs in ``ticc_ldmd_propagate``: energy-shared corrections,
reference propagators and both inversions per sector on the device, batched over
energies.  Inputs may be NumPy arrays or tensors on any device; they are copied to the
CUDA device once.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch
from loguru import logger

from .. import _native as nat

MAX_SECTORS_PER_CALL = 64


def _validate_square(name: str, value) -> tuple[int, ...]:
    shape = tuple(value.shape)
    if len(shape) < 2 or shape[-2] != shape[-1]:
        message = f"{name} must end with square matrix axes, but got shape={shape}"
        logger.error(message)
        raise ValueError(message)
    return shape


def _diagonal(W) -> torch.Tensor:
    return torch.diagonal(W if isinstance(W, torch.Tensor) else torch.as_tensor(np.asarray(W)), dim1=-2, dim2=-1).real.to(torch.float64)


def initialize_logD_inelastic(Wmat, device=None) -> torch.Tensor:
    """Y_ij(R0) = delta_ij sqrt|W_ii(R0)| (logd.py:48-65)."""
    _validate_square("Wmat", Wmat)
    dev = nat.require_cuda(device)
    d = _diagonal(Wmat).to(dev)
    return torch.diag_embed(torch.sqrt(torch.abs(d)))


def initialize_logD_capture(Wmat, device=None) -> torch.Tensor:
    """Y_ii = sqrt(W_ii) (W_ii >= 0), -i sqrt(-W_ii) (W_ii < 0) (logd.py:72-91)."""
    _validate_square("Wmat", Wmat)
    dev = nat.require_cuda(device)
    d = _diagonal(Wmat).to(dev)
    values = torch.where(d >= 0.0, torch.sqrt(torch.clamp(d, min=0.0)).to(torch.complex128), -1j * torch.sqrt(torch.clamp(-d, min=0.0)).to(torch.complex128))
    return torch.diag_embed(values)


def _is_complex(*values) -> bool:
    for v in values:
        if isinstance(v, torch.Tensor):
            if v.is_complex():
                return True
        elif np.iscomplexobj(np.asarray(v)):
            return True
    return False


def propagate_device(Y: torch.Tensor, energies: torch.Tensor, reduced_mass: float, half_steps: torch.Tensor, W_start: torch.Tensor, W_mid: torch.Tensor, W_end: torch.Tensor, *, stride=None, precision: int = nat.PRECISION_FP64, reduced_out: list | None = None) -> torch.Tensor:
    """Propagate device-resident Y (complex128 or float64, contiguous) in place through
    the sectors of one call.  ``stride`` overrides the element stride between consecutive
    sectors of the three W views (e.g. an interleaved point list).  In mixed precision,
    ``reduced_out`` (a list) receives a pinned host int32 tensor that the stream fills with
    the per-sector counts of 128-wide sweep blocks that took the TF32x3 product (read it
    after synchronising)."""
    lib = nat.load_library()
    n_energy, n, _ = Y.shape
    n_sector = half_steps.numel()
    is_complex = int(Y.is_complex())
    dev = Y.device
    with torch.cuda.device(dev):
        nbytes = nat.size_query(lib.ticc_ldmd_workspace_size, n, n_energy, n_sector, is_complex, precision)
        work = nat.Workspace.get(dev, nbytes)
        status = nat.DeviceStatus(dev)
        strides = stride if stride is not None else (n * n, n * n, n * n)
        nat.check(
            lib.ticc_ldmd_propagate(
                nat.ptr(Y), is_complex, nat.ptr(energies), n_energy, float(reduced_mass), nat.ptr(half_steps),
                nat.ptr(W_start), strides[0], nat.ptr(W_mid), strides[1], nat.ptr(W_end), strides[2],
                n_sector, n, precision, nat.ptr(work), work.numel(), status.pointer, nat.stream_handle(dev),
            ),
            "ticc_ldmd_propagate",
        )
        status.raise_if_failed("ticc_ldmd_propagate")
        if reduced_out is not None and precision == nat.PRECISION_MIXED:
            counts = torch.empty(n_sector, dtype=torch.int32, pin_memory=True)
            nat.check(lib.ticc_ldmd_reduced_blocks(nat.ptr(work), work.numel(), n, n_energy, 1, n_sector, is_complex, precision, ctypes.c_void_p(counts.data_ptr()), nat.stream_handle(dev)), "ticc_ldmd_reduced_blocks")
            reduced_out.append(counts)
    return Y


def blocks_workspace_bytes(n: int, n_energy: int, n_block: int, n_sector: int, is_complex: bool, precision: int) -> int:
    return nat.size_query(nat.load_library().ticc_ldmd_blocks_workspace_size, n, n_energy, n_block, n_sector, int(is_complex), precision)


def propagate_blocks_device(Y: torch.Tensor, energies: torch.Tensor, reduced_mass: float, half_steps: torch.Tensor, W_start: torch.Tensor, W_mid: torch.Tensor, W_end: torch.Tensor, *, stride, block_stride: int, precision: int = nat.PRECISION_FP64, workspace_slot: int = 0, status: "nat.DeviceStatus | None" = None) -> torch.Tensor:
    """Propagate device-resident Y of shape (n_block, n_energy, n, n) in place: block g
    reads its W at element offset g * block_stride from the three W views, whose
    consecutive sectors are ``stride`` elements apart.  Calls that may run concurrently on
    different streams pass different ``workspace_slot``s.  With ``status`` (a DeviceStatus
    the caller checks later) the call neither allocates a status word nor synchronises, so
    it can be captured into a CUDA graph once its workspace slot is large enough."""
    lib = nat.load_library()
    n_block, n_energy, n, _ = Y.shape
    n_sector = half_steps.numel()
    is_complex = int(Y.is_complex())
    dev = Y.device
    check_now = status is None
    with torch.cuda.device(dev):
        nbytes = blocks_workspace_bytes(n, n_energy, n_block, n_sector, bool(is_complex), precision)
        work = nat.Workspace.get(dev, nbytes, slot=workspace_slot)
        status = nat.DeviceStatus(dev) if status is None else status
        nat.check(
            lib.ticc_ldmd_propagate_blocks(
                nat.ptr(Y), is_complex, nat.ptr(energies), n_energy, float(reduced_mass), nat.ptr(half_steps),
                nat.ptr(W_start), stride[0], nat.ptr(W_mid), stride[1], nat.ptr(W_end), stride[2], int(block_stride),
                n_sector, n, n_block, precision, nat.ptr(work), work.numel(), status.pointer, nat.stream_handle(dev),
            ),
            "ticc_ldmd_propagate_blocks",
        )
        if check_now:
            status.raise_if_failed("ticc_ldmd_propagate_blocks")
    return Y


def propagate_logD(Y_initial, total_energies, reduced_mass: float, radial_half_steps, W_base_start, W_base_mid, W_base_end, *, device=None) -> torch.Tensor:
    """All energies through all LDMD sectors (logd.py:340-398).

    W_base(R) = U/R^2 + 2 mu [V(R) + diag(E_int)] is energy independent; the energy
    enters as W(R; E) = W_base(R) - 2 mu E I.  Shapes: Y_initial (n_energy, n, n),
    total_energies (n_energy,), radial_half_steps (n_sector,), W_base_* (n_sector, n, n).
    Returns Y at the last sector end, float64 (inelastic) or complex128 (capture)."""
    step_shape = tuple(np.shape(radial_half_steps))
    if len(step_shape) != 1:
        message = f"radial_half_steps must be one-dimensional, but got shape={step_shape}"
        logger.error(message)
        raise ValueError(message)
    shape = _validate_square("Y_initial", Y_initial)
    n_sector = step_shape[0]
    for name, W in (("W_base_start", W_base_start), ("W_base_mid", W_base_mid), ("W_base_end", W_base_end)):
        if tuple(W.shape) != (n_sector, shape[-1], shape[-1]):
            message = f"{name} must have shape {(n_sector, shape[-1], shape[-1])}, but got {tuple(W.shape)}"
            logger.error(message)
            raise ValueError(message)
    if np.any(np.asarray(torch.as_tensor(radial_half_steps).cpu() if isinstance(radial_half_steps, torch.Tensor) else radial_half_steps) <= 0.0):
        message = "radial_half_steps must be positive"
        logger.error(message)
        raise ValueError(message)
    dev = nat.require_cuda(device)
    complex_mode = _is_complex(Y_initial, W_base_start, W_base_mid, W_base_end)
    Y = nat.as_device(Y_initial, dev, torch.complex128 if complex_mode else torch.float64).clone()
    if Y.dim() == 2:
        Y = Y[None]
    energies = nat.as_device(np.atleast_1d(np.asarray(total_energies, dtype=np.float64)) if not isinstance(total_energies, torch.Tensor) else total_energies, dev, torch.float64)
    if energies.numel() != Y.shape[0]:
        message = f"total_energies has {energies.numel()} entries, but Y_initial holds {Y.shape[0]} matrices"
        logger.error(message)
        raise ValueError(message)
    halves = nat.as_device(radial_half_steps, dev, torch.float64)
    # the kernels take W_base exactly symmetric; caller-supplied matrices are symmetrised
    Ws, Wm, We = (_symmetrised(nat.as_device(W, dev, torch.float64)) for W in (W_base_start, W_base_mid, W_base_end))
    for s0 in range(0, n_sector, MAX_SECTORS_PER_CALL):
        s1 = min(n_sector, s0 + MAX_SECTORS_PER_CALL)
        propagate_device(Y, energies, reduced_mass, halves[s0:s1], Ws[s0:s1], Wm[s0:s1], We[s0:s1])
    return Y


def _symmetrised(W: torch.Tensor) -> torch.Tensor:
    return (0.5 * (W + W.transpose(-1, -2))).contiguous()


def propagate_logD_sector(Ymat, radial_half_step: float, W_start, W_mid, W_end, *, device=None) -> torch.Tensor:
    """One sector for one matrix with the energy already inside W (logd.py:232-281)."""
    shape = _validate_square("Ymat", Ymat)
    if radial_half_step <= 0.0:
        message = f"radial_half_step must be positive, but got radial_half_step={radial_half_step}"
        logger.error(message)
        raise ValueError(message)
    for name, value in (("W_start", W_start), ("W_mid", W_mid), ("W_end", W_end)):
        if _validate_square(name, value) != shape:
            message = f"Ymat and W matrices must have the same shape, but got Ymat.shape={shape}, {name}.shape={tuple(value.shape)}"
            logger.error(message)
            raise ValueError(message)
    out = propagate_logD(
        Ymat if isinstance(Ymat, torch.Tensor) else np.asarray(Ymat)[None],
        np.zeros(1),
        1.0,
        np.array([radial_half_step]),
        np.asarray(W_start)[None] if not isinstance(W_start, torch.Tensor) else W_start[None],
        np.asarray(W_mid)[None] if not isinstance(W_mid, torch.Tensor) else W_mid[None],
        np.asarray(W_end)[None] if not isinstance(W_end, torch.Tensor) else W_end[None],
        device=device,
    )
    return out[0]
