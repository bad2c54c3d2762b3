"""BF -> SF asymptotic transform (reference ``src/pyticc/match/asymptotic.py:16-110``).

``get_Bmat_BF_to_SF`` diagonalises U per (mis_X, mis_Y, j12) ladder on the host (setup,
once per block); ``transform_logD_BF_to_SF`` runs B^T Y B on the GPU."""

from __future__ import annotations

from collections.abc import Sequence

import numpy as np
import torch
from loguru import logger

from .. import _native as nat
from ..basis import get_Umat_BF


def get_Bmat_BF_to_SF(basis, channel_indices: Sequence[int] | None = None):
    """B with B^T U B = diag(L(L+1)), L = sqrt(lambda + 1/4) - 1/2; eigenvector signs fixed
    by the last component and the phase (-1)^(j12 + min(J, j12)) (asymptotic.py:16-75)."""
    indices = tuple(range(basis.n_channel)) if channel_indices is None else tuple(channel_indices)
    if not indices:
        message = "At least one channel is required for the BF-to-SF transformation"
        logger.error(message)
        raise ValueError(message)
    channels = [basis[i] for i in indices]
    U = get_Umat_BF(basis, indices)
    n = len(indices)
    B = np.zeros((n, n))
    L = np.empty(n)
    ladders: dict[tuple, list[int]] = {}
    for local, c in enumerate(channels):
        ladders.setdefault((c.mis_X, c.mis_Y, c.j_couple), []).append(local)
    for (_, _, j12), members in ladders.items():
        pos = np.asarray(members)
        values, vectors = np.linalg.eigh(U[np.ix_(pos, pos)])
        if np.min(values) < -1.0e-10:
            message = f"Centrifugal matrix has a negative eigenvalue {np.min(values)}"
            logger.error(message)
            raise ValueError(message)
        phase = (-1) ** (j12 + min(basis.Jtot, j12))
        vectors = vectors * np.where(vectors[-1] * phase < 0.0, -1.0, 1.0)
        B[np.ix_(pos, pos)] = vectors
        L[pos] = np.sqrt(np.maximum(values, 0.0) + 0.25) - 0.5
    return B, L


def transform_device(Y: torch.Tensor, B: torch.Tensor) -> torch.Tensor:
    """B^T Y B for a device batch (float64 or complex128), returned as a new tensor."""
    lib = nat.load_library()
    dev = Y.device
    batch, n, _ = Y.shape
    is_complex = int(Y.is_complex())
    out = torch.empty_like(Y)
    with torch.cuda.device(dev):
        nbytes = nat.size_query(lib.ticc_transform_workspace_size, n, batch, is_complex)
        work = nat.Workspace.get(dev, nbytes, slot=1)
        nat.check(lib.ticc_transform_bf_to_sf(nat.ptr(Y), nat.ptr(out), nat.ptr(B), n, batch, is_complex, nat.ptr(work), work.numel(), nat.stream_handle(dev)), "ticc_transform_bf_to_sf")
    return out


def transform_logD_BF_to_SF(Ymat, Bmat):
    """Y_SF = B^T Y_BF B for (..., n, n) inputs; returns the same kind of array it was given."""
    B_np = np.asarray(Bmat.cpu() if isinstance(Bmat, torch.Tensor) else Bmat, dtype=np.float64)
    if B_np.ndim != 2 or B_np.shape[0] != B_np.shape[1]:
        message = f"Bmat must be square, but got shape={B_np.shape}"
        logger.error(message)
        raise ValueError(message)
    shape = tuple(Ymat.shape)
    if len(shape) < 2 or shape[-2:] != B_np.shape:
        message = f"Ymat must end with matrix shape {B_np.shape}, but got shape={shape}"
        logger.error(message)
        raise ValueError(message)
    dev = Ymat.device if isinstance(Ymat, torch.Tensor) and Ymat.is_cuda else nat.require_cuda()
    complex_mode = Ymat.is_complex() if isinstance(Ymat, torch.Tensor) else np.iscomplexobj(np.asarray(Ymat))
    Y = nat.as_device(Ymat, dev, torch.complex128 if complex_mode else torch.float64).reshape(-1, *B_np.shape)
    out = transform_device(Y, nat.as_device(B_np, dev, torch.float64)).reshape(shape)
    return out if isinstance(Ymat, torch.Tensor) else out.cpu().numpy()
