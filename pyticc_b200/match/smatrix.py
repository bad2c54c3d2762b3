"""S matrices from SF log-derivatives on the GPU — drop-in for ``pyticc.match.get_Smat``
(``src/pyticc/match/smatrix.py:139-223``).

The kernels (``ticc_match_smatrix``) evaluate the open-channel Riccati–Bessel functions
and closed-channel K log-derivatives, eliminate the closed channels and solve for S in
one complex solve per energy; see ``csrc/match.cuh``.
"""

from __future__ import annotations

import numpy as np
import torch
from loguru import logger

from .. import _native as nat
from ..energy import get_Etot


def get_Smat_device(Y: torch.Tensor, Rmatch: float, energies: np.ndarray, reduced_mass: float, E_int: np.ndarray, L: np.ndarray) -> tuple[torch.Tensor, np.ndarray]:
    """Device S (n_energy, n, n) complex128 with each open block top-left, and n_open."""
    lib = nat.load_library()
    dev = Y.device
    n_energy, n, _ = Y.shape
    if np.any(np.asarray(E_int)[None, :] == np.asarray(energies)[:, None]):
        e_index = int(np.flatnonzero(np.any(np.asarray(E_int)[None, :] == np.asarray(energies)[:, None], axis=1))[0])
        message = f"Asymptotic matching is undefined exactly at a channel threshold Etot={energies[e_index]}"
        logger.error(message)
        raise ValueError(message)
    n_open_host = np.sum(np.asarray(E_int)[None, :] < np.asarray(energies)[:, None], axis=1)
    max_open = int(n_open_host.max()) if n_open_host.size else 0
    is_complex = int(Y.is_complex())
    S = torch.empty((n_energy, n, n), dtype=torch.complex128, device=dev)
    n_open = torch.empty(n_energy, dtype=torch.int32, device=dev)
    e_t = nat.as_device(energies, dev, torch.float64)
    ei_t = nat.as_device(E_int, dev, torch.float64)
    l_t = nat.as_device(L, dev, torch.float64)
    with torch.cuda.device(dev):
        nbytes = nat.size_query(lib.ticc_match_workspace_size, n, n_energy, is_complex, max_open)
        work = nat.Workspace.get(dev, nbytes, slot=2)
        status = nat.DeviceStatus(dev)
        nat.check(
            lib.ticc_match_smatrix(
                nat.ptr(Y), is_complex, float(Rmatch), nat.ptr(e_t), n_energy, float(reduced_mass), nat.ptr(ei_t), nat.ptr(l_t), n, max_open,
                nat.ptr(S), nat.ptr(n_open), nat.ptr(work), work.numel(), status.pointer, nat.stream_handle(dev),
            ),
            "ticc_match_smatrix",
        )
        status.raise_if_failed("get_Smat")
    return S, n_open_host


def get_Smat(Ymat, Rmatch: float, Etot, reduced_mass: float, E_int, L) -> tuple[np.ndarray, ...]:
    """One S matrix per energy, of shape (n_open, n_open) in the order of
    flatnonzero(E_int < Etot[i]); empty (0, 0) when no channel is open."""
    energies = get_Etot(Etot)
    E_int_a = np.asarray(E_int, dtype=np.float64)
    L_a = np.asarray(L, dtype=np.float64)
    n = E_int_a.size
    shape = tuple(Ymat.shape)
    if shape != (energies.size, n, n):
        message = f"Ymat must have shape {(energies.size, n, n)}, but got {shape}"
        logger.error(message)
        raise ValueError(message)
    if E_int_a.ndim != 1 or L_a.shape != E_int_a.shape:
        message = f"E_int and L must be one-dimensional arrays with the same shape, but got {E_int_a.shape} and {L_a.shape}"
        logger.error(message)
        raise ValueError(message)
    if Rmatch <= 0.0 or reduced_mass <= 0.0:
        message = f"Rmatch and reduced_mass must be positive, but got Rmatch={Rmatch}, reduced_mass={reduced_mass}"
        logger.error(message)
        raise ValueError(message)
    if np.any(L_a < 0.0):
        message = "Orbital angular momenta L must be non-negative"
        logger.error(message)
        raise ValueError(message)
    dev = Ymat.device if isinstance(Ymat, torch.Tensor) and Ymat.is_cuda else nat.require_cuda()
    complex_mode = Ymat.is_complex() if isinstance(Ymat, torch.Tensor) else np.iscomplexobj(np.asarray(Ymat))
    Y = nat.as_device(Ymat, dev, torch.complex128 if complex_mode else torch.float64)
    S, n_open = get_Smat_device(Y, Rmatch, energies, reduced_mass, E_int_a, L_a)
    return open_blocks_to_host(S, n_open)


def open_blocks_to_host(S: torch.Tensor, n_open: np.ndarray) -> tuple[np.ndarray, ...]:
    """Host copies of the open-open blocks of a device S batch; only the leading
    max(n_open) x max(n_open) corner of each matrix crosses to the host."""
    m = int(np.max(n_open)) if len(n_open) else 0
    S_host = S[:, :m, :m].cpu().numpy()
    return tuple(np.ascontiguousarray(S_host[e, : n_open[e], : n_open[e]]) for e in range(len(n_open)))
