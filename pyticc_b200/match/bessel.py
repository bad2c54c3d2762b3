"""Riccati–Bessel functions and the closed-channel K log-derivative, evaluated by the
device kernels of ``ticc_riccati_bessel_jy`` / ``ticc_bessel_k_logd`` (drop-in for
``src/pyticc/match/bessel.py:7-45,90-122``; scalars or arrays)."""

from __future__ import annotations

import numpy as np
import torch
from loguru import logger

from .. import _native as nat


def riccati_bessel_jy_device(ell: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    """(n, 4) tensor of (j, n, j', n') for device arrays ell, x."""
    lib = nat.load_library()
    dev = ell.device
    out = torch.empty((ell.numel(), 4), dtype=torch.float64, device=dev)
    status = nat.DeviceStatus(dev)
    with torch.cuda.device(dev):
        nat.check(lib.ticc_riccati_bessel_jy(nat.ptr(ell), nat.ptr(x), ell.numel(), nat.ptr(out), status.pointer, nat.stream_handle(dev)), "ticc_riccati_bessel_jy")
        status.raise_if_failed("riccati_bessel_jy")
    return out


def riccati_bessel_jy(ell, x):
    """(j_ell, y_ell, j'_ell, y'_ell) = sqrt(pi x/2) (J_nu, Y_nu, ...), nu = ell + 1/2."""
    ell_a, x_a = np.broadcast_arrays(np.asarray(ell, dtype=np.float64), np.asarray(x, dtype=np.float64))
    if np.any(x_a <= 0.0) or np.any(ell_a < 0.0):
        message = f"x must be positive and ell must be non-negative, but got x={x}, ell={ell}"
        logger.error(message)
        raise ValueError(message)
    dev = nat.require_cuda()
    out = riccati_bessel_jy_device(nat.as_device(ell_a.ravel(), dev, torch.float64), nat.as_device(x_a.ravel(), dev, torch.float64)).cpu().numpy()
    if not np.all(np.isfinite(out)):
        message = f"Riccati-Bessel functions and derivatives must be finite, but got {out}"
        logger.error(message)
        raise ValueError(message)
    if ell_a.ndim == 0:
        return tuple(float(v) for v in out[0])
    return tuple(out[:, k].reshape(ell_a.shape) for k in range(4))


def modified_bessel_K_logD(nu, x):
    """K'_nu(x)/K_nu(x) = -K_{nu-1}(x)/K_nu(x) - nu/x."""
    nu_a, x_a = np.broadcast_arrays(np.asarray(nu, dtype=np.float64), np.asarray(x, dtype=np.float64))
    if np.any(x_a <= 0.0) or np.any(nu_a < 0.0):
        message = f"x must be positive and nu must be non-negative, but got x={x}, nu={nu}"
        logger.error(message)
        raise ValueError(message)
    dev = nat.require_cuda()
    lib = nat.load_library()
    n_t = nat.as_device(nu_a.ravel(), dev, torch.float64)
    x_t = nat.as_device(x_a.ravel(), dev, torch.float64)
    out = torch.empty_like(n_t)
    status = nat.DeviceStatus(dev)
    with torch.cuda.device(dev):
        nat.check(lib.ticc_bessel_k_logd(nat.ptr(n_t), nat.ptr(x_t), n_t.numel(), nat.ptr(out), status.pointer, nat.stream_handle(dev)), "ticc_bessel_k_logd")
        status.raise_if_failed("modified_bessel_K_logD")
    values = out.cpu().numpy()
    return float(values[0]) if nu_a.ndim == 0 else values.reshape(nu_a.shape)
