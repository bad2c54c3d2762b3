"""NumPy restatement of the reference LDMD propagator (test infrastructure only).

Reference: ``src/pyticc/propagation/logd.py``.  The reference vectorises energies
with ``jax.vmap`` and sectors with ``jax.lax.scan``; here both are plain loops and
the linear solves are ``numpy.linalg.solve`` (LAPACK LU with partial pivoting),
which is what ``jnp.linalg.solve`` computes.
"""

from __future__ import annotations

import numpy as np


def initialize_inelastic(W: np.ndarray) -> np.ndarray:
    """Y_ii = sqrt|W_ii| (logd.py:48-65)."""
    diagonal = np.real(np.diagonal(W, axis1=-2, axis2=-1))
    values = np.sqrt(np.abs(diagonal))
    return values[..., :, None] * np.eye(W.shape[-1])


def initialize_capture(W: np.ndarray) -> np.ndarray:
    """Y_ii = sqrt(W_ii) for W_ii >= 0, else -i sqrt(-W_ii) (logd.py:72-91)."""
    diagonal = np.real(np.diagonal(W, axis1=-2, axis2=-1))
    values = np.where(diagonal >= 0.0, np.sqrt(np.maximum(diagonal, 0.0)) + 0j, -1j * np.sqrt(np.maximum(-diagonal, 0.0)))
    return values[..., :, None] * np.eye(W.shape[-1], dtype=np.complex128)


def reference_values(h: float, p2: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Diagonal reference propagators y1, y2 from p^2 (logd.py:98-132).

    p^2 >= 0: y1 = p coth(ph), y2 = p csch(ph); p^2 < 0: y1 = |p| cot(|p|h),
    y2 = |p| csc(|p|h); |p h| < 1e-5 uses the three-term Taylor series.
    """
    magnitude = np.sqrt(np.abs(p2))
    argument = magnitude * h
    small = np.abs(argument) < 1.0e-5
    safe = np.where(small, 1.0, argument)
    with np.errstate(divide="ignore", invalid="ignore"):
        y1 = np.where(p2 >= 0.0, magnitude / np.tanh(safe), magnitude / np.tan(safe))
        y2 = np.where(p2 >= 0.0, magnitude / np.sinh(safe), magnitude / np.sin(safe))
    y1_series = 1.0 / h + p2 * h / 3.0 - p2**2 * h**3 / 45.0
    y2_series = 1.0 / h - p2 * h / 6.0 + 7.0 * p2**2 * h**3 / 360.0
    return np.where(small, y1_series, y1), np.where(small, y2_series, y2)


def correction_matrices(h: float, W_start: np.ndarray, W_mid: np.ndarray, W_end: np.ndarray):
    """Energy-independent sector corrections (logd.py:143-164).

    ref = diag(W_mid); T = W - diag(ref); Q_start = h T_start / 3,
    Q_mid = (4/h) [(I - h^2 T_mid / 6)^-1 - I], Q_end = h T_end / 3.
    """
    n = W_mid.shape[-1]
    identity = np.eye(n)
    ref = np.real(np.diag(W_mid)).copy()
    reference = np.diag(ref)
    Q_start = h * (W_start - reference) / 3.0
    Q_mid = 4.0 / h * (np.linalg.solve(identity - h**2 * (W_mid - reference) / 6.0, identity) - identity)
    Q_end = h * (W_end - reference) / 3.0
    return ref, Q_start, Q_mid, Q_end


def propagate_with_corrections(Y, h, p2, Q_start, Q_mid, Q_end):
    """One energy through one sector with precomputed corrections (logd.py:168-194)."""
    dtype = np.result_type(Y.dtype, Q_start.dtype)
    y1, y2 = reference_values(h, p2)
    D = np.diag(y2).astype(dtype)
    start = Y + Q_start + np.diag(y1)
    Y_mid = Q_mid + np.diag(y1) - y2[:, None] * np.linalg.solve(start, D)
    mid = Y_mid + Q_mid + np.diag(y1)
    Y_end = Q_end + np.diag(y1) - y2[:, None] * np.linalg.solve(mid, D)
    return 0.5 * (Y_end + Y_end.T)


def propagate_logD(Y_initial, energies, reduced_mass, half_steps, W_start, W_mid, W_end):
    """All energies through all sectors (logd.py:288-330, 340-398)."""
    Y_initial = np.asarray(Y_initial)
    dtype = np.result_type(Y_initial.dtype, np.asarray(W_start).dtype)
    Y = np.array(Y_initial, dtype=dtype, copy=True)
    corrections = [correction_matrices(float(h), Ws, Wm, We) for h, Ws, Wm, We in zip(half_steps, W_start, W_mid, W_end, strict=True)]
    shift = 2.0 * reduced_mass * np.asarray(energies, dtype=np.float64)
    for e in range(Y.shape[0]):
        for h, (ref, Qs, Qm, Qe) in zip(half_steps, corrections, strict=True):
            Y[e] = propagate_with_corrections(Y[e], float(h), ref - shift[e], Qs, Qm, Qe)
    return Y
