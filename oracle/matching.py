"""NumPy/SciPy restatement of asymptotic matching (test infrastructure only).

References: ``src/pyticc/match/asymptotic.py:82-110`` (BF→SF transform),
``src/pyticc/match/bessel.py:7-45,90-122`` (Riccati–Bessel and K log-derivative,
which call ``scipy.special``), ``src/pyticc/match/smatrix.py:10-223`` (get_Smat).
"""

from __future__ import annotations

import numpy as np
from scipy import special


def transform_bf_to_sf(Y, B):
    """Y_SF = B^T Y_BF B (asymptotic.py:82-110)."""
    return np.einsum("ia,...ij,jb->...ab", B, Y, B, optimize=True)


def riccati_bessel_jy(ell: float, x: float):
    """(j, n, j', n') = sqrt(pi x/2) (J_nu, Y_nu, J'_nu + J_nu/(2x), ...), nu = ell + 1/2 (bessel.py:7-45)."""
    nu = ell + 0.5
    scale = np.sqrt(np.pi * x / 2.0)
    J, Y = special.jv(nu, x), special.yv(nu, x)
    Jp, Yp = special.jvp(nu, x), special.yvp(nu, x)
    return scale * J, scale * Y, scale * (Jp + 0.5 * J / x), scale * (Yp + 0.5 * Y / x)


def modified_bessel_K_logD(nu: float, x: float) -> float:
    """K'_nu/K_nu = -K_{nu-1}/K_nu - nu/x with exponentially scaled kve (bessel.py:90-122)."""
    return float(-special.kve(nu - 1.0, x) / special.kve(nu, x) - nu / x)


def reference_functions(energy, Rmatch, reduced_mass, E_int, L):
    """Open-channel J, N, J', N' and closed-channel Gamma (smatrix.py:10-79)."""
    difference = energy - np.asarray(E_int)
    if np.any(difference == 0.0):
        raise ValueError(f"Asymptotic matching is undefined exactly at a channel threshold Etot={energy}")
    open_idx = np.flatnonzero(difference > 0.0)
    closed_idx = np.flatnonzero(difference < 0.0)
    J = np.empty(open_idx.size)
    N = np.empty(open_idx.size)
    Jp = np.empty(open_idx.size)
    Np = np.empty(open_idx.size)
    Gamma = np.empty(closed_idx.size)
    for pos, i in enumerate(open_idx):
        k = np.sqrt(2.0 * reduced_mass * abs(difference[i]))
        j, n, jd, nd = riccati_bessel_jy(float(L[i]), k * Rmatch)
        J[pos], N[pos] = j / np.sqrt(k), n / np.sqrt(k)
        Jp[pos], Np[pos] = np.sqrt(k) * jd, np.sqrt(k) * nd
    for pos, i in enumerate(closed_idx):
        k = np.sqrt(2.0 * reduced_mass * abs(difference[i]))
        Gamma[pos] = 0.5 / Rmatch + k * modified_bessel_K_logD(float(L[i] + 0.5), k * Rmatch)
    return open_idx, closed_idx, J, N, Jp, Np, Gamma


def open_reaction_matrix(Y, open_idx, closed_idx, J, N, Jp, Np, Gamma):
    """Closed-channel elimination then K_oo (smatrix.py:86-132)."""
    Y_open = Y[np.ix_(open_idx, open_idx)]
    if closed_idx.size:
        Y_oc = Y[np.ix_(open_idx, closed_idx)]
        Y_co = Y[np.ix_(closed_idx, open_idx)]
        closed = Y[np.ix_(closed_idx, closed_idx)] - np.diag(Gamma)
        Y_open = Y_open - Y_oc @ np.linalg.solve(closed, Y_co)
    left = Y_open * N[None, :] - np.diag(Np)
    right = Y_open * J[None, :] - np.diag(Jp)
    return np.asarray(-np.linalg.solve(left, right), dtype=np.complex128)


def get_Smat(Y, Rmatch, energies, reduced_mass, E_int, L):
    """S = (I + iK)^-1 (I - iK) per energy (smatrix.py:139-223)."""
    Y = np.asarray(Y)
    out = []
    for e, energy in enumerate(np.asarray(energies, dtype=np.float64)):
        refs = reference_functions(float(energy), Rmatch, reduced_mass, E_int, L)
        open_idx = refs[0]
        if open_idx.size == 0:
            out.append(np.empty((0, 0), dtype=np.complex128))
            continue
        K = open_reaction_matrix(Y[e], *refs)
        identity = np.eye(open_idx.size, dtype=np.complex128)
        out.append(np.linalg.solve(identity + 1j * K, identity - 1j * K))
    return tuple(out)
