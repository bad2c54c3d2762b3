"""CPU restatement of the windowed radial driver and the full solve (test infrastructure only).

References: ``src/pyticc/propagation/runner.py:112-322`` (propagate / window loop:
initial Y from W(R0;E), W_base per window, LDMD per window),
``src/pyticc/match/finalize.py:32-98`` (BF→SF transform then get_Smat).
Windows only bound memory in the reference; their results agree with a one-shot
propagation to 1e-13 (reference ``test_propagation_runner.py:84-109``), so this
restatement propagates the whole grid at once unless ``window`` is given.
"""

from __future__ import annotations

import numpy as np

from . import contraction, ldmd, matching


def propagate(E_int, U, groups, B_real, B_imag, normalization, potential_values, radial_points, half_steps, reduced_mass, energies, mode="inelastic", window=None, sector_range=None, channel_indices=None):
    """Y at the last sector end for every energy (runner.py:165-322).

    With ``channel_indices`` the propagation covers that channel block only (the CS / NNCC
    block loop of runner.py:165-322 calls propagate_logD per block): ``E_int`` and ``U``
    are then the block's, and V is contracted over the block's channels."""
    energies = np.asarray(energies, dtype=np.float64)
    n = len(E_int)
    n_sector = len(half_steps)
    first, last = (0, n_sector) if sector_range is None else sector_range
    window = n_sector if window is None else window
    Y = None
    for start in range(first, last, window):
        stop = min(start + window, last)
        points = slice(2 * start, 2 * stop + 1)
        V = contraction.contract(groups, B_real, B_imag, normalization, potential_values[points], n, channel_indices)
        W = contraction.assemble_W_base(radial_points[points], U, E_int, reduced_mass, V)
        if Y is None:
            W0 = W[0][None] - 2.0 * reduced_mass * energies[:, None, None] * np.eye(n)
            Y = ldmd.initialize_inelastic(W0) if mode == "inelastic" else ldmd.initialize_capture(W0)
        Y = ldmd.propagate_logD(Y, energies, reduced_mass, half_steps[start:stop], W[0:-1:2], W[1::2], W[2::2])
    return Y


def solve(E_int, U, groups, B_real, B_imag, normalization, potential_values, radial_points, half_steps, reduced_mass, energies, Bmat, L, mode="inelastic", window=None, channel_indices=None):
    """Propagate then transform and match (solver.py:142-150, finalize.py:32-98; for one
    CS / NNCC block, finalize.py:168-225 with the block's Bmat and L)."""
    Y = propagate(E_int, U, groups, B_real, B_imag, normalization, potential_values, radial_points, half_steps, reduced_mass, energies, mode, window, channel_indices=channel_indices)
    Y_sf = matching.transform_bf_to_sf(Y, Bmat)
    Rmatch = float(radial_points[-1])
    return Y, matching.get_Smat(Y_sf, Rmatch, energies, reduced_mass, E_int, L)
