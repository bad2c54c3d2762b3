"""NumPy restatement of the V(R) contraction and W assembly (test infrastructure only).

References: ``src/pyticc/matrix/interaction/common.py:49-62,97-146`` (contract),
``src/pyticc/propagation/runner.py:265-281`` (W_base on device),
``src/pyticc/matrix/radial.py:7-57`` (get_Wmat).
"""

from __future__ import annotations

import numpy as np


def contract_block(B_real, B_imag, normalization, potential):
    """V_K = norm [(B_r v) B_r^T + (B_i v) B_i^T], then (V + V^T)/2 (common.py:49-62)."""
    V = (B_real * potential[None, :]) @ B_real.T
    if B_imag is not None:
        V = V + (B_imag * potential[None, :]) @ B_imag.T
    V = V * normalization
    return 0.5 * (V + V.T)


def contract(groups, B_real, B_imag, normalization, potential, n_channel, channel_indices=None):
    """Scatter every K block into the (n_R, N, N) block-diagonal V (common.py:97-146).

    ``groups`` maps K to the complete-basis positions of that K block;
    ``B_real[K]`` / ``B_imag[K]`` hold the matching weighted rows.
    """
    indices = tuple(range(n_channel)) if channel_indices is None else tuple(channel_indices)
    local = {g: i for i, g in enumerate(indices)}
    potential = np.asarray(potential, dtype=np.float64)
    batches = potential.reshape(potential.shape[0], -1)
    V = np.zeros((batches.shape[0], len(indices), len(indices)))
    for K, group in groups.items():
        selected = [(b, local[g]) for b, g in enumerate(group) if g in local]
        if not selected:
            continue
        rows, out = (np.asarray(x) for x in zip(*selected, strict=True))
        Br = B_real[K][rows]
        Bi = None if B_imag is None else B_imag[K][rows]
        for r in range(batches.shape[0]):
            V[r][np.ix_(out, out)] = contract_block(Br, Bi, normalization, batches[r])
    return V


def assemble_W_base(radial_points, U, E_int, reduced_mass, V):
    """W_base(R) = U/R^2 + 2 mu V(R) + 2 mu diag(E_int) (runner.py:269-271, radial.py:68-70)."""
    R = np.asarray(radial_points, dtype=np.float64)
    W = U[None, :, :] / R[:, None, None] ** 2 + 2.0 * reduced_mass * V
    W[:, np.arange(U.shape[0]), np.arange(U.shape[0])] += 2.0 * reduced_mass * np.asarray(E_int)[None, :]
    return W
