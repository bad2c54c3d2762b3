"""NumPy restatement of the learned sector-width proposer (test infrastructure only).

The reference has no learned part: it propagates on the fixed grid of
``src/pyticc/propagation/grid.py:193-239``.  This module is the CPU checker for this
project's own CUDA kernels (``pyticc_b200/csrc/learned.cuh``): the per-sector features,
the MLP forward pass, the gradient of the asymmetric weighted squared loss, one Adam
step, and the aligned power-of-two merge of fixed-step sectors.  Everything is float64,
so the GPU's FP32 results are compared with a relative tolerance.
"""

from __future__ import annotations

import numpy as np

N_FEATURE = 8
N_HIDDEN = 32


def split_params(params: np.ndarray) -> dict[str, np.ndarray]:
    """W1 (32, 8), b1 (32,), W2 (32, 32), b2 (32,), w3 (32,), b3 () from the packed vector."""
    p = np.asarray(params, dtype=np.float64)
    sizes = {"W1": N_HIDDEN * N_FEATURE, "b1": N_HIDDEN, "W2": N_HIDDEN * N_HIDDEN, "b2": N_HIDDEN, "w3": N_HIDDEN, "b3": 1}
    out, at = {}, 0
    for name, size in sizes.items():
        out[name] = p[at : at + size]
        at += size
    out["W1"] = out["W1"].reshape(N_HIDDEN, N_FEATURE)
    out["W2"] = out["W2"].reshape(N_HIDDEN, N_HIDDEN)
    out["b3"] = out["b3"][0]
    assert at == p.size, (at, p.size)
    return out


def step_features(Ws: np.ndarray, Wm: np.ndarray, We: np.ndarray, h: np.ndarray, two_mu_emax: float, two_mu_emin: float) -> np.ndarray:
    """(n_sector, 8) features, the same definitions as the CUDA feature kernel."""
    n_sector, n, _ = Wm.shape
    out = np.empty((n_sector, N_FEATURE))
    off_mask = ~np.eye(n, dtype=bool)
    for s in range(n_sector):
        a, b, c, hs = Ws[s], Wm[s], We[s], float(h[s])
        diag = np.diagonal(b)
        p2, q2 = diag - two_mu_emax, diag - two_mu_emin
        off = np.abs(b[off_mask]).max() if n > 1 else 0.0
        out[s] = [
            np.arcsinh(np.max(-p2)),
            np.log10(np.min(np.abs(p2)) + 1e-12),
            np.log10(np.min(np.abs(q2)) + 1e-12),
            np.log10(np.abs(c - a).max() / (2.0 * hs) + 1e-30),
            np.log10(np.abs(c - 2.0 * b + a).max() / (hs * hs) + 1e-30),
            np.log10(off + 1e-30),
            np.log10(hs),
            np.log10(np.max(np.abs(p2)) + 1e-12),
        ]
    return out


def forward(params: np.ndarray, norm: np.ndarray, X: np.ndarray) -> tuple[np.ndarray, tuple]:
    P = split_params(params)
    norm = np.asarray(norm, dtype=np.float64)
    x = (np.asarray(X, dtype=np.float64) - norm[:N_FEATURE]) * norm[N_FEATURE:]
    h1 = np.tanh(x @ P["W1"].T + P["b1"])
    h2 = np.tanh(h1 @ P["W2"].T + P["b2"])
    y = h2 @ P["w3"] + P["b3"]
    return y, (x, h1, h2)


def loss_and_gradient(params, norm, X, target, weight, over_weight: float, inv_weight_sum: float) -> tuple[float, np.ndarray]:
    """Loss = inv_weight_sum * sum w c (y - t)^2 with c = over_weight where y > t, and its
    gradient packed like ``params``."""
    P = split_params(params)
    y, (x, h1, h2) = forward(params, norm, X)
    r = y - np.asarray(target, dtype=np.float64)
    c = np.where(r > 0.0, over_weight, 1.0) * np.asarray(weight, dtype=np.float64) * inv_weight_sum
    loss = float(np.sum(c * r * r))
    g = 2.0 * c * r
    d2 = g[:, None] * P["w3"][None, :] * (1.0 - h2 * h2)
    d1 = (d2 @ P["W2"]) * (1.0 - h1 * h1)
    grads = np.concatenate([(d1.T @ x).ravel(), d1.sum(0), (d2.T @ h1).ravel(), d2.sum(0), h2.T @ g, [g.sum()]])
    return loss, grads


def adam(params, grads, m, v, step: int, lr: float, beta1: float, beta2: float, eps: float):
    m = beta1 * m + (1.0 - beta1) * grads
    v = beta2 * v + (1.0 - beta2) * grads * grads
    mhat = m / (1.0 - beta1**step)
    vhat = v / (1.0 - beta2**step)
    return params - lr * mhat / (np.sqrt(vhat) + eps), m, v


def merge_groups(levels: np.ndarray, run_id: np.ndarray, max_level: int, phase: np.ndarray | None = None, phase_limit: float = 2.8) -> list[tuple[int, int]]:
    """[(first base sector, count)] — at each position the largest power of two m <= 2^max_level
    that is aligned within its run of equal-width sectors, stays inside the run, whose
    sectors all carry a proposed level >= log2(m) and, when ``phase`` (max open |p| h per
    base sector) is given, with m * phase < phase_limit on all of them."""
    n = len(levels)
    starts = {}
    for s in range(n):
        starts.setdefault(int(run_id[s]), s)
    groups = []
    s = 0
    while s < n:
        m = 2**max_level
        while m > 1:
            offset = s - starts[int(run_id[s])]
            fits = offset % m == 0 and s + m <= n and run_id[s + m - 1] == run_id[s]
            if fits and np.min(levels[s : s + m]) >= np.log2(m) and (phase is None or m * np.max(phase[s : s + m]) < phase_limit):
                break
            m //= 2
        groups.append((s, m))
        s += m
    return groups
