"""The electric-field SF and diabatic contraction fixtures (made by the reference's own host
functions) restated in NumPy: pins what the CUDA path has to reproduce."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

DATA = np.load(Path(__file__).parent / "golden" / "contract_families.npz")
PARAMS = json.loads(str(DATA["params_json"]))


def test_electric_sf_is_the_symmetrised_two_component_contraction():
    Bc, Bs, pot = DATA["sf_B_cos"], DATA["sf_B_sin"], DATA["sf_pot"]
    for R in range(pot.shape[0]):
        v = pot[R].ravel()
        M = (Bc * v) @ Bc.T + (Bs * v) @ Bs.T
        np.testing.assert_allclose(DATA["sf_V"][R], 0.5 * (M + M.T), rtol=0, atol=1e-12 * np.abs(M).max())
    idx = PARAMS["sf_subset"]
    v = pot[1].ravel()
    M = (Bc[idx] * v) @ Bc[idx].T + (Bs[idx] * v) @ Bs[idx].T
    np.testing.assert_allclose(DATA["sf_V_subset"], 0.5 * (M + M.T), rtol=0, atol=1e-12 * np.abs(M).max())


def test_diabatic_is_blocks_of_state_weighted_products():
    groups = {tuple(int(x) for x in k.split(",")): v for k, v in PARAMS["groups"].items()}
    n = 12
    d = (DATA["dia_d0"], DATA["dia_d1"])
    c = DATA["dia_c"]
    for R in range(c.shape[0]):
        V = np.zeros((n, n))
        for (s, K), idx in groups.items():
            B = DATA[f"dia_Bd_{s}_{K}"]
            M = (B * d[s][R].ravel()) @ B.T
            V[np.ix_(idx, idx)] = 0.5 * (M + M.T)
        for K in (0, 1):
            A, B = DATA[f"dia_Bc_0_{K}"], DATA[f"dia_Bc_1_{K}"]
            X = (A * c[R, :, :, 0, 1].ravel()) @ B.T
            ia, ib = groups[(0, K)], groups[(1, K)]
            V[np.ix_(ia, ib)] = X
            V[np.ix_(ib, ia)] = X.T
        np.testing.assert_allclose(DATA["dia_V"][R], V, rtol=0, atol=1e-12 * np.abs(V).max())


FS = np.load(Path(__file__).parent / "golden" / "contract_fs.npz")
FS_PARAMS = json.loads(str(FS["params_json"]))


def _packed(n_channel, indices):
    pr, pc = np.tril_indices(len(indices))
    sel = np.asarray(indices)
    hi, lo = np.maximum(sel[pr], sel[pc]), np.minimum(sel[pr], sel[pc])
    return pr, pc, hi * (hi + 1) // 2 + lo, sel


def test_scalar_fs_is_a_packed_pair_product_scattered_symmetrically():
    n, idx = FS_PARAMS["n_channel"], FS_PARAMS["fs_subset"]
    for pot, want, indices in ((FS["fs_pot"].reshape(3, -1), FS["fs_V"], list(range(n))), (FS["fs_pot"][0].reshape(1, -1), FS["fs_V_subset"][None], idx)):
        pr, pc, packed, _ = _packed(n, indices)
        c = pot @ FS["fs_kernel"][:, packed]
        M = np.zeros((pot.shape[0], len(indices), len(indices)))
        M[:, pr, pc] = c
        M[:, pc, pr] = c
        np.testing.assert_allclose(want, M, rtol=0, atol=1e-12 * np.abs(M).max())


def test_spin_fs_is_a_packed_pair_product_scattered_hermitian():
    n, idx = FS_PARAMS["n_channel"], FS_PARAMS["spin_subset"]
    k = FS["spin_kernel"].reshape(-1, FS["spin_kernel"].shape[-1])
    for pot, want, indices in ((FS["spin_pot"].reshape(3, -1), FS["spin_V"], list(range(n))), (FS["spin_pot"][1].reshape(1, -1), FS["spin_V_subset"][None], idx)):
        pr, pc, packed, sel = _packed(n, indices)
        c = pot @ k[:, packed]
        rev = sel[pr] < sel[pc]
        c[:, rev] = np.conj(c[:, rev])
        M = np.zeros((pot.shape[0], len(indices), len(indices)), dtype=complex)
        M[:, pr, pc] = c
        off = pr != pc
        M[:, pc[off], pr[off]] = np.conj(c[:, off])
        M[:, pr[~off], pc[~off]] = np.real(c[:, ~off])
        np.testing.assert_allclose(want, M, rtol=0, atol=1e-12 * np.abs(M).max())
