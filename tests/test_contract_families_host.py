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
