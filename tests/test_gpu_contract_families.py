"""Electric-field SF and diabatic contractions on the GPU against the reference's own results
(tests/golden/contract_families.npz, made by tests/golden/make_golden.py)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest
import torch

from pyticc_b200.matrix import families as fam

pytestmark = pytest.mark.gpu

DATA = np.load(Path(__file__).parent / "golden" / "contract_families.npz")
PARAMS = json.loads(str(DATA["params_json"]))


def _close(got, want):
    got = got.cpu().numpy() if isinstance(got, torch.Tensor) else got
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_electric_sf_contraction_matches_reference():
    dev = torch.device("cuda", 0)
    grid_shape = tuple(PARAMS["grid_shape"])
    basis = fam.AtomDiatomVBasisElectricSF(DATA["sf_B_cos"].shape[0], grid_shape, np.zeros(3), np.zeros(1), DATA["sf_B_cos"], DATA["sf_B_sin"])
    basis_device = fam.device_basis_electric_sf(basis, dev)
    _close(fam.contract_electric_sf_device(basis, basis_device, DATA["sf_pot"], dev), DATA["sf_V"])
    _close(fam.contract_electric_sf_device(basis, None, DATA["sf_pot"][1], dev, PARAMS["sf_subset"]), DATA["sf_V_subset"])
    with pytest.raises(ValueError, match="unique"):
        fam.contract_electric_sf_device(basis, basis_device, DATA["sf_pot"], dev, (1, 1))


def _diabatic_basis():
    groups = {tuple(int(x) for x in k.split(",")): tuple(v) for k, v in PARAMS["groups"].items()}
    return fam.DiabaticVBasisBF(
        n_channel=12,
        n_state=2,
        theta=np.linspace(0.1, 3.0, PARAMS["n_theta"]),
        diagonal_grids=(DATA["dia_grid0"], DATA["dia_grid1"]),
        coupling_grid=DATA["dia_coupling_grid"],
        channel_indices=groups,
        B_diagonal={k: DATA[f"dia_Bd_{k[0]}_{k[1]}"] for k in groups},
        B_coupling={k: DATA[f"dia_Bc_{k[0]}_{k[1]}"] for k in groups},
    )


def test_diabatic_contraction_matches_reference():
    dev = torch.device("cuda", 0)
    basis = _diabatic_basis()
    basis_device = fam.device_basis_diabatic(basis, dev)
    grid = fam.DiabaticVGridBF(diagonal=(DATA["dia_d0"], DATA["dia_d1"]), coupling=DATA["dia_c"])
    V = fam.contract_diabatic_device(basis, basis_device, grid, dev)
    _close(V, DATA["dia_V"])
    Vc = V.cpu().numpy()
    np.testing.assert_array_equal(Vc, np.swapaxes(Vc, -2, -1))
    one = fam.DiabaticVGridBF(diagonal=(DATA["dia_d0"][2], DATA["dia_d1"][2]), coupling=DATA["dia_c"][2])
    _close(fam.contract_diabatic_device(basis, None, one, dev, PARAMS["dia_subset"]), DATA["dia_V_subset"])
    bad = DATA["dia_c"].copy()
    bad[..., 0, 1] += 1.0
    with pytest.raises(ValueError, match="symmetric"):
        fam.contract_diabatic_device(basis, basis_device, fam.DiabaticVGridBF(diagonal=(DATA["dia_d0"], DATA["dia_d1"]), coupling=bad), dev)


FS = np.load(Path(__file__).parent / "golden" / "contract_fs.npz")
FS_PARAMS = json.loads(str(FS["params_json"]))


class _FSBasis:
    def __init__(self, kernel, spin=False):
        n = FS_PARAMS["n_channel"]
        self.n_channel, self.grid_shape, self.kernel = n, tuple(FS_PARAMS["grid_shape"]), kernel
        self.pair_rows, self.pair_columns = np.tril_indices(n)
        if spin:
            self.two_total_spins, self.orbital_states = tuple(FS_PARAMS["two_total_spins"]), (None, None)


def test_scalar_fs_contraction_matches_reference():
    dev = torch.device("cuda", 0)
    basis = _FSBasis(FS["fs_kernel"])
    _close(fam.contract_fs_device(basis, fam.device_basis_fs(basis, dev), FS["fs_pot"], dev), FS["fs_V"])
    _close(fam.contract_fs_device(basis, None, FS["fs_pot"][0], dev, FS_PARAMS["fs_subset"]), FS["fs_V_subset"])


def test_spin_fs_contraction_matches_reference_and_is_hermitian():
    dev = torch.device("cuda", 0)
    basis = _FSBasis(FS["spin_kernel"], spin=True)
    V = fam.contract_fs_spin_device(basis, fam.device_basis_fs(basis, dev), FS["spin_pot"], dev)
    _close(V, FS["spin_V"])
    Vc = V.cpu().numpy()
    np.testing.assert_array_equal(Vc, np.conj(np.swapaxes(Vc, -2, -1)))
    _close(fam.contract_fs_spin_device(basis, None, FS["spin_pot"][1], dev, FS_PARAMS["spin_subset"]), FS["spin_V_subset"])
