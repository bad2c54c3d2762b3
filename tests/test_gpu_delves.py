"""Delves propagation on the GPU against the reference's own propagate_delves on the same
synthetic surface provider (tests/golden/delves.npz, made by tests/golden/make_golden.py)."""

from __future__ import annotations

import json
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

import pyticc_b200 as tb
from pyticc_b200.propagation import build_radial_sectors
from pyticc_b200.propagation.delves import propagate_delves

pytestmark = pytest.mark.gpu

DATA = np.load(Path(__file__).parent / "golden" / "delves.npz")
PARAMS = json.loads(str(DATA["params_json"]))


class _Provider:
    """The fixture's surfaces, looked up by sector midpoint; overlap C_a^T C_b."""

    def __init__(self):
        self.basis = SimpleNamespace(rho_min=PARAMS["rho_min"], mass=tuple(m * tb.AMU2AU for m in PARAMS["masses_amu"]), n_primitive=DATA["surface_coefficients"].shape[1])

    def surface(self, rho):
        i = int(np.argmin(np.abs(DATA["rho"] - rho)))
        assert abs(DATA["rho"][i] - rho) < 1e-12
        n = int(DATA["n_surface"][i])
        return SimpleNamespace(rho=rho, energies=DATA["surface_energies"][i, :n], coefficients=DATA["surface_coefficients"][i, :, :n])

    def transform(self, a, b):
        return a.coefficients.T @ b.coefficients


@pytest.mark.parametrize("mode", ["inelastic", "capture"])
def test_delves_propagation_matches_reference(mode):
    sectors = build_radial_sectors((PARAMS["rho_min"], PARAMS["rho_max"]), (PARAMS["half_step"],))
    result = propagate_delves(_Provider(), DATA["energies"], sectors, tb.Propagation(mode=mode))
    Y = result.Y_final.cpu().numpy()
    want = DATA[f"Y_{mode}"]
    assert Y.shape == want.shape == (3, 4, 4)
    assert np.abs(Y - want).max() <= 1e-10 * np.abs(want).max()
    assert result.surface_energies.size == 4 and result.rho_final == pytest.approx(PARAMS["rho_max"])
