"""Device evaluation of a Legendre-expansion PES (ticc_pes_legendre_grid) against its host
evaluation, the PotentialGrid it fills, and a solve on that grid."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import pyticc_b200 as tb
from pyticc_b200 import pes_analytic as pa
from pyticc_b200 import workloads
from pyticc_b200.pes import get_Vgrid_atom_diatom

pytestmark = pytest.mark.gpu


def test_device_grid_matches_host_evaluation():
    pes = pa.LegendrePES.build(
        [
            pa.LegendreTerm(0, (pa.Primitive("lj", 2e-3, 6.2), pa.Primitive("exp", 0.5, 1.1, 4.0)), (1.0, 0.2, -0.05)),
            pa.LegendreTerm(1, (pa.Primitive("power", -30.0, 6.0),), (0.3, 0.1)),
            pa.LegendreTerm(2, (pa.Primitive("gauss", 1e-3, 1.5, 7.0),)),
            pa.LegendreTerm(5, (pa.Primitive("lj", 1e-4, 6.0),), (0.1, 0.0, 0.02, 0.01)),
        ],
        re=1.3,
    )
    R = np.linspace(3.0, 25.0, 301)
    r = np.linspace(0.8, 2.2, 9)
    x, _ = np.polynomial.legendre.leggauss(20)
    V = pes.grid_device(R, r, x, torch.device("cuda", 0)).cpu().numpy().reshape(R.size, r.size, x.size)
    host = get_Vgrid_atom_diatom(pes, R, r, np.arccos(x))
    scale = np.abs(host).max(axis=(1, 2), keepdims=True)
    assert np.all(np.abs(V - host) <= 1e-13 * scale)


def test_prepare_potential_fills_the_grid_on_the_device_and_solves_the_same():
    """The rigid-rotor system with its surface as a LegendrePES: the grid equals the host
    evaluation, the device copy is the one the kernel wrote, and S equals the S of the same
    system with the surface as a plain callable."""
    plain = workloads.rigid_atom_diatom(jmax=10, J=6, n_theta=16, boundaries=(2.5, 20.0), half_steps=(0.05,), n_energy=4)
    system = tb.build_ScattSystem(
        tb.AtomSpec(), workloads.rigid_rotor(20.0, 10), Jtot=6, system_parity=1, potential=pa.lj_aniso_legendre(150.0 * tb.CM2AU, 6.5, 0.3, 0.2), reduced_mass=18.0 * tb.AMU2AU
    )
    grid = tb.prepare_potential(system, (2.5, 20.0), (0.05,), n_theta=16)
    assert (("cuda", 0) in grid._device_cache) or any(k[0] == "cuda" for k in grid._device_cache)
    np.testing.assert_allclose(grid.values, plain.grid.values, rtol=0, atol=1e-13 * np.abs(plain.grid.values).max())
    E = plain.energies
    a = tb.solve(plain.system, E, plain.grid, tb.Propagation())
    b = tb.solve(system, E, grid, tb.Propagation())
    for sa, sb in zip(a.Smat, b.Smat):
        assert sa.shape == sb.shape
        if sa.size:
            assert np.abs(sa - sb).max() <= 1e-10
