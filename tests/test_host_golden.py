"""Host-side setup (channels, U, B, L, weighted rows, sectors, windows) against the
reference's golden vectors.  No GPU needed."""

from __future__ import annotations

import numpy as np
import pytest

import pyticc_b200 as tb
from pyticc_b200 import workloads
from pyticc_b200.basis import DiatomSpec, build_ChannelBasis, gauss_legendre_dvr
from pyticc_b200.matrix.interaction import prepare_atom_diatom, prepare_diatom_diatom
from pyticc_b200.propagation.grid import build_radial_sectors, iter_radial_windows
from tests.conftest import golden_vrows, load_golden


def _system_for(name):
    g, p = load_golden(name)
    if name.startswith("solve_rigid"):
        diatom = workloads.rigid_rotor(p["B_cm"], p["jmax"])
        system = tb.build_ScattSystem(tb.AtomSpec(), diatom, Jtot=p["J"], system_parity=p["parity"], reduced_mass=p["mu_amu"] * tb.AMU2AU)
    elif name == "solve_morse":
        diatom = workloads.morse_diatom(p["De_cm"], p["re"], p["a"], p["diatom_mass_amu"], p["r_interval"], p["n_dvr"], p["vmax"], p["jmax"])
        system = tb.build_ScattSystem(tb.AtomSpec(), diatom, Jtot=p["J"], system_parity=1, reduced_mass=p["mu_amu"] * tb.AMU2AU)
    else:
        X = workloads.rigid_rotor(p["B1_cm"], p["jmax"])
        Y = workloads.rigid_rotor(p["B2_cm"], p["jmax"])
        system = tb.build_ScattSystem(X, Y, Jtot=p["J"], system_parity=1, reduced_mass=p["mu_amu"] * tb.AMU2AU)
    return g, p, system


@pytest.mark.parametrize("name", ["solve_rigid_p+", "solve_rigid_p-", "solve_morse", "solve_diatom_diatom"])
def test_channels_U_and_asymptotic_transform(name):
    g, p, system = _system_for(name)
    basis = system.basis
    channels = np.asarray([[c.mis_X.j, -1 if c.mis_X.v is None else c.mis_X.v, c.mis_Y.j, -1 if c.mis_Y.v is None else c.mis_Y.v, c.j_couple, c.K] for c in basis])
    np.testing.assert_array_equal(channels, g["channels"])
    np.testing.assert_allclose(basis.E_int, g["E_int"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(tb.get_Umat_BF(basis), g["U"], rtol=1e-14, atol=1e-14)
    B, L = tb.get_Bmat_BF_to_SF(basis)
    np.testing.assert_allclose(B, g["Bmat"], atol=1e-12)
    np.testing.assert_allclose(L, g["L"], atol=1e-10)


@pytest.mark.parametrize("name", ["solve_rigid_p+", "solve_morse", "solve_diatom_diatom"])
def test_weighted_rows_match_reference(name):
    g, p, system = _system_for(name)
    groups, B_real, B_imag, norm = golden_vrows(g)
    if name == "solve_diatom_diatom":
        cX, wX = gauss_legendre_dvr(-1.0, 1.0, p["n_theta_X"])
        cY, wY = gauss_legendre_dvr(-1.0, 1.0, p["n_theta_Y"])
        phi, wp = gauss_legendre_dvr(0.0, np.pi, p["n_phi"])
        vb = prepare_diatom_diatom(system.basis, system.monomer_X.rovib, system.monomer_Y.rovib, cX, wX, cY, wY, phi, wp)
    else:
        cos_theta, w = gauss_legendre_dvr(-1.0, 1.0, p["n_theta"])
        np.testing.assert_allclose(cos_theta, g["cos_theta"], atol=1e-15)
        vb = prepare_atom_diatom(system.basis, system.monomer_Y.rovib, cos_theta, w)
    assert vb.channel_indices == groups
    assert vb.normalization == pytest.approx(norm, rel=1e-15)
    for K in groups:
        np.testing.assert_allclose(vb.B_real[K], B_real[K], atol=1e-13)
        if B_imag is not None:
            np.testing.assert_allclose(vb.B_imag[K], B_imag[K], atol=1e-13)


def test_channel_counts_match_reference_builder():
    _, counts = load_golden("channel_counts")
    rotor = workloads.rigid_rotor(20.0, 20)
    for parity in (1, -1):
        assert build_ChannelBasis(tb.AtomSpec(), rotor, 20, parity).n_channel == counts[f"rigid_j20_J20_p{parity}"]
    table = DiatomSpec(Eint=np.zeros((4, 31)))
    for J in (0, 1, 2, 15, 30, 45, 60):
        for parity in (1, -1):
            assert build_ChannelBasis(tb.AtomSpec(), table, J, parity).n_channel == counts[f"vib_v3_j30_J{J}_p{parity}"]
    pair = DiatomSpec(Eint=np.zeros((1, 9)))
    for parity in (1, -1):
        assert build_ChannelBasis(pair, pair, 6, parity).n_channel == counts[f"pair_j8_J6_p{parity}"]
    slow = DiatomSpec(Eint=np.zeros((1, 41)))
    for J in (0, 5, 10):
        assert build_ChannelBasis(tb.AtomSpec(), slow, J, 1).n_channel == counts[f"capture_j40_J{J}_p1"]


def test_sectors_and_windows_match_reference():
    g, p = load_golden("grid")
    for index, (bounds, halves) in enumerate(p["cases"]):
        sectors = build_radial_sectors(bounds, halves)
        np.testing.assert_array_equal(np.asarray([[s.radial_start, s.radial_end] for s in sectors]), g[f"sectors_{index}"])
        windows = list(iter_radial_windows(sectors, n_grid=24, n_channel=231, n_energy=16, memory_limit_mb=64.0))
        np.testing.assert_array_equal([len(w) for w, _ in windows], g[f"window_sizes_{index}"])
        np.testing.assert_array_equal(np.concatenate([pts for _, pts in windows]), g[f"window_points_{index}"])


def test_potential_grid_points_and_values():
    g, p = load_golden("solve_rigid_p+")
    wl = workloads.rigid_atom_diatom(B_cm=p["B_cm"], jmax=p["jmax"], J=p["J"], parity=1, n_theta=p["n_theta"], boundaries=p["boundaries"], half_steps=p["half_steps"], n_energy=5)
    np.testing.assert_array_equal(wl.grid.radial_points, g["radial_points"])
    np.testing.assert_allclose(wl.grid.values, g["potential_values"], rtol=1e-13, atol=1e-18)


def test_validation_errors_match_reference():
    with pytest.raises(ValueError, match="strictly increasing"):
        build_radial_sectors((3.0, 2.0), (0.1,))
    with pytest.raises(ValueError, match="Propagation mode"):
        tb.Propagation(mode="elastic")
    with pytest.raises(ValueError, match="memory_mb"):
        tb.Propagation(memory_mb=0.0)
    with pytest.raises(ValueError, match="one-dimensional"):
        tb.get_Etot([[1.0]])
    with pytest.raises(ValueError, match="At least one total energy"):
        tb.get_Etot([])


def test_open_blocks_to_host_copies_only_the_open_corner():
    """The host copy of a matched batch keeps each energy's open-open block (in the
    reference's order) and nothing beyond the largest one."""
    import torch

    from pyticc_b200.match.smatrix import open_blocks_to_host

    rng = np.random.default_rng(7)
    S = torch.as_tensor(rng.normal(size=(3, 6, 6)) + 1j * rng.normal(size=(3, 6, 6)))
    n_open = np.array([2, 0, 4])
    out = open_blocks_to_host(S, n_open)
    assert [o.shape for o in out] == [(2, 2), (0, 0), (4, 4)]
    for e, o in enumerate(out):
        np.testing.assert_array_equal(o, S[e, : n_open[e], : n_open[e]].numpy())
    assert [o.shape for o in open_blocks_to_host(S[:1], np.array([0]))] == [(0, 0)]


def test_propagate_logD_keeps_the_reference_signature():
    """The parameter names and kinds of the reference's propagate_logD (recorded from the
    reference at the runner.py:293 call site) are this library's, so the runner's call binds."""
    import inspect

    from pyticc_b200.propagation.logd import propagate_logD

    _, params = load_golden("dropin_calls")
    ours = [[name, str(p.kind)] for name, p in inspect.signature(propagate_logD).parameters.items()]
    assert ours == params["parameters"]
