"""Partial cross sections from S (host arithmetic), checked on the reference's own S matrices.

The reference computes no cross sections, so they are pinned here by (1) an independent
channel-by-channel restatement of the Arthurs–Dalgarno sum applied to the reference's S,
(2) detailed balance g_i k_i^2 sigma_{i->f} = g_f k_f^2 sigma_{f->i}, which holds for a
symmetric S, and (3) the uncoupled limit, where only elastic terms survive.
"""

from __future__ import annotations

import numpy as np
import pytest

import pyticc_b200 as tb
from tests.test_host_golden import _system_for

FIXTURES = ["solve_rigid_p+", "solve_rigid_p-", "solve_morse", "solve_diatom_diatom"]


def build_case(name):
    return _system_for(name)[2]


def _data(name):
    return _system_for(name)[0]


def _fixture_smats(data) -> list[np.ndarray]:
    return [data["Smat"][e, :k, :k] for e, k in enumerate(data["n_open"])]


def _direct_sum(basis, energies, smats, mu):
    """sigma_{i->f} channel by channel (no level matrices)."""
    levels = []
    for c in basis:
        if (c.mis_X, c.mis_Y) not in levels:
            levels.append((c.mis_X, c.mis_Y))
    out = np.zeros((len(energies), len(levels), len(levels)))
    for e, (E, S) in enumerate(zip(energies, smats, strict=True)):
        open_channels = [c for c in range(basis.n_channel) if basis.E_int[c] < E]
        for a_pos, a in enumerate(open_channels):
            i = levels.index((basis[a].mis_X, basis[a].mis_Y))
            g = (2 * basis[a].mis_X.j + 1) * (2 * basis[a].mis_Y.j + 1)
            k2 = 2.0 * mu * (E - basis.E_int[a])
            for b_pos, b in enumerate(open_channels):
                f = levels.index((basis[b].mis_X, basis[b].mis_Y))
                t = (1.0 if a == b else 0.0) - S[a_pos, b_pos]
                out[e, i, f] += np.pi * (2 * basis.Jtot + 1) / (g * k2) * abs(t) ** 2
    return out


@pytest.mark.parametrize("name", FIXTURES)
def test_cross_sections_from_reference_S_match_a_direct_sum(name):
    data = _data(name)
    system = build_case(name)
    smats = _fixture_smats(data)
    cs = tb.partial_cross_sections(system.basis, data["energies"], smats, system.reduced_mass)
    want = _direct_sum(system.basis, data["energies"], smats, system.reduced_mass)
    np.testing.assert_allclose(cs.sigma, want, rtol=1e-13, atol=1e-13 * max(1.0, np.abs(want).max()))
    assert cs.sigma.shape[1] == len(cs.levels) == cs.thresholds.size


@pytest.mark.parametrize("name", FIXTURES)
def test_cross_sections_obey_detailed_balance(name):
    data = _data(name)
    system = build_case(name)
    cs = tb.partial_cross_sections(system.basis, data["energies"], _fixture_smats(data), system.reduced_mass)
    for e, E in enumerate(cs.Etot):
        idx = cs.open_levels(e)
        if idx.size < 2:
            continue
        flux = (cs.degeneracy * 2.0 * system.reduced_mass * (E - cs.thresholds))[idx]
        rate = flux[:, None] * cs.sigma[e][np.ix_(idx, idx)]
        np.testing.assert_allclose(rate, rate.T, rtol=1e-8, atol=1e-10 * np.abs(rate).max())


def test_uncoupled_S_gives_only_elastic_cross_sections():
    system = build_case("solve_rigid_p+")
    E = np.array([system.basis.E_int.max() + 1e-3])
    n = system.basis.n_channel
    phases = np.exp(2j * np.linspace(0.1, 1.3, n))
    cs = tb.partial_cross_sections(system.basis, E, [np.diag(phases)], system.reduced_mass)
    off = cs.sigma[0] - np.diag(np.diagonal(cs.sigma[0]))
    assert np.abs(off).max() == 0.0
    assert np.all(np.diagonal(cs.sigma[0]) > 0.0)


def test_cross_section_input_validation():
    system = build_case("solve_rigid_p+")
    with pytest.raises(ValueError, match="energies"):
        tb.partial_cross_sections(system.basis, [0.1, 0.2], [np.eye(1)], system.reduced_mass)
    with pytest.raises(ValueError, match="channels are open"):
        tb.partial_cross_sections(system.basis, [system.basis.E_int.max() + 1.0], [np.eye(1)], system.reduced_mass)
    with pytest.raises(ValueError, match="reduced_mass"):
        tb.partial_cross_sections(system.basis, [0.1], [np.eye(0)], -1.0)


def test_fixture_parameters_are_recorded():
    assert _system_for("solve_rigid_p+")[1]["J"] == 3
