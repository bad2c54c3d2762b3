"""Partial-wave sweep on the GPU against one solve per (J, parity) system.

Every block of a rigid-rotor sweep (J = 0..4, both parities, one empty block) must give the
same S matrices as solving its system alone, in FP64 (1e-10: same arithmetic, different
batching and padding) and in mixed precision (1e-6); a graph replay with new energies must
equal a fresh direct run bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

import pyticc_b200 as tb
from pyticc_b200 import workloads

pytestmark = pytest.mark.gpu


def _systems(jmax=6, Jmax=4):
    base = workloads.rigid_atom_diatom(jmax=jmax, J=0, n_energy=3, boundaries=(2.5, 14.0))
    rotor = workloads.rigid_rotor(20.0, jmax)
    pes = workloads.lj_aniso_pes(150.0, 6.5, 0.3, 0.2)
    systems = [tb.build_ScattSystem(tb.AtomSpec(), rotor, Jtot=J, system_parity=p, potential=pes, reduced_mass=18.0 * tb.AMU2AU) for J in range(Jmax + 1) for p in (1, -1)]
    return systems, base.grid


def _compare(results, systems, grid, energies, config, tol):
    worst = 0.0
    for system, result in zip(systems, results, strict=True):
        if system.basis.n_channel == 0:
            assert result is None
            continue
        alone = tb.solve(system, energies, grid, config)
        for a, b in zip(result.Smat, alone.Smat, strict=True):
            assert a.shape == b.shape
            if a.size:
                worst = max(worst, float(np.abs(a - b).max()))
    assert worst <= tol, worst
    return worst


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_sweep_equals_one_solve_per_system(precision, tol):
    systems, grid = _systems()
    assert any(s.basis.n_channel == 0 for s in systems)  # J = 0, parity -1 has no channels
    energies = np.array([37.0, 183.0, 425.0]) * tb.CM2AU
    config = tb.Propagation(precision=precision)
    results = tb.solve_sweep(systems, energies, grid, config)
    _compare(results, systems, grid, energies, config, tol)


def test_graph_replay_matches_a_direct_run():
    systems, grid = _systems()
    config = tb.Propagation()
    e1 = np.array([37.0, 183.0, 425.0]) * tb.CM2AU
    e2 = np.array([70.0, 250.0, 460.0]) * tb.CM2AU
    sweep = tb.PartialWaveSweep(systems, grid, config, n_energy=3, energy_bound=float(e2.max()), graph=True)
    sweep.run(e1)                     # direct, then captured
    assert sweep.graph is not None
    replayed = sweep.run(e2)          # graph replay with new energies
    direct = tb.PartialWaveSweep(systems, grid, config, n_energy=3, energy_bound=float(e2.max()), graph=False).run(e2)
    for a, b in zip(replayed, direct, strict=True):
        if a is None:
            assert b is None
            continue
        for x, y in zip(a.Smat, b.Smat, strict=True):
            np.testing.assert_array_equal(x, y)
