"""Coupled-states and NNCC block propagation on the GPU (``ticc_ldmd_propagate_blocks``)
against the reference's block solves, the oracle and the exact-CC limits.

Tolerances as for exact CC: Y and S of the plain FP64 path within 1e-8 of the reference
and the oracle; the limits where a block is the whole basis agree with the exact-CC
solve to 1e-12; mixed precision stays within 1e-6 of FP64.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import pyticc_b200 as tb
from oracle import pipeline as o_pipeline
from pyticc_b200 import workloads
from pyticc_b200.propagation.runner import propagate_blocks
from pyticc_b200.scattering import hamiltonian_for
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu

S_TOL = 1.0e-8
LIMIT_TOL = 1.0e-12
MIXED_TOL = 1.0e-6


def _fixture_workload(name):
    g, p = load_golden(name)
    approx = tb.Approx(p["approx"])
    energies_cm = g["energies"] * tb.AU2CM
    if name.startswith("solve_rigid"):
        wl = workloads.rigid_atom_diatom(
            B_cm=p["B_cm"], jmax=p["jmax"], J=p["J"], parity=p["parity"], n_theta=p["n_theta"], boundaries=p["boundaries"],
            half_steps=p["half_steps"], energies_cm=energies_cm, approx=approx, K_delta=p["K_delta"],
        )
    else:
        wl = workloads.rotor_pair(
            B1_cm=p["B1_cm"], B2_cm=p["B2_cm"], jmax=p["jmax"], J=p["J"], lmax=p["lmax"], seed=p["seed"], n_theta_X=p["n_theta_X"],
            n_theta_Y=p["n_theta_Y"], n_phi=p["n_phi"], boundaries=p["boundaries"], half_steps=p["half_steps"], energies_cm=energies_cm,
            approx=approx, K_delta=p["K_delta"],
        )
    return g, p, wl


@pytest.mark.parametrize("name", ["solve_rigid_cs", "solve_rigid_nncc", "solve_rigid_cs_capture", "solve_pair_nncc"])
def test_block_solve_matches_reference(name):
    g, p, wl = _fixture_workload(name)
    result = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation(mode=p["mode"]))
    assert isinstance(result, tb.CoupledStatesResult)
    assert len(result.blocks) == int(g["n_block"])
    for b, block in enumerate(result.blocks):
        assert list(block.block.channel_indices) == list(g[f"b{b}_channel_indices"])
        assert list(block.block.owned_channel_indices) == list(g[f"b{b}_owned"])
        np.testing.assert_allclose(block.Y_BF, g[f"b{b}_Y_BF"], rtol=1e-8, atol=1e-8)
        assert [s.shape[0] for s in block.Smat_asymptotic] == list(g[f"b{b}_n_open"])
        for e, (s, s_bf) in enumerate(zip(block.Smat_asymptotic, block.Smat_BF, strict=True)):
            n = s.shape[0]
            if n:
                assert np.abs(s - g[f"b{b}_Smat"][e, :n, :n]).max() <= S_TOL
                assert np.abs(s_bf - g[f"b{b}_Smat_BF"][e, :n, :n]).max() <= S_TOL


def _rigid(J, approx, K_cut=None, K_delta=1):
    """A small A+BC rigid rotor with an anisotropic LJ PES (3-5 bohr, h = 0.05)."""
    system = tb.build_ScattSystem(
        tb.AtomSpec(), workloads.rigid_rotor(20.0, 4), Jtot=J, system_parity=1, approx=approx, K_delta=K_delta,
        channel=tb.ChannelSpec(K_cut=K_cut), potential=workloads.lj_aniso_pes(150.0, 4.0, 0.3, 0.2), reduced_mass=2.0 * tb.AMU2AU,
    )
    grid = tb.prepare_potential(system, (3.0, 5.0), (0.05,), n_theta=8)
    return tb.solve(system, np.array([90.0, 260.0]) * tb.CM2AU, grid, tb.Propagation())


def _assert_exact_matches_single_block(exact, approximate):
    """Restates test_approximation_limits.py:64-77."""
    assert len(approximate.blocks) == 1
    block = approximate.blocks[0]
    assert block.block.channel_indices == tuple(range(exact.basis.n_channel))
    np.testing.assert_allclose(block.Y_BF, exact.Y_propagated, atol=LIMIT_TOL)
    np.testing.assert_allclose(block.Bmat, exact.asymptotic_transform, atol=LIMIT_TOL)
    np.testing.assert_allclose(block.L, exact.L, atol=LIMIT_TOL)
    np.testing.assert_allclose(block.Y_asymptotic, exact.Y_asymptotic, atol=LIMIT_TOL)
    for s_block, s_exact in zip(block.Smat_asymptotic, exact.Smat, strict=True):
        np.testing.assert_allclose(s_block, s_exact, atol=LIMIT_TOL)


def test_J_zero_exact_cs_and_nncc_are_identical():
    exact = _rigid(0, tb.Approx.EXACT)
    _assert_exact_matches_single_block(exact, _rigid(0, tb.Approx.CS))
    _assert_exact_matches_single_block(exact, _rigid(0, tb.Approx.NNCC))


def test_K_cut_zero_exact_and_cs_are_identical():
    _assert_exact_matches_single_block(_rigid(2, tb.Approx.EXACT, K_cut=0), _rigid(2, tb.Approx.CS, K_cut=0))


def test_nncc_covering_every_K_is_identical_to_exact():
    exact = _rigid(2, tb.Approx.EXACT)
    assert {c.K for c in exact.basis} == {0, 1, 2}
    _assert_exact_matches_single_block(exact, _rigid(2, tb.Approx.NNCC, K_delta=1))


def test_cs_blocks_are_unitary():
    result = _rigid(4, tb.Approx.CS)
    assert [b.block.K_values for b in result.blocks] == [(0,), (1,), (2,), (3,), (4,)]
    for block in result.blocks:
        for s, s_bf in zip(block.Smat_asymptotic, block.Smat_BF, strict=True):
            np.testing.assert_allclose(s.conj().T @ s, np.eye(s.shape[0]), atol=1e-12)
            np.testing.assert_allclose(s_bf.conj().T @ s_bf, np.eye(s_bf.shape[0]), atol=1e-12)


def _morse_nncc(approx=tb.Approx.NNCC, K_delta=1, **kw):
    """Vibrating A+BC, v <= 3, j <= 12, J = 8: NNCC windows of 72-144 channels (two 128-blocks
    for the largest, padding channels inside n for the others)."""
    args = dict(J=8, jmax=12, vmax=3, n_dvr=24, n_theta=16, boundaries=(2.5, 12.0), half_steps=(0.05,), energies_cm=[150.0, 1200.0, 2900.0])
    args.update(kw)
    return workloads.morse_atom_diatom(approx=approx, K_delta=K_delta, **args)


def test_batched_blocks_equal_one_block_at_a_time():
    """Padding a block with decoupled closed channels leaves its arithmetic unchanged."""
    wl = _morse_nncc(boundaries=(2.5, 6.0))
    ham = hamiltonian_for(wl.system, wl.grid)
    blocks = tuple(b.channel_indices for b in tb.build_nncc_blocks(wl.system.basis, K_delta=1))
    assert len({len(b) for b in blocks}) > 1
    together = propagate_blocks(ham, blocks, wl.energies, wl.grid.sectors, tb.Propagation())
    for block, Y in zip(blocks, together, strict=True):
        (alone,) = propagate_blocks(ham, (block,), wl.energies, wl.grid.sectors, tb.Propagation())
        assert torch.equal(Y, alone) or float((Y - alone).abs().max()) <= 1e-13


def test_nncc_blocks_match_oracle_across_padding():
    wl = _morse_nncc()
    result = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation())
    ham = hamiltonian_for(wl.system, wl.grid)
    vb = ham.V_basis
    U = tb.get_Umat_BF(wl.system.basis)
    values = wl.grid.values.reshape(wl.grid.radial_points.size, -1)
    halves = np.asarray([s.radial_half_step for s in wl.grid.sectors])
    sizes = [len(b.block.channel_indices) for b in result.blocks]
    assert max(sizes) > 128 > min(sizes)
    for block in result.blocks:
        idx = list(block.block.channel_indices)
        Y, S = o_pipeline.solve(
            wl.system.basis.E_int[idx], U[np.ix_(idx, idx)], vb.channel_indices, vb.B_real, None, 1.0, values, wl.grid.radial_points, halves,
            wl.system.reduced_mass, wl.energies, block.Bmat, block.L, channel_indices=idx,
        )
        np.testing.assert_allclose(block.Y_BF, Y, rtol=1e-8, atol=1e-8)
        for a, b in zip(block.Smat_asymptotic, S, strict=True):
            assert a.shape == b.shape
            if a.size:
                assert np.abs(a - b).max() <= S_TOL


def test_mixed_precision_blocks_match_fp64():
    wl = _morse_nncc(K_delta=2, J=10, jmax=16, boundaries=(2.5, 10.0), half_steps=(0.02,))
    plain = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation())
    mixed = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation(precision="mixed"))
    assert max(len(b.block.channel_indices) for b in plain.blocks) > 256
    for a, b in zip(plain.blocks, mixed.blocks, strict=True):
        for sa, sb in zip(a.Smat_asymptotic, b.Smat_asymptotic, strict=True):
            if sa.size:
                assert np.abs(sa - sb).max() <= MIXED_TOL


def test_learned_steps_are_refused_for_blocks():
    wl = workloads.rigid_atom_diatom(jmax=4, J=2, boundaries=(3.0, 4.0), n_theta=8, energies_cm=[100.0], approx=tb.Approx.CS)
    with pytest.raises(ValueError, match="exact coupled channels"):
        tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation(steps="learned"))
