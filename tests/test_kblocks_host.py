"""Coupled-states / NNCC host logic and oracle, pinned to the reference (no GPU).

The block builders and the block BF -> SF transforms are compared with the reference's
own outputs (``tests/golden/kblocks.npz``, ``solve_*_{cs,nncc}.npz``); the reference's
block-builder tests (``tests/unit/test_kblock.py``) are restated; and the oracle's
per-block propagation and matching is checked against the reference's block solves.
"""

from __future__ import annotations

import numpy as np
import pytest

import pyticc_b200 as tb
from oracle import pipeline
from pyticc_b200.basis import DiatomSpec, build_ChannelBasis
from tests.conftest import golden_vrows, load_golden

BLOCK_FIXTURES = ["solve_rigid_cs", "solve_rigid_nncc", "solve_rigid_cs_capture", "solve_pair_nncc"]


def _case_channels(name):
    X = tb.AtomSpec() if name.startswith("atom") else DiatomSpec(Eint=np.zeros((1, 4)))
    table = {
        "atom_j4_J4": (np.zeros((1, 5)), 4, 1, None),
        "atom_j6_J9_p-": (np.zeros((2, 7)), 9, -1, None),
        "atom_j8_J8_Kcut3": (np.zeros((1, 9)), 8, 1, 3),
        "pair_j3_J5": (np.zeros((1, 3)), 5, 1, None),
        "atom_j2_J0": (np.zeros((1, 3)), 0, 1, None),
    }
    Eint, J, parity, K_cut = table[name]
    return build_ChannelBasis(X, DiatomSpec(Eint=Eint), J, parity, tb.ChannelSpec(K_cut=K_cut))


def _as_lists(block):
    return [list(block.K_values), list(block.channel_indices), list(block.owned_K_values), list(block.owned_channel_indices), block.center_K]


@pytest.mark.parametrize("name", ["atom_j4_J4", "atom_j6_J9_p-", "atom_j8_J8_Kcut3", "pair_j3_J5", "atom_j2_J0"])
def test_block_builders_match_reference(name):
    _, p = load_golden("kblocks")
    expected = p["cases"][name]
    channels = _case_channels(name)
    assert [float(c.K) for c in channels] == expected["K"]
    assert [_as_lists(b) for b in tb.build_cs_blocks(channels)] == expected["cs"]
    for K_delta, blocks in expected["nncc"].items():
        assert [_as_lists(b) for b in tb.build_nncc_blocks(channels, K_delta=int(K_delta))] == blocks


def test_cs_builds_one_owned_block_per_K():
    """Restates test_kblock.py:15-22."""
    channels = build_ChannelBasis(tb.AtomSpec(), DiatomSpec(Eint=np.zeros((1, 5))), 4, 1)
    blocks = tb.build_cs_blocks(channels)
    assert [b.K_values for b in blocks] == [(0,), (1,), (2,), (3,), (4,)]
    assert [b.owned_K_values for b in blocks] == [(0,), (1,), (2,), (3,), (4,)]
    assert sorted(i for b in blocks for i in b.owned_channel_indices) == list(range(len(channels)))


def test_nncc_delta_one_builds_overlapping_three_K_windows():
    """Restates test_kblock.py:25-33."""
    channels = build_ChannelBasis(tb.AtomSpec(), DiatomSpec(Eint=np.zeros((1, 5))), 4, 1)
    blocks = tb.build_nncc_blocks(channels, K_delta=1)
    assert [b.K_values for b in blocks] == [(0, 1, 2), (1, 2, 3), (2, 3, 4)]
    assert [b.owned_K_values for b in blocks] == [(0, 1), (2,), (3, 4)]
    assert sorted(i for b in blocks for i in b.owned_channel_indices) == list(range(len(channels)))
    assert all(set(b.owned_channel_indices) <= set(b.channel_indices) for b in blocks)


def test_nncc_rejects_bad_K_delta_and_empty_channels():
    channels = build_ChannelBasis(tb.AtomSpec(), DiatomSpec(Eint=np.zeros((1, 3))), 2, 1)
    for bad in (0, -1, 1.5, True):
        with pytest.raises(ValueError, match="K_delta"):
            tb.build_nncc_blocks(channels, K_delta=bad)
    assert tb.build_nncc_blocks((), K_delta=1) == ()


def test_system_carries_the_approximation():
    rovib = tb.RovibBasis(grids=np.array([1.5]), E_vj=np.zeros((1, 3)), WF_vj=np.ones((1, 1, 3)))
    diatom = tb.DiatomBasis(rovib=rovib, energy_zero=0.0)
    system = tb.build_ScattSystem(tb.AtomSpec(), diatom, Jtot=2, system_parity=1, approx=tb.Approx.NNCC, K_delta=2)
    assert system.approx is tb.Approx.NNCC and system.K_delta == 2
    with pytest.raises(ValueError, match="K_delta"):
        tb.build_ScattSystem(tb.AtomSpec(), diatom, Jtot=2, system_parity=1, approx=tb.Approx.NNCC, K_delta=0)


def _fixture_basis(name, p):
    """The channel basis of a block fixture, rebuilt by the host code."""
    from pyticc_b200 import workloads

    if name.startswith("solve_rigid"):
        diatom = workloads.rigid_rotor(p["B_cm"], p["jmax"])
        return build_ChannelBasis(tb.AtomSpec(), diatom, p["J"], p["parity"])
    return build_ChannelBasis(workloads.rigid_rotor(p["B1_cm"], p["jmax"]), workloads.rigid_rotor(p["B2_cm"], p["jmax"]), p["J"], 1)


@pytest.mark.parametrize("name", BLOCK_FIXTURES)
def test_block_transforms_match_reference(name):
    g, p = load_golden(name)
    basis = _fixture_basis(name, p)
    np.testing.assert_allclose(basis.E_int, g["E_int"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(tb.get_Umat_BF(basis), g["U"], rtol=0, atol=1e-12)
    blocks = tb.build_cs_blocks(basis) if p["approx"] == "cs" else tb.build_nncc_blocks(basis, K_delta=p["K_delta"])
    assert len(blocks) == int(g["n_block"])
    for b, block in enumerate(blocks):
        assert list(block.channel_indices) == list(g[f"b{b}_channel_indices"])
        assert list(block.owned_channel_indices) == list(g[f"b{b}_owned"])
        B, L = tb.get_Bmat_BF_to_SF(basis, block.channel_indices)
        np.testing.assert_allclose(B, g[f"b{b}_Bmat"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(L, g[f"b{b}_L"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", BLOCK_FIXTURES)
def test_oracle_block_solve_matches_reference(name):
    g, p = load_golden(name)
    groups, B_real, B_imag, norm = golden_vrows(g)
    mu = p["mu_amu"] * 1822.888486209
    n_pts = g["radial_points"].size
    for b in range(int(g["n_block"])):
        idx = [int(i) for i in g[f"b{b}_channel_indices"]]
        Y, S = pipeline.solve(
            g["E_int"][idx], g["U"][np.ix_(idx, idx)], groups, B_real, B_imag, norm,
            g["potential_values"].reshape(n_pts, -1), g["radial_points"], g["half_steps_sectors"], mu, g["energies"],
            g[f"b{b}_Bmat"], g[f"b{b}_L"], p["mode"], window=9, channel_indices=idx,
        )
        np.testing.assert_allclose(Y, g[f"b{b}_Y_BF"], rtol=1e-9, atol=1e-9)
        for e, s in enumerate(S):
            n = s.shape[0]
            assert n == g[f"b{b}_n_open"][e]
            np.testing.assert_allclose(s, g[f"b{b}_Smat"][e, :n, :n], rtol=1e-10, atol=1e-10)


def test_blocks_are_batched_by_sweep_size():
    from pyticc_b200.propagation.runner import block_size_classes

    sizes = [4, 64, 65, 128, 129, 200, 360, 30, 300]
    blocks = [tuple(range(n)) for n in sizes]
    assert block_size_classes(blocks, "inelastic") == [[0, 1, 7], [2, 3], [4, 5], [6, 8]]
    # capture mode sweeps the 2n x 2n real embedding
    assert block_size_classes(blocks, "capture") == [[0, 7], [1], [2, 3], [4], [5], [8], [6]]
    assert block_size_classes([tuple(range(10))], "inelastic") == [[0]]

