"""The V(R) contraction at the AB+CD rotor pair's full size (N = 2610 channels in 7 K groups of
270-480 rows, 2700 complex grid rows, no channel cutoff) against a plain FP64 product of the
same rows (cuBLAS through torch): V_K = norm [(Br v) Br^T + (Bi v) Bi^T] per group, symmetrised
as the reference does (matrix/interaction/common.py:50-62)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pair_case():
    from pyticc_b200.scattering import build_hamiltonian
    from pyticc_b200.workloads import rotor_pair

    wl = rotor_pair()
    vb = build_hamiltonian(wl.system, wl.grid).V_basis
    points = wl.grid.radial_points[[0, wl.grid.radial_points.size // 3, wl.grid.radial_points.size - 1]]
    return wl, vb, points


def test_pair_case_has_the_full_size(pair_case):
    _, vb, _ = pair_case
    assert vb.n_channel == 2610 and int(np.prod(vb.grid_shape)) == 2700 and vb.B_imag is not None
    assert max(len(m) for m in vb.channel_indices.values()) == 480


def test_contraction_at_full_size_matches_fp64_product(pair_case):
    from pyticc_b200.matrix.interaction import contract_device

    wl, vb, points = pair_case
    dev = torch.device("cuda", 0)
    values = wl.grid.take_device(points, dev).reshape(points.size, -1)
    got = contract_device(vb, None, values, dev)
    want = torch.zeros_like(got)
    for K, members in vb.channel_indices.items():
        idx = torch.as_tensor(members, device=dev)
        Br = torch.as_tensor(vb.B_real[K], device=dev)
        Bi = torch.as_tensor(vb.B_imag[K], device=dev)
        for r in range(points.size):
            v = values[r]
            V = ((Br * v) @ Br.T + (Bi * v) @ Bi.T) * vb.normalization
            want[r][idx[:, None], idx[None, :]] = 0.5 * (V + V.T)
    for r in range(points.size):
        scale = want[r].abs().max().item()
        err = (got[r] - want[r]).abs().max().item()
        assert err <= 1e-12 * scale, (r, err, scale)
    assert torch.equal(got, got.transpose(1, 2))
