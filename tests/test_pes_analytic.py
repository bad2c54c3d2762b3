"""The Legendre-expansion analytic PES (host side): the declarative form reproduces the
benchmark systems' analytic surfaces, and malformed forms are rejected before any device call."""

from __future__ import annotations

import numpy as np
import pytest

import pyticc_b200 as tb
from pyticc_b200 import pes_analytic as pa
from pyticc_b200 import workloads
from pyticc_b200.pes import PESWrapper, get_Vgrid_atom_diatom


def _coordinates(r, theta):
    grids = np.meshgrid(r, theta, indexing="ij")
    return np.stack([g.ravel() for g in grids])


def test_lj_aniso_form_matches_the_workload_surface():
    ref = workloads.lj_aniso_pes(150.0, 6.5, 0.3, 0.2, 0.17, -0.31, 1.4)
    new = pa.lj_aniso_legendre(150.0 * tb.CM2AU, 6.5, 0.3, 0.2, 0.17, -0.31, 1.4)
    assert isinstance(new, PESWrapper)
    co = _coordinates(np.linspace(0.6, 2.8, 11), np.linspace(0.0, np.pi, 13))
    for R in (2.5, 4.0, 6.5, 9.0, 40.0):
        a, b = ref.interaction(R, co), new.interaction(R, co)
        assert np.abs(a - b).max() <= 1e-14 * np.abs(a).max()


def test_capture_form_matches_the_workload_surface():
    seed, C6, wall = 3, 1.0e4, 500.0
    g = tuple(np.random.default_rng(seed).uniform(0.2, 1.0, size=3))
    ref = workloads.capture_pes(C6, wall, seed)
    new = pa.capture_legendre(C6, wall * tb.CM2AU, g)
    co = _coordinates(np.array([1.1]), np.linspace(0.0, np.pi, 17))
    for R in (8.0, 7.0, 12.0, 300.0):
        a, b = ref.interaction(R, co), new.interaction(R, co)
        assert np.abs(a - b).max() <= 1e-14 * np.abs(a).max()


def test_tensor_grid_layout_is_the_reference_one():
    """get_Vgrid_atom_diatom (R x r x theta, meshgrid "ij") with the declarative PES."""
    pes = pa.lj_aniso_legendre(1e-3, 6.0, 0.4, 0.1)
    R, r, theta = np.array([5.0, 7.0]), np.array([1.2, 1.4, 1.6]), np.array([0.3, 1.2, 2.0, 2.9])
    V = get_Vgrid_atom_diatom(pes, R, r, theta)
    assert V.shape == (2, 3, 4)
    x = np.cos(theta[3])
    expected = 1e-3 * ((6.0 / 7.0) ** 12 - 2 * (6.0 / 7.0) ** 6) * (1 + 0.4 * x + 0.1 * 0.5 * (3 * x * x - 1))
    assert V[1, 1, 3] == pytest.approx(expected, rel=1e-14)


@pytest.mark.parametrize(
    "terms",
    [
        [],
        [pa.LegendreTerm(0, (pa.Primitive("lj", 1.0, 6.0),))] * 17,
        [pa.LegendreTerm(33, (pa.Primitive("lj", 1.0, 6.0),))],
        [pa.LegendreTerm(0, tuple(pa.Primitive("power", 1.0, 6.0) for _ in range(5)))],
        [pa.LegendreTerm(0, (pa.Primitive("lj", 1.0, 6.0),), (1.0, 0.0, 0.0, 0.0, 0.0))],
    ],
)
def test_forms_outside_the_kernel_are_rejected(terms):
    with pytest.raises(ValueError):
        pa.LegendrePES.build(terms)


def test_unknown_primitive_is_rejected():
    with pytest.raises(ValueError, match="unknown radial primitive"):
        pa.Primitive("yukawa", 1.0, 1.0)
