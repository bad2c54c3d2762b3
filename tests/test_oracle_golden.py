"""Pin the CPU oracle against the reference's golden vectors and known answers.

These run without a GPU.  The known-answer cases restate the reference's own
tests (``tests/unit/test_logd.py``, ``test_smatrix.py``, ``test_bessel.py``).
"""

from __future__ import annotations

import numpy as np
import pytest
from scipy import special

from oracle import contraction, ldmd, matching, pipeline
from tests.conftest import golden_vrows, load_golden


def _constant_logD(Y0, W, length):
    """Closed-form log derivative through a constant potential (test_logd.py:6-13)."""
    if W > 0.0:
        p = np.sqrt(W)
        t = np.tanh(p * length)
        return p * (Y0 + p * t) / (p + Y0 * t)
    k = np.sqrt(-W)
    t = np.tan(k * length)
    return k * (Y0 - k * t) / (k + Y0 * t)


@pytest.mark.parametrize("mode", ["real", "capture"])
def test_ldmd_matches_reference_golden(mode):
    g, p = load_golden(f"ldmd_{mode}")
    W = g["W_points"]
    Y = ldmd.propagate_logD(g["Y_initial"], g["energies"], p["reduced_mass"], g["half_steps"], W[0:-1:2], W[1::2], W[2::2])
    np.testing.assert_allclose(Y, g["Y_final"], rtol=1e-12, atol=1e-12)


def test_ldmd_constant_potential_is_exact():
    h, Y0, W = 0.15, 1.3, 4.0
    ref, Qs, Qm, Qe = ldmd.correction_matrices(h, np.array([[W]]), np.array([[W]]), np.array([[W]]))
    Y = ldmd.propagate_with_corrections(np.array([[Y0]]), h, ref, Qs, Qm, Qe)
    np.testing.assert_allclose(Y[0, 0], _constant_logD(Y0, W, 2 * h), rtol=1e-13)


def test_ldmd_capture_incoming_wave_is_invariant():
    W, h, Y0 = -9.0, 0.1, -3.0j
    ref, Qs, Qm, Qe = ldmd.correction_matrices(h, np.array([[W]]), np.array([[W]]), np.array([[W]]))
    Y = ldmd.propagate_with_corrections(np.array([[Y0]]), h, ref, Qs, Qm, Qe)
    np.testing.assert_allclose(Y[0, 0], Y0, rtol=1e-13, atol=1e-13)


def test_ldmd_batched_energies_equal_closed_form():
    energies = np.array([0.1, 0.2])
    mu = 2.0
    hs = np.array([0.05, 0.10])
    W = np.full((2, 1, 1), 3.0)
    Y = ldmd.propagate_logD(np.full((2, 1, 1), 1.25), energies, mu, hs, W, W, W)
    expected = [_constant_logD(1.25, 3.0 - 2 * mu * e, 2 * hs.sum()) for e in energies]
    np.testing.assert_allclose(Y[:, 0, 0], expected, rtol=1e-12)


@pytest.mark.parametrize("tag", ["real", "complex"])
def test_contraction_matches_reference_golden(tag):
    g, p = load_golden("contract")
    groups = {int(K): tuple(v) for K, v in p["groups"].items()}
    B_real = {K: g[f"B_real_{K}"] for K in groups}
    B_imag = {K: g[f"B_imag_{K}"] for K in groups} if tag == "complex" else None
    norm = p["norm_complex"] if tag == "complex" else 1.0
    V = contraction.contract(groups, B_real, B_imag, norm, g["potential"], p["n_channel"])
    np.testing.assert_allclose(V, g[f"V_{tag}"], rtol=1e-13, atol=1e-13)
    V = contraction.contract(groups, B_real, B_imag, norm, g["potential"], p["n_channel"], (7, 0, 5, 2))
    np.testing.assert_allclose(V, g[f"V_{tag}_subset"], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("tag", ["real", "complex"])
def test_smatrix_matches_reference_golden(tag):
    g, p = load_golden("smatrix")
    S = matching.get_Smat(g[f"Y_{tag}"], p["Rmatch"], g["energies"], p["reduced_mass"], g["E_int"], g["L"])
    for e, s in enumerate(S):
        n = s.shape[0]
        assert n == g["n_open"][e]
        np.testing.assert_allclose(s, g[f"S_{tag}"][e, :n, :n], rtol=1e-12, atol=1e-12)


def test_bessel_matches_reference_golden():
    g, _ = load_golden("bessel")
    for ell, x, *expected in g["riccati"]:
        np.testing.assert_allclose(matching.riccati_bessel_jy(ell, x), expected, rtol=1e-14, atol=1e-300)
    for nu, x, expected in g["k_logd"]:
        np.testing.assert_allclose(matching.modified_bessel_K_logD(nu, x), expected, rtol=1e-14)


def test_bessel_known_answers():
    x = 1.7
    j, n, jd, nd = matching.riccati_bessel_jy(0.0, x)
    np.testing.assert_allclose([j, n, jd, nd], [np.sin(x), -np.cos(x), np.cos(x), np.sin(x)], rtol=1e-14, atol=1e-14)
    j, n, jd, nd = matching.riccati_bessel_jy(2.3, 4.2)
    np.testing.assert_allclose(j * nd - jd * n, 1.0, rtol=1e-13)
    nu, x = 1.7, 3.1
    np.testing.assert_allclose(matching.modified_bessel_K_logD(nu, x), special.kvp(nu, x) / special.kv(nu, x), rtol=1e-13)


def test_smatrix_capture_boundary_known_answer():
    """An imposed K = -0.2i gives S00 = 2/3 (test_smatrix.py:148-161)."""
    energy, Rmatch, mu = 0.4, 6.0, 2.0
    k = np.sqrt(2 * mu * energy)
    j, n, jd, nd = matching.riccati_bessel_jy(0.0, k * Rmatch)
    J, N, Jp, Np = j / np.sqrt(k), n / np.sqrt(k), np.sqrt(k) * jd, np.sqrt(k) * nd
    K = -0.2j
    Y = (Jp + Np * K) / (J + N * K)
    (S,) = matching.get_Smat(np.array([[[Y]]]), Rmatch, [energy], mu, [0.0], [0.0])
    np.testing.assert_allclose(S[0, 0], 2.0 / 3.0, rtol=1e-12)


@pytest.mark.parametrize("name", ["solve_rigid_p+", "solve_rigid_p-", "solve_rigid_capture", "solve_morse", "solve_diatom_diatom"])
def test_pipeline_matches_reference_solve(name):
    g, p = load_golden(name)
    groups, B_real, B_imag, norm = golden_vrows(g)
    mu = p["mu_amu"] * 1822.888486209
    mode = "capture" if "capture" in name else "inelastic"
    n_pts = g["radial_points"].size
    Y, S = pipeline.solve(
        g["E_int"], g["U"], groups, B_real, B_imag, norm,
        g["potential_values"].reshape(n_pts, -1), g["radial_points"], g["half_steps_sectors"], mu, g["energies"], g["Bmat"], g["L"], mode,
        window=7,
    )
    np.testing.assert_allclose(Y, g["Y_propagated"], rtol=1e-9, atol=1e-9)
    for e, s in enumerate(S):
        n = s.shape[0]
        assert n == g["n_open"][e]
        np.testing.assert_allclose(s, g["Smat"][e, :n, :n], rtol=1e-10, atol=1e-10)
