"""Parity of the CUDA path (through the C ABI) with the oracle and the reference's golden vectors.

Tolerances: the plain FP64 path must reproduce the reference within max|dS| <= 1e-8 for
S matrices; intermediate quantities carry tighter bounds stated per test.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
from scipy import special

import pyticc_b200 as tb
from oracle import contraction as o_contraction
from oracle import ldmd as o_ldmd
from oracle import matching as o_matching
from oracle import pipeline as o_pipeline
from pyticc_b200 import _native as nat
from pyticc_b200 import workloads
from pyticc_b200.match.asymptotic import transform_device
from pyticc_b200.matrix.interaction import VBasisBF, contract_device
from pyticc_b200.propagation.logd import propagate_logD, propagate_logD_sector
from tests.conftest import golden_vrows, load_golden

pytestmark = pytest.mark.gpu

S_TOL = 1.0e-8


def _np(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def _sym_inverse(M: np.ndarray, is_complex: bool) -> np.ndarray:
    lib = nat.load_library()
    dev = nat.require_cuda()
    t = torch.as_tensor(M, device=dev).contiguous()
    nbytes = nat.size_query(lib.ticc_sym_inverse_workspace_size, M.shape[-1], M.shape[0], int(is_complex))
    work = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    status = nat.DeviceStatus(dev)
    nat.check(lib.ticc_sym_inverse(nat.ptr(t), M.shape[-1], M.shape[0], int(is_complex), nat.ptr(work), nbytes, status.pointer, nat.stream_handle(dev)), "sym_inverse")
    status.raise_if_failed("sym_inverse")
    return _np(t)


@pytest.mark.parametrize("n", [1, 7, 128, 129, 300, 520])
def test_symmetric_sweep_inverse_real(n):
    """Diagonally dominant symmetric matrices (the LDMD regime, y1 ~ 1/h on the diagonal)."""
    rng = np.random.default_rng(n)
    A = rng.normal(size=(3, n, n))
    A = A + A.transpose(0, 2, 1) + np.diag(rng.uniform(3.0, 6.0, n)) * np.sqrt(n) * np.sign(rng.normal(size=n))
    X = _sym_inverse(A, False)
    inv = np.linalg.inv(A)
    np.testing.assert_allclose(X, inv, rtol=0, atol=1e-13 * np.abs(inv).max())
    np.testing.assert_array_equal(X, X.transpose(0, 2, 1))


@pytest.mark.parametrize("n", [3584, 3713])
def test_symmetric_sweep_inverse_at_the_fused_step_limit(n):
    """28 pivot blocks (the largest sweep run as one persistent launch per step) and 30
    (separate row-panel and update kernels); both keep only the lower tiles current."""
    rng = np.random.default_rng(n)
    A = rng.normal(size=(1, n, n))
    A = A + A.transpose(0, 2, 1) + np.diag(rng.uniform(3.0, 6.0, n)) * np.sqrt(n) * np.sign(rng.normal(size=n))
    X = _sym_inverse(A, False)
    inv = np.linalg.inv(A)
    np.testing.assert_allclose(X, inv, rtol=0, atol=1e-12 * np.abs(inv).max())
    np.testing.assert_array_equal(X, X.transpose(0, 2, 1))


@pytest.mark.parametrize("n", [300, 520])
def test_symmetric_sweep_inverse_indefinite(n):
    """Random indefinite matrices: pivoting is local to each 128-wide block, so the error
    carries the conditioning of the pivot blocks (bound stated relative to max|A^-1|)."""
    rng = np.random.default_rng(n)
    A = rng.normal(size=(3, n, n))
    A = A + A.transpose(0, 2, 1) + np.eye(n) * 0.3 * np.sqrt(n)
    X = _sym_inverse(A, False)
    inv = np.linalg.inv(A)
    np.testing.assert_allclose(X, inv, rtol=0, atol=1e-8 * np.abs(inv).max())


@pytest.mark.parametrize("n", [5, 64, 200])
def test_symmetric_sweep_inverse_complex_symmetric(n):
    rng = np.random.default_rng(100 + n)
    A = rng.normal(size=(2, n, n)) + 1j * rng.normal(size=(2, n, n))
    A = A + A.transpose(0, 2, 1) + np.eye(n) * np.sqrt(n)
    X = _sym_inverse(A, True)
    np.testing.assert_allclose(X, np.linalg.inv(A), rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize("mode", ["real", "capture"])
def test_ldmd_matches_reference_golden(mode):
    g, p = load_golden(f"ldmd_{mode}")
    W = g["W_points"]
    Y = propagate_logD(g["Y_initial"], g["energies"], p["reduced_mass"], g["half_steps"], W[0:-1:2], W[1::2], W[2::2])
    np.testing.assert_allclose(_np(Y), g["Y_final"], rtol=1e-11, atol=1e-11)


def _constant_logD(Y0, W, length):
    if W > 0.0:
        p = np.sqrt(W)
        t = np.tanh(p * length)
        return p * (Y0 + p * t) / (p + Y0 * t)
    k = np.sqrt(-W)
    t = np.tan(k * length)
    return k * (Y0 - k * t) / (k + Y0 * t)


def test_ldmd_known_answers():
    """Constant potential is exact; the capture incoming wave is invariant (test_logd.py:46-80)."""
    W = np.array([[4.0]])
    Y = propagate_logD_sector(np.array([[1.3]]), 0.15, W, W, W)
    np.testing.assert_allclose(_np(Y)[0, 0], _constant_logD(1.3, 4.0, 0.3), rtol=1e-13)
    W = np.array([[-9.0]])
    Y = propagate_logD_sector(np.array([[-3.0j]]), 0.1, W, W, W)
    np.testing.assert_allclose(_np(Y)[0, 0], -3.0j, rtol=1e-13, atol=1e-13)
    energies = np.array([0.1, 0.2])
    hs = np.array([0.05, 0.10])
    Wb = np.full((2, 1, 1), 3.0)
    Y = propagate_logD(np.full((2, 1, 1), 1.25), energies, 2.0, hs, Wb, Wb, Wb)
    np.testing.assert_allclose(_np(Y)[:, 0, 0], [_constant_logD(1.25, 3.0 - 4.0 * e, 2 * hs.sum()) for e in energies], rtol=1e-12)


def test_ldmd_matches_oracle_on_a_padded_multi_block_size():
    """N = 150 spans two 128-wide pivot blocks; the oracle runs the same inputs."""
    rng = np.random.default_rng(9)
    n, n_sector, n_energy, mu = 150, 6, 4, 3.0
    base = rng.normal(size=(n, n)) * 0.2
    base = base + base.T + np.diag(np.linspace(-3.0, 40.0, n))
    W = np.asarray([base + 0.01 * k * np.eye(n) for k in range(2 * n_sector + 1)])
    hs = np.full(n_sector, 0.04)
    E = np.linspace(0.2, 1.1, n_energy)
    Y0 = o_ldmd.initialize_inelastic(W[0][None] - 2 * mu * E[:, None, None] * np.eye(n))
    got = _np(propagate_logD(Y0, E, mu, hs, W[0:-1:2], W[1::2], W[2::2]))
    want = o_ldmd.propagate_logD(Y0, E, mu, hs, W[0:-1:2], W[1::2], W[2::2])
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-9 * np.abs(want).max())


@pytest.mark.parametrize("tag", ["real", "complex"])
def test_contraction_matches_reference_golden(tag):
    g, p = load_golden("contract")
    groups = {int(K): tuple(v) for K, v in p["groups"].items()}
    B_real = {K: g[f"B_real_{K}"] for K in groups}
    B_imag = {K: g[f"B_imag_{K}"] for K in groups} if tag == "complex" else None
    vb = VBasisBF(p["n_channel"], tuple(p["grid_shape"]), groups, B_real, B_imag, p["norm_complex"] if tag == "complex" else 1.0)
    np.testing.assert_allclose(_np(contract_device(vb, None, g["potential"])), g[f"V_{tag}"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(_np(contract_device(vb, None, g["potential"], channel_indices=(7, 0, 5, 2))), g[f"V_{tag}_subset"], rtol=1e-12, atol=1e-12)


def test_bessel_matches_golden_and_scipy():
    g, _ = load_golden("bessel")
    R = g["riccati"]
    got = np.stack(tb.riccati_bessel_jy(R[:, 0], R[:, 1]), axis=1)
    envelope = np.hypot(R[:, 2], R[:, 3])[:, None]
    envelope_d = np.hypot(R[:, 4], R[:, 5])[:, None]
    err = np.abs(got - R[:, 2:]) / np.concatenate([envelope, envelope, envelope_d, envelope_d], axis=1)
    assert err.max() < 1e-11
    K = g["k_logd"]
    np.testing.assert_allclose(tb.modified_bessel_K_logD(K[:, 0], K[:, 1]), K[:, 2], rtol=1e-12)
    rng = np.random.default_rng(4)
    ell, x = rng.uniform(0, 60, 2000), np.exp(rng.uniform(np.log(0.05), np.log(2000.0), 2000))
    j, n, jd, nd = tb.riccati_bessel_jy(ell, x)
    np.testing.assert_allclose(j * nd - jd * n, 1.0, rtol=1e-10)
    nu = ell + 0.5
    np.testing.assert_allclose(tb.modified_bessel_K_logD(nu, x), -special.kve(nu - 1, x) / special.kve(nu, x) - nu / x, rtol=1e-12)


@pytest.mark.parametrize("tag", ["real", "complex"])
def test_smatrix_matches_reference_golden(tag):
    g, p = load_golden("smatrix")
    S = tb.get_Smat(g[f"Y_{tag}"], p["Rmatch"], g["energies"], p["reduced_mass"], g["E_int"], g["L"])
    for e, s in enumerate(S):
        n = g["n_open"][e]
        assert s.shape == (n, n)
        np.testing.assert_allclose(s, g[f"S_{tag}"][e, :n, :n], rtol=1e-10, atol=1e-10)


def test_smatrix_known_answers():
    energy, Rmatch, mu = 0.4, 6.0, 2.0
    k = np.sqrt(2 * mu * energy)
    j, n, jd, nd = o_matching.riccati_bessel_jy(0.0, k * Rmatch)
    J, N, Jp, Np = j / np.sqrt(k), n / np.sqrt(k), np.sqrt(k) * jd, np.sqrt(k) * nd
    Y = (Jp + Np * (-0.2j)) / (J + N * (-0.2j))
    (S,) = tb.get_Smat(np.array([[[Y]]]), Rmatch, [energy], mu, [0.0], [0.0])
    np.testing.assert_allclose(S[0, 0], 2.0 / 3.0, rtol=1e-12)
    with pytest.raises(ValueError, match="threshold"):
        tb.get_Smat(np.zeros((1, 2, 2)), 5.0, [0.1], 1.0, [0.0, 0.1], [0.0, 1.0])


def test_transform_matches_oracle():
    rng = np.random.default_rng(3)
    n = 140
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    Y = rng.normal(size=(3, n, n)) + 1j * rng.normal(size=(3, n, n))
    dev = nat.require_cuda()
    got = _np(transform_device(torch.as_tensor(Y, device=dev), torch.as_tensor(Q, device=dev)))
    np.testing.assert_allclose(got, o_matching.transform_bf_to_sf(Y, Q), rtol=1e-12, atol=1e-12)


def _golden_workload(name):
    g, p = load_golden(name)
    if name.startswith("solve_rigid"):
        wl = workloads.rigid_atom_diatom(B_cm=p["B_cm"], jmax=p["jmax"], J=p["J"], parity=p["parity"], n_theta=p["n_theta"], boundaries=p["boundaries"], half_steps=p["half_steps"], energies_cm=g["energies"] * tb.AU2CM)
    elif name == "solve_morse":
        wl = workloads.morse_atom_diatom(J=p["J"], seed=p["seed"], n_theta=p["n_theta"], boundaries=p["boundaries"], half_steps=p["half_steps"], energies_cm=g["energies"] * tb.AU2CM, De_cm=p["De_cm"], re=p["re"], a=p["a"], mass_amu=p["diatom_mass_amu"], r_interval=p["r_interval"], n_dvr=p["n_dvr"], vmax=p["vmax"], jmax=p["jmax"])
    else:
        wl = workloads.rotor_pair(B1_cm=p["B1_cm"], B2_cm=p["B2_cm"], jmax=p["jmax"], J=p["J"], lmax=p["lmax"], seed=p["seed"], n_theta_X=p["n_theta_X"], n_theta_Y=p["n_theta_Y"], n_phi=p["n_phi"], boundaries=p["boundaries"], half_steps=p["half_steps"], energies_cm=g["energies"] * tb.AU2CM)
    return g, p, wl


@pytest.mark.parametrize("name", ["solve_rigid_p+", "solve_rigid_p-", "solve_rigid_capture", "solve_morse", "solve_diatom_diatom"])
def test_solve_matches_reference(name):
    g, p, wl = _golden_workload(name)
    mode = "capture" if "capture" in name else "inelastic"
    result = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation(mode=mode))
    np.testing.assert_allclose(result.Y_propagated, g["Y_propagated"], rtol=1e-8, atol=1e-8)
    assert [s.shape[0] for s in result.Smat] == list(g["n_open"])
    for e, s in enumerate(result.Smat):
        n = s.shape[0]
        if n:
            assert np.abs(s - g["Smat"][e, :n, :n]).max() <= S_TOL


def test_solve_matches_oracle_on_cfg0_sized_block():
    """Full-size rigid rotor (N = 231, 275 sectors) at a few energies vs the oracle."""
    wl = workloads.rigid_atom_diatom(energies_cm=[37.0, 250.0, 480.0])
    result = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation())
    vb = tb.scattering.hamiltonian_for(wl.system, wl.grid).V_basis
    _, S = o_pipeline.solve(
        wl.system.basis.E_int, tb.get_Umat_BF(wl.system.basis), vb.channel_indices, vb.B_real, None, 1.0,
        wl.grid.values.reshape(wl.grid.radial_points.size, -1), wl.grid.radial_points,
        np.asarray([s.radial_half_step for s in wl.grid.sectors]), wl.system.reduced_mass, wl.energies, result.asymptotic_transform, result.L,
    )
    for a, b in zip(result.Smat, S, strict=True):
        assert a.shape == b.shape
        if a.size:
            assert np.abs(a - b).max() <= S_TOL
    assert result.unitarity_defect().max() < 1e-10


def test_device_status_reports_a_singular_pivot_block():
    """A symmetric matrix with an exactly zero 128-block is reported, not silently used."""
    M = np.zeros((1, 128, 128))
    with pytest.raises(RuntimeError, match="pivot block"):
        _sym_inverse(M, False)


MIXED_TOL = 1.0e-6


def test_mixed_precision_matches_fp64_on_vibrating_block():
    """v <= 3 puts channels > 4000 cm^-1 above the energies: their leading blocks take the
    TF32x3 product.  The mixed S must stay within 1e-6 of the plain FP64 S."""
    wl = workloads.morse_atom_diatom(J=8, jmax=12, vmax=3, n_dvr=24, n_theta=16, boundaries=(2.5, 20.0), half_steps=(0.02,), energies_cm=[150.0, 1200.0, 2900.0])
    assert wl.system.basis.n_channel > 256
    plain = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation())
    mixed = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation(precision="mixed"))
    worst = max(float(np.abs(a - b).max()) for a, b in zip(plain.Smat, mixed.Smat, strict=True) if a.size)
    assert worst <= MIXED_TOL
    assert worst > 0.0  # the reduced-precision blocks did run
    assert mixed.unitarity_defect().max() < 1e-6


def test_mixed_precision_matches_oracle_where_reduced_steps_run():
    """A vibrating block of more than 256 channels over a short inner grid (2.5-4.5 bohr,
    inside the repulsive wall, where every leading block is strongly closed): the mixed
    solve takes TF32x3 steps (counted through ticc_ldmd_reduced_blocks) and still matches
    the oracle's all-FP64 LAPACK propagation and matching within 1e-6."""
    wl = workloads.morse_atom_diatom(J=8, jmax=12, vmax=3, n_dvr=24, n_theta=16, boundaries=(2.5, 4.5), half_steps=(0.02,), energies_cm=[150.0, 2900.0])
    assert wl.system.basis.n_channel > 256
    stats: dict = {}
    mixed = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation(precision="mixed"), stats=stats)
    assert stats["reduced_steps"] >= stats["sweep_steps"] // 2, stats
    vb = tb.scattering.hamiltonian_for(wl.system, wl.grid).V_basis
    _, S = o_pipeline.solve(
        wl.system.basis.E_int, tb.get_Umat_BF(wl.system.basis), vb.channel_indices, vb.B_real, None, 1.0,
        wl.grid.values.reshape(wl.grid.radial_points.size, -1), wl.grid.radial_points,
        np.asarray([s.radial_half_step for s in wl.grid.sectors]), wl.system.reduced_mass, wl.energies, mixed.asymptotic_transform, mixed.L,
    )
    for a, b in zip(mixed.Smat, S, strict=True):
        assert a.shape == b.shape
        if a.size:
            assert np.abs(a - b).max() <= MIXED_TOL


def test_fused_step_wait_gives_up_reports_status_and_the_context_survives():
    """With the poll limit at 0 every wait of the fused sweep step gives up at once: the
    call reports device status 6 instead of hanging, and the next call (default limit)
    computes the right inverse on the same context."""
    lib = nat.load_library()
    rng = np.random.default_rng(6)
    A = rng.normal(size=(4, 300, 300))
    A = A + A.transpose(0, 2, 1) + np.diag(rng.uniform(3.0, 6.0, 300)) * np.sqrt(300)
    nat.check(lib.ticc_debug_set_step_poll_limit(0), "ticc_debug_set_step_poll_limit")
    try:
        with pytest.raises(RuntimeError, match="gave up waiting"):
            _sym_inverse(A, False)
    finally:
        nat.check(lib.ticc_debug_set_step_poll_limit(1 << 22), "ticc_debug_set_step_poll_limit")
    X = _sym_inverse(A, False)
    inv = np.linalg.inv(A)
    np.testing.assert_allclose(X, inv, rtol=0, atol=1e-13 * np.abs(inv).max())


def test_learned_schedule_is_judged_inside_solve():
    """solve(steps='learned') runs the fixed-step judge: an accepted schedule is used (fewer
    sectors, within 1e-6 of the fixed-step S) and its verdict is cached; with a tolerance no
    schedule can meet, the solve falls back to the fixed grid and equals the fixed-step solve."""
    from pyticc_b200.propagation.learned import train_proposer, training_set
    from pyticc_b200.scattering import hamiltonian_for

    wl = workloads.ultracold_capture(jmax=6, J=1, parity=-1, boundaries=(8.0, 300.0), n_energy=6)
    base = tb.Propagation(mode="capture")
    X, T = training_set([(hamiltonian_for(wl.system, wl.grid), wl.grid.sectors, wl.energies[[0, 5]], base)], max_level=8)
    proposer, _ = train_proposer(X, T, steps=2000)
    energies = wl.energies[[2, 3]]
    fixed = tb.solve(wl.system, energies, wl.grid, base)
    stats: dict = {}
    learned = tb.solve(wl.system, energies, wl.grid, tb.Propagation(mode="capture", steps="learned", proposer=proposer), stats=stats)
    record = stats["learned"]
    assert record["accepted"] and record["judged"] and record["n_learned"] < record["n_fixed"]
    assert max(float(np.abs(a - b).max()) for a, b in zip(fixed.Smat, learned.Smat, strict=True) if a.size) <= MIXED_TOL
    again: dict = {}
    tb.solve(wl.system, energies, wl.grid, tb.Propagation(mode="capture", steps="learned", proposer=proposer), stats=again)
    assert not again["learned"]["judged"]  # the cached verdict
    span = (float(wl.energies.min()), float(wl.energies.max()))
    ranged: list = []
    for batch in (wl.energies[[1, 2]], wl.energies[[3, 4]]):  # one schedule for the whole range
        st: dict = {}
        tb.solve(wl.system, batch, wl.grid, tb.Propagation(mode="capture", steps="learned", proposer=proposer, learned_range=span), stats=st)
        ranged.append(st["learned"])
    assert ranged[0]["n_learned"] == ranged[1]["n_learned"] and not ranged[1]["judged"]
    with pytest.raises(ValueError, match="learned_range"):
        tb.solve(wl.system, wl.energies[[0, 5]] * 2.0, wl.grid, tb.Propagation(mode="capture", steps="learned", proposer=proposer, learned_range=span))
    strict: dict = {}
    refused = tb.solve(wl.system, energies, wl.grid, tb.Propagation(mode="capture", steps="learned", proposer=proposer, judge_tol=1e-300), stats=strict)
    assert not strict["learned"]["accepted"] and strict["sectors"] == record["n_fixed"]
    for a, b in zip(fixed.Smat, refused.Smat, strict=True):
        np.testing.assert_array_equal(a, b)


def test_audit_attaches_max_dS_against_plain_fp64():
    wl = workloads.morse_atom_diatom(J=8, jmax=12, vmax=3, n_dvr=24, n_theta=16, boundaries=(2.5, 12.0), half_steps=(0.02,), energies_cm=[150.0, 2900.0])
    audited = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation(precision="mixed", audit=True))
    plain = tb.solve(wl.system, wl.energies, wl.grid, tb.Propagation())
    want = [float(np.abs(a - b).max()) if a.size else 0.0 for a, b in zip(audited.Smat, plain.Smat, strict=True)]
    np.testing.assert_array_equal(audited.max_dS, want)
    assert audited.max_dS.max() <= MIXED_TOL


def test_assembled_W_base_is_exactly_symmetric():
    """The LDMD kernels read W_base[i][j] only; the device assembly must be symmetric bit for bit."""
    from pyticc_b200 import scattering
    from pyticc_b200.propagation import runner

    for wl in (workloads.rigid_atom_diatom(jmax=8, J=4, n_energy=2), workloads.morse_atom_diatom(J=8, jmax=10, vmax=1, n_dvr=16, n_theta=12, boundaries=(2.5, 6.0), n_energy=2)):
        ham = scattering.hamiltonian_for(wl.system, wl.grid)
        for closed_first in (False, True):
            dh = runner.device_hamiltonian(ham, nat.require_cuda(), closed_first=closed_first)
            W = dh.W_base(wl.grid.radial_points[:7])
            assert torch.equal(W, W.transpose(-1, -2))
