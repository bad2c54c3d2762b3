"""Generate golden input/output vectors from the unmodified PyTICC reference.

Run once in a container that has the reference checked out (JAX itself is not
needed: ``tests/golden/_jaxshim`` is a NumPy-backed stand-in for the few JAX calls
the reference makes)::

    python tests/golden/make_golden.py /path/to/PyTICC/src [fixture names...]

Every fixture is a small ``.npz`` written next to this script.  The product never
reads these files; ``tests/`` uses them to pin the oracle and the CUDA path.

Synthetic systems follow the shapes of the benchmark configurations at reduced
sizes (fewer rotor states, shorter radial grids, fewer energies) so that the
reference finishes in seconds.  The parameters are stored in each fixture's
``params_json`` entry and are mirrored by ``pyticc_b200.workloads``.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "_jaxshim"))
sys.path.insert(1, sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")

from loguru import logger  # noqa: E402

logger.remove()

import pyticc as ticc  # noqa: E402
from pyticc.basis.angle import gauss_legendre_dvr  # noqa: E402
from pyticc.basis.dvr import build_RovibDVR, build_SineDVR  # noqa: E402
from pyticc.basis.rovib import RovibBasis  # noqa: E402
from pyticc.match import bessel as ref_bessel  # noqa: E402
from pyticc.match import get_Smat  # noqa: E402
from pyticc.matrix.interaction.common import VBasisBF, contract  # noqa: E402
from pyticc.propagation.grid import build_radial_sectors, iter_radial_windows  # noqa: E402
from pyticc.propagation.logd import propagate_logD  # noqa: E402

CM = ticc.CM2AU
AMU = 1822.888486209
K2AU = 1.0 / 315775.02480407


def _save(name: str, params: dict, **arrays) -> None:
    payload = {key: np.asarray(value) for key, value in arrays.items()}
    payload["params_json"] = np.asarray(json.dumps(params))
    np.savez_compressed(HERE / f"{name}.npz", **payload)
    size = (HERE / f"{name}.npz").stat().st_size
    print(f"wrote {name}.npz ({size / 1024:.1f} KiB)")


def _legendre(n: int, x: np.ndarray) -> np.ndarray:
    from numpy.polynomial import legendre

    coefficients = np.zeros(n + 1)
    coefficients[n] = 1.0
    return legendre.legval(x, coefficients)


# ----------------------------------------------------------------------------------------
# Unit-level fixtures
# ----------------------------------------------------------------------------------------
def make_ldmd() -> None:
    rng = np.random.default_rng(1234)
    for mode, n_channel in (("real", 6), ("capture", 5)):
        n_sector, n_energy = 9, 3
        reduced_mass = 1.7
        half_steps = rng.uniform(0.03, 0.08, size=n_sector)
        base = rng.normal(size=(n_channel, n_channel)) * 0.4
        base = 0.5 * (base + base.T) + np.diag(rng.uniform(-2.0, 6.0, size=n_channel))
        W = []
        for point in range(2 * n_sector + 1):
            drift = rng.normal(size=(n_channel, n_channel)) * 0.05
            W.append(base + 0.5 * (drift + drift.T) + 0.02 * point * np.eye(n_channel))
        W = np.asarray(W)
        energies = rng.uniform(0.05, 0.9, size=n_energy)
        W0 = W[0][None] - 2.0 * reduced_mass * energies[:, None, None] * np.eye(n_channel)
        if mode == "real":
            Y0 = np.asarray(ticc.propagation.initialize_logD_inelastic(W0))
        else:
            Y0 = np.asarray(ticc.propagation.initialize_logD_capture(W0))
        Y = np.asarray(propagate_logD(Y0, energies, reduced_mass, half_steps, W[0:-1:2], W[1::2], W[2::2]))
        _save(
            f"ldmd_{mode}",
            {"mode": mode, "reduced_mass": reduced_mass},
            Y_initial=Y0,
            energies=energies,
            half_steps=half_steps,
            W_points=W,
            Y_final=Y,
        )


def make_contract() -> None:
    rng = np.random.default_rng(77)
    grid_shape = (3, 5)
    n_grid = 15
    groups = {0: (0, 3, 4), 1: (1, 5), 2: (2, 6, 7, 8)}
    n_channel = 9
    B_real = {K: rng.normal(size=(len(idx), n_grid)) for K, idx in groups.items()}
    B_imag = {K: rng.normal(size=(len(idx), n_grid)) for K, idx in groups.items()}
    potential = rng.normal(size=(4, *grid_shape))
    out = {}
    for tag, imag, norm in (("real", None, 1.0), ("complex", B_imag, 0.3)):
        basis = VBasisBF(n_channel=n_channel, grid_shape=grid_shape, channel_indices=groups, B_real=B_real, B_imag=imag, normalization=norm)
        out[f"V_{tag}"] = contract(basis, potential)
        out[f"V_{tag}_subset"] = contract(basis, potential, (7, 0, 5, 2))
    _save(
        "contract",
        {"groups": {str(K): list(v) for K, v in groups.items()}, "n_channel": n_channel, "grid_shape": list(grid_shape), "norm_complex": 0.3},
        potential=potential,
        **{f"B_real_{K}": v for K, v in B_real.items()},
        **{f"B_imag_{K}": v for K, v in B_imag.items()},
        **out,
    )


def make_smatrix() -> None:
    rng = np.random.default_rng(5)
    n_channel = 6
    E_int = np.array([0.0, 0.05, 0.11, 0.3, 0.45, 0.8])
    L = np.array([0.0, 1.0, 2.35, 1.7, 4.2, 6.0])
    energies = np.array([0.2, 0.5, 0.07])
    reduced_mass = 2.5
    Rmatch = 9.0
    real = []
    for _ in energies:
        M = rng.normal(size=(n_channel, n_channel)) * 0.3
        real.append(0.5 * (M + M.T) + np.diag(rng.uniform(-1.5, 1.0, size=n_channel)))
    real = np.asarray(real)
    S_real = get_Smat(real, Rmatch, energies, reduced_mass, E_int, L)
    imag = np.asarray([-0.2 * np.diag(rng.uniform(0.1, 1.0, size=n_channel)) for _ in energies])
    S_complex = get_Smat(real + 1j * imag, Rmatch, energies, reduced_mass, E_int, L)

    def pad(mats):
        outp = np.zeros((len(mats), n_channel, n_channel), dtype=np.complex128)
        for i, m in enumerate(mats):
            outp[i, : m.shape[0], : m.shape[1]] = m
        return outp

    _save(
        "smatrix",
        {"reduced_mass": reduced_mass, "Rmatch": Rmatch},
        E_int=E_int,
        L=L,
        energies=energies,
        Y_real=real,
        Y_complex=real + 1j * imag,
        S_real=pad(S_real),
        S_complex=pad(S_complex),
        n_open=np.array([m.shape[0] for m in S_real]),
    )


def make_bessel() -> None:
    ells = np.array([0.0, 0.3, 1.0, 2.7, 10.0, 25.5, 60.0, 3.0000000000001])
    xs = np.array([0.01, 0.5, 1.9, 2.1, 5.0, 20.0, 100.0, 500.0, 1500.0])
    rows = []
    for ell in ells:
        for x in xs:
            try:
                values = ref_bessel.riccati_bessel_jy(float(ell), float(x))
            except ValueError:
                continue
            rows.append([ell, x, *values])
    nus = np.array([0.5, 0.8, 1.5, 3.2, 10.5, 30.5, 60.5])
    krows = []
    for nu in nus:
        for x in np.array([0.01, 0.5, 1.9, 2.1, 5.0, 40.0, 300.0, 2500.0]):
            try:
                krows.append([nu, x, ref_bessel.modified_bessel_K_logD(float(nu), float(x))])
            except ValueError:
                continue
    _save("bessel", {}, riccati=np.asarray(rows), k_logd=np.asarray(krows))


def make_grid() -> None:
    cases = [((2.5, 30.0), (0.05,)), ((2.5, 40.0), (0.02,)), ((3.0, 3.37, 5.0), (0.1, 0.07)), ((1.0, 1.05), (0.1,))]
    payload = {}
    for index, (boundaries, halves) in enumerate(cases):
        sectors = build_radial_sectors(boundaries, halves)
        payload[f"sectors_{index}"] = np.asarray([[s.radial_start, s.radial_end] for s in sectors])
        windows = list(iter_radial_windows(sectors, n_grid=24, n_channel=231, n_energy=16, memory_limit_mb=64.0))
        payload[f"window_sizes_{index}"] = np.asarray([len(w) for w, _ in windows])
        payload[f"window_points_{index}"] = np.concatenate([p for _, p in windows])
    _save("grid", {"cases": [[list(b), list(h)] for b, h in cases]}, **payload)


# ----------------------------------------------------------------------------------------
# End-to-end fixtures through ticc.prepare_potential / ticc.solve
# ----------------------------------------------------------------------------------------
def _rigid_rotor(B_cm: float, jmax: int) -> ticc.DiatomBasis:
    energies = B_cm * CM * np.arange(jmax + 1) * (np.arange(jmax + 1) + 1.0)
    rovib = RovibBasis(grids=np.array([1.5]), E_vj=energies[None, :], WF_vj=np.ones((1, 1, jmax + 1)))
    return ticc.DiatomBasis(rovib=rovib, energy_zero=0.0)


def _lj_aniso_pes(eps_cm: float, Rm: float, a1: float, a2: float, c1: float = 0.0, c2: float = 0.0, re: float = 1.4):
    def interaction(R, coordinates):
        r, theta = coordinates
        x = np.cos(theta)
        radial = eps_cm * CM * ((Rm / R) ** 12 - 2.0 * (Rm / R) ** 6)
        aniso = 1.0 + a1 * (1.0 + c1 * (r - re)) * x + a2 * (1.0 + c2 * (r - re)) * 0.5 * (3.0 * x * x - 1.0)
        return radial * aniso

    return ticc.PESWrapper(interaction=interaction)


def _pad_smat(smats, n_channel):
    out = np.zeros((len(smats), n_channel, n_channel), dtype=np.complex128)
    for i, m in enumerate(smats):
        out[i, : m.shape[0], : m.shape[1]] = m
    return out


def _vbasis_rows(system, grid):
    """The reference's own weighted contraction rows, grouped by K."""
    from pyticc.matrix.interaction import atom_diatom as vmat_ad
    from pyticc.matrix.interaction import diatom_diatom as vmat_dd

    if grid.scattering_type is ticc.ScatteringType.ATOM_DIATOM:
        vb = vmat_ad.prepare(system.basis, system.monomer_Y.rovib, grid.coordinate("cos_theta"), grid.weight("theta"))
    else:
        vb = vmat_dd.prepare(
            system.basis,
            system.monomer_X.rovib,
            system.monomer_Y.rovib,
            grid.coordinate("cos_theta_X"),
            grid.weight("theta_X"),
            grid.coordinate("cos_theta_Y"),
            grid.weight("theta_Y"),
            grid.coordinate("phi"),
            grid.weight("phi"),
        )
    rows = {}
    for K, indices in vb.channel_indices.items():
        rows[f"vrows_idx_{K}"] = np.asarray(indices)
        rows[f"vrows_real_{K}"] = vb.B_real[K]
        if vb.B_imag is not None:
            rows[f"vrows_imag_{K}"] = vb.B_imag[K]
    rows["vrows_norm"] = np.asarray(vb.normalization)
    return rows


def _solve_and_save(name, params, system, boundaries, halves, energies, mode, memory_mb, **quad):
    grid = ticc.prepare_potential(system, boundaries, halves, **quad)
    result = ticc.solve(system, energies, grid, ticc.Propagation(mode=mode, memory_mb=memory_mb, device="cpu"))
    basis = system.basis
    vrows = _vbasis_rows(system, grid)
    channels = np.asarray([[c.mis_X.j, -1 if c.mis_X.v is None else c.mis_X.v, c.mis_Y.j, -1 if c.mis_Y.v is None else c.mis_Y.v, c.j_couple, c.K] for c in basis])
    _save(
        name,
        params,
        energies=np.asarray(energies),
        E_int=basis.E_int,
        channels=channels,
        radial_points=grid.radial_points,
        potential_values=np.asarray(grid.values),
        U=ticc.scattering.ScattHamiltonian(basis=basis, reduced_mass=system.reduced_mass, interaction=lambda R: None).U,
        Bmat=result.asymptotic_transform,
        L=result.L,
        Y_propagated=np.asarray(result.Y_propagated),
        Smat=_pad_smat(result.Smat, basis.n_channel),
        n_open=np.asarray([m.shape[0] for m in result.Smat]),
        cos_theta=grid.coordinate("cos_theta") if grid.scattering_type is ticc.ScatteringType.ATOM_DIATOM else np.zeros(0),
        half_steps_sectors=np.asarray([s.radial_half_step for s in grid.sectors]),
        **vrows,
    )


def make_solve_rigid() -> None:
    params = {"B_cm": 20.0, "jmax": 5, "J": 3, "mu_amu": 18.0, "eps_cm": 150.0, "Rm": 6.5, "a1": 0.3, "a2": 0.2, "n_theta": 8, "boundaries": [2.5, 10.0], "half_steps": [0.05]}
    energies = np.linspace(10.0, 500.0, 5) * CM
    for parity in (1, -1):
        system = ticc.build_ScattSystem(
            ticc.AtomSpec(),
            _rigid_rotor(params["B_cm"], params["jmax"]),
            Jtot=params["J"],
            system_parity=parity,
            potential=_lj_aniso_pes(params["eps_cm"], params["Rm"], params["a1"], params["a2"]),
            reduced_mass=params["mu_amu"] * AMU,
        )
        _solve_and_save(f"solve_rigid_p{'+' if parity > 0 else '-'}", {**params, "parity": parity}, system, params["boundaries"], params["half_steps"], energies, "inelastic", 512.0, n_theta=params["n_theta"])
    # the same system in capture mode, with a memory budget small enough to force several windows
    system = ticc.build_ScattSystem(
        ticc.AtomSpec(),
        _rigid_rotor(params["B_cm"], params["jmax"]),
        Jtot=params["J"],
        system_parity=1,
        potential=_lj_aniso_pes(params["eps_cm"], params["Rm"], params["a1"], params["a2"]),
        reduced_mass=params["mu_amu"] * AMU,
    )
    _solve_and_save("solve_rigid_capture", {**params, "parity": 1, "memory_mb": 0.05}, system, params["boundaries"], params["half_steps"], energies, "capture", 0.05, n_theta=params["n_theta"])


def make_solve_morse() -> None:
    params = {
        "De_cm": 40000.0,
        "re": 1.4,
        "a": 1.2,
        "diatom_mass_amu": 1.0,
        "r_interval": [0.5, 3.5],
        "n_dvr": 16,
        "vmax": 1,
        "jmax": 4,
        "J": 2,
        "mu_amu": 18.0,
        "eps_cm": 150.0,
        "Rm": 6.5,
        "a1": 0.3,
        "a2": 0.2,
        "seed": 2024,
        "n_theta": 6,
        "boundaries": [2.5, 8.0],
        "half_steps": [0.05],
    }
    c1, c2 = np.random.default_rng(params["seed"]).uniform(-0.5, 0.5, size=2)
    params["c1"], params["c2"] = float(c1), float(c2)
    mass = params["diatom_mass_amu"] * AMU

    def morse(r):
        return params["De_cm"] * CM * (1.0 - np.exp(-params["a"] * (r - params["re"]))) ** 2

    dvr = build_SineDVR(params["r_interval"][0], params["r_interval"][1], params["n_dvr"], mass, morse)
    rovib = build_RovibDVR(dvr, params["vmax"], params["jmax"], mass)
    diatom = ticc.DiatomBasis(rovib=rovib, energy_zero=float(rovib.E_vj[0, 0]))
    energies = np.array([100.0, 1100.0, 2500.0, 3000.0]) * CM
    system = ticc.build_ScattSystem(
        ticc.AtomSpec(),
        diatom,
        Jtot=params["J"],
        system_parity=1,
        potential=_lj_aniso_pes(params["eps_cm"], params["Rm"], params["a1"], params["a2"], c1, c2, params["re"]),
        reduced_mass=params["mu_amu"] * AMU,
    )
    _solve_and_save("solve_morse", params, system, params["boundaries"], params["half_steps"], energies, "inelastic", 512.0, n_theta=params["n_theta"])
    np.savez_compressed(HERE / "morse_rovib.npz", grids=rovib.grids, E_vj=rovib.E_vj, WF_vj=rovib.WF_vj)


def _bispherical_pes(params):
    """sum_(l1,l2,l) c strength exp(-0.8 (R-6)) A_{l1 l2 l} + LJ, c ~ N(0,1) seeded, with the
    reference's own angular functions."""
    from pyticc.basis.angle import clebsch_gordan, norm_YjK

    rng = np.random.default_rng(params["seed"])
    terms = []
    for l1 in range(params["lmax"] + 1):
        for l2 in range(params["lmax"] + 1):
            for lam in range(abs(l1 - l2), min(l1 + l2, params["lmax"]) + 1):
                if (l1 + l2 + lam) % 2 == 0 and (l1, l2, lam) != (0, 0, 0):
                    terms.append((l1, l2, lam, float(rng.normal())))

    def interaction(R, coordinates):
        _, _, t1, t2, phi = coordinates
        x1, x2 = np.cos(t1), np.cos(t2)
        total = np.zeros_like(x1)
        for l1, l2, lam, c in terms:
            angular = np.zeros_like(x1)
            for m in range(-min(l1, l2), min(l1, l2) + 1):
                angular += float(clebsch_gordan(l1, m, l2, -m, lam)) * norm_YjK(l1, m, x1) * norm_YjK(l2, -m, x2) * np.cos(m * phi)
            total += c * angular
        radial = params["strength_cm"] * CM * np.exp(-0.8 * (R - 6.0))
        lj = params["lj_eps_cm"] * CM * ((params["lj_Rm"] / R) ** 12 - 2.0 * (params["lj_Rm"] / R) ** 6)
        return radial * total + lj

    return terms, interaction


def make_solve_diatom_diatom() -> None:
    params = {"B1_cm": 60.0, "B2_cm": 2.0, "jmax": 2, "J": 1, "mu_amu": 3.6, "lmax": 2, "seed": 11, "strength_cm": 40.0, "lj_eps_cm": 100.0, "lj_Rm": 6.0, "n_theta_X": 6, "n_theta_Y": 6, "n_phi": 5, "boundaries": [4.0, 10.0], "half_steps": [0.05]}
    terms, interaction = _bispherical_pes(params)
    params["terms"] = terms
    diatom_X = _rigid_rotor(params["B1_cm"], params["jmax"])
    diatom_Y = _rigid_rotor(params["B2_cm"], params["jmax"])
    energies = np.array([5.0, 200.0, 800.0]) * CM
    system = ticc.build_ScattSystem(diatom_X, diatom_Y, Jtot=params["J"], system_parity=1, potential=ticc.PESWrapper(interaction=interaction), reduced_mass=params["mu_amu"] * AMU)
    _solve_and_save(
        "solve_diatom_diatom",
        params,
        system,
        params["boundaries"],
        params["half_steps"],
        energies,
        "inelastic",
        512.0,
        n_theta_X=params["n_theta_X"],
        n_theta_Y=params["n_theta_Y"],
        n_phi=params["n_phi"],
    )


def make_channel_counts() -> None:
    """Channel counts per (J, parity) from the reference's own channel builder."""
    counts = {}
    rigid = _rigid_rotor(20.0, 20)
    for parity in (1, -1):
        system = ticc.build_ScattSystem(ticc.AtomSpec(), rigid, Jtot=20, system_parity=parity)
        counts[f"rigid_j20_J20_p{parity}"] = system.basis.n_channel
    table = np.zeros((4, 31))
    spec = ticc.DiatomSpec(Eint=table) if hasattr(ticc, "DiatomSpec") else None
    from pyticc.basis.monomer import DiatomSpec

    spec = DiatomSpec(Eint=table)
    for J in (0, 1, 2, 15, 30, 45, 60):
        for parity in (1, -1):
            system = ticc.ScattSystem(ticc.AtomSpec(), spec, Jtot=J, system_parity=parity)
            from pyticc.basis.channel import build_ChannelBasis

            counts[f"vib_v3_j30_J{J}_p{parity}"] = build_ChannelBasis(system, ticc.ChannelSpec()).n_channel
    pair = DiatomSpec(Eint=np.zeros((1, 9)))
    for parity in (1, -1):
        system = ticc.ScattSystem(pair, pair, Jtot=6, system_parity=parity)
        counts[f"pair_j8_J6_p{parity}"] = build_ChannelBasis(system, ticc.ChannelSpec()).n_channel
    slow = DiatomSpec(Eint=np.zeros((1, 41)))
    for J in (0, 5, 10):
        system = ticc.ScattSystem(ticc.AtomSpec(), slow, Jtot=J, system_parity=1)
        counts[f"capture_j40_J{J}_p1"] = build_ChannelBasis(system, ticc.ChannelSpec()).n_channel
    _save("channel_counts", counts)


def make_kblocks() -> None:
    """CS and NNCC block structures from the reference's own block builders."""
    from pyticc.basis.channel import build_ChannelBasis
    from pyticc.basis.kblock import build_cs_blocks, build_nncc_blocks
    from pyticc.basis.monomer import DiatomSpec

    cases = {
        "atom_j4_J4": (ticc.AtomSpec(), DiatomSpec(Eint=np.zeros((1, 5))), 4, 1, None),
        "atom_j6_J9_p-": (ticc.AtomSpec(), DiatomSpec(Eint=np.zeros((2, 7))), 9, -1, None),
        "atom_j8_J8_Kcut3": (ticc.AtomSpec(), DiatomSpec(Eint=np.zeros((1, 9))), 8, 1, 3),
        "pair_j3_J5": (DiatomSpec(Eint=np.zeros((1, 4))), DiatomSpec(Eint=np.zeros((1, 3))), 5, 1, None),
        "atom_j2_J0": (ticc.AtomSpec(), DiatomSpec(Eint=np.zeros((1, 3))), 0, 1, None),
    }
    table = {}
    for name, (X, Y, J, parity, K_cut) in cases.items():
        system = ticc.ScattSystem(X, Y, Jtot=J, system_parity=parity)
        channels = build_ChannelBasis(system, ticc.ChannelSpec(K_cut=K_cut))
        entry = {"K": [float(c.K) for c in channels], "cs": [], "nncc": {}}
        for block in build_cs_blocks(channels):
            entry["cs"].append([list(block.K_values), list(block.channel_indices), list(block.owned_K_values), list(block.owned_channel_indices), block.center_K])
        for K_delta in (1, 2, 3):
            entry["nncc"][str(K_delta)] = [
                [list(b.K_values), list(b.channel_indices), list(b.owned_K_values), list(b.owned_channel_indices), b.center_K]
                for b in build_nncc_blocks(channels, K_delta=K_delta)
            ]
        table[name] = entry
    _save("kblocks", {"cases": table})


def _solve_blocks_and_save(name, params, system, boundaries, halves, energies, mode, **quad):
    grid = ticc.prepare_potential(system, boundaries, halves, **quad)
    result = ticc.solve(system, energies, grid, ticc.Propagation(mode=mode, device="cpu"))
    basis = system.basis
    payload = {
        "energies": np.asarray(energies),
        "n_block": np.asarray(len(result.blocks)),
        "E_int": basis.E_int,
        "radial_points": grid.radial_points,
        "potential_values": np.asarray(grid.values),
        "half_steps_sectors": np.asarray([s.radial_half_step for s in grid.sectors]),
        "U": ticc.scattering.ScattHamiltonian(basis=basis, reduced_mass=system.reduced_mass, interaction=lambda R: None).U,
        **_vbasis_rows(system, grid),
    }
    for b, block in enumerate(result.blocks):
        n = len(block.block.channel_indices)
        payload[f"b{b}_channel_indices"] = np.asarray(block.block.channel_indices)
        payload[f"b{b}_owned"] = np.asarray(block.block.owned_channel_indices)
        payload[f"b{b}_K_values"] = np.asarray(block.block.K_values)
        payload[f"b{b}_Y_BF"] = np.asarray(block.Y_BF)
        payload[f"b{b}_Bmat"] = np.asarray(block.Bmat)
        payload[f"b{b}_L"] = np.asarray(block.L)
        payload[f"b{b}_Smat"] = _pad_smat(block.Smat_asymptotic, n)
        payload[f"b{b}_n_open"] = np.asarray([m.shape[0] for m in block.Smat_asymptotic])
        payload[f"b{b}_Smat_BF"] = _pad_smat(block.Smat_BF, n)
    _save(name, params, **payload)


def make_solve_kblocks() -> None:
    """CS and NNCC solves of the rigid A+BC, vibrating A+BC and AB+CD fixtures' systems."""
    rigid = {"B_cm": 20.0, "jmax": 5, "J": 3, "mu_amu": 18.0, "eps_cm": 150.0, "Rm": 6.5, "a1": 0.3, "a2": 0.2, "n_theta": 8, "boundaries": [2.5, 10.0], "half_steps": [0.05]}
    energies = np.linspace(10.0, 500.0, 5) * CM
    for approx, K_delta, mode, tag in ((ticc.Approx.CS, 1, "inelastic", "cs"), (ticc.Approx.NNCC, 1, "inelastic", "nncc"), (ticc.Approx.CS, 1, "capture", "cs_capture")):
        system = ticc.build_ScattSystem(
            ticc.AtomSpec(),
            _rigid_rotor(rigid["B_cm"], rigid["jmax"]),
            Jtot=rigid["J"],
            system_parity=1,
            approx=approx,
            K_delta=K_delta,
            potential=_lj_aniso_pes(rigid["eps_cm"], rigid["Rm"], rigid["a1"], rigid["a2"]),
            reduced_mass=rigid["mu_amu"] * AMU,
        )
        _solve_blocks_and_save(f"solve_rigid_{tag}", {**rigid, "parity": 1, "approx": approx.value, "K_delta": K_delta, "mode": mode}, system, rigid["boundaries"], rigid["half_steps"], energies, mode, n_theta=rigid["n_theta"])
    # rotor pair (AB+CD) under NNCC with K_delta = 1 and J = 3 (K = 0..3)
    pair = {"B1_cm": 60.0, "B2_cm": 2.0, "jmax": 2, "J": 3, "mu_amu": 3.6, "lmax": 2, "seed": 11, "strength_cm": 40.0, "lj_eps_cm": 100.0, "lj_Rm": 6.0, "n_theta_X": 6, "n_theta_Y": 6, "n_phi": 5, "boundaries": [4.0, 10.0], "half_steps": [0.05]}
    from pyticc.basis.angle import clebsch_gordan, norm_YjK

    rng = np.random.default_rng(pair["seed"])
    terms = []
    for l1 in range(pair["lmax"] + 1):
        for l2 in range(pair["lmax"] + 1):
            for lam in range(abs(l1 - l2), min(l1 + l2, pair["lmax"]) + 1):
                if (l1 + l2 + lam) % 2 == 0 and (l1, l2, lam) != (0, 0, 0):
                    terms.append((l1, l2, lam, float(rng.normal())))

    def interaction(R, coordinates):
        _, _, t1, t2, phi = coordinates
        x1, x2 = np.cos(t1), np.cos(t2)
        total = np.zeros_like(x1)
        for l1, l2, lam, c in terms:
            angular = np.zeros_like(x1)
            for m in range(-min(l1, l2), min(l1, l2) + 1):
                angular += float(clebsch_gordan(l1, m, l2, -m, lam)) * norm_YjK(l1, m, x1) * norm_YjK(l2, -m, x2) * np.cos(m * phi)
            total += c * angular
        radial = pair["strength_cm"] * CM * np.exp(-0.8 * (R - 6.0))
        lj = pair["lj_eps_cm"] * CM * ((pair["lj_Rm"] / R) ** 12 - 2.0 * (pair["lj_Rm"] / R) ** 6)
        return radial * total + lj

    system = ticc.build_ScattSystem(
        _rigid_rotor(pair["B1_cm"], pair["jmax"]),
        _rigid_rotor(pair["B2_cm"], pair["jmax"]),
        Jtot=pair["J"],
        system_parity=1,
        approx=ticc.Approx.NNCC,
        K_delta=1,
        potential=ticc.PESWrapper(interaction=interaction),
        reduced_mass=pair["mu_amu"] * AMU,
    )
    _solve_blocks_and_save(
        "solve_pair_nncc",
        {**pair, "terms": terms, "approx": "nncc", "K_delta": 1, "mode": "inelastic"},
        system,
        pair["boundaries"],
        pair["half_steps"],
        np.array([5.0, 200.0, 800.0]) * CM,
        "inelastic",
        n_theta_X=pair["n_theta_X"],
        n_theta_Y=pair["n_theta_Y"],
        n_phi=pair["n_phi"],
    )


# ----------------------------------------------------------------------------------------
# Benchmark-size fixtures (minutes of CPU each; only S, open counts and energies are kept)
# ----------------------------------------------------------------------------------------
BENCH_ENERGIES_CM = np.linspace(100.0, 3000.0, 256)  # the vibrating A+BC energy grid


def _solve_full_and_save(name, params, system, boundaries, halves, energies, mode, **quad):
    import time

    grid = ticc.prepare_potential(system, boundaries, halves, **quad)
    started = time.perf_counter()
    result = ticc.solve(system, energies, grid, ticc.Propagation(mode=mode, memory_mb=2048.0, device="cpu"))
    params = {**params, "reference_wall_s": time.perf_counter() - started, "n_channel": int(system.basis.n_channel), "n_sector": len(grid.sectors)}
    n_open = np.asarray([m.shape[0] for m in result.Smat])
    width = int(max(n_open.max(), 1))
    _save(name, params, energies=np.asarray(energies), n_open=n_open, Smat=_pad_smat(result.Smat, width), E_int=system.basis.E_int)


def make_full_rigid() -> None:
    """The CPU-runnable rigid-rotor configuration at full size: N=231, 275 sectors, 16 energies."""
    params = {"B_cm": 20.0, "jmax": 20, "J": 20, "parity": 1, "mu_amu": 18.0, "eps_cm": 150.0, "Rm": 6.5, "a1": 0.3, "a2": 0.2, "n_theta": 24, "boundaries": [2.5, 30.0], "half_steps": [0.05]}
    system = ticc.build_ScattSystem(
        ticc.AtomSpec(),
        _rigid_rotor(params["B_cm"], params["jmax"]),
        Jtot=params["J"],
        system_parity=1,
        potential=_lj_aniso_pes(params["eps_cm"], params["Rm"], params["a1"], params["a2"]),
        reduced_mass=params["mu_amu"] * AMU,
    )
    energies = np.linspace(10.0, 500.0, 16) * CM
    _solve_full_and_save("full_rigid_J20", params, system, params["boundaries"], params["half_steps"], energies, "inelastic", n_theta=params["n_theta"])


def make_full_morse() -> None:
    """The vibrating A+BC benchmark blocks at full size (N=1984 / 1860, 938 sectors) at two of
    the benchmark energies, one low and one near the top of the grid."""
    params = {
        "De_cm": 40000.0, "re": 1.4, "a": 1.2, "diatom_mass_amu": 1.0, "r_interval": [0.5, 3.5], "n_dvr": 32, "vmax": 3, "jmax": 30, "J": 30,
        "mu_amu": 18.0, "eps_cm": 150.0, "Rm": 6.5, "a1": 0.3, "a2": 0.2, "seed": 2024, "n_theta": 32, "boundaries": [2.5, 40.0], "half_steps": [0.02],
        "energy_indices": [0, 250],
    }
    c1, c2 = np.random.default_rng(params["seed"]).uniform(-0.5, 0.5, size=2)
    params["c1"], params["c2"] = float(c1), float(c2)
    mass = params["diatom_mass_amu"] * AMU

    def morse(r):
        return params["De_cm"] * CM * (1.0 - np.exp(-params["a"] * (r - params["re"]))) ** 2

    dvr = build_SineDVR(params["r_interval"][0], params["r_interval"][1], params["n_dvr"], mass, morse)
    rovib = build_RovibDVR(dvr, params["vmax"], params["jmax"], mass)
    diatom = ticc.DiatomBasis(rovib=rovib, energy_zero=float(rovib.E_vj[0, 0]))
    energies = BENCH_ENERGIES_CM[params["energy_indices"]] * CM
    parities = [int(p) for p in sys.argv[3:]] if len(sys.argv) > 3 and sys.argv[2] == "full_morse" else [1, -1]
    for parity in parities:
        system = ticc.build_ScattSystem(
            ticc.AtomSpec(),
            diatom,
            Jtot=params["J"],
            system_parity=parity,
            potential=_lj_aniso_pes(params["eps_cm"], params["Rm"], params["a1"], params["a2"], c1, c2, params["re"]),
            reduced_mass=params["mu_amu"] * AMU,
        )
        tag = "+" if parity > 0 else "-"
        _solve_full_and_save(f"full_morse_J30_p{tag}", {**params, "parity": parity}, system, params["boundaries"], params["half_steps"], energies, "inelastic", n_theta=params["n_theta"])


def make_full_pair() -> None:
    """The AB+CD rigid-rotor pair at full size: j1, j2 <= 8, J = 6, parity +1, no channel or
    energy cutoff (N = 2610), 275 sectors, three energies of its 5-800 cm^-1 grid (5, 105.2 and
    555.9 cm^-1; 3, 28 and 345 open channels)."""
    params = {"B1_cm": 60.0, "B2_cm": 2.0, "jmax": 8, "J": 6, "parity": 1, "mu_amu": 3.6, "lmax": 4, "seed": 11, "strength_cm": 40.0, "lj_eps_cm": 100.0, "lj_Rm": 6.0,
              "n_theta_X": 15, "n_theta_Y": 15, "n_phi": 12, "boundaries": [2.5, 30.0], "half_steps": [0.05], "energy_indices": [0, 16, 88]}
    terms, interaction = _bispherical_pes(params)
    params["terms"] = terms
    energies = np.linspace(5.0, 800.0, 128)[params["energy_indices"]] * CM
    system = ticc.build_ScattSystem(_rigid_rotor(params["B1_cm"], params["jmax"]), _rigid_rotor(params["B2_cm"], params["jmax"]), Jtot=params["J"], system_parity=1,
                                    potential=ticc.PESWrapper(interaction=interaction), reduced_mass=params["mu_amu"] * AMU)
    _solve_full_and_save("full_pair_J6", params, system, params["boundaries"], params["half_steps"], energies, "inelastic", n_theta_X=params["n_theta_X"],
                         n_theta_Y=params["n_theta_Y"], n_phi=params["n_phi"])


def make_full_capture() -> None:
    """The ultracold capture block at full size: rigid rotor B=0.03 cm^-1, j<=40, J=10 (N=396;
    optional other J values after the name: ``make_golden.py <src> full_capture 0 1``),
    capture boundary at 8 bohr, fixed step h=0.05 to 1500 bohr, at 1 uK and 1 mK."""
    J_values = [int(v) for v in sys.argv[3:]] if len(sys.argv) > 3 and sys.argv[2] == "full_capture" else [10]
    for J in J_values:
        _make_full_capture(J)


def _make_full_capture(J: int) -> None:
    params = {"B_cm": 0.03, "jmax": 40, "J": J, "parity": 1, "mu_amu": 100.0, "C6": 1.0e4, "wall_cm": 500.0, "seed": 3, "n_theta": 48, "boundaries": [8.0, 1500.0], "half_steps": [0.05], "energies_K": [1.0e-6, 1.0e-3]}
    g = np.random.default_rng(params["seed"]).uniform(0.2, 1.0, size=3)

    def interaction(R, coordinates):
        _, theta = coordinates
        x = np.cos(theta)
        p2 = 0.5 * (3.0 * x * x - 1.0)
        wall = params["wall_cm"] * CM * np.exp(-(((R - 7.0) / 1.5) ** 2)) * (g[0] + g[1] * x + g[2] * p2)
        return -params["C6"] / R**6 * (1.0 + 0.1 * p2) + wall

    system = ticc.build_ScattSystem(
        ticc.AtomSpec(),
        _rigid_rotor(params["B_cm"], params["jmax"]),
        Jtot=params["J"],
        system_parity=params["parity"],
        potential=ticc.PESWrapper(interaction=interaction),
        reduced_mass=params["mu_amu"] * AMU,
    )
    energies = np.asarray(params["energies_K"]) * K2AU
    _solve_full_and_save(f"full_capture_J{J}", params, system, params["boundaries"], params["half_steps"], energies, "capture", n_theta=params["n_theta"])


def make_dropin() -> None:
    """Every call the reference's own runner makes to ``propagate_logD`` (runner.py:293) during
    a solve split into several radial windows: arguments and result, for a replay through the
    CUDA ``propagate_logD``, plus the solve's S matrices."""
    import pyticc.propagation.runner as ref_runner

    params = {"B_cm": 20.0, "jmax": 7, "J": 5, "parity": 1, "mu_amu": 18.0, "eps_cm": 150.0, "Rm": 6.5, "a1": 0.3, "a2": 0.2, "n_theta": 10, "boundaries": [2.5, 5.0, 9.0], "half_steps": [0.04, 0.08], "memory_mb": 3.0}
    system = ticc.build_ScattSystem(
        ticc.AtomSpec(),
        _rigid_rotor(params["B_cm"], params["jmax"]),
        Jtot=params["J"],
        system_parity=params["parity"],
        potential=_lj_aniso_pes(params["eps_cm"], params["Rm"], params["a1"], params["a2"]),
        reduced_mass=params["mu_amu"] * AMU,
    )
    energies = np.array([20.0, 260.0, 480.0]) * CM
    grid = ticc.prepare_potential(system, params["boundaries"], params["half_steps"], n_theta=params["n_theta"])
    calls = []
    original = ref_runner.propagate_logD

    def recording(Y_initial, total_energies, reduced_mass, radial_half_steps, W_base_start, W_base_mid, W_base_end, **kwargs):
        out = original(Y_initial, total_energies, reduced_mass, radial_half_steps, W_base_start, W_base_mid, W_base_end, **kwargs)
        calls.append({k: np.asarray(v) for k, v in (("Y_initial", Y_initial), ("total_energies", total_energies), ("radial_half_steps", radial_half_steps), ("W_base_start", W_base_start), ("W_base_mid", W_base_mid), ("W_base_end", W_base_end), ("Y_final", out))} | {"reduced_mass": np.asarray(reduced_mass)})
        return out

    ref_runner.propagate_logD = recording
    try:
        result = ticc.solve(system, energies, grid, ticc.Propagation(mode="inelastic", memory_mb=params["memory_mb"], device="cpu"))
    finally:
        ref_runner.propagate_logD = original
    import inspect

    arrays = {f"call{i}_{k}": v for i, c in enumerate(calls) for k, v in c.items()}
    params["n_calls"] = len(calls)
    params["signature"] = str(inspect.signature(original))
    params["parameters"] = [[name, str(parameter.kind)] for name, parameter in inspect.signature(original).parameters.items()]
    _save(
        "dropin_calls",
        params,
        energies=energies,
        E_int=system.basis.E_int,
        Bmat=result.asymptotic_transform,
        L=result.L,
        Rmatch=np.asarray(grid.sectors[-1].radial_end),
        Smat=_pad_smat(result.Smat, system.basis.n_channel),
        n_open=np.asarray([m.shape[0] for m in result.Smat]),
        **arrays,
    )


def make_contract_families() -> None:
    """Electric-field SF and diabatic contractions: the reference's host functions on seeded
    synthetic bases (atom_diatom.py:208-267, diabatic_atom_diatom.py:325-440)."""
    from pyticc.matrix.interaction import atom_diatom as ref_ad
    from pyticc.matrix.interaction import diabatic_atom_diatom as ref_dia

    rng = np.random.default_rng(404)
    grid_shape = (3, 4, 5, 2)
    n_grid, n_channel = int(np.prod(grid_shape)), 11
    B_cos, B_sin = rng.normal(size=(n_channel, n_grid)), rng.normal(size=(n_channel, n_grid))
    sf = ref_ad.AtomDiatomVBasisElectricSF(n_channel=n_channel, grid_shape=grid_shape, r=np.zeros(3), gamma=np.zeros((4, 5, 2)), B_cos=B_cos, B_sin=B_sin)
    sf_pot = rng.normal(size=(3, *grid_shape))
    sf_V = ref_ad.contract_electric_sf(sf, sf_pot)
    sf_V_subset = ref_ad.contract_electric_sf(sf, sf_pot[1], (9, 2, 4, 0))

    n_theta, grids = 6, (np.linspace(1.0, 2.0, 4), np.linspace(1.2, 2.4, 5))
    coupling_grid = np.linspace(1.0, 2.4, 7)
    groups = {(0, 0): (0, 3, 5), (0, 1): (1, 6), (1, 0): (2, 7, 8, 9), (1, 1): (4, 10, 11)}
    n_dia = 12
    B_diag = {k: rng.normal(size=(len(v), grids[k[0]].size * n_theta)) for k, v in groups.items()}
    B_coup = {k: rng.normal(size=(len(v), coupling_grid.size * n_theta)) for k, v in groups.items()}
    dia = ref_dia.DiabaticVBasisBF(n_channel=n_dia, n_state=2, theta=np.linspace(0.1, 3.0, n_theta), diagonal_grids=grids, coupling_grid=coupling_grid,
                                   channel_indices=groups, B_diagonal=B_diag, B_coupling=B_coup)
    d0, d1 = rng.normal(size=(3, grids[0].size, n_theta)), rng.normal(size=(3, grids[1].size, n_theta))
    c = rng.normal(size=(3, coupling_grid.size, n_theta, 2, 2))
    c = 0.5 * (c + np.swapaxes(c, -2, -1))
    dia_V = ref_dia.contract(dia, ref_dia.DiabaticVGridBF(diagonal=(d0, d1), coupling=c))
    dia_V_subset = ref_dia.contract(dia, ref_dia.DiabaticVGridBF(diagonal=(d0[2], d1[2]), coupling=c[2]), (11, 3, 7, 0, 10, 2))
    _save(
        "contract_families",
        {"grid_shape": list(grid_shape), "groups": {f"{k[0]},{k[1]}": list(v) for k, v in groups.items()}, "n_theta": n_theta, "sf_subset": [9, 2, 4, 0],
         "dia_subset": [11, 3, 7, 0, 10, 2]},
        sf_B_cos=B_cos, sf_B_sin=B_sin, sf_pot=sf_pot, sf_V=sf_V, sf_V_subset=sf_V_subset,
        dia_grid0=grids[0], dia_grid1=grids[1], dia_coupling_grid=coupling_grid, dia_d0=d0, dia_d1=d1, dia_c=c, dia_V=dia_V, dia_V_subset=dia_V_subset,
        **{f"dia_Bd_{k[0]}_{k[1]}": v for k, v in B_diag.items()}, **{f"dia_Bc_{k[0]}_{k[1]}": v for k, v in B_coup.items()},
    )



def make_contract_fs() -> None:
    """Fine-structure diatom-diatom contractions, scalar and spin-resolved: the reference's host
    functions on seeded synthetic packed kernels (fs_diatom_diatom.py:356-391,
    fs_diatom_diatom_spin.py:459-482)."""
    from pyticc.matrix.interaction import fs_diatom_diatom as ref_fs
    from pyticc.matrix.interaction import fs_diatom_diatom_spin as ref_spin
    from pyticc.pes.spin_resolved_diatom_diatom import OrbitalState

    rng = np.random.default_rng(505)
    grid_shape = (2, 2, 3, 2, 2)
    n_grid, n_channel = int(np.prod(grid_shape)), 7
    n_packed = n_channel * (n_channel + 1) // 2
    pr, pc = np.tril_indices(n_channel)
    kernel = rng.normal(size=(n_grid, n_packed))
    fs = ref_fs.FSDiatomDiatomVBasis(n_channel=n_channel, grid_shape=grid_shape, pair_rows=pr, pair_columns=pc, kernel=kernel)
    fs_pot = rng.normal(size=(3, *grid_shape))
    fs_V = ref_fs.contract(fs, fs_pot)
    fs_V_subset = ref_fs.contract(fs, fs_pot[0], (5, 1, 6, 2))
    spins, orbitals = (0, 2), (OrbitalState(0, 0), OrbitalState(2, -2))
    n_el = len(spins) * len(orbitals) ** 2
    skernel = rng.normal(size=(n_grid, n_el, n_packed)) + 1j * rng.normal(size=(n_grid, n_el, n_packed))
    spin = ref_spin.SpinResolvedFSDiatomDiatomVBasis(n_channel=n_channel, grid_shape=grid_shape, two_total_spins=spins, orbital_states=orbitals, pair_rows=pr,
                                                     pair_columns=pc, kernel=skernel)
    spin_pot = rng.normal(size=(3, *grid_shape, 2, 2, 2)) + 1j * rng.normal(size=(3, *grid_shape, 2, 2, 2))
    spin_V = ref_spin.contract(spin, spin_pot)
    spin_V_subset = ref_spin.contract(spin, spin_pot[1], (6, 0, 3, 4))
    _save("contract_fs", {"grid_shape": list(grid_shape), "n_channel": n_channel, "fs_subset": [5, 1, 6, 2], "spin_subset": [6, 0, 3, 4], "two_total_spins": list(spins)},
          fs_kernel=kernel, fs_pot=fs_pot, fs_V=fs_V, fs_V_subset=fs_V_subset, spin_kernel=skernel, spin_pot=spin_pot, spin_V=spin_V, spin_V_subset=spin_V_subset)


def make_delves() -> None:
    """Delves propagation (propagation/delves.py:54-286) driven by a seeded synthetic surface
    provider: surfaces whose energies and coefficients vary smoothly with rho and whose count
    drops from 5 to 4 halfway (a rectangular overlap); inelastic and capture starts."""
    from pyticc.propagation.delves import propagate_delves as ref_propagate_delves
    from pyticc.scattering.reactive.delves import DelvesHamiltonian, DelvesSurface

    n_primitive = 6

    class _Basis:
        rho_min = 2.0
        mass = (1.0 * AMU, 2.0 * AMU, 19.0 * AMU)

    _Basis.n_primitive = n_primitive

    def surface_at(rho):
        n = 5 if rho < 4.0 else 4
        e = np.array([0.02 + 0.01 * k + 0.05 * np.exp(-(rho - 2.0)) * (k + 1) for k in range(n)])
        th, ph = 0.3 * np.sin(rho), 0.2 * np.cos(0.7 * rho)
        G = np.eye(n_primitive)
        for (a, b, ang) in ((0, 1, th), (2, 3, ph), (1, 4, 0.5 * th)):
            R = np.eye(n_primitive)
            R[a, a] = R[b, b] = np.cos(ang)
            R[a, b], R[b, a] = -np.sin(ang), np.sin(ang)
            G = G @ R
        return e, G[:, :n].copy()

    class _Synthetic(DelvesHamiltonian):
        def __post_init__(self):
            pass

        def surface(self, rho):
            e, C = surface_at(rho)
            return DelvesSurface(rho=rho, energies=e, coefficients=C, overlap_eigenvalues=np.ones(e.size))

        def transform(self, a, b):
            return a.coefficients.T @ b.coefficients

    ham = _Synthetic(basis=_Basis(), total_potential=None)
    sectors = build_radial_sectors((2.0, 6.0), (0.05,))
    energies = np.array([0.035, 0.05, 0.08])
    rho = np.array([s.radial_mid for s in sectors])
    E_s = np.zeros((rho.size, 5))
    C_s = np.zeros((rho.size, n_primitive, 5))
    n_s = np.zeros(rho.size, dtype=np.int64)
    for i, r in enumerate(rho):
        e, C = surface_at(r)
        n_s[i] = e.size
        E_s[i, : e.size] = e
        C_s[i, :, : e.size] = C
    out = {}
    for mode in ("inelastic", "capture"):
        res = ref_propagate_delves(ham, energies, sectors, ticc.Propagation(mode=mode))
        out[f"Y_{mode}"] = np.asarray(res.Y_final)
    _save("delves", {"rho_min": 2.0, "rho_max": 6.0, "half_step": 0.05, "masses_amu": [1.0, 2.0, 19.0]},
          energies=energies, rho=rho, surface_energies=E_s, surface_coefficients=C_s, n_surface=n_s, **out)

MAKERS = {
    "ldmd": make_ldmd,
    "contract": make_contract,
    "smatrix": make_smatrix,
    "bessel": make_bessel,
    "grid": make_grid,
    "solve_rigid": make_solve_rigid,
    "solve_morse": make_solve_morse,
    "solve_diatom_diatom": make_solve_diatom_diatom,
    "channel_counts": make_channel_counts,
    "kblocks": make_kblocks,
    "solve_kblocks": make_solve_kblocks,
    "dropin": make_dropin,
    "contract_families": make_contract_families,
    "contract_fs": make_contract_fs,
    "delves": make_delves,
}
# benchmark-size fixtures: run by name only (tens of minutes of CPU in total);
# ``full_morse`` takes optional parities after its name: ``make_golden.py <src> full_morse -1``
FULL_SIZE_MAKERS = {
    "full_rigid": make_full_rigid,
    "full_morse": make_full_morse,
    "full_capture": make_full_capture,
    "full_pair": make_full_pair,
}

if __name__ == "__main__":
    # python make_golden.py <reference src> [fixture names...]  (default: all small fixtures)
    names = sys.argv[2:] or list(MAKERS)
    if names and names[0] in ("full_morse", "full_capture"):
        names = names[:1]
    for key in names:
        {**MAKERS, **FULL_SIZE_MAKERS}[key]()
