"""Synthetic scattering systems with the shapes of the benchmark configurations.

No public dataset is involved: each workload is an analytic PES on a model monomer,
built from parameters (and a NumPy seed) so that tests and the benchmark construct
identical inputs.  The same parameter sets, at reduced sizes, produced the committed
golden fixtures through the reference's own API.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .basis import AtomSpec, DiatomBasis, RovibBasis, build_RovibDVR, build_SineDVR, clebsch_gordan, norm_YjK
from .constants import AMU2AU, CM2AU, K2AU
from .pes import PESWrapper
from .scattering import PotentialGrid, prepare_potential
from .system import Approx, ScattSystem, build_ScattSystem


def rigid_rotor(B_cm: float, jmax: int) -> DiatomBasis:
    """Rigid rotor as a one-point rovibrational basis: E_j = B j(j+1), WF = 1."""
    j = np.arange(jmax + 1)
    rovib = RovibBasis(grids=np.array([1.5]), E_vj=(B_cm * CM2AU * j * (j + 1.0))[None, :], WF_vj=np.ones((1, 1, jmax + 1)))
    return DiatomBasis(rovib=rovib, energy_zero=0.0)


def morse_diatom(De_cm: float, re: float, a: float, mass_amu: float, r_interval, n_dvr: int, vmax: int, jmax: int) -> DiatomBasis:
    """Morse oscillator in a sine DVR; thresholds relative to (v=0, j=0)."""
    mass = mass_amu * AMU2AU

    def morse(r):
        return De_cm * CM2AU * (1.0 - np.exp(-a * (r - re))) ** 2

    rovib = build_RovibDVR(build_SineDVR(r_interval[0], r_interval[1], n_dvr, mass, morse), vmax, jmax, mass)
    return DiatomBasis(rovib=rovib, energy_zero=float(rovib.E_vj[0, 0]))


def lj_aniso_pes(eps_cm: float, Rm: float, a1: float, a2: float, c1: float = 0.0, c2: float = 0.0, re: float = 1.4) -> PESWrapper:
    """V = eps[(Rm/R)^12 - 2(Rm/R)^6] (1 + a1(r) P1(cos t) + a2(r) P2(cos t)), a_k(r) = a_k (1 + c_k (r - re))."""

    def interaction(R, coordinates):
        r, theta = coordinates
        x = np.cos(theta)
        radial = eps_cm * CM2AU * ((Rm / R) ** 12 - 2.0 * (Rm / R) ** 6)
        return radial * (1.0 + a1 * (1.0 + c1 * (r - re)) * x + a2 * (1.0 + c2 * (r - re)) * 0.5 * (3.0 * x * x - 1.0))

    return PESWrapper(interaction=interaction)


def bispherical_pes(terms, strength_cm: float, lj_eps_cm: float, lj_Rm: float) -> PESWrapper:
    """sum_(l1,l2,l) c strength exp(-0.8 (R-6)) A_{l1 l2 l}(t1, t2, phi) + LJ(eps, Rm), with
    A = sum_m <l1 m l2 -m | l 0> Ybar_{l1 m}(t1) Ybar_{l2 -m}(t2) cos(m phi)."""

    def interaction(R, coordinates):
        _, _, t1, t2, phi = coordinates
        x1, x2 = np.cos(t1), np.cos(t2)
        total = np.zeros_like(x1)
        for l1, l2, lam, c in terms:
            angular = np.zeros_like(x1)
            for m in range(-min(l1, l2), min(l1, l2) + 1):
                angular += clebsch_gordan(l1, m, l2, -m, lam) * norm_YjK(l1, m, x1) * norm_YjK(l2, -m, x2) * np.cos(m * phi)
            total += c * angular
        lj = lj_eps_cm * CM2AU * ((lj_Rm / R) ** 12 - 2.0 * (lj_Rm / R) ** 6)
        return strength_cm * CM2AU * np.exp(-0.8 * (R - 6.0)) * total + lj

    return PESWrapper(interaction=interaction)


def bispherical_terms(lmax: int, seed: int) -> list[tuple[int, int, int, float]]:
    rng = np.random.default_rng(seed)
    terms = []
    for l1 in range(lmax + 1):
        for l2 in range(lmax + 1):
            for lam in range(abs(l1 - l2), min(l1 + l2, lmax) + 1):
                if (l1 + l2 + lam) % 2 == 0 and (l1, l2, lam) != (0, 0, 0):
                    terms.append((l1, l2, lam, float(rng.normal())))
    return terms


def capture_pes(C6: float, wall_cm: float, seed: int) -> PESWrapper:
    """-C6/R^6 (1 + 0.1 P2) plus a seeded anisotropic Gaussian wall exp(-((R-7)/1.5)^2) sum_k g_k P_k."""
    g = np.random.default_rng(seed).uniform(0.2, 1.0, size=3)

    def interaction(R, coordinates):
        _, theta = coordinates
        x = np.cos(theta)
        p2 = 0.5 * (3.0 * x * x - 1.0)
        wall = wall_cm * CM2AU * np.exp(-(((R - 7.0) / 1.5) ** 2)) * (g[0] + g[1] * x + g[2] * p2)
        return -C6 / R**6 * (1.0 + 0.1 * p2) + wall

    return PESWrapper(interaction=interaction)


@dataclass
class Workload:
    """One (J, parity) block: system, PES grid and energies (hartree)."""

    name: str
    system: ScattSystem
    grid: PotentialGrid
    energies: np.ndarray
    mode: str = "inelastic"


def rigid_atom_diatom(*, B_cm=20.0, jmax=20, J=20, parity=1, mu_amu=18.0, eps_cm=150.0, Rm=6.5, a1=0.3, a2=0.2, n_theta=24, boundaries=(2.5, 30.0), half_steps=(0.05,), energies_cm=None, n_energy=16, approx=Approx.EXACT, K_delta=1) -> Workload:
    """Plain A+BC rigid rotor (the CPU-runnable configuration at full size)."""
    energies = np.linspace(10.0, 500.0, n_energy) * CM2AU if energies_cm is None else np.asarray(energies_cm) * CM2AU
    system = build_ScattSystem(AtomSpec(), rigid_rotor(B_cm, jmax), Jtot=J, system_parity=parity, potential=lj_aniso_pes(eps_cm, Rm, a1, a2), reduced_mass=mu_amu * AMU2AU, approx=approx, K_delta=K_delta)
    return Workload("rigid_atom_diatom", system, prepare_potential(system, boundaries, half_steps, n_theta=n_theta), energies)


MORSE_DEFAULTS = dict(De_cm=40000.0, re=1.4, a=1.2, mass_amu=1.0, r_interval=(0.5, 3.5), n_dvr=32, vmax=3, jmax=30)


def morse_atom_diatom(*, J=30, parity=1, mu_amu=18.0, eps_cm=150.0, Rm=6.5, a1=0.3, a2=0.2, seed=2024, n_theta=32, boundaries=(2.5, 40.0), half_steps=(0.02,), energies_cm=None, n_energy=256, diatom=None, approx=Approx.EXACT, K_delta=1, **diatom_args) -> Workload:
    """Vibrating A+BC: Morse diatom (v <= 3, j <= 30) with r-dependent anisotropy c_k ~ U(-1/2, 1/2)."""
    params = {**MORSE_DEFAULTS, **diatom_args}
    c1, c2 = np.random.default_rng(seed).uniform(-0.5, 0.5, size=2)
    diatom = morse_diatom(**params) if diatom is None else diatom
    energies = np.linspace(100.0, 3000.0, n_energy) * CM2AU if energies_cm is None else np.asarray(energies_cm) * CM2AU
    system = build_ScattSystem(AtomSpec(), diatom, Jtot=J, system_parity=parity, potential=lj_aniso_pes(eps_cm, Rm, a1, a2, c1, c2, params["re"]), reduced_mass=mu_amu * AMU2AU, approx=approx, K_delta=K_delta)
    return Workload("morse_atom_diatom", system, prepare_potential(system, boundaries, half_steps, n_theta=n_theta), energies)


def rotor_pair(*, B1_cm=60.0, B2_cm=2.0, jmax=8, J=6, parity=1, mu_amu=3.6, lmax=4, seed=11, strength_cm=40.0, lj_eps_cm=100.0, lj_Rm=6.0, n_theta_X=15, n_theta_Y=15, n_phi=12, boundaries=(2.5, 30.0), half_steps=(0.05,), energies_cm=None, n_energy=128, approx=Approx.EXACT, K_delta=1) -> Workload:
    """AB+CD rigid rotors with a seeded bispherical expansion plus isotropic LJ."""
    terms = bispherical_terms(lmax, seed)
    energies = np.linspace(5.0, 800.0, n_energy) * CM2AU if energies_cm is None else np.asarray(energies_cm) * CM2AU
    system = build_ScattSystem(rigid_rotor(B1_cm, jmax), rigid_rotor(B2_cm, jmax), Jtot=J, system_parity=parity, potential=bispherical_pes(terms, strength_cm, lj_eps_cm, lj_Rm), reduced_mass=mu_amu * AMU2AU, approx=approx, K_delta=K_delta)
    grid = prepare_potential(system, boundaries, half_steps, n_theta_X=n_theta_X, n_theta_Y=n_theta_Y, n_phi=n_phi)
    return Workload("rotor_pair", system, grid, energies)


def ultracold_capture(*, B_cm=0.03, jmax=40, J=10, parity=1, mu_amu=100.0, C6=1.0e4, wall_cm=500.0, seed=3, n_theta=48, boundaries=(8.0, 1500.0), half_steps=(0.05,), energies_K=None, n_energy=512, approx=Approx.EXACT, K_delta=1) -> Workload:
    """Capture-mode A+BC: ultracold energies log-uniform over 1 uK .. 1 mK."""
    energies = np.geomspace(1.0e-6, 1.0e-3, n_energy) * K2AU if energies_K is None else np.asarray(energies_K) * K2AU
    system = build_ScattSystem(AtomSpec(), rigid_rotor(B_cm, jmax), Jtot=J, system_parity=parity, potential=capture_pes(C6, wall_cm, seed), reduced_mass=mu_amu * AMU2AU, approx=approx, K_delta=K_delta)
    return Workload("ultracold_capture", system, prepare_potential(system, boundaries, half_steps, n_theta=n_theta), energies, mode="capture")


def _time_contraction(system: str, n_points: int, repeat: int) -> None:
    """Best-of-``repeat`` time of one ``ticc_contract`` call over ``n_points`` radial points of the
    vibrating A+BC system (N = 1984, 1024 grid points, real rows) or the AB+CD rotor pair (N = 2610,
    2700 grid points, complex rows); the rate counts the lower-triangle multiply-adds of every K
    group, 2 n_grid (x2 for complex rows) flops per channel pair."""
    import torch

    from .matrix.interaction import contract_rows, device_rows
    from .scattering import build_hamiltonian

    wl = morse_atom_diatom() if system == "morse" else rotor_pair()
    vb = build_hamiltonian(wl.system, wl.grid).V_basis
    dev = torch.device("cuda", 0)
    rows = device_rows(vb, dev)
    points = wl.grid.radial_points[np.linspace(0, wl.grid.radial_points.size - 1, n_points).astype(int)]
    values = wl.grid.take_device(points, dev).reshape(n_points, -1).contiguous()
    out = contract_rows(rows, values)
    torch.cuda.synchronize()
    best = None
    for _ in range(repeat):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        contract_rows(rows, values, out=out)
        end.record()
        torch.cuda.synchronize()
        best = start.elapsed_time(end) if best is None else min(best, start.elapsed_time(end))
    parts = 2 if vb.B_imag is not None else 1
    pairs = sum(len(m) * (len(m) + 1) // 2 for m in vb.channel_indices.values())
    flops = 2.0 * rows.n_grid * parts * pairs * n_points
    print(f"contract {system}: N={vb.n_channel} n_grid={rows.n_grid} parts={parts} points={n_points}: {best:.3f} ms ({best / n_points * 1e3:.1f} us/point), "
          f"{flops / (best * 1e-3) / 1e12:.2f} TF/s FP64 (lower-triangle work)")


def _time_pair_solve(n_energy: int) -> None:
    """Wall time of one ``solve`` of the AB+CD rotor pair (N = 2610, 275 sectors) over every
    128/n_energy-th of its 128 energies, plain FP64 then mixed precision, after a one-energy
    warm-up solve that builds the Hamiltonian and its device caches."""
    from time import perf_counter

    import torch

    from .propagation.config import Propagation
    from .scattering import solve

    wl = rotor_pair()
    energies = wl.energies[:: max(1, wl.energies.size // n_energy)][:n_energy]
    solve(wl.system, energies[:1], wl.grid, Propagation(precision="fp64"))
    results = {}
    for precision in ("fp64", "mixed"):
        stats: dict = {}
        torch.cuda.synchronize()
        started = perf_counter()
        result = solve(wl.system, energies, wl.grid, Propagation(precision=precision), stats=stats)
        torch.cuda.synchronize()
        wall = perf_counter() - started
        results[precision] = result
        print(f"pair N={wl.system.basis.n_channel} sectors={len(wl.grid.sectors)} {precision}: {energies.size} energies in {wall:.2f} s = {energies.size / wall:.2f} solves/s, "
              f"reduced sweep steps {stats.get('reduced_steps', 0)} of {stats.get('sweep_steps', 0)}, unitarity defect {result.unitarity_defect().max():.1e}")
    dS = max((float(np.abs(a - b).max()) for a, b in zip(results["fp64"].Smat, results["mixed"].Smat) if a.size), default=0.0)
    print(f"pair mixed vs fp64 max|dS| {dS:.2e}")


def _propagate_window(argv=None) -> None:
    """Propagate a window of the bench system's sectors once (a small, fixed case for
    profilers): ``python -m pyticc_b200.workloads --precision mixed --first 100 --sectors 8``."""
    import argparse

    import torch

    from .propagation.config import Propagation
    from .propagation.runner import propagate
    from .scattering import hamiltonian_for

    p = argparse.ArgumentParser(description=_propagate_window.__doc__)
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    p.add_argument("--first", type=int, default=100, help="first sector")
    p.add_argument("--sectors", type=int, default=8)
    p.add_argument("--energies", type=int, default=16, help="every 256/energies-th of the bench energies")
    p.add_argument("--repeat", type=int, default=0, help="also time the LDMD launches this many times (CUDA events) and print the best ms per sector")
    p.add_argument("--contract", choices=["morse", "pair"], default=None, help="time the V(R) contraction of this system instead (CUDA events, --points radial points per call)")
    p.add_argument("--points", type=int, default=64, help="radial points per contraction call")
    p.add_argument("--solve-pair", action="store_true", help="time whole solves of the AB+CD rotor pair (N = 2610) for --energies energies, FP64 and mixed")
    args = p.parse_args(argv)
    if args.contract is not None:
        _time_contraction(args.contract, args.points, max(args.repeat, 1))
        return
    if args.solve_pair:
        _time_pair_solve(args.energies)
        return
    wl = morse_atom_diatom()
    ham = hamiltonian_for(wl.system, wl.grid)
    energies = wl.energies[:: max(1, wl.energies.size // args.energies)][: args.energies]
    sectors = wl.grid.sectors[args.first : args.first + args.sectors]
    config = Propagation(precision=args.precision)
    propagate(ham, energies, sectors, config)
    torch.cuda.synchronize()
    best = None
    for _ in range(args.repeat):
        windows: list = []
        propagate(ham, energies, sectors, config, window_timing=windows)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b, _ in windows)
        best = ms if best is None else min(best, ms)
    if best is not None:
        flops = 2.0 * wl.system.basis.n_channel**3 * energies.size * len(sectors)
        print(f"{args.precision}: {best / len(sectors):.2f} ms/sector (best of {args.repeat} x {len(sectors)} sectors), {flops / (best * 1e-3) / 1e12:.1f} TF/s")
    print("ok")


if __name__ == "__main__":
    _propagate_window()
