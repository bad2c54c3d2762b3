"""PotentialGrid preparation, Hamiltonian construction and the ``solve`` driver.

Mirrors ``src/pyticc/scattering/{potential,hamiltonian,solver}.py`` and the A+BC / AB+CD
models of ``scattering/energy_transfer/{atom_diatom,diatom_diatom}.py``.  PES evaluation,
channel and row construction are host setup; propagation and matching run on the GPU.
"""

from __future__ import annotations

from collections import OrderedDict
from collections.abc import Sequence
from dataclasses import dataclass, field, replace
from time import perf_counter, process_time

import numpy as np
import torch
from loguru import logger

from .. import _native as nat
from ..basis import gauss_legendre_dvr, get_Umat_BF
from ..energy import get_Etot
from ..match.asymptotic import get_Bmat_BF_to_SF, transform_device
from ..match.smatrix import get_Smat_device, open_blocks_to_host
from ..matrix.interaction import DeviceBasisCache, VBasisBF, contract_device, prepare_atom_diatom, prepare_diatom_diatom
from ..pes import PESWrapper, get_Vgrid_atom_diatom, get_Vgrid_diatom_diatom
from ..pes_analytic import LegendrePES
from ..propagation.config import Propagation
from ..propagation.grid import RadialSector, build_radial_sectors, radial_points_of
from ..kblock import KBlock, build_cs_blocks, build_nncc_blocks
from ..result import CoupledStatesResult, KBlockResult, ScatteringResult, Timing
from ..system import Approx, ScatteringType, ScattSystem


@dataclass(frozen=True, slots=True)
class PotentialGrid:
    """Raw PES values on every sector start/mid/end point and quadrature node, with a
    per-device copy made once (reference ``scattering/potential.py:26-163``)."""

    boundaries: tuple[float, ...]
    half_steps: tuple[float, ...]
    sectors: tuple[RadialSector, ...]
    radial_points: np.ndarray
    scattering_type: ScatteringType
    coordinates: tuple[tuple[str, np.ndarray], ...]
    weights: tuple[tuple[str, np.ndarray], ...]
    values: np.ndarray
    _device_cache: dict = field(default_factory=dict, init=False, repr=False, compare=False)

    @property
    def Rmatch(self) -> float:
        return self.sectors[-1].radial_end

    def coordinate(self, name: str) -> np.ndarray:
        return self._named(self.coordinates, name, "coordinate")

    def weight(self, name: str) -> np.ndarray:
        return self._named(self.weights, name, "weight")

    @staticmethod
    def _named(arrays, name, label):
        for key, value in arrays:
            if key == name:
                return value
        message = f"Potential grid has no {label} named {name!r}"
        logger.error(message)
        raise KeyError(message)

    def selection(self, radial_points) -> np.ndarray:
        """Grid indices of the requested points (1e-12 bohr tolerance)."""
        requested = np.atleast_1d(np.asarray(radial_points, dtype=np.float64))
        positions = np.searchsorted(self.radial_points, requested)
        clipped = np.clip(positions, 0, self.radial_points.size - 1)
        lower = np.clip(positions - 1, 0, self.radial_points.size - 1)
        best = np.where(np.abs(self.radial_points[clipped] - requested) <= np.abs(self.radial_points[lower] - requested), clipped, lower)
        matched = np.abs(self.radial_points[best] - requested) <= 1.0e-12
        if not np.all(matched):
            message = f"Potential grid does not contain radial points {requested[~matched].tolist()}"
            logger.error(message)
            raise ValueError(message)
        return best.astype(np.int64)

    def take(self, radial_points) -> np.ndarray:
        index = self.selection(radial_points)
        return self.values[index] if np.ndim(radial_points) else self.values[index[0]]

    def device_values(self, device: torch.device) -> torch.Tensor:
        """The complete raw grid on one device, (n_points, n_grid), copied once."""
        key = (device.type, device.index)
        values = self._device_cache.get(key)
        if values is None:
            values = torch.as_tensor(np.ascontiguousarray(self.values.reshape(self.radial_points.size, -1)), device=device)
            self._device_cache[key] = values
            logger.info(f"Potential grid resident on gpu:{device.index}, size={values.numel() * 8 / 1024**2:.1f} MiB")
        return values

    def take_device(self, radial_points, device) -> torch.Tensor:
        index = torch.as_tensor(self.selection(radial_points), device=device)
        return self.device_values(torch.device(device)).index_select(0, index)


def _radial_grid(boundaries, half_steps):
    b = tuple(float(v) for v in boundaries)
    h = tuple(float(v) for v in half_steps)
    sectors = build_radial_sectors(b, h)
    return b, h, sectors, radial_points_of(sectors)


def prepare_potential(system: ScattSystem, boundaries: Sequence[float], half_steps: Sequence[float], *, processes: int = 1, **quadrature) -> PotentialGrid:
    """Evaluate the PES on the complete propagation grid (reference potential.py:182-222,
    energy_transfer/atom_diatom.py:28-73, diatom_diatom.py:28-90)."""
    if not isinstance(system, ScattSystem) or system.scattering_type is None:
        message = "prepare_potential requires a system built by build_ScattSystem"
        logger.error(message)
        raise TypeError(message)
    if not isinstance(system.potential, PESWrapper):
        message = "Potential preparation requires a scalar PESWrapper"
        logger.error(message)
        raise TypeError(message)
    b, h, sectors, points = _radial_grid(boundaries, half_steps)
    started = perf_counter()
    logger.info(f"Potential preparation started: type={system.scattering_type.value}, radial_points={points.size}, processes={processes}")
    if system.scattering_type is ScatteringType.ATOM_DIATOM:
        n_theta = int(quadrature.get("n_theta", 16))
        parity = system.channel_spec.exchange_parity_Y
        cos_theta, w = gauss_legendre_dvr(-1.0, 1.0, n_theta, symmetry=parity != 0)
        radial = system.monomer_Y.rovib.grids
        device_values = None
        if isinstance(system.potential, LegendrePES) and torch.cuda.is_available():
            # an analytic PES in the Legendre form is evaluated on the device, straight into
            # the grid the propagation reads (pes_analytic.py, ticc_pes_legendre_grid)
            device = torch.device("cuda", torch.cuda.current_device())
            device_values = system.potential.grid_device(points, radial, cos_theta, device)
            values = device_values.cpu().numpy().reshape(points.size, radial.size, cos_theta.size)
        else:
            values = get_Vgrid_atom_diatom(system.potential, points, radial, np.arccos(cos_theta))
        grid = PotentialGrid(b, h, sectors, points, system.scattering_type, (("r", radial), ("cos_theta", cos_theta)), (("theta", w),), values)
        if device_values is not None:
            grid._device_cache[(device.type, device.index)] = device_values
    else:
        cX, wX = gauss_legendre_dvr(-1.0, 1.0, int(quadrature.get("n_theta_X", 15)))
        cY, wY = gauss_legendre_dvr(-1.0, 1.0, int(quadrature.get("n_theta_Y", 15)))
        phi, wp = gauss_legendre_dvr(0.0, np.pi, int(quadrature.get("n_phi", 12)))
        rX, rY = system.monomer_X.rovib.grids, system.monomer_Y.rovib.grids
        values = get_Vgrid_diatom_diatom(system.potential, points, rX, rY, np.arccos(cX), np.arccos(cY), phi)
        grid = PotentialGrid(
            b, h, sectors, points, system.scattering_type,
            (("r_X", rX), ("r_Y", rY), ("cos_theta_X", cX), ("cos_theta_Y", cY), ("phi", phi)),
            (("theta_X", wX), ("theta_Y", wY), ("phi", wp)),
            values,
        )
    logger.info(f"Potential preparation complete: type={system.scattering_type.value}, radial_points={points.size}, wall={perf_counter() - started:.3f} s")
    return grid


@dataclass(frozen=True)
class ScattHamiltonian:
    """Projected channel Hamiltonian: H(R) = diag(E_int) + U/(2 mu R^2) + V(R)
    (reference ``scattering/hamiltonian.py:36-180``).  ``device_block_interaction`` is the
    reference's GPU contraction hook, served by ``ticc_contract``."""

    basis: object
    reduced_mass: float
    V_basis: VBasisBF
    potential_grid: PotentialGrid
    approx: Approx = Approx.EXACT
    K_delta: int = 1
    _device_cache: DeviceBasisCache = field(default_factory=DeviceBasisCache, compare=False, repr=False)
    # device-resident propagation state (rows, U, E_int, channel order) per device and
    # channel selection; it lives and dies with this Hamiltonian
    _runner_cache: dict = field(default_factory=dict, compare=False, repr=False)

    def __post_init__(self) -> None:
        if self.K_delta < 1:
            message = f"K_delta must be positive, but got {self.K_delta}"
            logger.error(message)
            raise ValueError(message)

    @property
    def E_int(self) -> np.ndarray:
        return self.basis.E_int

    def centrifugal(self, channel_indices: Sequence[int] | None = None) -> np.ndarray:
        """U over the selected channels in the given order (hamiltonian.py:87-110): the
        field-free BF matrix keeps the K -> K+1 Coriolis couplings inside the selection, so
        a single-K (CS) block has none and an NNCC window keeps those between its K."""
        return get_Umat_BF(self.basis, channel_indices)

    @property
    def U(self) -> np.ndarray:
        return get_Umat_BF(self.basis)

    @property
    def potential_grid_size(self) -> int:
        return int(np.prod(self.V_basis.grid_shape))

    def device_block_interaction(self, radial_points, channel_blocks, device=None):
        """V for each channel block at the given points, on the device (atom_diatom.py:147-157)."""
        dev = nat.require_cuda(device)
        values = self.potential_grid.take_device(radial_points, dev)
        return tuple(contract_device(self.V_basis, self._device_cache, values, dev, indices) for indices in channel_blocks)


def build_hamiltonian(system: ScattSystem, potential_grid: PotentialGrid) -> ScattHamiltonian:
    """Weighted rows for the grid's quadrature (atom_diatom.py:80-168, diatom_diatom.py:97-217)."""
    if potential_grid.scattering_type is not system.scattering_type:
        message = f"System type {system.scattering_type.value} cannot use a {potential_grid.scattering_type.value} potential grid"
        logger.error(message)
        raise TypeError(message)
    if system.reduced_mass is None:
        message = "The Hamiltonian requires a collision reduced mass"
        logger.error(message)
        raise ValueError(message)
    if system.scattering_type is ScatteringType.ATOM_DIATOM:
        vb = prepare_atom_diatom(system.basis, system.monomer_Y.rovib, potential_grid.coordinate("cos_theta"), potential_grid.weight("theta"))
    else:
        g = potential_grid
        vb = prepare_diatom_diatom(
            system.basis, system.monomer_X.rovib, system.monomer_Y.rovib,
            g.coordinate("cos_theta_X"), g.weight("theta_X"), g.coordinate("cos_theta_Y"), g.weight("theta_Y"), g.coordinate("phi"), g.weight("phi"),
        )
    return ScattHamiltonian(system.basis, float(system.reduced_mass), vb, potential_grid, system.approx, system.K_delta)


HAMILTONIAN_CACHE_SIZE = 8
_HAMILTONIANS: OrderedDict[tuple[int, int], tuple[ScattSystem, PotentialGrid, ScattHamiltonian]] = OrderedDict()


def hamiltonian_for(system: ScattSystem, potential_grid: PotentialGrid) -> ScattHamiltonian:
    """Build once per (system, grid) pair and reuse (the rows only depend on geometry).

    The cache holds the system and grid it was built from and checks their identity, so an
    object id reused after garbage collection can never be served another system's
    Hamiltonian; it keeps the most recent HAMILTONIAN_CACHE_SIZE pairs, and an evicted
    Hamiltonian frees its device state with it."""
    key = (id(system), id(potential_grid))
    entry = _HAMILTONIANS.get(key)
    if entry is not None and entry[0] is system and entry[1] is potential_grid:
        _HAMILTONIANS.move_to_end(key)
        return entry[2]
    hamiltonian = build_hamiltonian(system, potential_grid)
    _HAMILTONIANS[key] = (system, potential_grid, hamiltonian)
    _HAMILTONIANS.move_to_end(key)
    while len(_HAMILTONIANS) > HAMILTONIAN_CACHE_SIZE:
        _HAMILTONIANS.popitem(last=False)
    return hamiltonian


def build_k_blocks(hamiltonian: ScattHamiltonian) -> tuple[KBlock, ...]:
    """CS or NNCC propagation blocks of one Hamiltonian (solver.py:203-216)."""
    if hamiltonian.approx is Approx.CS:
        return build_cs_blocks(hamiltonian.basis)
    if hamiltonian.approx is Approx.NNCC:
        return build_nncc_blocks(hamiltonian.basis, hamiltonian.K_delta)
    message = f"Coupled-states blocks require approx='cs' or 'nncc', but got {hamiltonian.approx.value!r}"
    logger.error(message)
    raise ValueError(message)


def _match(Y: torch.Tensor, B: np.ndarray, L: np.ndarray, E_int: np.ndarray, Rmatch: float, energies: np.ndarray, reduced_mass: float) -> tuple[np.ndarray, ...]:
    """BF -> SF transform and matching on the device; one open-open S per energy."""
    Y_sf = transform_device(Y, nat.as_device(B, Y.device, torch.float64))
    S, n_open = get_Smat_device(Y_sf, Rmatch, energies, reduced_mass, E_int, L)
    return open_blocks_to_host(S, n_open)


def finalize_K_block(basis, block: KBlock, Y_BF: torch.Tensor, Etot, reduced_mass: float, Rmatch: float, *, approx: Approx = Approx.NNCC) -> KBlockResult:
    """Transform, match and package one CS or NNCC block (finalize.py:168-225); ``Y_BF`` is
    the block's device log-derivative batch (n_energy, n_b, n_b)."""
    energies = get_Etot(Etot)
    indices = np.asarray(block.channel_indices, dtype=np.int64)
    E_int = basis.E_int[indices]
    B, L = get_Bmat_BF_to_SF(basis, block.channel_indices)
    smats = _match(Y_BF, B, L, E_int, Rmatch, energies, reduced_mass)
    open_indices = tuple(indices[np.flatnonzero(E_int < e)] for e in energies)
    return KBlockResult(block, open_indices, Y_BF.cpu().numpy(), B, L, smats)


def solve(problem: ScattSystem, Etot, potential_grid: PotentialGrid, propagation: Propagation, *, sectors: Sequence[RadialSector] | None = None, stats: dict | None = None) -> ScatteringResult | CoupledStatesResult:
    """Build (or reuse), propagate and match one (J, parity) system (reference
    solver.py:57-178): exact CC returns a ScatteringResult; CS and NNCC propagate their K
    blocks together and return a CoupledStatesResult.

    ``sectors`` optionally replaces the grid's fixed-step sectors by another schedule whose
    start/mid/end points all lie on the grid (e.g. a learned step schedule).  ``stats``
    (optional dict, exact CC) receives the sectors propagated, the reduced-precision sweep
    steps among all sweep steps, and the learned-schedule judge's record."""
    from ..propagation.runner import propagate, propagate_blocks

    if not isinstance(problem, ScattSystem):
        message = "solve requires a ScattSystem"
        logger.error(message)
        raise TypeError(message)
    if not isinstance(potential_grid, PotentialGrid):
        message = "A ScattSystem solve requires a PotentialGrid"
        logger.error(message)
        raise TypeError(message)
    energies = get_Etot(Etot)
    wall, cpu = perf_counter(), process_time()
    basis = problem.basis
    logger.info(f"Solving Jtot={basis.Jtot}, system_parity={basis.system_parity:+d}, approx={problem.approx.value}, channels={basis.n_channel}, energies={energies.size}")
    if basis.n_channel == 0:
        message = "At least one non-empty channel block is required for propagation"
        logger.error(message)
        raise ValueError(message)
    hamiltonian = hamiltonian_for(problem, potential_grid)
    run_sectors = potential_grid.sectors if sectors is None else tuple(sectors)
    if problem.approx is not Approx.EXACT:
        if sectors is None and propagation.steps == "learned":
            message = "Learned sector widths are trained for exact coupled channels; use steps='fixed' with CS/NNCC"
            logger.error(message)
            raise ValueError(message)
        blocks = build_k_blocks(hamiltonian)
        Y_blocks = propagate_blocks(hamiltonian, tuple(b.channel_indices for b in blocks), energies, run_sectors, propagation)
        Rmatch = run_sectors[-1].radial_end
        results = tuple(
            finalize_K_block(basis, block, Y_b, energies, hamiltonian.reduced_mass, Rmatch, approx=problem.approx)
            for block, Y_b in zip(blocks, Y_blocks, strict=True)
        )
        timing = Timing(perf_counter() - wall, process_time() - cpu)
        logger.info(f"Solver complete: {timing}")
        return CoupledStatesResult(basis, energies, problem.approx, results, timing)
    if sectors is None and propagation.steps == "learned":
        from ..propagation.learned import judged_learned_sectors

        run_sectors, record = judged_learned_sectors(problem, potential_grid, energies, propagation)
        if stats is not None:
            stats["learned"] = record
    Y = propagate(hamiltonian, energies, run_sectors, propagation, stats=stats)
    B, L = get_Bmat_BF_to_SF(basis)
    smats = _match(Y, B, L, basis.E_int, run_sectors[-1].radial_end, energies, hamiltonian.reduced_mass)
    max_dS = None
    if propagation.audit:
        plain = solve(problem, energies, potential_grid, replace(propagation, precision="fp64", steps="fixed", audit=False))
        max_dS = np.asarray([float(np.abs(a - b).max()) if a.shape == b.shape and a.size else (0.0 if a.shape == b.shape else np.inf) for a, b in zip(smats, plain.Smat, strict=True)])
    if stats is not None:
        from ..propagation.runner import finish_stats

        finish_stats(stats)
    timing = Timing(perf_counter() - wall, process_time() - cpu)
    logger.info(f"Solver complete: {timing}")
    return ScatteringResult(basis, energies, Y.cpu().numpy(), B, L, smats, timing, hamiltonian.reduced_mass, max_dS)
