"""Partial-wave sweep: every (J, parity) block of a system, batched, in one CUDA graph.

The reference solves one (J, parity) system per ``ticc.solve`` call (``scattering/solver.py:
57-178``); a partial-wave sum loops over J and parity outside it, and inside a call
``_propagate_blocks`` (``propagation/runner.py:165-322``) runs one ``propagate_logD`` per block
and window.  Here a ``PartialWaveSweep`` takes all blocks at once:

* blocks without channels are skipped up front (the reference raises on an empty exact
  block, ``runner.py:206-209``) and give ``None`` results;
* the others are grouped by the size of their sweep matrix (64 rows, then multiples of 128)
  and each group is padded to its size with decoupled closed channels and propagated as one
  batch of (block, energy) matrices per radial window (``ticc_ldmd_propagate_blocks``);
* an autotuner decides, per size class, whether the class runs on its own or padded into the
  next larger class (fewer, larger launches against more padded flops), by timing a probe of
  two sectors of each option on the device; decisions are cached per class signature;
* groups larger than the memory budget are split into several launches;
* the window loop of every launch (contraction of W_base, initial Y, batched LDMD) is
  enqueued with preallocated buffers and no host synchronisation, so that it is captured
  once into one CUDA graph and replayed for each new set of energies.

Matching stays outside the graph (its open-channel counts depend on the energies).
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass

import numpy as np
import torch
from loguru import logger

from .. import _native as nat
from ..energy import get_Etot
from ..matrix.interaction import contract_rows
from .config import Propagation, resolve_device
from .grid import MAX_SECTORS_PER_WINDOW, RadialSector, radial_points_of
from .logd import blocks_workspace_bytes, propagate_blocks_device
from .runner import BlockState, DeviceBlocks, initial_logD

SWEEP_WORKSPACE_SLOT = 32     # workspace slot shared by the sweep's launches (they run in order)
PROBE_SECTORS = 2             # sectors timed per option by the autotuner
_AUTOTUNE: dict = {}          # (device name, mode, precision, n_energy, class signature) -> merge decisions


def size_class(n_channel: int, mode: str) -> int:
    """Rows of the sweep matrix a block of n_channel channels is propagated in: 64 (the 64-wide
    single-block inversion) when they fit, else a multiple of 128."""
    rows = (2 if mode == "capture" else 1) * n_channel
    return 64 if rows <= 64 else -(-rows // 128) * 128


def class_channels(size: int, mode: str) -> int:
    """Largest channel count a class of the given sweep size holds."""
    return size // (2 if mode == "capture" else 1)


@dataclass
class LaunchPlan:
    """One batched launch: block positions (into the sweep's list) padded to n channels."""

    members: tuple[int, ...]
    n: int


def plan_launches(sizes: Sequence[int], mode: str, merged_into_next: dict[int, bool], bytes_per_block, budget: float) -> list[LaunchPlan]:
    """Group blocks (channel counts ``sizes``; 0 = empty, skipped) by size class, merge a class
    into the next larger one where ``merged_into_next[class]`` says so, and split each group
    into launches of at most ``budget`` bytes (``bytes_per_block(n, count)`` estimates one
    launch's device memory)."""
    classes: dict[int, list[int]] = {}
    for i, n in enumerate(sizes):
        if n > 0:
            classes.setdefault(size_class(n, mode), []).append(i)
    keys = sorted(classes)
    groups: list[tuple[int, list[int]]] = []
    carry: list[int] = []
    for k, key in enumerate(keys):
        members = carry + classes[key]
        if k + 1 < len(keys) and merged_into_next.get(key, False):
            carry = members
            continue
        carry = []
        groups.append((key, members))
    launches = []
    for key, members in groups:
        n = class_channels(key, mode)
        per = max(1, int(budget // max(bytes_per_block(n, 1), 1)))
        while per > 1 and bytes_per_block(n, per) > budget:
            per -= 1
        for start in range(0, len(members), per):
            launches.append(LaunchPlan(tuple(members[start : start + per]), n))
    return launches


class _Launch:
    """Device state of one launch: blocks padded to n, windows precomputed, buffers allocated;
    ``enqueue`` issues the whole radial traversal without a host synchronisation."""

    def __init__(self, states, n: int, sectors: Sequence[RadialSector], n_energy: int, energy_bound: float, config: Propagation, device: torch.device):
        self.device = device
        self.config = config
        self.db = DeviceBlocks(None, device, states=states, n=n)
        self.n = n
        self.n_block = len(states)
        self.n_energy = n_energy
        self.complex = config.mode == "capture"
        self.precision = nat.PRECISION_MIXED if config.precision == "mixed" else nat.PRECISION_FP64
        self.E_pad = self.db.thresholds(np.array([energy_bound]), device)
        n_sector = len(sectors)
        size = max(1, min(n_sector, MAX_SECTORS_PER_WINDOW, 65535 // self.n_block, window_sectors(n, self.n_block, n_energy, self.complex)))
        self.windows = []
        for s0 in range(0, n_sector, size):
            window = tuple(sectors[s0 : s0 + size])
            points = radial_points_of(window)
            index = torch.as_tensor(self.db.grid.selection(points), device=device)
            R = torch.as_tensor(np.ascontiguousarray(points), device=device)
            halves = torch.as_tensor(np.asarray([s.radial_half_step for s in window]), device=device)
            self.windows.append((len(window), index, R, halves))
        self.points_max = 2 * size + 1
        self.W = torch.empty((self.n_block, self.points_max, n, n), dtype=torch.float64, device=device)
        dtype = torch.complex128 if self.complex else torch.float64
        self.Y = torch.empty((self.n_block, n_energy, n, n), dtype=dtype, device=device)
        self.energies = torch.zeros(n_energy, dtype=torch.float64, device=device)
        self.status = nat.DeviceStatus(device)
        self.workspace_bytes = blocks_workspace_bytes(n, n_energy, self.n_block, size, self.complex, self.precision)

    def enqueue(self) -> None:
        db = self.db
        stride = 2 * self.n * self.n
        for w, (count, index, R, halves) in enumerate(self.windows):
            potential = db.values.index_select(0, index)
            npts = 2 * count + 1
            for g in range(self.n_block):
                contract_rows(db.rows[g], potential, radial_points=R, U=db.U[g], E_int=self.E_pad[g], reduced_mass=db.reduced_mass, out=self.W[g, :npts])
            if w == 0:
                for g in range(self.n_block):
                    self.Y[g].copy_(initial_logD(self.W[g, 0], self.energies, db.reduced_mass, self.config.mode))
            propagate_blocks_device(self.Y, self.energies, db.reduced_mass, halves, self.W[0, 0], self.W[0, 1], self.W[0, 2], stride=(stride, stride, stride),
                                    block_stride=self.points_max * self.n * self.n, precision=self.precision, workspace_slot=SWEEP_WORKSPACE_SLOT, status=self.status)

    def block_Y(self, g: int) -> torch.Tensor:
        size = self.db.sizes[g]
        pos = self.db.position[g]
        return self.Y[g, :, :size, :size][:, pos][:, :, pos].contiguous()


def window_sectors(n: int, n_block: int, n_energy: int, is_complex: bool, budget: float = 4 * 1024**3) -> int:
    """Sectors per window so that the W points and per-sector Q_mid / y1 / y2 of a launch stay
    within ``budget`` bytes."""
    padded = -(-(2 * n if is_complex else n) // 128) * 128
    per_sector = 8 * n_block * (2 * n * n + padded * padded + 2 * n_energy * n)
    return max(1, int(budget // per_sector))


def launch_bytes(n: int, n_block: int, n_energy: int, n_sector: int, mode: str, precision: str) -> int:
    """Device bytes of one launch: work matrices, sweep scratch and split panels (the
    workspace), the W window, Y and the energies."""
    is_complex = mode == "capture"
    size = max(1, min(n_sector, MAX_SECTORS_PER_WINDOW, window_sectors(n, n_block, n_energy, is_complex)))
    work = blocks_workspace_bytes(n, n_energy, n_block, size, is_complex, nat.PRECISION_MIXED if precision == "mixed" else nat.PRECISION_FP64)
    W = 8 * n_block * (2 * size + 1) * n * n
    Y = (16 if is_complex else 8) * n_block * n_energy * n * n
    return work + W + Y


class PartialWaveSweep:
    """Exact-CC solves of many (J, parity) systems that share one PotentialGrid and reduced
    mass, for batches of ``n_energy`` energies not above ``energy_bound`` (hartree).

    ``graph=True``: the first ``run`` propagates directly and then records the propagation of
    every block into one CUDA graph, which every later ``run`` replays (new energies are
    copied into the captured buffers first); ``autotune=True`` times the class-merging options once
    per class signature; ``memory_fraction`` of the free device memory bounds the launches
    (all of them are resident together in the graph)."""

    def __init__(self, systems: Sequence, potential_grid, propagation: Propagation, *, n_energy: int, energy_bound: float, sectors: Sequence[RadialSector] | None = None,
                 graph: bool = True, autotune: bool = True, memory_fraction: float = 0.6):
        from ..scattering import build_hamiltonian
        from ..system import Approx

        if propagation.steps != "fixed":
            message = "A partial-wave sweep propagates on the fixed grid (steps='fixed')"
            logger.error(message)
            raise ValueError(message)
        if n_energy < 1:
            message = f"n_energy must be positive, but got {n_energy}"
            logger.error(message)
            raise ValueError(message)
        self.device = resolve_device(propagation.device)
        self.config = propagation
        self.systems = tuple(systems)
        self.grid = potential_grid
        self.sectors = tuple(potential_grid.sectors if sectors is None else sectors)
        self.n_energy = int(n_energy)
        self.energy_bound = float(energy_bound)
        for system in self.systems:
            if system.approx is not Approx.EXACT:
                message = "A partial-wave sweep solves exact coupled channels; use solve() for CS/NNCC"
                logger.error(message)
                raise ValueError(message)
        masses = {float(s.reduced_mass) for s in self.systems if s.basis.n_channel}
        if len(masses) > 1:
            message = f"Systems of one sweep must share a reduced mass, but got {sorted(masses)}"
            logger.error(message)
            raise ValueError(message)
        self.sizes = tuple(s.basis.n_channel for s in self.systems)
        skipped = sum(1 for n in self.sizes if n == 0)
        if skipped:
            logger.info(f"Partial-wave sweep: {skipped} block(s) without channels skipped")
        closed_first = True  # the propagation order at every precision (runner.DeviceHamiltonian)
        self.states = {}
        for i, system in enumerate(self.systems):
            if self.sizes[i]:
                ham = build_hamiltonian(system, potential_grid)
                self.states[i] = BlockState(ham, tuple(range(self.sizes[i])), self.device, closed_first)
        free, _ = torch.cuda.mem_get_info(self.device)
        self.budget = memory_fraction * free
        merges = self._autotune() if autotune else {}
        n_sector = len(self.sectors)
        per_block = lambda n, count: launch_bytes(n, count, self.n_energy, n_sector, propagation.mode, propagation.precision)  # noqa: E731
        plans = plan_launches(self.sizes, propagation.mode, merges, per_block, self.budget / max(1, len(set(self.sizes))))
        self.merges = merges
        self.launches = [_Launch([self.states[i] for i in p.members], p.n, self.sectors, self.n_energy, self.energy_bound, propagation, self.device) for p in plans]
        self.members = [p.members for p in plans]
        nat.Workspace.get(self.device, max(l.workspace_bytes for l in self.launches), slot=SWEEP_WORKSPACE_SLOT)
        self.use_graph = graph
        self.graph = None
        self.graph_launches = 0  # library kernels recorded in the graph (each replay launches them)
        logger.info(f"Partial-wave sweep: {len(self.states)} blocks in {len(self.launches)} launches, classes merged: {sorted(k for k, v in merges.items() if v)}, graph={graph}")

    # ---- autotuning --------------------------------------------------------------------------
    def _signature(self) -> tuple:
        counts: dict[int, int] = {}
        for n in self.sizes:
            if n:
                key = size_class(n, self.config.mode)
                counts[key] = counts.get(key, 0) + 1
        return tuple(sorted(counts.items()))

    def _probe(self, members: Sequence[int], n: int) -> float:
        """Device milliseconds of PROBE_SECTORS sectors of one launch of these blocks."""
        launch = _Launch([self.states[i] for i in members], n, self.sectors[:PROBE_SECTORS], self.n_energy, self.energy_bound, self.config, self.device)
        nat.Workspace.get(self.device, launch.workspace_bytes, slot=SWEEP_WORKSPACE_SLOT)
        launch.energies.fill_(0.5 * self.energy_bound)
        launch.enqueue()  # warm
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        launch.enqueue()
        stop.record()
        torch.cuda.synchronize(self.device)
        launch.status.raise_if_failed("partial-wave sweep autotune probe")
        return start.elapsed_time(stop)

    def _autotune(self) -> dict[int, bool]:
        mode = self.config.mode
        key = (torch.cuda.get_device_name(self.device), mode, self.config.precision, self.n_energy, self._signature())
        cached = _AUTOTUNE.get(key)
        if cached is not None:
            return dict(cached)
        classes: dict[int, list[int]] = {}
        for i, n in enumerate(self.sizes):
            if n:
                classes.setdefault(size_class(n, mode), []).append(i)
        keys = sorted(classes)
        decisions: dict[int, bool] = {}
        carry: list[int] = []
        n_sector = len(self.sectors)
        for k in range(len(keys) - 1):
            small, large = keys[k], keys[k + 1]
            members_small = carry + classes[small]
            n_large = class_channels(large, mode)
            fits = launch_bytes(n_large, len(members_small) + len(classes[large]), self.n_energy, n_sector, mode, self.config.precision) <= self.budget / 2
            if not fits:
                decisions[small], carry = False, []
                continue
            separate = self._probe(members_small, class_channels(small, mode)) + self._probe(classes[large], n_large)
            merged = self._probe(members_small + classes[large], n_large)
            decisions[small] = merged < separate
            carry = members_small if decisions[small] else []
            logger.info(f"Autotune class {small} -> {large}: separate {separate:.2f} ms, merged {merged:.2f} ms per {PROBE_SECTORS} sectors: {'merge' if decisions[small] else 'keep'}")
        _AUTOTUNE[key] = dict(decisions)
        return decisions

    # ---- running -----------------------------------------------------------------------------
    def _enqueue_all(self) -> None:
        for launch in self.launches:
            launch.enqueue()

    def propagate(self, Etot) -> list[torch.Tensor | None]:
        """Y at the last sector end for every block (device, original channel order)."""
        energies = get_Etot(Etot)
        if energies.size != self.n_energy:
            message = f"This sweep was planned for {self.n_energy} energies, but got {energies.size}"
            logger.error(message)
            raise ValueError(message)
        if float(energies.max()) > self.energy_bound:
            message = f"Energy {float(energies.max())} is above the sweep's bound {self.energy_bound}"
            logger.error(message)
            raise ValueError(message)
        host = torch.as_tensor(energies)
        with torch.cuda.device(self.device):
            for launch in self.launches:
                launch.energies.copy_(host)
                launch.status.tensor.zero_()
            if self.graph is not None:
                self.graph.replay()
            else:
                self._enqueue_all()
            torch.cuda.synchronize(self.device)
            for launch in self.launches:
                launch.status.raise_if_failed("partial-wave sweep")
            out: list[torch.Tensor | None] = [None] * len(self.systems)
            for launch, members in zip(self.launches, self.members, strict=True):
                for g, i in enumerate(members):
                    out[i] = launch.block_Y(g)
            if self.use_graph and self.graph is None:
                # the first call ran directly (its kernels set their attributes outside any
                # capture); record the same traversal once for the later calls to replay.  The
                # library sets kernel attributes and queries the device while enqueueing, which
                # the relaxed capture mode allows.
                self.graph = torch.cuda.CUDAGraph()
                lib = nat.load_library()
                before = lib.ticc_kernel_launches()
                with torch.cuda.graph(self.graph, capture_error_mode="relaxed"):
                    self._enqueue_all()
                self.graph_launches = int(lib.ticc_kernel_launches() - before)
        return out
    def run(self, Etot) -> list:
        """ScatteringResult per system (None for a system without channels)."""
        from ..match.asymptotic import get_Bmat_BF_to_SF
        from ..result import ScatteringResult, Timing
        from ..scattering import _match

        energies = get_Etot(Etot)
        Ys = self.propagate(energies)
        results = []
        Rmatch = self.sectors[-1].radial_end
        for i, (system, Y) in enumerate(zip(self.systems, Ys, strict=True)):
            if Y is None:
                results.append(None)
                continue
            B, L = get_Bmat_BF_to_SF(system.basis)
            smats = _match(Y, B, L, system.basis.E_int, Rmatch, energies, float(system.reduced_mass))
            results.append(ScatteringResult(system.basis, energies, Y.cpu().numpy(), B, L, smats, Timing(0.0, 0.0), float(system.reduced_mass)))
        return results


def solve_sweep(systems: Sequence, Etot, potential_grid, propagation: Propagation, **options) -> list:
    """One-call partial-wave sweep: every system at every energy (see PartialWaveSweep)."""
    energies = get_Etot(Etot)
    plan = PartialWaveSweep(systems, potential_grid, propagation, n_energy=energies.size, energy_bound=float(energies.max()), **options)
    return plan.run(energies)
