"""Windowed radial driver on the GPU (reference ``src/pyticc/propagation/runner.py:112-322``).

Per window of sectors: W_base at every start/mid/end point is built on the device by the
fused contraction (``ticc_contract`` with the U/R^2 + 2 mu [V + E_int] epilogue) straight
from the device-resident PES grid, then ``ticc_ldmd_propagate`` advances all energies.
Y stays on the device for the whole traversal.  Windows are sized by device memory
(W points plus per-sector Q_mid), not by the reference's host transient-memory model.
"""

from __future__ import annotations

from collections.abc import Sequence
from copy import copy
from concurrent.futures import ThreadPoolExecutor
from math import ceil
from time import perf_counter

import numpy as np
import torch
from loguru import logger

from .. import _native as nat
from ..energy import get_Etot
from ..matrix.interaction import contract_rows, device_rows
from .config import Propagation, resolve_device
from .grid import MAX_SECTORS_PER_WINDOW, RadialSector, radial_points_of
from .logd import propagate_blocks_device, propagate_device

WINDOW_BYTES = 6 * 1024**3  # device budget for one window's W points and Q_mid


def device_window(n_channel: int, n_sector: int) -> int:
    """Sectors per window so that (2w+1) W points + w Q_mid fit the window budget."""
    padded = -(-n_channel // 128) * 128
    per_sector = 8 * (2 * n_channel * n_channel + padded * padded)
    return max(1, min(n_sector, MAX_SECTORS_PER_WINDOW, WINDOW_BYTES // per_sector))


class DeviceHamiltonian:
    """Device-resident pieces of one channel block: rows, U, E_int and the PES grid.

    With ``closed_first`` the channels are reordered once so that the most strongly closed
    ones (largest W_ii at the outermost grid point) come first; the mixed-precision sweep
    takes its reduced-precision blocks from the front of that order.  ``position[c]`` is
    the propagated index of original channel c.

    The propagation uses that order at every precision: the sweep pivots only inside each
    64-wide sub-block of a 128-block, so the order decides which channels share a pivot
    block.  Eliminating the strongly closed (diagonally dominant) channels first keeps the
    pivot blocks better conditioned.  On the AB+CD rotor pair (N = 2610) at 556 cm^-1,
    against the reference's fully pivoted LU: a CPU emulation of the blocked sweep loses
    3.7e-8 in S in this order and 4.3e-7 in the basis order; on the device the basis order
    lost 6e-3 and this order 2.4e-7 (FP64) and 2.3e-7 (mixed precision)."""

    def __init__(self, hamiltonian, device: torch.device, closed_first: bool = False) -> None:
        self.rows = device_rows(hamiltonian.V_basis, device)
        U = np.ascontiguousarray(hamiltonian.U)
        E_int = np.ascontiguousarray(hamiltonian.E_int)
        self.values = hamiltonian.potential_grid.device_values(device)
        self.grid = hamiltonian.potential_grid
        self.reduced_mass = hamiltonian.reduced_mass
        self.n = hamiltonian.basis.n_channel
        self.U = torch.as_tensor(U, device=device)
        self.E_int = torch.as_tensor(E_int, device=device)
        self.position = None
        if closed_first:
            outer = self.W_base(self.grid.radial_points[-1:])[0]
            order = np.argsort(-torch.diagonal(outer).cpu().numpy(), kind="stable")
            position = np.empty_like(order)
            position[order] = np.arange(order.size)
            self.U = torch.as_tensor(np.ascontiguousarray(U[np.ix_(order, order)]), device=device)
            self.E_int = torch.as_tensor(np.ascontiguousarray(E_int[order]), device=device)
            self.rows.row_out = torch.as_tensor(position, device=device, dtype=torch.int32)[self.rows.row_out.long()].to(torch.int32).contiguous()
            self.position = torch.as_tensor(position, device=device)

    def W_base(self, radial_points: np.ndarray, out: torch.Tensor | None = None) -> torch.Tensor:
        dev = self.U.device
        index = torch.as_tensor(self.grid.selection(radial_points), device=dev)
        potential = self.values.index_select(0, index)
        R = torch.as_tensor(np.ascontiguousarray(radial_points), device=dev)
        return contract_rows(self.rows, potential, radial_points=R, U=self.U, E_int=self.E_int, reduced_mass=self.reduced_mass, out=out)


def _device_state(hamiltonian, key, build):
    """Device state cached on the Hamiltonian object itself (its ``_runner_cache``), so the
    state lives exactly as long as the Hamiltonian; objects without that attribute get a
    fresh build on every call."""
    cache = getattr(hamiltonian, "_runner_cache", None)
    if cache is None:
        return build()
    state = cache.get(key)
    if state is None:
        state = build()
        cache[key] = state
    return state


def release_device_state(hamiltonian) -> None:
    """Drop every device-resident copy this Hamiltonian holds (they are rebuilt on use)."""
    cache = getattr(hamiltonian, "_runner_cache", None)
    if cache is not None:
        cache.clear()


def device_hamiltonian(hamiltonian, device: torch.device, closed_first: bool = False) -> DeviceHamiltonian:
    return _device_state(hamiltonian, ("exact", device.index, closed_first), lambda: DeviceHamiltonian(hamiltonian, device, closed_first))


def finish_stats(stats: dict) -> dict:
    """Synchronise and fold the pending reduced-block counts of ``propagate(stats=...)``
    into stats["reduced_steps"] (two sweeps per sector take the same count)."""
    pending = stats.pop("_reduced", [])
    if pending:
        torch.cuda.synchronize()
    stats["reduced_steps"] = stats.get("reduced_steps", 0) + sum(2 * int(c.sum()) for c in pending)
    return stats


def initial_logD(W0: torch.Tensor, energies: torch.Tensor, reduced_mass: float, mode: str) -> torch.Tensor:
    """Y(R0) from diag W(R0; E) = diag W_base(R0) - 2 mu E (logd.py:48-91)."""
    d = torch.diagonal(W0)[None, :] - 2.0 * reduced_mass * energies[:, None]
    if mode == "inelastic":
        return torch.diag_embed(torch.sqrt(torch.abs(d))).contiguous()
    values = torch.where(d >= 0.0, torch.sqrt(torch.clamp(d, min=0.0)).to(torch.complex128), -1j * torch.sqrt(torch.clamp(-d, min=0.0)).to(torch.complex128))
    return torch.diag_embed(values).contiguous()


def propagate(hamiltonian, Etot, radial_sectors: Sequence[RadialSector], config: Propagation, *, Y_initial: torch.Tensor | None = None, window_timing: list | None = None, stats: dict | None = None) -> torch.Tensor:
    """Y at the last sector end for every energy, on the device (runner.py:112-161).

    ``window_timing`` (optional list) receives (start event, stop event, algorithmic
    flops) per LDMD launch: two symmetric N x N inversions (N^3 each) per (sector, energy).
    ``stats`` (optional dict) receives the sector count, the sweep steps and, in mixed
    precision, the device's per-sector reduced-block counts as pending host copies;
    ``finish_stats`` turns them into "reduced_steps" (no synchronisation until then)."""
    energies_np = get_Etot(Etot)
    dev = resolve_device(config.device)
    if not radial_sectors:
        message = "Propagation produced no radial windows"
        logger.error(message)
        raise RuntimeError(message)
    mixed = config.precision == "mixed"
    dh = device_hamiltonian(hamiltonian, dev, closed_first=True)
    n = dh.n
    energies = torch.as_tensor(np.array(energies_np), device=dev)
    n_sector = len(radial_sectors)
    size = device_window(n, n_sector)
    precision = nat.PRECISION_MIXED if mixed else nat.PRECISION_FP64
    if Y_initial is not None and dh.position is not None:
        Y_initial = Y_initial[:, dh.position.argsort()][:, :, dh.position.argsort()].contiguous()
    logger.info(f"Propagation device: gpu:{dev.index}, x64=True")
    if config.print_verbose:
        logger.info(f"Propagation started: blocks=1, sectors={n_sector}, channels={n}, energies={energies_np.size}, pes_prefetch=False")
    started = perf_counter()
    interval = max(1, ceil(n_sector / 10))
    next_report = interval
    Y = Y_initial
    W = torch.empty((2 * size + 1, n, n), dtype=torch.float64, device=dev)
    done = 0
    for s0 in range(0, n_sector, size):
        window = tuple(radial_sectors[s0 : s0 + size])
        points = radial_points_of(window)
        Wv = dh.W_base(points, out=W[: points.size])
        if Y is None:
            Y = initial_logD(Wv[0], energies, dh.reduced_mass, config.mode)
        halves = torch.as_tensor(np.asarray([s.radial_half_step for s in window]), device=dev)
        stride = 2 * n * n
        if window_timing is not None:
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record()
        reduced = stats.setdefault("_reduced", []) if stats is not None and mixed else None
        propagate_device(Y, energies, dh.reduced_mass, halves, Wv[0::2], Wv[1::2], Wv[2::2], stride=(stride, stride, stride), precision=precision, reduced_out=reduced)
        if window_timing is not None:
            t1.record()
            window_timing.append((t0, t1, 2.0 * float(n) ** 3 * len(window) * energies.numel()))
        if stats is not None:
            blocks = -(-(2 * n if config.mode == "capture" else n) // 128)
            stats["sectors"] = stats.get("sectors", 0) + len(window)
            stats["sweep_steps"] = stats.get("sweep_steps", 0) + 2 * blocks * len(window)
        done += len(window)
        if config.print_verbose and (done == n_sector or done >= next_report):
            torch.cuda.synchronize(dev)
            logger.info(f"Propagation: {done}/{n_sector} sectors, R={window[-1].radial_end:.6f} bohr, wall={perf_counter() - started:.3f} s")
            while next_report <= done:
                next_report += interval
    if dh.position is not None:
        Y = Y[:, dh.position][:, :, dh.position].contiguous()
    return Y


# ---- several channel blocks (coupled states, NNCC) -------------------------------------------
DUMMY_P2 = 3600.0  # local wavenumber^2 (bohr^-2) of the closed channels that pad a smaller block
CLASS_WORKSPACE_SLOT = 16  # first workspace slot of the concurrently propagated size classes


class BlockState:
    """One channel block on a device, built once: rows (output positions inside the block),
    centrifugal matrix U and thresholds E_int in propagation order, and ``position`` (the
    propagated index of each block channel).  With ``closed_first`` the order is most-closed
    first (by W_ii at the outermost grid point), as for one exact-CC block."""

    def __init__(self, hamiltonian, block: tuple[int, ...], device: torch.device, closed_first: bool = False) -> None:
        grid = hamiltonian.potential_grid
        indices = np.asarray(block, dtype=np.int64)
        U = np.asarray(hamiltonian.centrifugal(block))
        E_int = np.asarray(hamiltonian.E_int)[indices]
        order = np.arange(indices.size)
        if closed_first:
            rows = device_rows(hamiltonian.V_basis, device, block)
            outer = grid.radial_points[-1:]
            index = torch.as_tensor(grid.selection(outer), device=device)
            W = contract_rows(rows, grid.device_values(device).index_select(0, index), radial_points=torch.as_tensor(outer, device=device),
                              U=torch.as_tensor(U, device=device), E_int=torch.as_tensor(E_int, device=device), reduced_mass=hamiltonian.reduced_mass)[0]
            order = np.argsort(-torch.diagonal(W).cpu().numpy(), kind="stable")
        self.hamiltonian = hamiltonian
        self.size = int(indices.size)
        self.rows = device_rows(hamiltonian.V_basis, device, tuple(int(c) for c in indices[order]))
        self.U = U[np.ix_(order, order)]
        self.E_int = E_int[order]
        position = np.empty_like(order)
        position[order] = np.arange(order.size)
        self.position = torch.as_tensor(position, device=device)


class DeviceBlocks:
    """Device-resident pieces of several channel blocks, padded to the largest block size n:
    per block its rows (output positions inside the block), its centrifugal matrix U and
    thresholds E_int.  ``entries`` lists (hamiltonian, channel indices) pairs: the K blocks of
    one Hamiltonian (coupled states, NNCC) or whole systems of a partial-wave sweep, which
    must share one PotentialGrid and reduced mass (or ``states``: prebuilt BlockStates, and
    ``n``: a padded size at least their largest).  Padding channels have no coupling, U = 0
    and a threshold set per call far above the highest energy, so they stay closed and
    decoupled.  With ``closed_first`` each block's channels are ordered most-closed first."""

    def __init__(self, entries, device: torch.device, closed_first: bool = False, *, states=None, n: int | None = None) -> None:
        if states is None:
            states = [BlockState(h, tuple(b), device, closed_first) for h, b in entries]
        first = states[0].hamiltonian
        self.grid = first.potential_grid
        self.values = self.grid.device_values(device)
        self.reduced_mass = first.reduced_mass
        if any(st.hamiltonian.potential_grid is not self.grid or st.hamiltonian.reduced_mass != self.reduced_mass for st in states):
            message = "Blocks propagated together must share one PotentialGrid and reduced mass"
            logger.error(message)
            raise ValueError(message)
        self.sizes = tuple(st.size for st in states)
        self.n = max(self.sizes) if n is None else int(n)
        if self.n < max(self.sizes):
            message = f"Padded block size {self.n} is below the largest block ({max(self.sizes)} channels)"
            logger.error(message)
            raise ValueError(message)
        self.rows, self.U, self.E_int, self.position = [], [], [], []
        for st in states:
            rows = copy(st.rows)
            rows.n_channel = self.n
            U_pad = np.zeros((self.n, self.n))
            U_pad[: st.size, : st.size] = st.U
            self.rows.append(rows)
            self.U.append(torch.as_tensor(U_pad, device=device))
            self.E_int.append(st.E_int)
            self.position.append(st.position)

    def _contract(self, rows, radial_points, U, E_int, out=None):
        dev = U.device
        index = torch.as_tensor(self.grid.selection(radial_points), device=dev)
        potential = self.values.index_select(0, index)
        R = torch.as_tensor(np.ascontiguousarray(radial_points), device=dev)
        return contract_rows(rows, potential, radial_points=R, U=U, E_int=E_int, reduced_mass=self.reduced_mass, out=out)

    def thresholds(self, energies: np.ndarray, device: torch.device) -> list[torch.Tensor]:
        """Per block E_int padded with the closed padding thresholds for these energies."""
        dummy = float(np.max(energies)) + DUMMY_P2 / (2.0 * self.reduced_mass)
        out = []
        for E_int in self.E_int:
            padded = np.full(self.n, dummy)
            padded[: E_int.size] = E_int
            out.append(torch.as_tensor(padded, device=device))
        return out

    def W_base(self, g: int, radial_points: np.ndarray, E_int: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        return self._contract(self.rows[g], radial_points, self.U[g], E_int, out=out)


def device_blocks(hamiltonian, blocks, device: torch.device, closed_first: bool = False) -> DeviceBlocks:
    return _device_state(hamiltonian, ("blocks", blocks, device.index, closed_first), lambda: DeviceBlocks([(hamiltonian, b) for b in blocks], device, closed_first))


def blocks_window(n_channel: int, n_block: int, n_sector: int) -> int:
    """Sectors per window so that every block's W points and Q_mid fit the window budget."""
    padded = -(-n_channel // 128) * 128
    per_sector = 8 * n_block * (2 * n_channel * n_channel + padded * padded)
    return max(1, min(n_sector, MAX_SECTORS_PER_WINDOW, WINDOW_BYTES // per_sector, 65535 // n_block))


def block_size_classes(blocks, mode: str) -> list[list[int]]:
    """Positions of the blocks grouped by the size of their sweep matrix, smallest first, so
    that no block is padded to a larger class: 64 rows (the 64-wide single-block sweep: 64
    real channels, or 32 complex ones in capture mode), then multiples of 128 rows."""
    rows = 2 if mode == "capture" else 1

    def size_class(b) -> int:
        m = rows * len(b)
        return 64 if m <= 64 else -(-m // 128) * 128

    keys = sorted({size_class(b) for b in blocks})
    return [[g for g, b in enumerate(blocks) if size_class(b) == key] for key in keys]


def propagate_blocks(hamiltonian, channel_blocks, Etot, radial_sectors: Sequence[RadialSector], config: Propagation, *, window_timing: list | None = None, workspace_slot: int = 0) -> tuple[torch.Tensor, ...]:
    """Y at the last sector end of every channel block, one (n_energy, n_b, n_b) device
    tensor per block (reference runner.py:165-322).  All blocks of a size class share each
    radial window and advance together in one batched LDMD call per window; the size
    classes run concurrently, each on its own CUDA stream (host thread), so that a small
    class fills the SMs a larger one leaves idle."""
    energies_np = get_Etot(Etot)
    blocks = tuple(tuple(int(i) for i in b) for b in channel_blocks)
    if not blocks or any(not b for b in blocks):
        message = "At least one non-empty channel block is required for propagation"
        logger.error(message)
        raise ValueError(message)
    if not radial_sectors:
        message = "Propagation produced no radial windows"
        logger.error(message)
        raise RuntimeError(message)
    classes = block_size_classes(blocks, config.mode)
    if len(classes) > 1:
        dev = resolve_device(config.device)
        main = torch.cuda.current_stream(dev)
        streams = [torch.cuda.Stream(dev) for _ in classes]

        def run(k: int):
            streams[k].wait_stream(main)
            with torch.cuda.device(dev), torch.cuda.stream(streams[k]):
                members = tuple(blocks[g] for g in classes[k])
                return propagate_blocks(hamiltonian, members, Etot, radial_sectors, config, window_timing=window_timing, workspace_slot=CLASS_WORKSPACE_SLOT + k)

        with ThreadPoolExecutor(max_workers=len(classes)) as pool:
            results = list(pool.map(run, range(len(classes))))
        out: list = [None] * len(blocks)
        for k, members in enumerate(classes):
            main.wait_stream(streams[k])
            for g, Y in zip(members, results[k], strict=True):
                Y.record_stream(main)  # made on the class's stream, used on the caller's
                out[g] = Y
        return tuple(out)
    dev = resolve_device(config.device)
    db = device_blocks(hamiltonian, blocks, dev, closed_first=True)
    n, n_block = db.n, len(blocks)
    energies = torch.as_tensor(np.array(energies_np), device=dev)
    E_pad = db.thresholds(energies_np, dev)
    n_sector = len(radial_sectors)
    size = blocks_window(n, n_block, n_sector)
    precision = nat.PRECISION_MIXED if config.precision == "mixed" else nat.PRECISION_FP64
    logger.info(f"Propagation device: gpu:{dev.index}, x64=True")
    if config.print_verbose:
        logger.info(f"Propagation started: blocks={n_block}, sectors={n_sector}, channels={max(db.sizes)}, energies={energies_np.size}, pes_prefetch=False")
    started = perf_counter()
    interval = max(1, ceil(n_sector / 10))
    next_report = interval
    points_max = 2 * size + 1
    W = torch.empty((n_block, points_max, n, n), dtype=torch.float64, device=dev)
    Y = None
    done = 0
    flops_per_unit = sum(2.0 * float(m) ** 3 for m in db.sizes)
    for s0 in range(0, n_sector, size):
        window = tuple(radial_sectors[s0 : s0 + size])
        points = radial_points_of(window)
        for g in range(n_block):
            db.W_base(g, points, E_pad[g], W[g, : points.size])
        if Y is None:
            Y = torch.stack([initial_logD(W[g, 0], energies, db.reduced_mass, config.mode) for g in range(n_block)]).contiguous()
        halves = torch.as_tensor(np.asarray([s.radial_half_step for s in window]), device=dev)
        stride = 2 * n * n
        if window_timing is not None:
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record()
        propagate_blocks_device(Y, energies, db.reduced_mass, halves, W[0, 0], W[0, 1], W[0, 2], stride=(stride, stride, stride), block_stride=points_max * n * n, precision=precision, workspace_slot=workspace_slot)
        if window_timing is not None:
            t1.record()
            window_timing.append((t0, t1, flops_per_unit * len(window) * energies.numel()))
        done += len(window)
        if config.print_verbose and (done == n_sector or done >= next_report):
            torch.cuda.synchronize(dev)
            logger.info(f"Propagation: {done}/{n_sector} sectors, R={window[-1].radial_end:.6f} bohr, wall={perf_counter() - started:.3f} s")
            while next_report <= done:
                next_report += interval
    out = []
    for g, size_g in enumerate(db.sizes):
        pos = db.position[g]
        out.append(Y[g, :, :size_g, :size_g][:, pos][:, :, pos].contiguous())
    return tuple(out)

