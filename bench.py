"""Benchmark: S-matrix solves/s for the vibrating A+BC coupled-channel workload.

Workload (synthetic, built by ``pyticc_b200.workloads.morse_atom_diatom``): Morse diatom
(De = 40000 cm^-1, re = 1.4, a = 1.2) in a 32-point sine DVR, v <= 3, j <= 30, J = 30, both
parities (N = 1984 / 1860 channels), cfg0-form PES with seeded r-dependent anisotropy,
32-point theta quadrature, LDMD from 2.5 to 40 bohr at h = 0.02 (938 sectors), 256 energies
uniform over 100-3000 cm^-1.  One step = one parity block x one batch of energies,
propagated through every sector and matched: it yields `batch` S matrices.  Steps cycle
over (parity, energy batch); every rank of a multi-GPU run owns different batches (weak
scaling, no collective on the data path).

Output: one JSON line on rank 0 (see the repository's benchmark contract).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "S-matrix solves/s on 1 B200: mixed+learned vs plain FP64 LogD at max|dS|<=1e-6"
STEP_KERNEL_DRAM_BYTES = 342_238_208 + 278_014_208  # ncu: one FP64 sweep step launch, 16 matrices of 2048^2
WORKLOAD = "vibrating A+BC exact CC: Morse diatom v<=3 j<=30, J=30, both parities (N=1984/1860), 938 LDMD sectors 2.5-40 bohr h=0.02, 256 energies 100-3000 cm^-1"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["native", "reference"], default="native")
    p.add_argument("--batch", type=int, default=32, help="energies per step (per solve call); 256 / batch batches per parity block")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="mixed", help="headline arm precision")
    p.add_argument("--schedule", choices=["fixed", "learned"], default="learned", help="headline arm sector schedule")
    p.add_argument("--plain-steps", type=int, default=None, help="timed steps of the plain FP64 fixed-step arm (default: steps - 1, at least 1)")
    p.add_argument("--sectors", type=int, default=0, help="limit sectors (0 = all 938); for quick checks only")
    p.add_argument("--approx", choices=["exact", "cs", "nncc"], default="exact", help="exact CC (the metric) or the coupled-states / NNCC (K_delta=1) blocks of the same system")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [line for line in out.splitlines() if line.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            parts = [x.strip() for x in line.split(",")]
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except (ValueError, IndexError):
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(args):
    import pyticc_b200 as tb
    from pyticc_b200 import workloads

    halves = (0.02,)
    bounds = (2.5, 40.0)
    blocks = []
    diatom = workloads.morse_diatom(**workloads.MORSE_DEFAULTS)
    approx = tb.Approx(getattr(args, "approx", "exact"))
    for parity in (1, -1):
        wl = workloads.morse_atom_diatom(parity=parity, diatom=diatom, boundaries=bounds, half_steps=halves, n_energy=256, approx=approx, K_delta=1)
        blocks.append(wl)
    return blocks


def units(blocks, batch, rank, world, count):
    """(block index, energy slice) for this rank's `count` steps (disjoint across ranks)."""
    from pyticc_b200.replicas import rank_units

    return [(u.block, slice(u.start, u.stop)) for u in rank_units(len(blocks), 256, batch, rank, world, count)]


def fp64_peak_tflops(torch, dev) -> float:
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(5):
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192**3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def cpu_baseline(block, batch_energies, sample_sectors: int = 6) -> dict:
    """Oracle (NumPy/LAPACK port of the reference) on a bounded sample: one energy through
    `sample_sectors` sectors, extrapolated linearly to all sectors and energies."""
    import torch

    from oracle import contraction, ldmd
    from pyticc_b200 import scattering

    wl = block
    ham = scattering.hamiltonian_for(wl.system, wl.grid)
    n = wl.system.basis.n_channel
    U = ham.U
    pts = 2 * sample_sectors + 1
    V = contraction.contract(ham.V_basis.channel_indices, ham.V_basis.B_real, None, 1.0, wl.grid.values.reshape(wl.grid.radial_points.size, -1)[:pts], n)
    W = contraction.assemble_W_base(wl.grid.radial_points[:pts], U, wl.system.basis.E_int, wl.system.reduced_mass, V)
    hs = np.asarray([s.radial_half_step for s in wl.grid.sectors[:sample_sectors]])
    E = np.asarray(batch_energies[:1])
    Y0 = ldmd.initialize_inelastic(W[0][None] - 2 * wl.system.reduced_mass * E[:, None, None] * np.eye(n))
    t0 = time.perf_counter()
    ldmd.propagate_logD(Y0, E, wl.system.reduced_mass, hs, W[0:-1:2], W[1::2], W[2::2])
    elapsed = time.perf_counter() - t0
    per_sector = elapsed / sample_sectors
    n_sector = len(wl.grid.sectors)
    solves_per_s = 1.0 / (per_sector * n_sector)
    return {
        "value": solves_per_s,
        "unit": "solves/s",
        "cores": torch.get_num_threads(),
        "kind": "port",
        "sample": f"1 energy x {sample_sectors} of {n_sector} sectors at N={n} ({elapsed:.1f} s), extrapolated linearly in sectors; NumPy/LAPACK LDMD restatement of the reference",
    }


def run_reference(args, rank, world):
    if rank != 0:
        return
    import torch

    torch.set_num_threads(os.cpu_count() or 1)
    blocks = build_workload(args)
    steps = []
    for k in range(args.warmup + args.steps):
        b = k % 2
        base = cpu_baseline(blocks[b], blocks[b].energies, sample_sectors=3)
        if k >= args.warmup:
            steps.append(base["value"])
    value = statistics.mean(steps)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch": 1, "precision": "fp64"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": torch.get_num_threads(), "kind": "port", "sample": "per step: 1 energy x 3 sectors of 938 at N=1984/1860, extrapolated linearly in sectors"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.approx != "exact":
        run_blocks(args, rank, world, local)
        return
    import torch

    import pyticc_b200 as tb
    from pyticc_b200 import _native as nat
    from pyticc_b200 import scattering
    from pyticc_b200.propagation import runner
    from pyticc_b200.propagation.learned import learned_sectors, resolve_proposer
    from pyticc_b200.replicas import max_over_ranks

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    group = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        group = dist
    lib = nat.load_library()
    blocks = build_workload(args)
    sectors_of = [b.grid.sectors if args.sectors == 0 else b.grid.sectors[: args.sectors] for b in blocks]
    proposer = resolve_proposer(None)
    headline = tb.Propagation(precision=args.precision)
    plain = tb.Propagation(precision="fp64")
    plain_steps = args.plain_steps if args.plain_steps is not None else max(1, args.steps - 1)
    n_total = args.warmup + args.steps
    plan = units(blocks, args.batch, rank, world, n_total)

    def one_step(block_index, energy_slice, config, schedule, timing_list=None, used=None):
        """One solve batch through the library's device path: schedule, propagate, match."""
        wl = blocks[block_index]
        ham = scattering.hamiltonian_for(wl.system, wl.grid)
        energies = wl.energies[energy_slice]
        sectors = sectors_of[block_index]
        if schedule == "learned":
            sectors = learned_sectors(ham, sectors, energies, proposer, "auto")
        if used is not None:
            used.append(len(sectors))
        Y = runner.propagate(ham, energies, sectors, config, window_timing=timing_list)
        B, L = tb.get_Bmat_BF_to_SF(wl.system.basis)
        Y_sf = tb.match.asymptotic.transform_device(Y, nat.as_device(B, dev, torch.float64))
        S, n_open = tb.match.smatrix.get_Smat_device(Y_sf, sectors[-1].radial_end, energies, ham.reduced_mass, wl.system.basis.E_int, L)
        return S, n_open

    def timed(config, schedule, steps, warmup, windows=None, used=None):
        for k in range(warmup):
            one_step(*plan[k], config, schedule)
        torch.cuda.synchronize()
        if group:
            group.barrier()
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        first = None
        start.record()
        for k in range(warmup, warmup + steps):
            out = one_step(*plan[k], config, schedule, timing_list=windows, used=used)
            first = out if first is None else first
        stop.record()
        torch.cuda.synchronize()
        if group:
            group.barrier()
        return max_over_ranks(start.elapsed_time(stop) * 1e-3, group), first

    # headline arm: mixed precision + learned sector widths (warm-up also builds the
    # Hamiltonian rows and device PES grids)
    launches0 = None
    windows: list = []
    used: list = []
    for k in range(args.warmup):
        one_step(*plan[k], headline, args.schedule)
    torch.cuda.synchronize()
    launches0 = lib.ticc_kernel_launches()
    with ClockSampler(local) as clocks:
        elapsed, head_first = timed(headline, args.schedule, args.steps, 0, windows, used)
    launches = lib.ticc_kernel_launches() - launches0
    solves = args.steps * args.batch * world
    value = solves / elapsed
    # plain FP64 fixed-step arm on the same first units (its kernels are warm)
    plain_elapsed, plain_first = timed(plain, "fixed", plain_steps, 0)
    plain_value = plain_steps * args.batch * world / plain_elapsed

    # roofline: the LDMD propagate launches (window x energy batch), two symmetric
    # N x N inversions (N^3 flops each) per (sector, energy)
    prop_seconds = sum(a.elapsed_time(b) * 1e-3 for a, b, _ in windows)
    prop_flops = sum(f for _, _, f in windows)
    peak = fp64_peak_tflops(torch, dev) if rank == 0 else 0.0

    # accuracy of the headline arm against plain FP64 fixed step on the first timed unit
    S_h, n_h = head_first
    S_p, n_p = plain_first
    counts_equal = bool(np.array_equal(np.asarray(n_h), np.asarray(n_p)))
    max_dS = float((S_h - S_p).abs().max().item())

    # end-to-end through the public API: host energies in, host S and Y out, fresh device PES copy
    e2e_value = None
    h2d = d2h = 0
    cpu = None
    if rank == 0:
        wl = blocks[plan[args.warmup][0]]
        energies = np.ascontiguousarray(wl.energies[plan[args.warmup][1]])
        wl.grid._device_cache.clear()
        runner._DEVICE_HAMILTONIANS.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_config = tb.Propagation(precision=args.precision, steps=args.schedule)
        result = tb.solve(wl.system, energies, wl.grid, e2e_config, sectors=None if args.sectors == 0 else sectors_of[plan[args.warmup][0]])
        e2e_seconds = time.perf_counter() - t0
        e2e_value = len(energies) / e2e_seconds
        h2d = int(energies.nbytes + wl.grid.values.nbytes)
        d2h = int(result.Y_propagated.nbytes + sum(x.nbytes for x in result.Smat))
        cpu = cpu_baseline(wl, energies)
    if group:
        group.barrier()
        group.destroy_process_group()
    if rank != 0:
        return
    n_channel = blocks[0].system.basis.n_channel
    achieved = prop_flops / prop_seconds / 1e12 if prop_seconds else None
    n_fixed = len(sectors_of[0])
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f64+tf32x3",
        "data": "synthetic",
        "config": {
            "workload": WORKLOAD,
            "batch": args.batch,
            "precision": args.precision,
            "schedule": args.schedule,
            "sectors_fixed": n_fixed,
            "sectors_used_per_step": used,
            "l2": "inputs larger than L2 (per-energy work matrices 32 MiB each, W windows > 1 GiB)",
        },
        "plain_fp64": {"value": plain_value, "unit": "solves/s", "steps": plain_steps, "ms_per_step": plain_elapsed / plain_steps * 1e3, "schedule": "fixed h=0.02",
                       "speedup_of_value": value / plain_value},
        "accuracy": {"max_dS_vs_plain_fp64": max_dS, "open_counts_equal": counts_equal, "tolerance": 1e-6, "energies": args.batch},
        "roofline": {
            "bound": "tensor",
            "achieved": achieved,
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": achieved / peak if achieved and peak else None,
            # DRAM bytes per launch of the dominant kernel (sweep_step_kernel, one sweep step of
            # 16 matrices of 2048^2) from one ncu capture; the algorithmic bytes are 595 MB
            "traffic": STEP_KERNEL_DRAM_BYTES * args.batch / 16,
            "traffic_note": f"dram__bytes_read.sum + dram__bytes_write.sum of one sweep_step_kernel launch from an ncu capture of 16 matrices of 2048^2 (342 + 278 MB, algorithmic 595 MB), scaled to the {args.batch} matrices of a launch here (the traffic is per matrix)",
            "kernel": "ticc_ldmd_propagate of the headline arm (batched symmetric sweeps; FP64 DMMA, TF32x3 on strongly closed blocks in mixed precision); peak = cuBLAS DGEMM 8192^3 measured in this run (no measured FP64 peak is supplied)",
            "flops_per_unit": f"2 N^3 per (sector, energy), N={n_channel}, counted in FP64-equivalent flops",
        },
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def run_blocks(args, rank, world, local):
    """Coupled-states or NNCC solves of the benchmark system: every K block of one parity
    block propagated together (one batched LDMD call per window) and matched per block."""
    import torch

    import pyticc_b200 as tb
    from oracle import contraction, ldmd
    from pyticc_b200 import _native as nat
    from pyticc_b200 import scattering
    from pyticc_b200.propagation import runner
    from pyticc_b200.replicas import max_over_ranks

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    group = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        group = dist
    lib = nat.load_library()
    blocks = build_workload(args)
    sectors_of = [b.grid.sectors if args.sectors == 0 else b.grid.sectors[: args.sectors] for b in blocks]
    config = tb.Propagation(precision="fp64")
    plan = units(blocks, args.batch, rank, world, args.warmup + args.steps)
    k_blocks = [scattering.build_k_blocks(scattering.hamiltonian_for(b.system, b.grid)) for b in blocks]

    def one_step(block_index, energy_slice, windows=None):
        wl = blocks[block_index]
        ham = scattering.hamiltonian_for(wl.system, wl.grid)
        energies = wl.energies[energy_slice]
        sectors = sectors_of[block_index]
        kb = k_blocks[block_index]
        # the size classes run concurrently on their own streams, so the roofline takes the
        # whole propagation on the caller's stream (after the join), not the sum of windows
        inner = None if windows is None else []
        if windows is not None:
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record()
        Ys = runner.propagate_blocks(ham, tuple(b.channel_indices for b in kb), energies, sectors, config, window_timing=inner)
        if windows is not None:
            t1.record()
            windows.append((t0, t1, sum(f for _, _, f in inner)))
        return [scattering.finalize_K_block(wl.system.basis, b, Y, energies, ham.reduced_mass, sectors[-1].radial_end, approx=wl.system.approx) for b, Y in zip(kb, Ys, strict=True)]

    for k in range(args.warmup):
        one_step(*plan[k])
    torch.cuda.synchronize()
    if group:
        group.barrier()
    launches0 = lib.ticc_kernel_launches()
    windows: list = []
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record()
        for k in range(args.warmup, args.warmup + args.steps):
            one_step(*plan[k], windows)
        stop.record()
        torch.cuda.synchronize()
    launches = lib.ticc_kernel_launches() - launches0
    elapsed = max_over_ranks(start.elapsed_time(stop) * 1e-3, group)
    value = args.steps * args.batch * world / elapsed
    prop_seconds = sum(a.elapsed_time(b) * 1e-3 for a, b, _ in windows)
    prop_flops = sum(f for _, _, f in windows)
    peak = fp64_peak_tflops(torch, dev) if rank == 0 else 0.0
    e2e_value, h2d, d2h, cpu = None, 0, 0, None
    if rank == 0:
        wl = blocks[plan[args.warmup][0]]
        energies = np.ascontiguousarray(wl.energies[plan[args.warmup][1]])
        wl.grid._device_cache.clear()
        runner._DEVICE_BLOCKS.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        result = tb.solve(wl.system, energies, wl.grid, config)
        e2e_seconds = time.perf_counter() - t0
        e2e_value = len(energies) / e2e_seconds
        h2d = int(energies.nbytes + wl.grid.values.nbytes)
        d2h = int(sum(b.Y_BF.nbytes + sum(x.nbytes for x in b.Smat_asymptotic) for b in result.blocks))
        # oracle: one energy through 4 sectors for every block, extrapolated in sectors
        ham = scattering.hamiltonian_for(wl.system, wl.grid)
        U = ham.U
        pts, n_s = 9, 4
        values = wl.grid.values.reshape(wl.grid.radial_points.size, -1)[:pts]
        hs = np.asarray([s.radial_half_step for s in wl.grid.sectors[:n_s]])
        E = energies[:1]
        t0 = time.perf_counter()
        for b in k_blocks[plan[args.warmup][0]]:
            idx = list(b.channel_indices)
            V = contraction.contract(ham.V_basis.channel_indices, ham.V_basis.B_real, None, 1.0, values, len(idx), idx)
            W = contraction.assemble_W_base(wl.grid.radial_points[:pts], U[np.ix_(idx, idx)], wl.system.basis.E_int[idx], wl.system.reduced_mass, V)
            Y0 = ldmd.initialize_inelastic(W[0][None] - 2 * wl.system.reduced_mass * E[:, None, None] * np.eye(len(idx)))
            ldmd.propagate_logD(Y0, E, wl.system.reduced_mass, hs, W[0:-1:2], W[1::2], W[2::2])
        cpu_s = time.perf_counter() - t0
        cpu = {"value": 1.0 / (cpu_s / n_s * len(wl.grid.sectors)), "unit": "solves/s", "cores": torch.get_num_threads(), "kind": "port",
               "sample": f"1 energy x {n_s} of {len(wl.grid.sectors)} sectors for all {len(k_blocks[0])} blocks ({cpu_s:.1f} s), extrapolated linearly in sectors; NumPy/LAPACK LDMD restatement of the reference"}
    if group:
        group.barrier()
        group.destroy_process_group()
    if rank != 0:
        return
    sizes = [len(b.channel_indices) for b in k_blocks[0]]
    achieved = prop_flops / prop_seconds / 1e12 if prop_seconds else None
    line = {
        "metric": f"{args.approx.upper()} S-matrix solves/s on 1 B200 (one solve = every K block of one (J, parity) block at one energy)",
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD.replace("exact CC", f"{args.approx.upper()} blocks (K_delta=1)" if args.approx == "nncc" else "CS blocks"), "batch": args.batch,
                   "blocks": len(sizes), "block_channels": [min(sizes), max(sizes)], "sectors": len(sectors_of[0]), "l2": "inputs larger than L2 (W windows of every block > 1 GiB)"},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if achieved and peak else None, "traffic": None,
                     "kernel": "ticc_ldmd_propagate_blocks (all K blocks batched; pivot-block inversions dominate for blocks of <= 128 channels)",
                     "flops_per_unit": "sum over blocks of 2 n_b^3 per (sector, energy)"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
