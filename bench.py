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
    p.add_argument("--config", choices=["vibrating", "sweep", "capture"], default="vibrating",
                   help="vibrating: the headline J=30 blocks; sweep: the batched partial-wave sweep of the same system; capture: the ultracold capture system with learned widths")
    p.add_argument("--sweep-J-step", type=int, default=12, help="sweep: every n-th J of 0..60 (1 = all 61)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region, written to a temporary file
    (a pipe read only at the end fills up and stalls the sampler)."""

    QUERY = "timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        import tempfile

        self.file = tempfile.TemporaryFile(mode="w+")
        self.started = time.perf_counter()
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.span = time.perf_counter() - self.started
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
        self.file.seek(0)
        self.lines = [line for line in self.file.read().splitlines() if line.strip()]
        self.file.close()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except (ValueError, IndexError):
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm), "sampled_s": round(getattr(self, "span", 0.0), 1)}


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


def _best_gemm_tflops(torch, dev, dtype, allow_tf32=False) -> float:
    previous = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = allow_tf32
    try:
        a = torch.randn(8192, 8192, dtype=dtype, device=dev)
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
    finally:
        torch.backends.cuda.matmul.allow_tf32 = previous


def blas_threads() -> int:
    from threadpoolctl import threadpool_info

    counts = [info["num_threads"] for info in threadpool_info() if info.get("user_api") == "blas"]
    return max(counts) if counts else 1


def cpu_sample(block, energies_all, n_energy: int = 4, sample_sectors: int = 3) -> dict:
    """The oracle (the reference's NumPy/LAPACK algorithm, restated) on a bounded sample of
    the workload, charged per solve the way the reference spends it: per-energy sector
    updates (``n_energy`` energies through ``sample_sectors`` sectors), the energy-shared
    Q_mid corrections and the V(R) contraction amortised over the block's 256 energies (the
    reference solves all energies of a block in one call, logd.py:305-310), and one
    energy's BF -> SF transform and matching.  Extrapolated linearly in sectors."""
    from threadpoolctl import threadpool_limits

    import pyticc_b200 as tb
    from oracle import contraction, ldmd, matching
    from pyticc_b200 import scattering

    wl = block
    ham = scattering.hamiltonian_for(wl.system, wl.grid)
    basis = wl.system.basis
    n = basis.n_channel
    mu = wl.system.reduced_mass
    pts = 2 * sample_sectors + 1
    n_sector = len(wl.grid.sectors)
    n_points = wl.grid.radial_points.size
    E = np.asarray(energies_all[np.linspace(0, len(energies_all) - 1, n_energy).astype(int)])
    cores = os.cpu_count() or 1
    with threadpool_limits(cores, user_api="blas"):
        threads = blas_threads()
        t0 = time.perf_counter()
        V = contraction.contract(ham.V_basis.channel_indices, ham.V_basis.B_real, None, 1.0, wl.grid.values.reshape(n_points, -1)[:pts], n)
        W = contraction.assemble_W_base(wl.grid.radial_points[:pts], ham.U, basis.E_int, mu, V)
        t_contract = time.perf_counter() - t0
        hs = [s.radial_half_step for s in wl.grid.sectors[:sample_sectors]]
        t0 = time.perf_counter()
        corrections = [ldmd.correction_matrices(h, W[2 * s], W[2 * s + 1], W[2 * s + 2]) for s, h in enumerate(hs)]
        t_corr = time.perf_counter() - t0
        Y = ldmd.initialize_inelastic(W[0][None] - 2 * mu * E[:, None, None] * np.eye(n))
        t0 = time.perf_counter()
        for e in range(E.size):
            for h, (ref, Qs, Qm, Qe) in zip(hs, corrections, strict=True):
                Y[e] = ldmd.propagate_with_corrections(Y[e], h, ref - 2.0 * mu * E[e], Qs, Qm, Qe)
        t_prop = time.perf_counter() - t0
        B, L = tb.get_Bmat_BF_to_SF(basis)
        t0 = time.perf_counter()
        Y_sf = matching.transform_bf_to_sf(Y[-1:], B)
        matching.get_Smat(Y_sf, wl.grid.sectors[-1].radial_end, E[-1:], mu, basis.E_int, L)
        t_match = time.perf_counter() - t0
    per_solve = (t_prop / (E.size * sample_sectors) + t_corr / (sample_sectors * 256)) * n_sector + t_contract / pts * n_points / 256 + t_match
    wall = t_contract + t_corr + t_prop + t_match
    return {
        "value": 1.0 / per_solve,
        "unit": "solves/s",
        "cores": threads,
        "kind": "port",
        "wall_s": wall,
        "sample": (f"N={n}: {E.size} energies x {sample_sectors} of {n_sector} sectors ({t_prop:.1f} s), Q_mid corrections of those sectors ({t_corr:.1f} s) and "
                   f"V(R) at {pts} of {n_points} points ({t_contract:.1f} s) amortised over the block's 256 energies, one energy's transform and matching ({t_match:.1f} s); "
                   f"extrapolated linearly in sectors; NumPy/LAPACK LDMD restatement of the reference, {threads} BLAS threads"),
    }


def run_reference(args, rank, world):
    """The reference's CPU algorithm (oracle port) on the host cores: every step is one
    bounded sample of the workload (alternating parity blocks); ms_per_step is that
    sample's measured wall time and value its extrapolated solves/s."""
    if rank != 0:
        return
    blocks = build_workload(args)
    rates, walls = [], []
    sample = None
    for k in range(args.warmup + args.steps):
        b = k % 2
        sample = cpu_sample(blocks[b], blocks[b].energies)
        if k >= args.warmup:
            rates.append(sample["value"])
            walls.append(sample["wall_s"])
    value = statistics.mean(rates)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": statistics.mean(walls) * 1e3,
        "ms_per_step_note": "measured wall time of one step's bounded CPU sample; value is that sample's cost extrapolated to whole solves",
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch": 1, "precision": "fp64", "extrapolated": True},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": sample["cores"], "kind": "port", "sample": "per step: " + sample["sample"]},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_fixtures() -> list[tuple[int, dict]]:
    """The reference's own S at full size for two benchmark energies per parity block
    (tests/golden/full_morse_J30_p+/-.npz, made by tests/golden/make_golden.py)."""
    out = []
    for b, tag in enumerate("+-"):
        path = ROOT / "tests" / "golden" / f"full_morse_J30_p{tag}.npz"
        if path.exists():
            data = np.load(path)
            out.append((b, {"energy_indices": json.loads(str(data["params_json"]))["energy_indices"], "Smat": data["Smat"], "n_open": data["n_open"], "file": path.name}))
    return out


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.approx != "exact":
        run_blocks(args, rank, world, local)
        return
    if args.config == "sweep":
        run_sweep(args, rank, world, local)
        return
    if args.config == "capture":
        run_capture(args, rank, world, local)
        return
    import torch

    import pyticc_b200 as tb
    from pyticc_b200 import _native as nat
    from pyticc_b200 import scattering
    from pyticc_b200.propagation import runner
    from pyticc_b200.propagation.learned import judged_learned_sectors
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
    headline = tb.Propagation(precision=args.precision, steps=args.schedule)
    plain = tb.Propagation(precision="fp64")
    plain_steps = args.plain_steps if args.plain_steps is not None else max(1, args.steps - 1)
    n_total = args.warmup + args.steps
    plan = units(blocks, args.batch, rank, world, n_total)
    B_dev = [nat.as_device(tb.get_Bmat_BF_to_SF(b.system.basis)[0], dev, torch.float64) for b in blocks]
    L_of = [tb.get_Bmat_BF_to_SF(b.system.basis)[1] for b in blocks]

    def one_step(block_index, energy_slice, config, timing_list=None, used=None, stats=None):
        """One solve batch through the library's device path: the learned schedule (judged
        against the fixed step inside solve's logic), propagation and matching.  Returns the
        open-open corners of S (device) and the open counts."""
        wl = blocks[block_index]
        ham = scattering.hamiltonian_for(wl.system, wl.grid)
        energies = wl.energies[energy_slice]
        sectors = sectors_of[block_index]
        if config.steps == "learned" and args.sectors == 0:
            sectors, _ = judged_learned_sectors(wl.system, wl.grid, energies, config)
        if used is not None:
            used.append(len(sectors))
        Y = runner.propagate(ham, energies, sectors, config, window_timing=timing_list, stats=stats)
        Y_sf = tb.match.asymptotic.transform_device(Y, B_dev[block_index])
        S, n_open = tb.match.smatrix.get_Smat_device(Y_sf, sectors[-1].radial_end, energies, ham.reduced_mass, wl.system.basis.E_int, L_of[block_index])
        m = int(np.count_nonzero(wl.system.basis.E_int < energies.max()))
        return S[:, :m, :m].clone(), n_open

    def timed(config, steps, windows=None, used=None, stats=None):
        torch.cuda.synchronize()
        if group:
            group.barrier()
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        outs = []
        start.record()
        for k in range(args.warmup, args.warmup + steps):
            outs.append(one_step(*plan[k], config, timing_list=windows, used=used, stats=stats))
        stop.record()
        torch.cuda.synchronize()
        if group:
            group.barrier()
        return max_over_ranks(start.elapsed_time(stop) * 1e-3, group), outs

    # headline arm (warm-up also builds the Hamiltonian rows, device PES grids and judge verdicts)
    for k in range(args.warmup):
        one_step(*plan[k], headline)
    torch.cuda.synchronize()
    launches0 = lib.ticc_kernel_launches()
    windows: list = []
    used: list = []
    head_stats: dict = {}
    with ClockSampler(local) as clocks:
        elapsed, head_out = timed(headline, args.steps, windows, used, head_stats)
    launches = lib.ticc_kernel_launches() - launches0
    runner.finish_stats(head_stats)
    value = args.steps * args.batch * world / elapsed
    # plain FP64 fixed-step arm on the same units (its kernels are warm)
    plain_windows: list = []
    plain_elapsed, plain_out = timed(plain, plain_steps, plain_windows)
    plain_value = plain_steps * args.batch * world / plain_elapsed

    # every headline S against the plain FP64 S of the same unit, and its unitarity defect
    per_S_dS, per_S_unitarity, counts_equal = [], [], True
    for k, ((S_h, n_h), out_p) in enumerate(zip(head_out, plain_out + [None] * (len(head_out) - len(plain_out)))):
        n_h = np.asarray(n_h)
        S_h = S_h.cpu().numpy()
        if out_p is not None:
            S_p, n_p = out_p[0].cpu().numpy(), np.asarray(out_p[1])
            counts_equal &= bool(np.array_equal(n_h, n_p))
        for e, m in enumerate(n_h):
            s = S_h[e, :m, :m]
            per_S_unitarity.append(float(np.abs(s.conj().T @ s - np.eye(m)).max()) if m else 0.0)
            if out_p is not None and m:
                per_S_dS.append(float(np.abs(s - S_p[e, :m, :m]).max()))

    # accuracy against the reference's own S at full size (both arms, untimed)
    accuracy = {"tolerance": 1e-6, "fp64_tolerance": 1e-8, "max_dS_vs_plain_fp64_per_S": {"max": max(per_S_dS, default=None), "compared": len(per_S_dS)},
                "unitarity_defect_per_S": {"max": max(per_S_unitarity, default=None), "count": len(per_S_unitarity)}, "open_counts_equal": counts_equal}
    if rank == 0 and args.sectors == 0:
        ref = {}
        for b, fixture in reference_fixtures():
            idx = np.asarray(fixture["energy_indices"])
            for name, config in (("headline", headline), ("plain_fp64", plain)):
                S, n_open = one_step(b, idx, config)
                S, n_open = S.cpu().numpy(), np.asarray(n_open)
                worst = max(float(np.abs(S[e, :m, :m] - fixture["Smat"][e, :m, :m]).max()) for e, m in enumerate(n_open) if m)
                entry = ref.setdefault(name, {"max_dS": 0.0, "open_counts_equal": True, "fixtures": []})
                entry["max_dS"] = max(entry["max_dS"], worst)
                entry["open_counts_equal"] &= bool(np.array_equal(n_open, fixture["n_open"]))
                entry["fixtures"].append(fixture["file"])
        accuracy["vs_reference_full_size"] = ref

    # roofline: the LDMD propagate launches (window x energy batch), two symmetric
    # N x N inversions (N^3 flops each) per (sector, energy), FP64-equivalent
    def achieved(win):
        seconds = sum(a.elapsed_time(b) * 1e-3 for a, b, _ in win)
        return sum(f for _, _, f in win) / seconds / 1e12 if seconds else None

    peak = _best_gemm_tflops(torch, dev, torch.float64) if rank == 0 else 0.0
    tf32 = _best_gemm_tflops(torch, dev, torch.float32, allow_tf32=True) if rank == 0 else 0.0
    head_achieved, plain_achieved = achieved(windows), achieved(plain_windows)
    reduced_fraction = head_stats.get("reduced_steps", 0) / head_stats["sweep_steps"] if head_stats.get("sweep_steps") else 0.0
    # the headline's ceiling: FP64 steps at the DGEMM rate, reduced steps at a third of the
    # TF32 GEMM rate (three TF32 products per FP64-equivalent product)
    mixed_peak = 1.0 / ((1.0 - reduced_fraction) / peak + reduced_fraction / (tf32 / 3.0)) if peak and tf32 else None
    head_peak = mixed_peak if args.precision == "mixed" else peak

    # end-to-end through the public API: host energies in, host S and Y out, fresh device PES copy
    e2e_value = None
    h2d = d2h = 0
    cpu = None
    if rank == 0:
        wl = blocks[plan[args.warmup][0]]
        energies = np.ascontiguousarray(wl.energies[plan[args.warmup][1]])
        wl.grid._device_cache.clear()
        runner.release_device_state(scattering.hamiltonian_for(wl.system, wl.grid))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        result = tb.solve(wl.system, energies, wl.grid, headline, sectors=None if args.sectors == 0 else sectors_of[plan[args.warmup][0]])
        e2e_seconds = time.perf_counter() - t0
        e2e_value = len(energies) / e2e_seconds
        h2d = int(energies.nbytes + wl.grid.values.nbytes)
        d2h = int(result.Y_propagated.nbytes + sum(x.nbytes for x in result.Smat))
        cpu = cpu_sample(wl, wl.energies)
        cpu.pop("wall_s")
    if group:
        group.barrier()
        group.destroy_process_group()
    if rank != 0:
        return
    n_channel = blocks[0].system.basis.n_channel
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
            "reduced_sweep_steps": {"reduced": head_stats.get("reduced_steps", 0), "of": head_stats.get("sweep_steps", 0)},
            "l2": "inputs larger than L2 (per-energy work matrices 32 MiB each, W windows > 1 GiB)",
        },
        "plain_fp64": {
            "value": plain_value, "unit": "solves/s", "steps": plain_steps, "ms_per_step": plain_elapsed / plain_steps * 1e3, "schedule": "fixed h=0.02",
            "speedup_of_value": value / plain_value,
            "roofline": {"bound": "tensor", "achieved": plain_achieved, "peak": peak, "unit": "TFLOP/s", "frac": plain_achieved / peak if plain_achieved and peak else None,
                         "peak_note": "cuBLAS DGEMM 8192^3 measured in this run"},
        },
        "accuracy": accuracy,
        "roofline": {
            "bound": "tensor",
            "achieved": head_achieved,
            "peak": head_peak,
            "unit": "TFLOP/s",
            "frac": head_achieved / head_peak if head_achieved and head_peak else None,
            # DRAM bytes per launch of the dominant kernel (sweep_step_kernel, one sweep step of
            # 16 matrices of 2048^2) from one ncu capture; the algorithmic bytes are 595 MB
            "traffic": STEP_KERNEL_DRAM_BYTES * args.batch / 16,
            "traffic_note": f"dram__bytes_read.sum + dram__bytes_write.sum of one sweep_step_kernel launch from an ncu capture of 16 matrices of 2048^2 (342 + 278 MB, algorithmic 595 MB), scaled to the {args.batch} matrices of a launch here (the traffic is per matrix)",
            "kernel": "ticc_ldmd_propagate of the headline arm (batched symmetric sweeps; FP64 DMMA, TF32x3 on strongly closed blocks in mixed precision)",
            "peak_note": (f"measured in this run: cuBLAS DGEMM {peak:.1f} TF/s for the FP64 steps, cuBLAS TF32 GEMM {tf32:.0f} TF/s / 3 for the {reduced_fraction:.1%} of sweep steps "
                          "that take the TF32x3 product (harmonic mix by step count)") if args.precision == "mixed" else "cuBLAS DGEMM 8192^3 measured in this run",
            "flops_per_unit": f"2 N^3 per (sector, energy), N={n_channel}, counted in FP64-equivalent flops",
        },
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def _timed_loop(torch, fn, steps):
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    outs = [fn(k) for k in range(steps)]
    stop.record()
    torch.cuda.synchronize()
    return start.elapsed_time(stop) * 1e-3, outs


def run_sweep(args, rank, world, local):
    """The batched partial-wave sweep of the vibrating A+BC system: J = 0..60 (every
    --sweep-J-step-th), both parities, 64 energies log-uniform over 1-3000 cm^-1 per block,
    --batch of them per step (one step = every block at one energy batch); all blocks in one
    CUDA graph (first run direct, then replays).  Headline: mixed precision; then plain FP64."""
    import torch

    import pyticc_b200 as tb
    from pyticc_b200 import _native as nat
    from pyticc_b200 import workloads
    from pyticc_b200.replicas import max_over_ranks

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = nat.load_library()
    diatom = workloads.morse_diatom(**workloads.MORSE_DEFAULTS)
    base = workloads.morse_atom_diatom(parity=1, diatom=diatom, n_energy=1)
    Js = list(range(0, 61, max(1, args.sweep_J_step)))
    pes = base.system.potential
    systems = [tb.build_ScattSystem(tb.AtomSpec(), diatom, Jtot=J, system_parity=p, potential=pes, reduced_mass=base.system.reduced_mass) for J in Js for p in (1, -1)]
    energies_all = np.geomspace(1.0, 3000.0, 64) * tb.CM2AU
    batch = min(args.batch, 64)
    batches = [energies_all[(np.arange(batch) * (64 // batch) + k) % 64] for k in range(64 // batch)]
    sizes = [s.basis.n_channel for s in systems]
    flops_per_energy = sum(2.0 * n**3 for n in sizes) * len(base.grid.sectors)
    from pyticc_b200.match.asymptotic import get_Bmat_BF_to_SF
    from pyticc_b200.scattering import _match

    BL = [get_Bmat_BF_to_SF(s.basis) if s.basis.n_channel else None for s in systems]
    Rmatch = base.grid.sectors[-1].radial_end

    def matched(Ys, E):
        return [None if Y is None else _match(Y, BL[i][0], BL[i][1], systems[i].basis.E_int, Rmatch, E, float(systems[i].reduced_mass)) for i, Y in enumerate(Ys)]

    arms = {}
    for precision in ("mixed", "fp64"):
        config = tb.Propagation(precision=precision)
        sweep = tb.PartialWaveSweep(systems, base.grid, config, n_energy=batch, energy_bound=float(energies_all.max()), graph=True)
        for k in range(args.warmup):
            sweep.propagate(batches[k % len(batches)])  # the first run also captures the graph
        launches0 = lib.ticc_kernel_launches()

        def step(k, sweep=sweep):
            E = batches[(args.warmup + k) % len(batches)]
            return matched(sweep.propagate(E), E)

        with ClockSampler(local) as clocks:
            elapsed, outs = _timed_loop(torch, step, args.steps)
        elapsed = max_over_ranks(elapsed, None)
        # kernels inside graph replays do not pass the library's launch counter: add the
        # captured launches once per replay
        launches = lib.ticc_kernel_launches() - launches0 + args.steps * sweep.graph_launches
        arms[precision] = {"seconds": elapsed, "launches": launches, "clocks": clocks.summary(), "S": outs[0], "sweep": sweep}
    n_solves = sum(1 for n in sizes if n) * batch * args.steps
    head, plain = arms["mixed"], arms["fp64"]
    value = n_solves / head["seconds"]
    plain_value = n_solves / plain["seconds"]
    # accuracy: the first timed batch in both arms, every S
    worst, defect = 0.0, 0.0
    for Sh, Sp in zip(head["S"], plain["S"], strict=True):
        if Sh is None:
            continue
        for a, b in zip(Sh, Sp, strict=True):
            if a.size:
                worst = max(worst, float(np.abs(a - b).max()))
                defect = max(defect, float(np.abs(a.conj().T @ a - np.eye(a.shape[0])).max()))
    peak = _best_gemm_tflops(torch, dev, torch.float64)
    achieved = flops_per_energy * batch * args.steps / head["seconds"] / 1e12
    plain_achieved = flops_per_energy * batch * args.steps / plain["seconds"] / 1e12
    line = {
        "metric": "S-matrix solves/s on 1 B200, batched partial-wave sweep (one solve = one (J, parity) block at one energy)",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": head["seconds"] / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64+tf32x3", "data": "synthetic",
        "config": {"workload": f"vibrating A+BC sweep: Morse diatom v<=3 j<=30, J in {Js[0]}..{Js[-1]} step {Js[1] - Js[0] if len(Js) > 1 else 1}, both parities ({len(systems)} blocks, {sum(1 for n in sizes if not n)} empty, N {min(n for n in sizes if n)}-{max(sizes)}), 938 sectors, 64 energies log-uniform 1-3000 cm^-1",
                   "batch": batch, "launches": len(head["sweep"].launches), "classes_merged": sorted(k for k, v in head["sweep"].merges.items() if v), "graph": True,
                   "l2": "inputs larger than L2 (work matrices of the large blocks 32 MiB each per energy)"},
        "plain_fp64": {"value": plain_value, "ms_per_step": plain["seconds"] / args.steps * 1e3, "speedup_of_value": value / plain_value,
                       "roofline": {"bound": "tensor", "achieved": plain_achieved, "peak": peak, "unit": "TFLOP/s", "frac": plain_achieved / peak}},
        "accuracy": {"max_dS_vs_plain_fp64": worst, "unitarity_defect_max": defect, "tolerance": 1e-6, "energies": batch},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_note": "cuBLAS DGEMM measured in this run; flops are FP64-equivalent (sum over blocks of 2 N^3 per (sector, energy))"},
        "e2e": None,
        "gpu_launches": int(head["launches"]),
        "clocks": head["clocks"],
    }
    print(json.dumps(line), flush=True)


def run_capture(args, rank, world, local):
    """The ultracold capture system (rigid rotor B=0.03 cm^-1, j<=40, capture boundary at 8
    bohr, fixed step h=0.05 to 1500 bohr) at J = 0, 5, 10 with energies log-uniform over
    1 uK-1 mK, --batch per step: learned sector widths (judged inside solve) against the fixed
    grid, both timed; accuracy against the reference's full-size S at J = 0 and J = 10."""
    import torch

    import pyticc_b200 as tb
    from pyticc_b200 import _native as nat
    from pyticc_b200 import workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = nat.load_library()
    Js = (0, 5, 10)
    blocks = [workloads.ultracold_capture(J=J, n_energy=512) for J in Js]
    batch = min(args.batch, 512)
    arms = {}
    span = (min(float(wl.energies.min()) for wl in blocks), max(float(wl.energies.max()) for wl in blocks))
    for steps_kind in ("learned", "fixed"):
        # the learned schedule is built and judged once for the whole energy range
        config = tb.Propagation(mode="capture", precision="mixed", steps=steps_kind, learned_range=span if steps_kind == "learned" else None)
        used: list = []

        def step(k, config=config, used=used):
            out = []
            for wl in blocks:
                E = wl.energies[(np.arange(batch) * (512 // batch) + k) % 512]
                stats: dict = {}
                out.append(tb.solve(wl.system, E, wl.grid, config, stats=stats))
                used.append(stats.get("sectors"))
            return out

        for k in range(args.warmup):
            step(k)
        used.clear()
        launches0 = lib.ticc_kernel_launches()
        with ClockSampler(local) as clocks:
            elapsed, _ = _timed_loop(torch, lambda k: step(args.warmup + k), args.steps)
        arms[steps_kind] = {"seconds": elapsed, "sectors": list(used), "launches": lib.ticc_kernel_launches() - launches0, "clocks": clocks.summary()}
    accuracy = {}
    for J, name in ((0, "full_capture_J0.npz"), (10, "full_capture_J10.npz")):
        path = ROOT / "tests" / "golden" / name
        if not path.exists():
            continue
        data = np.load(path)
        wl = blocks[Js.index(J)]
        result = tb.solve(wl.system, data["energies"], wl.grid, tb.Propagation(mode="capture", precision="mixed", steps="learned", learned_range=span))
        accuracy[f"J{J}"] = max((float(np.abs(s - data["Smat"][e, : s.shape[0], : s.shape[0]]).max()) for e, s in enumerate(result.Smat) if s.size), default=0.0)
    n_solves = len(blocks) * batch * args.steps
    head, fixed = arms["learned"], arms["fixed"]
    line = {
        "metric": "S-matrix solves/s on 1 B200, ultracold capture with learned sector widths (one solve = one (J, parity) block at one energy)",
        "value": n_solves / head["seconds"], "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": head["seconds"] / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128 via real embedding, f64+tf32x3", "data": "synthetic",
        "config": {"workload": "ultracold capture: rigid rotor B=0.03 cm^-1 j<=40, J=0,5,10 parity +1 (N=41..396 complex), C6 tail + Gaussian wall, capture boundary 8 bohr, fixed h=0.05 to 1500 bohr (14920 sectors), 512 energies log-uniform 1 uK-1 mK",
                   "batch": batch, "sectors_fixed": len(blocks[0].grid.sectors), "sectors_learned_per_block": head["sectors"][: len(blocks)]},
        "fixed_grid": {"value": n_solves / fixed["seconds"], "ms_per_step": fixed["seconds"] / args.steps * 1e3, "speedup_of_learned": fixed["seconds"] / head["seconds"]},
        "accuracy": {"max_dS_vs_reference_fixed_step": accuracy, "tolerance": 1e-6},
        "e2e": None,
        "gpu_launches": int(head["launches"]),
        "clocks": head["clocks"],
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
    peak = _best_gemm_tflops(torch, dev, torch.float64) if rank == 0 else 0.0
    e2e_value, h2d, d2h, cpu = None, 0, 0, None
    if rank == 0:
        wl = blocks[plan[args.warmup][0]]
        energies = np.ascontiguousarray(wl.energies[plan[args.warmup][1]])
        wl.grid._device_cache.clear()
        runner.release_device_state(scattering.hamiltonian_for(wl.system, wl.grid))
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
        cpu = {"value": 1.0 / (cpu_s / n_s * len(wl.grid.sectors)), "unit": "solves/s", "cores": blas_threads(), "kind": "port",
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
