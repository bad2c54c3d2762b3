"""Train the default sector-width proposer on the GPU and write its weights.

    python -m pyticc_b200.propagation.train_proposer --out proposer_default.npz [--report r.json]

Training labels come from step doubling with the plain FP64 propagator on three systems
of the shapes this library is benchmarked on (the rigid-rotor A+BC block, the vibrating
Morse A+BC block at J=30, and ultracold capture at J=10), at the lowest and highest
energy of each range.  The fitted network is then checked against the fixed-step solve on
held-out energies of every system (max|dS| and the sector counts are reported).
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from ..constants import CM2AU, K2AU
from ..workloads import morse_atom_diatom, rigid_atom_diatom, ultracold_capture
from .config import Propagation
from .learned import training_set, train_proposer, validate_learned


def cases(names):
    out = []
    if "rigid" in names:
        wl = rigid_atom_diatom(n_energy=4)
        out.append(("rigid", wl, np.array([10.0, 500.0]) * CM2AU, np.array([180.0, 420.0]) * CM2AU))
    if "morse" in names:
        wl = morse_atom_diatom(n_energy=4)
        out.append(("morse", wl, np.array([100.0, 3000.0]) * CM2AU, np.array([900.0, 2400.0]) * CM2AU))
    if "capture" in names:
        wl = ultracold_capture(n_energy=4)
        out.append(("capture", wl, np.array([1.0e-6, 1.0e-3]) * K2AU, np.array([1.0e-5, 2.0e-4]) * K2AU))
    return out


def main(argv=None) -> int:
    from ..scattering import hamiltonian_for

    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--out", required=True)
    parser.add_argument("--report", default=None)
    parser.add_argument("--cases", default="rigid,morse,capture")
    parser.add_argument("--steps", type=int, default=4000)
    parser.add_argument("--max-level", type=int, default=8)
    parser.add_argument("--tol", type=float, default=1e-9)
    args = parser.parse_args(argv)
    report = {"cases": {}}
    selected = cases(args.cases.split(","))
    data = []
    for name, wl, train_E, _ in selected:
        t0 = time.perf_counter()
        config = Propagation(mode=wl.mode)
        X, T = training_set([(hamiltonian_for(wl.system, wl.grid), wl.grid.sectors, train_E, config)], max_level=args.max_level, tol=args.tol)
        data.append((X, T))
        report["cases"][name] = {"n_channel": wl.system.basis.n_channel, "base_sectors": len(wl.grid.sectors), "label_mean": float(T.mean()), "label_min": float(T.min()),
                                 "label_seconds": time.perf_counter() - t0}
        print(name, report["cases"][name], flush=True)
    X = np.concatenate([d[0] for d in data])
    T = np.concatenate([d[1] for d in data])
    t0 = time.perf_counter()
    proposer, history = train_proposer(X, T, steps=args.steps, max_level=args.max_level)
    report["train"] = {"samples": int(X.shape[0]), "steps": args.steps, "loss_first": float(history[0]), "loss_last": float(history[-1]), "seconds": time.perf_counter() - t0}
    print(report["train"], flush=True)
    proposer.save(args.out)
    for name, wl, _, held_out in selected:
        t0 = time.perf_counter()
        accepted, dS, n_fixed, n_learned, _ = validate_learned(wl.system, held_out, wl.grid, Propagation(mode=wl.mode), proposer)
        report["cases"][name].update({"accepted": accepted, "max_dS": dS, "fixed_sectors": n_fixed, "learned_sectors": n_learned, "validate_seconds": time.perf_counter() - t0})
        print(name, report["cases"][name], flush=True)
    if args.report:
        with open(args.report, "w") as handle:
            json.dump(report, handle, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
