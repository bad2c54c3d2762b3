"""Propagation runtime settings (reference ``src/pyticc/propagation/config.py:47-74``)."""

from __future__ import annotations

import re
from dataclasses import dataclass
from typing import Literal

import numpy as np
import torch
from loguru import logger

PropagationMode = Literal["inelastic", "capture"]
_DEVICE_PATTERN = re.compile(r"(?:auto|cpu(?::\d+)?|gpu(?::\d+)?|cuda(?::\d+)?)")


def normalize_device_spec(value: object) -> str:
    """Normalise 'auto', 'gpu[:i]' / 'cuda[:i]' (and 'cpu[:i]', which is rejected at resolve time)."""
    if not isinstance(value, str) or _DEVICE_PATTERN.fullmatch(value.strip().lower()) is None:
        message = f"Propagation device must be 'auto', 'cpu', 'gpu', or '<platform>:<index>', but got {value!r}"
        logger.error(message)
        raise ValueError(message)
    return value.strip().lower().replace("cuda", "gpu")


def resolve_device(value: str) -> torch.device:
    """The CUDA device for a request; a CPU request or a missing GPU raises RuntimeError
    (this library has no CPU path)."""
    requested = normalize_device_spec(value)
    platform, _, index_text = requested.partition(":")
    if platform == "cpu":
        message = f"Propagation requested {requested!r}, but this library runs on CUDA devices only"
        logger.error(message)
        raise RuntimeError(message)
    count = torch.cuda.device_count() if torch.cuda.is_available() else 0
    index = int(index_text) if index_text else (torch.cuda.current_device() if count else 0)
    if index >= count:
        available = ", ".join(f"gpu:{i}" for i in range(count)) or "none"
        message = f"Propagation requested {requested!r}, but available gpu devices are: {available}"
        logger.error(message)
        raise RuntimeError(message)
    return torch.device("cuda", index)


@dataclass(frozen=True, slots=True)
class Propagation:
    """mode: inner boundary condition; memory_mb: transient-memory target of the host
    window iterator; device: 'auto' | 'gpu[:i]'; print_verbose: progress logging;
    precision: 'fp64' (plain) or 'mixed' (closed channels swept in FP32);
    steps: 'fixed' (the PotentialGrid's sectors) or 'learned' (aligned merges of them
    proposed by ``proposer``, a StepProposer or a path to its weights; None = the
    packaged default), used only once a fixed-step solve at the lowest and highest energy
    of the call agrees with it within ``judge_tol`` (max|dS|, equal open counts);
    learned_range: (E_min, E_max) in hartree the learned schedule is built and judged for;
    every call whose energies lie inside reuses that one schedule and its cached verdict
    (without it each call's own lowest and highest energy define the schedule);
    audit: also solve every energy in plain FP64 with fixed steps and attach max|dS| per
    energy to the result (doubles the cost; for validation runs)."""

    mode: PropagationMode = "inelastic"
    memory_mb: float = 512.0
    device: str = "auto"
    print_verbose: bool = False
    precision: str = "fp64"
    steps: str = "fixed"
    proposer: object = None
    judge_tol: float = 1.0e-6
    learned_range: tuple | None = None
    audit: bool = False

    def __post_init__(self) -> None:
        object.__setattr__(self, "device", normalize_device_spec(self.device))
        if self.mode not in ("inelastic", "capture"):
            message = f"Propagation mode must be 'inelastic' or 'capture', but got {self.mode!r}"
            logger.error(message)
            raise ValueError(message)
        if not np.isfinite(self.memory_mb) or self.memory_mb <= 0.0:
            message = f"Propagation memory_mb must be positive, but got {self.memory_mb}"
            logger.error(message)
            raise ValueError(message)
        if not isinstance(self.print_verbose, bool):
            message = f"Propagation print_verbose must be a boolean, but got {self.print_verbose!r}"
            logger.error(message)
            raise ValueError(message)
        if self.precision not in ("fp64", "mixed"):
            message = f"Propagation precision must be 'fp64' or 'mixed', but got {self.precision!r}"
            logger.error(message)
            raise ValueError(message)
        if self.steps not in ("fixed", "learned"):
            message = f"Propagation steps must be 'fixed' or 'learned', but got {self.steps!r}"
            logger.error(message)
            raise ValueError(message)
        if not (np.isfinite(self.judge_tol) and self.judge_tol > 0.0):
            message = f"Propagation judge_tol must be positive, but got {self.judge_tol}"
            logger.error(message)
            raise ValueError(message)
        if self.learned_range is not None:
            lo, hi = (float(v) for v in self.learned_range)
            if not (np.isfinite(lo) and np.isfinite(hi) and lo <= hi):
                message = f"Propagation learned_range must be (E_min, E_max) with E_min <= E_max, but got {self.learned_range!r}"
                logger.error(message)
                raise ValueError(message)
            object.__setattr__(self, "learned_range", (lo, hi))
        if not isinstance(self.audit, bool):
            message = f"Propagation audit must be a boolean, but got {self.audit!r}"
            logger.error(message)
            raise ValueError(message)
