"""Learned LDMD sector widths (no counterpart in the reference).

The reference propagates on the fixed grid of ``build_radial_sectors``
(``src/pyticc/propagation/grid.py:193-239``).  Here a small MLP proposes, for every
fixed-step (base) sector, log2 of how many aligned base sectors may be merged into one
LDMD sector.  A merged sector of m base sectors of half-step h has half-step m h and its
start, mid and end points are base grid points, so the PotentialGrid is unchanged and
no PES is evaluated anywhere new.

* ``sector_features``      per-base-sector features from W_base (CUDA kernel)
* ``StepProposer``         the network: FP32 parameters, forward / gradient / Adam on the
                           GPU through the C ABI (hand-written kernels)
* ``step_doubling_labels`` training targets from the plain FP64 propagator itself: a
                           merged sector is compared with the base sectors it replaces
* ``merge_sectors``        the schedule: the widest aligned power-of-two group whose
                           sectors all allow it, capped so that a merged sector keeps
                           |p| h below 2.8 for every open channel (the reference
                           propagators cot/csc of an LDMD sector have poles at
                           |p| h = n pi; the cap keeps merged sectors below the first)
* ``validate_learned``     the fixed-step solve checks the learned one: accepted only if
                           max|dS| is within tolerance and the open-channel counts agree.
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence
from dataclasses import dataclass, field, replace
from pathlib import Path

import numpy as np
import torch
from loguru import logger

from .. import _native as nat
from ..energy import get_Etot
from .config import Propagation, resolve_device
from .grid import RadialSector, radial_points_of

N_FEATURE = 8
N_HIDDEN = 32
N_PARAM = N_HIDDEN * N_FEATURE + N_HIDDEN + N_HIDDEN * N_HIDDEN + N_HIDDEN + N_HIDDEN + 1
OPEN_PHASE_LIMIT = 2.8
DEFAULT_PROPOSER = Path(__file__).with_name("proposer_default.npz")


def library_shape() -> tuple[int, int, int]:
    """(n_feature, n_hidden, n_param) as compiled into the CUDA library."""
    lib = nat.load_library()
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    nat.check(lib.ticc_mlp_shape(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "ticc_mlp_shape")
    return a.value, b.value, c.value


# ---- schedules (host) -----------------------------------------------------------------------
def sector_runs(sectors: Sequence[RadialSector]) -> np.ndarray:
    """Run index of each sector: consecutive, touching sectors of equal width share a run
    (the shortened last sector of an interval starts a run of its own)."""
    run = np.zeros(len(sectors), dtype=np.int64)
    for k in range(1, len(sectors)):
        prev, cur = sectors[k - 1], sectors[k]
        w0, w1 = prev.radial_end - prev.radial_start, cur.radial_end - cur.radial_start
        same = abs(w1 - w0) <= 1e-9 * w0 and abs(cur.radial_start - prev.radial_end) <= 1e-12
        run[k] = run[k - 1] + (0 if same else 1)
    return run


def open_phase(features: np.ndarray, sectors: Sequence[RadialSector]) -> np.ndarray:
    """max over open channels of |p| h per base sector, from feature 0 = asinh(max -p^2)."""
    k2 = np.sinh(np.asarray(features, dtype=np.float64)[:, 0])
    halves = np.array([s.radial_half_step for s in sectors])
    return np.sqrt(np.maximum(k2, 0.0)) * halves


def merge_groups(levels: np.ndarray, runs: np.ndarray, max_level: int, phase: np.ndarray | None = None) -> list[tuple[int, int]]:
    """[(first base sector, count)]: at each position the largest m = 2^l <= 2^max_level that
    is aligned within its run, stays inside it, has levels >= l on all its sectors and keeps
    m * phase below OPEN_PHASE_LIMIT."""
    levels = np.asarray(levels, dtype=np.float64)
    n = levels.size
    run_start = np.zeros(n, dtype=np.int64)
    for s in range(1, n):
        run_start[s] = run_start[s - 1] if runs[s] == runs[s - 1] else s
    groups = []
    s = 0
    while s < n:
        m = 2**max_level
        while m > 1:
            if (s - run_start[s]) % m == 0 and s + m <= n and runs[s + m - 1] == runs[s] and levels[s : s + m].min() >= np.log2(m):
                if phase is None or m * phase[s : s + m].max() < OPEN_PHASE_LIMIT:
                    break
            m //= 2
        groups.append((s, m))
        s += m
    return groups


def merge_sectors(sectors: Sequence[RadialSector], levels: np.ndarray, max_level: int, phase: np.ndarray | None = None) -> tuple[RadialSector, ...]:
    runs = sector_runs(sectors)
    return tuple(RadialSector(sectors[s].radial_start, sectors[s + m - 1].radial_end) for s, m in merge_groups(levels, runs, max_level, phase))


# ---- features (device) ----------------------------------------------------------------------
def sector_features(hamiltonian, sectors: Sequence[RadialSector], Etot, device: str = "auto") -> torch.Tensor:
    """(n_sector, 8) FP32 features of every base sector for the energy set ``Etot``."""
    from .runner import device_hamiltonian, device_window

    dev = resolve_device(device)
    lib = nat.load_library()
    energies = get_Etot(Etot)
    dh = device_hamiltonian(hamiltonian, dev)
    n = dh.n
    n_sector = len(sectors)
    two_mu = 2.0 * dh.reduced_mass
    out = torch.empty((n_sector, N_FEATURE), dtype=torch.float32, device=dev)
    size = device_window(n, n_sector)
    W = torch.empty((2 * size + 1, n, n), dtype=torch.float64, device=dev)
    stride = 2 * n * n
    with torch.cuda.device(dev):
        for s0 in range(0, n_sector, size):
            window = tuple(sectors[s0 : s0 + size])
            points = radial_points_of(window)
            Wv = dh.W_base(points, out=W[: points.size])
            halves = torch.as_tensor(np.asarray([s.radial_half_step for s in window]), device=dev)
            nat.check(
                lib.ticc_step_features(
                    nat.ptr(Wv[0::2]), stride, nat.ptr(Wv[1::2]), stride, nat.ptr(Wv[2::2]), stride, nat.ptr(halves), len(window), n,
                    two_mu * float(energies.max()), two_mu * float(energies.min()), ctypes.c_void_p(out.data_ptr() + 4 * N_FEATURE * s0), nat.stream_handle(dev),
                ),
                "ticc_step_features",
            )
    return out


# ---- the network ----------------------------------------------------------------------------------
@dataclass
class StepProposer:
    """MLP proposer.  ``params`` (N_PARAM,) and ``norm`` (mean[8], 1/scale[8]) are FP32;
    ``margin`` is subtracted from every prediction before a width is taken."""

    params: np.ndarray
    norm: np.ndarray
    max_level: int = 8
    margin: float = 0.5
    _cache: dict = field(default_factory=dict, repr=False, compare=False)

    @classmethod
    def initialize(cls, features: np.ndarray, *, seed: int = 0, max_level: int = 8, margin: float = 0.5) -> StepProposer:
        """Glorot-uniform weights; inputs standardised with the statistics of ``features``."""
        rng = np.random.default_rng(seed)
        features = np.asarray(features, dtype=np.float64)

        def glorot(fan_out, fan_in):
            return rng.uniform(-1.0, 1.0, (fan_out, fan_in)) * np.sqrt(6.0 / (fan_in + fan_out))

        params = np.concatenate([glorot(N_HIDDEN, N_FEATURE).ravel(), np.zeros(N_HIDDEN), glorot(N_HIDDEN, N_HIDDEN).ravel(), np.zeros(N_HIDDEN), glorot(1, N_HIDDEN).ravel(), [0.0]])
        mean = features.mean(axis=0)
        scale = np.maximum(features.std(axis=0), 1e-3)
        norm = np.concatenate([mean, 1.0 / scale])
        return cls(params.astype(np.float32), norm.astype(np.float32), max_level, margin)

    @classmethod
    def load(cls, path: str | Path = DEFAULT_PROPOSER) -> StepProposer:
        data = np.load(path)
        return cls(data["params"].astype(np.float32), data["norm"].astype(np.float32), int(data["max_level"]), float(data["margin"]))

    def save(self, path: str | Path) -> None:
        np.savez(path, params=self.params, norm=self.norm, max_level=self.max_level, margin=self.margin)

    def _device(self, dev: torch.device) -> tuple[torch.Tensor, torch.Tensor]:
        key = (dev.index, self.params.tobytes(), self.norm.tobytes())
        cached = self._cache.get("device")
        if cached is None or cached[0] != key:
            cached = (key, torch.as_tensor(self.params, device=dev), torch.as_tensor(self.norm, device=dev))
            self._cache["device"] = cached
        return cached[1], cached[2]

    def predict(self, features: torch.Tensor) -> torch.Tensor:
        """Raw network output (log2 of the admissible merge) for (n, 8) device features."""
        X = features.to(torch.float32).contiguous()
        dev = X.device
        lib = nat.load_library()
        params, norm = self._device(dev)
        y = torch.empty(X.shape[0], dtype=torch.float32, device=dev)
        with torch.cuda.device(dev):
            nat.check(lib.ticc_mlp_forward(nat.ptr(params), nat.ptr(norm), nat.ptr(X), X.shape[0], nat.ptr(y), nat.stream_handle(dev)), "ticc_mlp_forward")
        return y

    def gradient(self, X: torch.Tensor, target: torch.Tensor, weight: torch.Tensor, *, over_weight: float = 4.0) -> tuple[float, torch.Tensor]:
        """(loss, gradient) of the asymmetric weighted squared loss on the device."""
        dev = X.device
        lib = nat.load_library()
        params, norm = self._device(dev)
        grads = torch.empty(N_PARAM, dtype=torch.float32, device=dev)
        loss = torch.empty(1, dtype=torch.float32, device=dev)
        n = X.shape[0]
        with torch.cuda.device(dev):
            work = nat.Workspace.get(dev, nat.size_query(lib.ticc_mlp_workspace_size, n), slot=4)
            nat.check(
                lib.ticc_mlp_gradient(nat.ptr(params), nat.ptr(norm), nat.ptr(X), nat.ptr(target), nat.ptr(weight), n, over_weight, float(1.0 / float(weight.sum())),
                                      nat.ptr(grads), nat.ptr(loss), nat.ptr(work), work.numel(), nat.stream_handle(dev)),
                "ticc_mlp_gradient",
            )
        return float(loss.item()), grads

    def fit(self, features, target, weight=None, *, steps: int = 3000, lr: float = 3e-3, over_weight: float = 4.0, beta1: float = 0.9, beta2: float = 0.999,
            eps: float = 1e-8, device: str = "auto") -> np.ndarray:
        """Full-batch Adam on the GPU; returns the loss before every step."""
        dev = resolve_device(device)
        lib = nat.load_library()
        X = torch.as_tensor(np.asarray(features, dtype=np.float32), device=dev).contiguous() if not isinstance(features, torch.Tensor) else features.to(dev, torch.float32).contiguous()
        T = torch.as_tensor(np.asarray(target, dtype=np.float32), device=dev).contiguous()
        Wt = torch.ones_like(T) if weight is None else torch.as_tensor(np.asarray(weight, dtype=np.float32), device=dev).contiguous()
        n = X.shape[0]
        params = torch.as_tensor(self.params, device=dev).clone()
        norm = torch.as_tensor(self.norm, device=dev)
        moments = torch.zeros(2 * N_PARAM, dtype=torch.float32, device=dev)
        grads = torch.empty(N_PARAM, dtype=torch.float32, device=dev)
        history = torch.empty(steps, dtype=torch.float32, device=dev)
        inv_wsum = float(1.0 / float(Wt.sum()))
        with torch.cuda.device(dev):
            work = nat.Workspace.get(dev, nat.size_query(lib.ticc_mlp_workspace_size, n), slot=4)
            stream = nat.stream_handle(dev)
            for k in range(steps):
                nat.check(
                    lib.ticc_mlp_gradient(nat.ptr(params), nat.ptr(norm), nat.ptr(X), nat.ptr(T), nat.ptr(Wt), n, over_weight, inv_wsum, nat.ptr(grads),
                                          ctypes.c_void_p(history.data_ptr() + 4 * k), nat.ptr(work), work.numel(), stream),
                    "ticc_mlp_gradient",
                )
                nat.check(lib.ticc_mlp_adam(nat.ptr(params), nat.ptr(grads), nat.ptr(moments), k + 1, lr, beta1, beta2, eps, stream), "ticc_mlp_adam")
        self.params = params.cpu().numpy()
        self._cache.clear()
        return history.cpu().numpy()


# ---- training labels from the plain propagator -------------------------------------------------
def _local_s_distance(Ya: torch.Tensor, Yb: torch.Tensor, diag_w: torch.Tensor, energies: torch.Tensor, reduced_mass: float) -> tuple[np.ndarray, np.ndarray]:
    """Per energy: (max over the channels open at the comparison point, max over all
    channels) of |C(Ya) - C(Yb)|, with C(Y) = I - 2i s K^1/2 (Y + i s K)^-1 K^1/2 the local S
    matrix there (K = diag sqrt|p^2|, floor 1e-4 bohr^-1; s = -1 when Y carries incoming
    flux, Im Y < 0, so that Y + i s K stays far from singular).  For a closed channel, where
    Y ~ p, C measures the relative error of Y; such errors decay outwards, so the labels
    hold them to a looser tolerance than the open block."""
    from ..linalg import symmetric_inverse

    p2 = diag_w[None, :] - 2.0 * reduced_mass * energies[:, None]
    k = torch.sqrt(torch.clamp(p2.abs(), min=1e-8))
    sign = -1.0 if (Ya.is_complex() and float(torch.diagonal(Ya, dim1=-2, dim2=-1).imag.sum()) < 0.0) else 1.0
    shift = torch.diag_embed(1j * sign * k.to(torch.complex128))
    inv = symmetric_inverse(torch.cat([Ya.to(torch.complex128) + shift, Yb.to(torch.complex128) + shift]))
    n_e = Ya.shape[0]
    root = torch.sqrt(k)
    D = ((inv[:n_e] - inv[n_e:]) * root[:, :, None] * root[:, None, :]).abs()
    open_ = (p2 < 0.0).to(torch.float64)
    open_err = (D * open_[:, :, None] * open_[:, None, :]).amax(dim=(1, 2))
    return (2.0 * open_err).cpu().numpy(), (2.0 * D.amax(dim=(1, 2))).cpu().numpy()


def step_doubling_errors(hamiltonian, sectors: Sequence[RadialSector], Etot, propagation: Propagation, *, max_level: int = 8) -> tuple[np.ndarray, np.ndarray]:
    """errors[b, l-1, s]: local-S distance between one merged sector of 2^l base sectors and
    the base sectors it replaces, for the aligned group holding sector s (max over
    energies), over the open block (b = 0) and over all channels (b = 1); NaN where the
    group does not exist (run edges) and +inf where the merge breaks the open-phase cap.
    Also returns the (n_sector, 8) features for the same energies."""
    from .runner import device_hamiltonian, initial_logD, propagate

    config = replace(propagation, precision="fp64")
    dev = resolve_device(config.device)
    energies_np = get_Etot(Etot)
    energies = torch.as_tensor(np.array(energies_np), device=dev)
    dh = device_hamiltonian(hamiltonian, dev)
    n_sector = len(sectors)
    features = sector_features(hamiltonian, sectors, energies_np, config.device)
    phase = open_phase(features.cpu().numpy(), sectors)
    runs = sector_runs(sectors)
    run_start = np.zeros(n_sector, dtype=np.int64)
    run_end = np.zeros(n_sector, dtype=np.int64)
    for s in range(1, n_sector):
        run_start[s] = run_start[s - 1] if runs[s] == runs[s - 1] else s
    run_end[-1] = n_sector
    for s in range(n_sector - 2, -1, -1):
        run_end[s] = run_end[s + 1] if runs[s] == runs[s + 1] else s + 1
    errors = np.full((2, max_level, n_sector), np.nan)
    Y = initial_logD(dh.W_base(np.array([sectors[0].radial_start]))[0], energies, dh.reduced_mass, config.mode)
    pending: dict[int, tuple[int, torch.Tensor]] = {}
    s = 0
    while s < n_sector:
        for level in range(1, max_level + 1):
            m = 2**level
            if (s - run_start[s]) % m or s + m > run_end[s]:
                continue
            if m * phase[s : s + m].max() >= OPEN_PHASE_LIMIT:
                errors[:, level - 1, s : s + m] = np.inf
                continue
            merged = RadialSector(sectors[s].radial_start, sectors[s + m - 1].radial_end)
            pending[level] = (s + m, propagate(hamiltonian, energies_np, [merged], config, Y_initial=Y.clone()))
        step = 2 if (s - run_start[s]) % 2 == 0 and s + 2 <= run_end[s] else 1
        Y = propagate(hamiltonian, energies_np, list(sectors[s : s + step]), config, Y_initial=Y)
        s += step
        done = [level for level, (end, _) in pending.items() if end == s]
        if done:
            diag_w = torch.diagonal(dh.W_base(np.array([sectors[s - 1].radial_end]))[0]).contiguous()
            for level in done:
                _, Yc = pending.pop(level)
                open_err, all_err = _local_s_distance(Yc, Y, diag_w, energies, dh.reduced_mass)
                errors[0, level - 1, s - 2**level : s] = open_err.max()
                errors[1, level - 1, s - 2**level : s] = all_err.max()
    return errors, features.cpu().numpy()


def labels_from_errors(errors: np.ndarray, *, tol: float = 1e-9, closed_tol: float = 1e-5, order: float = 5.0, noise: float = 1e-12) -> np.ndarray:
    """Continuous admissible level per base sector: min over levels l of
    l + log2(tol / err_l) / order (local error ~ width^order), ignoring errors at the noise
    floor, l - 1 where the merge is forbidden (+inf), clipped to [0, max_level].  With
    errors of shape (2, L, n) (open block, all channels) both bounds apply, the second
    with ``closed_tol``."""
    if errors.ndim == 3:
        return np.minimum(labels_from_errors(errors[0], tol=tol, order=order, noise=noise), labels_from_errors(errors[1], tol=closed_tol, order=order, noise=noise))
    max_level, n = errors.shape
    label = np.full(n, float(max_level))
    for level in range(1, max_level + 1):
        e = errors[level - 1]
        forbidden = np.isinf(e)
        label[forbidden] = np.minimum(label[forbidden], level - 1.0)
        valid = np.isfinite(e) & (e > noise)
        label[valid] = np.minimum(label[valid], level + np.log2(tol / e[valid]) / order)
    return np.clip(label, 0.0, float(max_level))


# ---- use ---------------------------------------------------------------------------------------------
_LOADED: dict[str, StepProposer] = {}


def resolve_proposer(proposer) -> StepProposer:
    """A StepProposer from an instance, a weights path, or None (the packaged default)."""
    if isinstance(proposer, StepProposer):
        return proposer
    path = str(DEFAULT_PROPOSER if proposer is None else proposer)
    if path not in _LOADED:
        _LOADED[path] = StepProposer.load(path)
    return _LOADED[path]


def learned_sectors(hamiltonian, sectors: Sequence[RadialSector], Etot, proposer: StepProposer, device: str = "auto") -> tuple[RadialSector, ...]:
    """The learned schedule for one energy set: features -> network -> aligned merges."""
    features = sector_features(hamiltonian, sectors, Etot, device)
    levels = proposer.predict(features).cpu().numpy().astype(np.float64) - proposer.margin
    phase = open_phase(features.cpu().numpy(), sectors)
    merged = merge_sectors(sectors, levels, proposer.max_level, phase)
    logger.info(f"Learned schedule: {len(merged)} sectors in place of {len(sectors)}")
    return merged


def judged_learned_sectors(problem, potential_grid, Etot, propagation: Propagation) -> tuple[tuple[RadialSector, ...], dict]:
    """The learned schedule for these energies if the fixed step accepts it, else the fixed
    grid.  The schedule is built for the call's lowest and highest energy, or for
    ``propagation.learned_range`` (then built once and cached); the judge solves those two
    energies with both schedules (same precision and mode) and accepts when the open counts
    are equal and max|dS| <= ``propagation.judge_tol``.  Verdicts are cached per schedule on
    the Hamiltonian, so repeated calls with the same schedule are judged once; a schedule
    equal to the fixed grid needs no judge.  Returns (sectors, record) with record holding the
    decision, max|dS| of the judge and both sector counts."""
    from ..scattering import hamiltonian_for, solve

    hamiltonian = hamiltonian_for(problem, potential_grid)
    fixed = tuple(potential_grid.sectors)
    energies = np.atleast_1d(np.asarray(Etot, dtype=np.float64))
    cache = getattr(hamiltonian, "_runner_cache", {})
    span = (float(energies.min()), float(energies.max()))
    if propagation.learned_range is not None:
        lo, hi = propagation.learned_range
        if span[0] < lo or span[1] > hi:
            message = f"Energies {span} lie outside the learned_range {propagation.learned_range}"
            logger.error(message)
            raise ValueError(message)
        span = (lo, hi)
    proposer = resolve_proposer(propagation.proposer)
    schedule_key = ("learned_schedule", span, len(fixed))
    cached = cache.get(schedule_key)
    if cached is not None and cached[0] is proposer:
        schedule = cached[1]
    else:
        schedule = learned_sectors(hamiltonian, fixed, np.asarray(span), proposer, propagation.device)
        if propagation.learned_range is not None:
            cache[schedule_key] = (proposer, schedule)
    record = {"n_fixed": len(fixed), "n_learned": len(schedule), "accepted": True, "max_dS": 0.0, "judged": False}
    if len(schedule) == len(fixed):
        return fixed, record
    key = ("learned_judge", propagation.precision, propagation.mode, propagation.judge_tol, tuple((s.radial_start, s.radial_end) for s in schedule))
    verdict = cache.get(key)
    if verdict is None:
        probe = np.unique(np.asarray(span))
        plain = replace(propagation, steps="fixed", audit=False)
        a = solve(problem, probe, potential_grid, plain, sectors=fixed)
        b = solve(problem, probe, potential_grid, plain, sectors=schedule)
        same_counts = all(x.shape == y.shape for x, y in zip(a.Smat, b.Smat, strict=True))
        dS = max((float(np.abs(x - y).max()) for x, y in zip(a.Smat, b.Smat, strict=True) if x.size and x.shape == y.shape), default=0.0)
        verdict = (bool(same_counts and dS <= propagation.judge_tol), dS)
        cache[key] = verdict
        if not verdict[0]:
            logger.warning(f"Learned schedule rejected by the fixed-step judge: max|dS|={dS:.3e}, open counts equal={same_counts}; using the fixed grid")
        record["judged"] = True
    record["accepted"], record["max_dS"] = verdict
    return (schedule if verdict[0] else fixed), record


def validate_learned(problem, Etot, potential_grid, propagation: Propagation, proposer: StepProposer, *, tol: float = 1e-6):
    """Solve with the fixed grid and with the learned schedule; return (accepted, max|dS|,
    n_fixed, n_learned, result) where result is the learned solve when accepted and the
    fixed-step one otherwise (same open-channel counts and max|dS| <= tol required)."""
    from ..scattering import hamiltonian_for, solve

    hamiltonian = hamiltonian_for(problem, potential_grid)
    propagation = replace(propagation, steps="fixed")
    fixed = solve(problem, Etot, potential_grid, propagation)
    schedule = learned_sectors(hamiltonian, potential_grid.sectors, Etot, proposer, propagation.device)
    learned = solve(problem, Etot, potential_grid, propagation, sectors=schedule)
    same_counts = all(a.shape == b.shape for a, b in zip(fixed.Smat, learned.Smat, strict=True))
    if not any(a.size for a in fixed.Smat):
        logger.warning("No open channel at any energy: the S matrices give no test of the learned schedule")
    dS = max((float(np.abs(a - b).max()) for a, b in zip(fixed.Smat, learned.Smat, strict=True) if a.size and a.shape == b.shape), default=0.0)
    accepted = same_counts and dS <= tol
    if not accepted:
        logger.warning(f"Learned schedule rejected: max|dS|={dS:.3e}, open counts equal={same_counts}; keeping the fixed-step result")
    return accepted, dS, len(potential_grid.sectors), len(schedule), (learned if accepted else fixed)


def training_set(cases, *, max_level: int = 8, tol: float = 1e-9, closed_tol: float = 1e-5, order: float = 5.0) -> tuple[np.ndarray, np.ndarray]:
    """Features and labels from step doubling on every case (hamiltonian, sectors, Etot,
    propagation), stacked."""
    X, T = [], []
    logger.disable("pyticc_b200")  # thousands of short propagations: keep their progress lines quiet
    try:
        for hamiltonian, sectors, Etot, propagation in cases:
            errors, features = step_doubling_errors(hamiltonian, sectors, Etot, propagation, max_level=max_level)
            X.append(features)
            T.append(labels_from_errors(errors, tol=tol, closed_tol=closed_tol, order=order))
    finally:
        logger.enable("pyticc_b200")
    return np.concatenate(X), np.concatenate(T)


def train_proposer(features: np.ndarray, labels: np.ndarray, *, seed: int = 0, steps: int = 4000, lr: float = 3e-3, over_weight: float = 4.0, max_level: int = 8,
                   margin: float = 0.5, device: str = "auto") -> tuple[StepProposer, np.ndarray]:
    """A proposer fitted on the GPU (own gradient and Adam kernels); returns it and the loss history."""
    proposer = StepProposer.initialize(features, seed=seed, max_level=max_level, margin=margin)
    history = proposer.fit(features, labels, steps=steps, lr=lr, over_weight=over_weight, device=device)
    return proposer, history
