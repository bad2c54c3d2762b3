"""LDMD propagation on the GPU (reference ``src/pyticc/propagation``)."""

from .config import Propagation, PropagationMode, resolve_device
from .delves import DelvesPropagationResult, propagate_delves
from .grid import RadialSector, build_radial_sectors, iter_radial_windows
from .logd import initialize_logD_capture, initialize_logD_inelastic, propagate_logD, propagate_logD_sector
from .runner import propagate, propagate_blocks
from .sweep import PartialWaveSweep, solve_sweep

__all__ = [
    "DelvesPropagationResult", "propagate_delves",
    "PartialWaveSweep",
    "Propagation",
    "PropagationMode",
    "RadialSector",
    "build_radial_sectors",
    "initialize_logD_capture",
    "initialize_logD_inelastic",
    "iter_radial_windows",
    "propagate",
    "propagate_blocks",
    "propagate_logD",
    "propagate_logD_sector",
    "resolve_device",
    "solve_sweep",
]
