"""pyticc_b200 — B200-native coupled-channel hot path behind PyTICC's public API.

``solve`` / ``prepare_potential`` / ``Propagation`` / ``build_ScattSystem`` follow the
reference's signatures for exact coupled-channel A+BC and AB+CD scattering; LDMD
propagation, the PotentialGrid contraction and asymptotic matching run in the sm_100a
CUDA library ``pyticc_b200/_lib/libticc_b200.so`` (C ABI in ``include/ticc_b200.h``).
"""

from .basis import AtomSpec, Channel, ChannelBasis, DiatomBasis, DiatomSpec, RovibBasis, build_ChannelBasis, build_RovibDVR, build_SineDVR, get_Umat_BF
from .constants import AMU2AU, AU2CM, AU2K, CM2AU, K2AU
from .cross_section import PartialCrossSections, partial_cross_sections
from .energy import get_Etot
from .match import get_Bmat_BF_to_SF, get_Smat, modified_bessel_K_logD, riccati_bessel_jy, transform_logD_BF_to_SF
from .pes import PESWrapper
from .pes_analytic import LegendrePES, LegendreTerm, Primitive
from .propagation import PartialWaveSweep, Propagation, build_radial_sectors, propagate_logD, solve_sweep
from .kblock import KBlock, build_cs_blocks, build_nncc_blocks
from .result import CoupledStatesResult, KBlockResult, ScatteringResult, Timing
from .scattering import PotentialGrid, ScattHamiltonian, build_k_blocks, finalize_K_block, prepare_potential, solve
from .system import Approx, ChannelSpec, ScatteringType, ScattSystem, build_ScattSystem, reduced_mass

__all__ = [
    "AMU2AU", "AU2CM", "AU2K", "CM2AU", "K2AU",
    "Approx", "AtomSpec", "Channel", "ChannelBasis", "ChannelSpec", "CoupledStatesResult", "DiatomBasis", "DiatomSpec", "KBlock", "KBlockResult", "LegendrePES", "LegendreTerm",
    "PESWrapper", "Primitive", "PartialCrossSections", "PartialWaveSweep", "PotentialGrid",
    "Propagation", "RovibBasis", "ScattHamiltonian", "ScattSystem", "ScatteringResult", "ScatteringType", "Timing",
    "build_ChannelBasis", "build_RovibDVR", "build_ScattSystem", "build_SineDVR", "build_cs_blocks", "build_k_blocks", "build_nncc_blocks",
    "build_radial_sectors", "finalize_K_block", "get_Bmat_BF_to_SF",
    "get_Etot", "get_Smat", "get_Umat_BF", "modified_bessel_K_logD", "partial_cross_sections", "prepare_potential", "propagate_logD", "reduced_mass",
    "riccati_bessel_jy", "solve", "solve_sweep", "transform_logD_BF_to_SF",
]
