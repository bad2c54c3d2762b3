"""Channel matrices: centrifugal U, W assembly and the V(R) contraction."""

from ..basis import get_Umat_BF
from .interaction import VBasisBF, contract_device, device_basis, prepare_atom_diatom, prepare_diatom_diatom

__all__ = ["VBasisBF", "contract_device", "device_basis", "get_Umat_BF", "prepare_atom_diatom", "prepare_diatom_diatom"]
