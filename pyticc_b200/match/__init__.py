"""Asymptotic matching on the GPU: BF->SF transform, Riccati–Bessel functions, S matrices."""

from .asymptotic import get_Bmat_BF_to_SF, transform_logD_BF_to_SF
from .bessel import modified_bessel_K_logD, riccati_bessel_jy
from .smatrix import get_Smat, get_Smat_device

__all__ = ["get_Bmat_BF_to_SF", "transform_logD_BF_to_SF", "riccati_bessel_jy", "modified_bessel_K_logD", "get_Smat", "get_Smat_device"]
