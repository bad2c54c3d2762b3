"""Batched symmetric (real or complex-symmetric) inverse through the C ABI.

The same blocked sweep the LDMD sectors use; here for host code that needs A^{-1}
outside a propagation (the step-doubling error measure of the learned proposer)."""

from __future__ import annotations

import torch

from . import _native as nat


def symmetric_inverse(A: torch.Tensor) -> torch.Tensor:
    """A^{-1} for a (batch, n, n) symmetric float64 or complex-symmetric complex128 CUDA tensor
    (A itself is left unchanged)."""
    if A.dim() != 3 or A.shape[-1] != A.shape[-2]:
        raise ValueError(f"symmetric_inverse needs a (batch, n, n) tensor, got {tuple(A.shape)}")
    if A.dtype not in (torch.float64, torch.complex128) or A.device.type != "cuda":
        raise ValueError(f"symmetric_inverse needs float64 or complex128 CUDA data, got {A.dtype} on {A.device}")
    lib = nat.load_library()
    batch, n, _ = A.shape
    is_complex = int(A.is_complex())
    out = A.clone().contiguous()
    dev = A.device
    with torch.cuda.device(dev):
        nbytes = nat.size_query(lib.ticc_sym_inverse_workspace_size, n, batch, is_complex)
        work = nat.Workspace.get(dev, nbytes, slot=3)
        status = nat.DeviceStatus(dev)
        nat.check(lib.ticc_sym_inverse(nat.ptr(out), n, batch, is_complex, nat.ptr(work), work.numel(), status.pointer, nat.stream_handle(dev)), "ticc_sym_inverse")
        status.raise_if_failed("ticc_sym_inverse")
    return out.neg_()
