"""ctypes binding of ``libticc_b200.so`` and the device-buffer helpers around it.

The CUDA library is the only compute path: there is no CPU fallback.  Loading fails
loudly when the shared object is missing (build it with
``python -c "import __graft_entry__ as g; g.build()"`` or ``pyticc_b200._build.build()``),
and every entry point's status is turned into the exception the reference raises
for the same condition (``ValueError`` for bad shapes or values, ``RuntimeError``
for device failures).
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import numpy as np
import torch
from loguru import logger

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libticc_b200.so"
HEADER_PATH = Path(__file__).resolve().parents[1] / "include" / "ticc_b200.h"

OK, ERR_INVALID_ARGUMENT, ERR_CUDA, ERR_WORKSPACE, ERR_UNSUPPORTED = 0, 1, 2, 3, 4
PRECISION_FP64, PRECISION_MIXED = 0, 1

DEVICE_STATUS_TEXT = {
    1: "a 128-wide pivot block of the symmetric sweep is singular or non-finite",
    2: "a non-finite value reached an S matrix",
    3: "a Bessel continued fraction did not converge or produced a non-finite value",
    4: "asymptotic matching is undefined exactly at a channel threshold",
    5: "more open channels than the workspace was sized for",
    6: "a fused sweep step gave up waiting for a row-panel tile (internal error; the wait is bounded)",
}

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_LL = ctypes.c_longlong
_SZ = ctypes.c_size_t
_PSZ = ctypes.POINTER(ctypes.c_size_t)
_F = ctypes.c_float

SIGNATURES: dict[str, tuple[list, type]] = {
    "ticc_version": ([], _I),
    "ticc_kernel_launches": ([], _LL),
    "ticc_last_error": ([ctypes.c_char_p, _SZ], _I),
    "ticc_sym_inverse_workspace_size": ([_I, _I, _I, _PSZ], _I),
    "ticc_sym_inverse": ([_P, _I, _I, _I, _P, _SZ, _P, _P], _I),
    "ticc_sym_inverse_noalloc": ([_P, _I, _I, _I, _P, _P], _I),
    "ticc_debug_set_step_poll_limit": ([_LL], _I),
    "ticc_debug_tc_update_workspace_size": ([_I, _I, _PSZ], _I),
    "ticc_debug_tc_update": ([_P, _I, _I, _P, _P, _P, _I, _P, _SZ, _P, _P], _I),
    "ticc_ldmd_workspace_size": ([_I, _I, _I, _I, _I, _PSZ], _I),
    "ticc_ldmd_propagate": ([_P, _I, _P, _I, _D, _P, _P, _LL, _P, _LL, _P, _LL, _I, _I, _I, _P, _SZ, _P, _P], _I),
    "ticc_ldmd_reduced_blocks": ([_P, _SZ, _I, _I, _I, _I, _I, _I, _P, _P], _I),
    "ticc_ldmd_blocks_workspace_size": ([_I, _I, _I, _I, _I, _I, _PSZ], _I),
    "ticc_ldmd_propagate_blocks": ([_P, _I, _P, _I, _D, _P, _P, _LL, _P, _LL, _P, _LL, _LL, _I, _I, _I, _I, _P, _SZ, _P, _P], _I),
    "ticc_contract": ([_P, _P, ctypes.POINTER(_I), _I, _P, _I, _D, _P, _LL, _I, _I, _P, _P, _P, _D, _P, _P], _I),
    "ticc_contract_block": ([_P, _I, _P, _I, _I, _P, _LL, _I, _P, _P, _I, _I, _I, _P, _P], _I),
    "ticc_pairs_to_matrix": ([_P, _I, _LL, _I, _P, _P, _P, _I, _I, _P, _P], _I),
    "ticc_pes_legendre_grid": ([_P, _I, _P, _I, _P, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_D), ctypes.POINTER(_I), ctypes.POINTER(_D), _D, _P, _P], _I),
    "ticc_transform_workspace_size": ([_I, _I, _I, _PSZ], _I),
    "ticc_transform_bf_to_sf": ([_P, _P, _P, _I, _I, _I, _P, _SZ, _P], _I),
    "ticc_riccati_bessel_jy": ([_P, _P, _I, _P, _P, _P], _I),
    "ticc_bessel_k_logd": ([_P, _P, _I, _P, _P, _P], _I),
    "ticc_match_workspace_size": ([_I, _I, _I, _I, _PSZ], _I),
    "ticc_match_smatrix": ([_P, _I, _D, _P, _I, _D, _P, _P, _I, _I, _P, _P, _P, _SZ, _P, _P], _I),
    "ticc_mlp_shape": ([ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "ticc_step_features": ([_P, _LL, _P, _LL, _P, _LL, _P, _I, _I, _D, _D, _P, _P], _I),
    "ticc_mlp_forward": ([_P, _P, _P, _I, _P, _P], _I),
    "ticc_mlp_workspace_size": ([_I, _PSZ], _I),
    "ticc_mlp_gradient": ([_P, _P, _P, _P, _P, _I, _F, _F, _P, _P, _P, _SZ, _P], _I),
    "ticc_mlp_adam": ([_P, _P, _P, _I, _F, _F, _F, _F, _P], _I),
}

_lib = None
_lock = threading.Lock()


def load_library() -> ctypes.CDLL:
    """Load the CUDA library once; raise RuntimeError if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                message = f"CUDA library {LIB_PATH} is missing; build it with pyticc_b200._build.build()"
                logger.error(message)
                raise RuntimeError(message)
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (argtypes, restype) in SIGNATURES.items():
                function = getattr(lib, name)
                function.argtypes = argtypes
                function.restype = restype
            _lib = lib
    return _lib


def last_error() -> str:
    buffer = ctypes.create_string_buffer(512)
    load_library().ticc_last_error(buffer, 512)
    return buffer.value.decode()


def check(code: int, where: str) -> None:
    """Raise the reference's exception type for a failed C-ABI call."""
    if code == OK:
        return
    message = f"{where}: {last_error()}"
    logger.error(message)
    if code == ERR_INVALID_ARGUMENT:
        raise ValueError(message)
    if code == ERR_UNSUPPORTED:
        raise NotImplementedError(message)
    raise RuntimeError(message)


def require_cuda(device: torch.device | None = None) -> torch.device:
    """The CUDA device the kernels run on; raise if none is available."""
    if not torch.cuda.is_available():
        message = "pyticc_b200 needs a CUDA device (B200, sm_100a); none is available"
        logger.error(message)
        raise RuntimeError(message)
    return torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)


def stream_handle(device: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(tensor: torch.Tensor | None) -> ctypes.c_void_p | None:
    return None if tensor is None else ctypes.c_void_p(tensor.data_ptr())


def as_device(value, device: torch.device, dtype: torch.dtype) -> torch.Tensor:
    """Contiguous device tensor of the requested dtype (copies only when needed)."""
    if isinstance(value, torch.Tensor):
        return value.to(device=device, dtype=dtype).contiguous()
    array = np.array(value, copy=True, order="C")
    if np.iscomplexobj(array) and dtype == torch.float64:
        array = array.real
    return torch.as_tensor(array, device=device, dtype=dtype).contiguous()


class DeviceStatus:
    """int[4] device status word shared by the kernels of one call."""

    def __init__(self, device: torch.device) -> None:
        self.tensor = torch.zeros(4, dtype=torch.int32, device=device)

    @property
    def pointer(self) -> ctypes.c_void_p:
        return ptr(self.tensor)

    def raise_if_failed(self, where: str) -> None:
        code, item, detail, _ = (int(v) for v in self.tensor.cpu())
        if code == 0:
            return
        text = DEVICE_STATUS_TEXT.get(code, f"device status {code}")
        message = f"{where}: {text} (batch item {item}, detail {detail})"
        logger.error(message)
        if code == 4:
            raise ValueError(message)
        raise RuntimeError(message)


class Workspace:
    """Per-device cached scratch buffer, grown on demand (never shrunk)."""

    _buffers: dict[tuple[int, int], torch.Tensor] = {}

    @classmethod
    def get(cls, device: torch.device, nbytes: int, slot: int = 0) -> torch.Tensor:
        key = (device.index if device.index is not None else torch.cuda.current_device(), slot)
        buffer = cls._buffers.get(key)
        if buffer is None or buffer.numel() < nbytes:
            cls._buffers.pop(key, None)
            buffer = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)
            cls._buffers[key] = buffer
        return buffer

    @classmethod
    def release(cls) -> None:
        cls._buffers.clear()


def size_query(function, *args) -> int:
    out = ctypes.c_size_t(0)
    check(function(*args, ctypes.byref(out)), function.__name__)
    return int(out.value)
