"""The allocation-free inversion entry point against the workspace one.

Some callers cannot allocate device memory (plugin hosts that pass only their own buffers,
runtimes that fix their device memory budget at start-up, C/Fortran drivers without a
device allocator);
``ticc_sym_inverse_noalloc`` serves them from a fixed device array inside the library.
This file is collected last on purpose: it must pass both alone in a fresh process and
after every other test has used the library.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from pyticc_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _with_workspace(A: np.ndarray, is_complex: bool) -> np.ndarray:
    lib = nat.load_library()
    dev = nat.require_cuda()
    t = torch.as_tensor(A, device=dev).contiguous()
    nbytes = nat.size_query(lib.ticc_sym_inverse_workspace_size, A.shape[-1], A.shape[0], int(is_complex))
    work = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    status = nat.DeviceStatus(dev)
    nat.check(lib.ticc_sym_inverse(nat.ptr(t), A.shape[-1], A.shape[0], int(is_complex), nat.ptr(work), nbytes, status.pointer, nat.stream_handle(dev)), "ticc_sym_inverse")
    status.raise_if_failed("ticc_sym_inverse")
    return t.cpu().numpy()


def _no_alloc(A: np.ndarray, is_complex: bool) -> np.ndarray:
    lib = nat.load_library()
    dev = nat.require_cuda()
    t = torch.as_tensor(A, device=dev).contiguous()
    status = nat.DeviceStatus(dev)
    nat.check(lib.ticc_sym_inverse_noalloc(nat.ptr(t), A.shape[-1], A.shape[0], int(is_complex), status.pointer, nat.stream_handle(dev)), "ticc_sym_inverse_noalloc")
    status.raise_if_failed("ticc_sym_inverse_noalloc")
    return t.cpu().numpy()


def _matrices(seed: int, n: int, batch: int, is_complex: bool) -> np.ndarray:
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(batch, n, n))
    if is_complex:
        A = A + 1j * rng.normal(size=(batch, n, n))
    A = A + A.transpose(0, 2, 1) + np.diag(rng.uniform(3.0, 6.0, n) * np.sqrt(n) * np.sign(rng.normal(size=n)))
    return A


@pytest.mark.parametrize("is_complex", [False, True])
def test_no_alloc_inverse_matches_workspace_inverse_on_two_calls(is_complex):
    # 300 and 200: several pivot blocks (fused sweep steps); 100: one pivot block (real) or
    # two (complex); 40: the 64-wide single-block inversion (real) or one 128 block (complex)
    for call, (n, batch) in enumerate([(300, 3), (200, 2), (100, 4), (40, 3)]):
        A = _matrices(10 + call, n, batch, is_complex)
        want = _with_workspace(A, is_complex)
        got = _no_alloc(A, is_complex)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-13 * np.abs(want).max())
        np.testing.assert_allclose(got, np.linalg.inv(A), rtol=0, atol=1e-12 * np.abs(want).max())


def test_no_alloc_rejects_requests_beyond_its_fixed_scratch():
    lib = nat.load_library()
    dev = nat.require_cuda()
    t = torch.zeros(1, dtype=torch.float64, device=dev)
    code = lib.ticc_sym_inverse_noalloc(nat.ptr(t), 4096, 4, 0, None, nat.stream_handle(dev))
    assert code == nat.ERR_INVALID_ARGUMENT
    assert "fixed device array holds" in nat.last_error()
