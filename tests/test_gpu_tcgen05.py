"""The tcgen05 TF32x3 trailing-update tile (TMA-fed, TMEM-accumulated) against FP64.

C <- C - A^T B on 128 x 128 tiles with A, B given as FP32 panels, split in shared memory
as hi + lo TF32 words, and the three products hi*hi + hi*lo + lo*hi accumulated in FP32: the error must stay at the FP32 level
(bound: 1e-5 of sum |a||b| per element, mean relative error below 2e-6, far from the 1e-3
of a single TF32 product), untouched tiles must not change, and a diagonal tile must come
out exactly symmetric (lower half mirrored).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from pyticc_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _run(M, cold, U, tiles):
    lib = nat.load_library()
    dev = nat.require_cuda()
    batch, np_, _ = M.shape
    Mt = torch.as_tensor(M, device=dev).contiguous()
    ct = torch.as_tensor(cold, device=dev).contiguous()
    ut = torch.as_tensor(U, device=dev).contiguous()
    tt = torch.as_tensor(np.asarray(tiles, dtype=np.int32).reshape(-1), device=dev)
    nbytes = nat.size_query(lib.ticc_debug_tc_update_workspace_size, np_, batch)
    work = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    status = nat.DeviceStatus(dev)
    nat.check(lib.ticc_debug_tc_update(nat.ptr(Mt), np_, batch, nat.ptr(ct), nat.ptr(ut), nat.ptr(tt), len(tiles), nat.ptr(work), nbytes, status.pointer, nat.stream_handle(dev)), "ticc_debug_tc_update")
    status.raise_if_failed("ticc_debug_tc_update")
    return Mt.cpu().numpy()


def _expected(M, cold, U, tiles):
    out = M.copy()
    bound = np.zeros_like(M)
    for b, ta, tb in tiles:
        rs, cs = slice(128 * ta, 128 * ta + 128), slice(128 * tb, 128 * tb + 128)
        out[b, rs, cs] = M[b, rs, cs] - cold[b][:, rs].T @ U[b][:, cs]
        bound[b, rs, cs] = np.abs(cold[b][:, rs]).T @ np.abs(U[b][:, cs])
        if ta == tb:
            block = out[b, rs, cs]
            out[b, rs, cs] = np.tril(block) + np.tril(block, -1).T
            bb = bound[b, rs, cs]
            bound[b, rs, cs] = np.tril(bb) + np.tril(bb, -1).T
    return out, bound


@pytest.mark.parametrize("np_,batch", [(256, 1), (512, 2)])
def test_tcgen05_update_tiles_match_fp64(np_, batch):
    rng = np.random.default_rng(np_ + batch)
    M = rng.normal(size=(batch, np_, np_))
    cold = rng.normal(size=(batch, 128, np_))
    U = rng.normal(size=(batch, 128, np_)) * np.exp(rng.uniform(-3, 3, size=(batch, 128, 1)))
    nt = np_ // 128
    tiles = [(b, ta, tb) for b in range(batch) for ta in range(nt) for tb in range(nt) if (ta + tb + b) % 2 == 0 or ta == tb]
    got = _run(M, cold, U, tiles)
    want, bound = _expected(M, cold, U, tiles)
    err = np.abs(got - want)
    assert np.all(err <= 1e-5 * bound + 1e-12), float((err / (bound + 1e-300)).max())
    touched = bound > 0
    rel = err[touched] / bound[touched]
    assert rel.mean() < 2e-6, rel.mean()
    np.testing.assert_array_equal(got[~touched], M[~touched])
    for b, ta, tb in tiles:
        if ta == tb:
            block = got[b, 128 * ta : 128 * ta + 128, 128 * tb : 128 * tb + 128]
            np.testing.assert_array_equal(block, block.T)


def test_tcgen05_update_repeats_on_the_same_ctas():
    """More tiles than SMs: every CTA runs several units, so barrier phases, the stage ring
    and the TMEM accumulator are reused across tiles."""
    rng = np.random.default_rng(3)
    batch, np_ = 20, 512
    M = rng.normal(size=(batch, np_, np_))
    cold = rng.normal(size=(batch, 128, np_))
    U = rng.normal(size=(batch, 128, np_))
    tiles = [(b, ta, tb) for b in range(batch) for ta in range(4) for tb in range(ta + 1)]
    got = _run(M, cold, U, tiles)
    want, bound = _expected(M, cold, U, tiles)
    assert np.all(np.abs(got - want) <= 1e-5 * bound + 1e-12)
