"""Learned sector widths on the GPU: feature kernel, MLP forward / gradient / Adam against
the CPU oracle, training, and what the trained proposer gains over the fixed grid."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import learned as oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from pyticc_b200 import _native as nat

    return nat.require_cuda()


def _random_params(rng, scale=0.4):
    from pyticc_b200.propagation.learned import N_PARAM

    return (rng.standard_normal(N_PARAM) * scale).astype(np.float32)


def test_library_shape_matches_host_constants():
    from pyticc_b200.propagation.learned import N_FEATURE, N_HIDDEN, N_PARAM, library_shape

    assert library_shape() == (N_FEATURE, N_HIDDEN, N_PARAM)


@pytest.mark.parametrize("n", [1, 37, 300])
def test_features_match_oracle(dev, n):
    import ctypes

    from pyticc_b200 import _native as nat

    rng = np.random.default_rng(n)
    n_sector = 5
    points = rng.standard_normal((2 * n_sector + 1, n, n))
    points = 0.5 * (points + points.transpose(0, 2, 1))
    points[:, np.arange(n), np.arange(n)] += np.linspace(-3.0, 40.0, n)
    h = rng.uniform(0.01, 0.1, n_sector)
    W = torch.as_tensor(points, device=dev)
    hd = torch.as_tensor(h, device=dev)
    out = torch.empty((n_sector, 8), dtype=torch.float32, device=dev)
    lib = nat.load_library()
    stride = 2 * n * n
    nat.check(lib.ticc_step_features(nat.ptr(W[0::2]), stride, nat.ptr(W[1::2]), stride, nat.ptr(W[2::2]), stride, nat.ptr(hd), n_sector, n, 7.5, 0.25, nat.ptr(out), nat.stream_handle(dev)), "features")
    expect = oracle.step_features(points[0:-1:2], points[1::2], points[2::2], h, 7.5, 0.25)
    if n == 1:
        expect[:, 5] = -30.0  # no off-diagonal element: log10(0 + 1e-30)
    np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=2e-6, atol=2e-6)


def test_forward_matches_oracle(dev):
    from pyticc_b200.propagation.learned import StepProposer

    rng = np.random.default_rng(1)
    X = rng.standard_normal((1000, 8)).astype(np.float32) * 3.0
    proposer = StepProposer.initialize(X, seed=3)
    proposer.params = _random_params(rng)
    y = proposer.predict(torch.as_tensor(X, device=dev)).cpu().numpy()
    expect, _ = oracle.forward(proposer.params, proposer.norm, X)
    np.testing.assert_allclose(y, expect, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("n", [1, 127, 1000])
def test_gradient_matches_oracle(dev, n):
    from pyticc_b200.propagation.learned import StepProposer

    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, 8)).astype(np.float32)
    T = rng.uniform(0.0, 6.0, n).astype(np.float32)
    Wt = rng.uniform(0.5, 2.0, n).astype(np.float32)
    proposer = StepProposer.initialize(X if n > 1 else np.vstack([X, X + 1]), seed=5)
    proposer.params = _random_params(rng)
    loss, grads = proposer.gradient(torch.as_tensor(X, device=dev), torch.as_tensor(T, device=dev), torch.as_tensor(Wt, device=dev), over_weight=4.0)
    exp_loss, exp_grads = oracle.loss_and_gradient(proposer.params, proposer.norm, X, T, Wt, 4.0, 1.0 / float(Wt.astype(np.float32).sum()))
    assert loss == pytest.approx(exp_loss, rel=2e-4)
    g = grads.cpu().numpy()
    scale = np.abs(exp_grads).max()
    np.testing.assert_allclose(g, exp_grads, rtol=0, atol=2e-4 * scale)


def test_adam_step_matches_oracle(dev):
    import ctypes

    from pyticc_b200 import _native as nat
    from pyticc_b200.propagation.learned import N_PARAM

    rng = np.random.default_rng(7)
    p = rng.standard_normal(N_PARAM).astype(np.float32)
    g = rng.standard_normal(N_PARAM).astype(np.float32)
    m = rng.standard_normal(N_PARAM).astype(np.float32) * 0.1
    v = rng.uniform(0.0, 0.1, N_PARAM).astype(np.float32)
    P = torch.as_tensor(p, device=dev)
    moments = torch.as_tensor(np.concatenate([m, v]), device=dev)
    lib = nat.load_library()
    nat.check(lib.ticc_mlp_adam(nat.ptr(P), nat.ptr(torch.as_tensor(g, device=dev)), nat.ptr(moments), 3, 1e-2, 0.9, 0.999, 1e-8, nat.stream_handle(dev)), "adam")
    ep, em, ev = oracle.adam(p.astype(np.float64), g, m, v, 3, 1e-2, 0.9, 0.999, 1e-8)
    np.testing.assert_allclose(P.cpu().numpy(), ep, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(moments.cpu().numpy(), np.concatenate([em, ev]), rtol=1e-5, atol=1e-7)


def test_training_fits_a_smooth_target(dev):
    from pyticc_b200.propagation.learned import train_proposer

    rng = np.random.default_rng(11)
    X = rng.standard_normal((4000, 8)).astype(np.float32)
    T = (3.0 + 1.5 * np.tanh(X[:, 0] - 0.5 * X[:, 3]) + 0.5 * X[:, 6]).astype(np.float32)
    proposer, history = train_proposer(X, T, steps=1500, lr=3e-3)
    assert history[-1] < 0.02 * history[0]
    y = proposer.predict(torch.as_tensor(X, device=dev)).cpu().numpy()
    assert np.sqrt(np.mean((y - T) ** 2)) < 0.15


def test_learned_schedule_gains_over_fixed_grid(dev):
    """Capture from 8 to 300 bohr at ultracold energies: the proposer, trained on step-doubling
    labels of two energies, merges long-range sectors for two held-out energies (about
    2.3x fewer sectors), and the fixed-step solve accepts the result (max|dS| <= 1e-6)."""
    from pyticc_b200 import Propagation
    from pyticc_b200.propagation.learned import training_set, train_proposer, validate_learned
    from pyticc_b200.scattering import hamiltonian_for
    from pyticc_b200.workloads import ultracold_capture

    wl = ultracold_capture(jmax=6, J=1, parity=-1, boundaries=(8.0, 300.0), n_energy=6)
    config = Propagation(mode="capture")
    hamiltonian = hamiltonian_for(wl.system, wl.grid)
    X, T = training_set([(hamiltonian, wl.grid.sectors, wl.energies[[0, 5]], config)], max_level=8)
    proposer, history = train_proposer(X, T, steps=2000)
    assert history[-1] < 0.25 * history[0]
    accepted, dS, n_fixed, n_learned, _ = validate_learned(wl.system, wl.energies[[2, 3]], wl.grid, config, proposer)
    print(f"fixed sectors {n_fixed}, learned {n_learned}, max|dS| {dS:.2e}")
    assert accepted and dS <= 1e-6
    assert n_learned < n_fixed / 1.8
