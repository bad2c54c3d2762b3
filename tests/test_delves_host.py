"""Host pieces of the Delves propagation: the hyperradial mass and the exact hard-wall
log-derivative (reference propagation/delves.py:197-236, matrix/delves/geometry.py:14-50)."""

from __future__ import annotations

import numpy as np
import pytest

from pyticc_b200.propagation.delves import delves_reduced_mass, hard_wall_logD


def test_reduced_mass_is_the_three_body_hyperradial_mass():
    assert delves_reduced_mass((1.0, 2.0, 19.0)) == pytest.approx(np.sqrt(38.0 / 22.0), rel=1e-15)
    with pytest.raises(ValueError):
        delves_reduced_mass((1.0, -2.0, 3.0))


def test_hard_wall_branches():
    mu, w = 3.0, 0.1
    eps = np.array([1.0, 0.2, 0.5 + 1e-14])
    E = np.array([0.5])
    Y = hard_wall_logD(E, mu, eps, w)
    assert Y.shape == (1, 3, 3) and np.count_nonzero(Y - np.diag(np.diag(Y[0]))[None]) == 0
    p = np.sqrt(2 * mu * (1.0 - 0.5))
    q = np.sqrt(2 * mu * (0.5 - 0.2))
    assert Y[0, 0, 0] == pytest.approx(p / np.tanh(p * w), rel=1e-14)
    assert Y[0, 1, 1] == pytest.approx(q / np.tan(q * w), rel=1e-14)
    assert Y[0, 2, 2] == pytest.approx(1.0 / w, rel=1e-10)
