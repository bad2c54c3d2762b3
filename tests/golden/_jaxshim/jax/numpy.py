"""NumPy forwarding module standing in for ``jax.numpy`` (test infrastructure only)."""

from __future__ import annotations

import numpy as _np

from . import _wrap


class _Linalg:
    def __getattr__(self, name):
        function = getattr(_np.linalg, name)
        return lambda *args, **kwargs: _wrap(function(*args, **kwargs))


linalg = _Linalg()


def asarray(value, dtype=None):
    return _wrap(_np.array(value, dtype=dtype, copy=False) if dtype is None else _np.asarray(value, dtype=dtype))


def zeros(shape, dtype=None, device=None):
    return _wrap(_np.zeros(shape, dtype=dtype))


def __getattr__(name):
    attribute = getattr(_np, name)
    if callable(attribute) and not isinstance(attribute, type):
        return lambda *args, **kwargs: _wrap(attribute(*args, **kwargs))
    return attribute
