"""NumPy-backed stand-in for the small part of ``jax`` that PyTICC touches.

Test infrastructure only: it lets ``tests/golden/make_golden.py`` import the
unmodified reference package in a container where JAX is not installed, so that
golden input/output vectors can be generated from the reference's own code.
Nothing in the product imports this package.

Semantics: ``jit`` is the identity, ``vmap`` and ``lax.scan`` are Python loops,
``device_put`` converts to an ndarray subclass that supports ``.at[...]``
updates, and a single fake CPU device exists.
"""

from __future__ import annotations

import types

import numpy as np


class _AtUpdater:
    def __init__(self, array: "Array", index) -> None:
        self._array = array
        self._index = index

    def add(self, values):
        out = np.array(self._array, copy=True)
        np.add.at(out, self._index, values) if _is_fancy(self._index) else out.__setitem__(self._index, out[self._index] + values)
        return out.view(Array)

    def set(self, values):
        out = np.array(self._array, copy=True)
        out[self._index] = values
        return out.view(Array)


def _is_fancy(index) -> bool:
    if not isinstance(index, tuple):
        index = (index,)
    return any(isinstance(item, np.ndarray) and item.ndim > 0 for item in index)


class _AtIndexer:
    def __init__(self, array: "Array") -> None:
        self._array = array

    def __getitem__(self, index) -> _AtUpdater:
        return _AtUpdater(self._array, index)


class _Device:
    def __init__(self, platform: str, index: int) -> None:
        self.platform = platform
        self.id = index

    def __repr__(self) -> str:
        return f"FakeDevice({self.platform}:{self.id})"


_CPU = _Device("cpu", 0)


class Array(np.ndarray):
    """ndarray subclass standing in for ``jax.Array``."""

    @property
    def at(self) -> _AtIndexer:
        return _AtIndexer(self)

    def block_until_ready(self) -> "Array":
        return self

    def devices(self) -> set:
        return {_CPU}

    def copy(self, *args, **kwargs) -> "Array":
        return np.array(self, copy=True).view(Array)


def _wrap(value):
    if isinstance(value, np.ndarray) and not isinstance(value, Array):
        return value.view(Array)
    if isinstance(value, tuple):
        return tuple(_wrap(item) for item in value)
    if isinstance(value, list):
        return [_wrap(item) for item in value]
    return value


def device_put(value, device=None):
    return np.array(value, copy=True).view(Array) if isinstance(value, np.ndarray) or np.isscalar(value) or isinstance(value, (list, tuple)) else value


def devices(platform: str | None = None):
    if platform in (None, "cpu"):
        return [_CPU]
    raise RuntimeError(f"Unknown backend {platform}")


def jit(function=None, **kwargs):
    if function is None:
        return lambda f: f
    return function


def _take(value, axis, index):
    if axis is None:
        return value
    return np.take(np.asarray(value), index, axis=axis)


def vmap(function, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        sizes = {np.asarray(arg).shape[axis] for arg, axis in zip(args, axes, strict=True) if axis is not None}
        (size,) = sizes
        results = [function(*(_wrap(_take(arg, axis, i)) for arg, axis in zip(args, axes, strict=True))) for i in range(size)]
        if isinstance(results[0], tuple):
            return tuple(_wrap(np.stack([np.asarray(r[k]) for r in results])) for k in range(len(results[0])))
        return _wrap(np.stack([np.asarray(r) for r in results]))

    return mapped


class _Config:
    def __init__(self) -> None:
        self._values = {"jax_enable_x64": True}

    def update(self, name, value) -> None:
        self._values[name] = value

    def read(self, name):
        return self._values.get(name)


config = _Config()


def _scan(function, init, xs, length=None):
    carry = init
    if isinstance(xs, tuple):
        n = np.asarray(xs[0]).shape[0]
        slices = [tuple(_wrap(np.asarray(x)[i]) for x in xs) for i in range(n)]
    else:
        n = np.asarray(xs).shape[0]
        slices = [_wrap(np.asarray(xs)[i]) for i in range(n)]
    outputs = []
    for item in slices:
        carry, out = function(carry, item)
        outputs.append(out)
    if outputs and outputs[0] is not None:
        return carry, _wrap(np.stack([np.asarray(o) for o in outputs]))
    return carry, None


lax = types.SimpleNamespace(scan=_scan)

from . import numpy  # noqa: E402
from . import typing  # noqa: E402

__all__ = ["Array", "config", "device_put", "devices", "jit", "lax", "numpy", "typing", "vmap"]
