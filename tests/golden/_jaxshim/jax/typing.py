"""Type aliases for the NumPy-backed ``jax`` stand-in (test infrastructure only)."""

from numpy.typing import DTypeLike  # noqa: F401
