"""Process-wide precision control: the reference's ``dense_evolution.config``
(``dense_evolution/config.py:29-62``: ``set_precision``, ``ensure_x64``,
``with_x64``) for code written against it.

The reference switches JAX's process-wide ``jax_enable_x64`` flag; with x64
off its complex128 states silently become complex64.  This engine has no JAX:
precision is a property of each simulator / energy function.  The flag kept
here plays the same role for the constructors that are not told a precision
(``DenseSVSimulator(n)``, ``circuit_to_energy_fn(circ, n)``): with float64 on
(the default) they use complex128, after an explicit ``set_precision(False)``
complex64.  ``ensure_x64()`` turns float64 back on unless a caller chose
explicitly, exactly as in the reference.
"""
from __future__ import annotations

import functools

_float64 = True
_explicit = False


def set_precision(float64: bool = True) -> None:
    """Choose the default precision explicitly; later ensure_x64() calls then
    leave the choice alone."""
    global _float64, _explicit
    _float64 = bool(float64)
    _explicit = True


def ensure_x64() -> None:
    """Turn float64 on unless set_precision() chose explicitly."""
    global _float64
    if not _explicit:
        _float64 = True


def with_x64(fn):
    """Wrap fn so ensure_x64() runs before every call."""
    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        ensure_x64()
        return fn(*args, **kwargs)
    return wrapper


def float64_enabled() -> bool:
    """The current default: True -> complex128, False -> complex64."""
    return _float64


def default_use_float32(use_float32) -> bool:
    """Resolve a constructor's ``use_float32`` argument (None: the default)."""
    return (not _float64) if use_float32 is None else bool(use_float32)
