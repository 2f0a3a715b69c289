"""Flat import path kept from the reference (``dense_evolution/random_circuit.py``).

Importing this submodule rebinds ``dense_evolution.random_circuit`` to the
module object; the module is therefore made callable so that
``dense_evolution.random_circuit(...)`` keeps working either way."""
import sys
import types

from .circuits.random_circuit import random_circuit  # noqa: F401


class _CallableModule(types.ModuleType):
    def __call__(self, *args, **kwargs):
        return random_circuit(*args, **kwargs)


sys.modules[__name__].__class__ = _CallableModule
