"""Flat import path kept from the reference (``dense_evolution/compiler.py``)."""
from .circuits.compiler import QuantumTranspiler  # noqa: F401
