"""Flat import path kept from the reference (``dense_evolution/random_circuit.py``)."""
from .circuits.random_circuit import random_circuit  # noqa: F401
