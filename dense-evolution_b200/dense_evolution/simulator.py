"""Flat import path kept from the reference (``dense_evolution/simulator.py``)."""
from .backends.statevector import DenseSVSimulator  # noqa: F401
