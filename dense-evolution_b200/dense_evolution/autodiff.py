"""Flat import path kept from the reference (``dense_evolution/autodiff.py``)."""
from .solvers.autodiff import circuit_to_energy_fn  # noqa: F401
