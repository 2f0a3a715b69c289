"""Flat import path kept from the reference (``dense_evolution/measurement.py``)."""
from .utils.measurement import sample_counts, statevector_fidelity  # noqa: F401
