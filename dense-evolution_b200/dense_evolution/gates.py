"""Flat import path kept from the reference (``dense_evolution/gates.py``)."""
from .circuits.gates import GATES, PARAMETRIC_GATES, GATE_IDS, INV2  # noqa: F401
