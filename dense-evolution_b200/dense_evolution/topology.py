"""Flat import path kept from the reference (``dense_evolution/topology.py``)."""
from .circuits.topology import entangling_layer, VALID_PATTERNS  # noqa: F401
