"""Flat import path kept from the reference (``dense_evolution/parser.py``)."""
from .circuits.parser import QASMParser, QASMCircuit  # noqa: F401
