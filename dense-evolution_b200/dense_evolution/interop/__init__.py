"""Interop with Qiskit / PennyLane (the reference's dense_evolution.interop)."""
from .qiskit_pennylane import (_to_qiskit_bit_order, from_pennylane, from_qiskit, run_qiskit_circuit,
                               to_little_endian)

__all__ = ['from_qiskit', 'from_pennylane', 'run_qiskit_circuit', 'to_little_endian', '_to_qiskit_bit_order']
