"""Flat import path kept from the reference (``dense_evolution/observables.py``)."""
from .physics.observables import pauli_expectation, pauli_sum_expectation, pauli_hamiltonian_to_matrix, pauli_sum_matvec, multiply_pauli_terms, pauli_sum_matvec_jax, pauli_sum_expectation_jax, PauliSumOperator  # noqa: F401
