"""dense_evolution -- B200-native dense statevector engine with the public API
of tatopenn-cell/Dense-Evolution's dense path (``DenseSVSimulator``,
``QASMParser``, Pauli observables, ``circuit_to_energy_fn``).

Every statevector lives in HBM as a torch CUDA tensor and every kernel is
hand-written CUDA for sm_100a in ``libdesv.so`` (``_lib/``), reached through a
C ABI (``include/desv.h``).  There is no CPU fallback.
"""
__version__ = "8.3.4+b200.1"

from .circuits.gates import GATES, PARAMETRIC_GATES, GATE_IDS
from .circuits.parser import QASMParser, QASMCircuit
from .circuits.compiler import QuantumTranspiler, CompiledCircuit
from .circuits.topology import entangling_layer, VALID_PATTERNS
from .circuits.random_circuit import random_circuit
from .backends.statevector import DenseSVSimulator
from .physics.observables import (pauli_expectation, pauli_sum_expectation, pauli_hamiltonian_to_matrix,
                                  pauli_sum_matvec, multiply_pauli_terms, pauli_sum_matvec_jax,
                                  pauli_sum_expectation_jax, PauliSumOperator)
from .utils.measurement import sample_counts, statevector_fidelity
from .solvers.autodiff import circuit_to_energy_fn
from .noise import NoiseModel, NoiseSpec
from . import config
from .config import set_precision


__all__ = ['DenseSVSimulator', 'QASMParser', 'QASMCircuit', 'QuantumTranspiler', 'CompiledCircuit', 'GATES',
           'PARAMETRIC_GATES', 'GATE_IDS', 'entangling_layer', 'VALID_PATTERNS', 'random_circuit',
           'pauli_expectation', 'pauli_sum_expectation', 'pauli_hamiltonian_to_matrix', 'pauli_sum_matvec',
           'multiply_pauli_terms', 'pauli_sum_matvec_jax', 'pauli_sum_expectation_jax', 'PauliSumOperator',
           'sample_counts', 'statevector_fidelity', 'circuit_to_energy_fn', 'set_precision', 'NoiseModel',
           'NoiseSpec', 'config', '__version__']
