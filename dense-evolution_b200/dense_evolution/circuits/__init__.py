from .gates import GATES, PARAMETRIC_GATES, GATE_IDS
from .parser import QASMParser, QASMCircuit
from .compiler import QuantumTranspiler, CompiledCircuit
from .topology import entangling_layer, VALID_PATTERNS
from .random_circuit import random_circuit
