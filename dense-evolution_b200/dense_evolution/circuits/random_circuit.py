"""Seeded random circuits (the reference's ``circuits/random_circuit.py:15-85``).

The generator makes the same NumPy ``Generator`` draws in the same order as
the reference -- per gate: a ``random()`` for the 1q/2q choice (only when both
pools are non-empty), an ``integers`` for the gate name, then either
``choice(n, 2, replace=False)`` or ``integers(n)`` (+ ``uniform(0, 2pi)`` for
rx/ry/rz) -- so a seed yields the same circuit in both libraries.
"""
import numpy as np

__all__ = ['random_circuit']

_1Q_STATIC = ('h', 'x', 'y', 'z', 's', 'sdg', 't', 'tdg', 'sx')
_1Q_PARAMETRIC = ('rx', 'ry', 'rz')
_2Q_STATIC = ('cx', 'cz', 'cy', 'swap')
_KNOWN = frozenset(_1Q_STATIC + _1Q_PARAMETRIC + _2Q_STATIC)


def random_circuit(n_qubits, n_gates, seed=None, gate_set=None, two_qubit_prob=0.4):
    if n_qubits < 1:
        raise ValueError(f"random_circuit needs at least 1 qubit, got {n_qubits}")
    if n_gates < 0:
        raise ValueError(f"n_gates must be >= 0, got {n_gates}")
    if not 0.0 <= two_qubit_prob <= 1.0:
        raise ValueError(f"two_qubit_prob must be in [0, 1], got {two_qubit_prob}")
    rng = seed if isinstance(seed, np.random.Generator) else np.random.default_rng(seed)
    if gate_set is None:
        singles = list(_1Q_STATIC) + list(_1Q_PARAMETRIC)
        doubles = list(_2Q_STATIC) if n_qubits >= 2 else []
    else:
        gate_set = list(gate_set)
        bad = set(gate_set) - _KNOWN
        if bad:
            raise ValueError(f"unknown gate name(s) in gate_set: {sorted(bad)}")
        singles = [g for g in gate_set if g in _1Q_STATIC] + [g for g in gate_set if g in _1Q_PARAMETRIC]
        doubles = [g for g in gate_set if g in _2Q_STATIC]
    if not singles and not doubles:
        raise ValueError("gate_set leaves no usable gates for this n_qubits")
    ops = []
    for _ in range(n_gates):
        two = bool(doubles) and n_qubits >= 2 and (not singles or rng.random() < two_qubit_prob)
        if two:
            name = doubles[rng.integers(len(doubles))]
            a, b = rng.choice(n_qubits, size=2, replace=False)
            ops.append((name, int(a), int(b)))
        else:
            name = singles[rng.integers(len(singles))]
            q = int(rng.integers(n_qubits))
            if name in _1Q_PARAMETRIC:
                ops.append((name, q, float(rng.uniform(0, 2 * np.pi))))
            else:
                ops.append((name, q))
    return ops
