"""Seeded synthetic workloads of the engine's benchmarks and tests.

* ``brick_u3_circuit`` -- U3(theta, phi, lambda) on every qubit, angles i.i.d.
  U[0, 2pi) drawn in gate order, then a brick wall of CZ on (2i, 2i+1) in even
  layers and (2i+1, 2i+2) in odd layers (the ``'brick'`` halves of the
  reference's ``entangling_layer``, circuits/topology.py:71-74).
* ``hea_circuit`` -- hardware-efficient ansatz: per layer RY then RZ on every
  qubit, then CX(i, i+1); parameter index l*2n + 2q (+1 for RZ).
* ``tfim_terms`` / ``xxz_terms`` / ``xxx_terms`` -- open-chain Hamiltonians as
  (coefficient, {qubit: letter}) Pauli terms.
"""
from __future__ import annotations

import numpy as np


def brick_u3_circuit(n: int, layers: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    ops = []
    for layer in range(layers):
        for q in range(n):
            th, ph, lam = rng.uniform(0.0, 2 * np.pi, 3)
            ops.append(('u3', q, float(th), float(ph), float(lam)))
        for a in range(layer % 2, n - 1, 2):
            ops.append(('cz', a, a + 1))
    return ops


def hea_circuit(n: int, layers: int, theta=None):
    """Gate tuples of the ansatz; theta (length 2*n*layers) or zeros."""
    theta = np.zeros(2 * n * layers) if theta is None else np.asarray(theta, dtype=np.float64)
    ops, k = [], 0
    for _ in range(layers):
        for q in range(n):
            ops.append(('ry', q, float(theta[k])))
            ops.append(('rz', q, float(theta[k + 1])))
            k += 2
        for q in range(n - 1):
            ops.append(('cx', q, q + 1))
    return ops


def hea_qasm(n: int, layers: int, theta=None) -> str:
    theta = np.zeros(2 * n * layers) if theta is None else np.asarray(theta, dtype=np.float64)
    lines = ['OPENQASM 2.0;', 'include "qelib1.inc";', f'qreg q[{n}];']
    k = 0
    for _ in range(layers):
        for q in range(n):
            lines.append(f'ry({float(theta[k])!r}) q[{q}];')
            lines.append(f'rz({float(theta[k + 1])!r}) q[{q}];')
            k += 2
        for q in range(n - 1):
            lines.append(f'cx q[{q}],q[{q + 1}];')
    return '\n'.join(lines)


def tfim_terms(n: int, h: float = 1.0):
    """H = -sum_i Z_i Z_{i+1} - h sum_i X_i (open chain)."""
    t = [(-1.0, {i: 'Z', i + 1: 'Z'}) for i in range(n - 1)]
    return t + [(-h, {i: 'X'}) for i in range(n)]


def xxz_terms(n: int, jz: float, jxy: float = 1.0):
    """H = sum_i [jxy (X_i X_{i+1} + Y_i Y_{i+1}) + jz Z_i Z_{i+1}] (open chain)."""
    t = []
    for i in range(n - 1):
        t += [(jxy, {i: 'X', i + 1: 'X'}), (jxy, {i: 'Y', i + 1: 'Y'}), (jz, {i: 'Z', i + 1: 'Z'})]
    return t


def xxx_terms(n: int):
    return xxz_terms(n, 1.0, 1.0)
