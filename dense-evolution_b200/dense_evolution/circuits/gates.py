"""Gate tables of the drop-in API (same names and values as the reference's
``dense_evolution/circuits/gates.py:11-91``).

Matrices act on the gate's qubits in argument order with the FIRST qubit as
the most significant bit of the row index (``apply_gate_2q`` convention,
``backends/statevector.py:188-203``).  They are plain complex128 NumPy arrays;
the engine builds every device matrix from them on the host in FP64.
"""
import numpy as np

INV2 = 1.0 / np.sqrt(2.0)


def _m(rows):
    return np.array(rows, dtype=np.complex128)


_E4 = np.exp(0.25j * np.pi)

GATES = {
    'h': INV2 * _m([[1, 1], [1, -1]]),
    'x': _m([[0, 1], [1, 0]]),
    'y': _m([[0, -1j], [1j, 0]]),
    'z': _m([[1, 0], [0, -1]]),
    's': _m([[1, 0], [0, 1j]]),
    'sdg': _m([[1, 0], [0, -1j]]),
    't': _m([[1, 0], [0, _E4]]),
    'tdg': _m([[1, 0], [0, np.conj(_E4)]]),
    'sx': 0.5 * _m([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]]),
    'id': np.eye(2, dtype=np.complex128),
    'cx': _m([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]]),
    'cz': np.diag([1, 1, 1, -1]).astype(np.complex128),
    'cy': _m([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, -1j], [0, 0, 1j, 0]]),
    'swap': _m([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]]),
    'iswap': _m([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]]),
    'ecr': INV2 * _m([[0, 0, 1, 1j], [0, 0, 1j, 1], [1, -1j, 0, 0], [-1j, 1, 0, 0]]),
    'ccx': np.eye(8, dtype=np.complex128)[[0, 1, 2, 3, 4, 5, 7, 6]],
}

# Integer ids of the compiled path (1-qubit: 0..14, 2-qubit: 20..25; 23 =
# swap is reserved and never dispatched because transpile() decomposes it).
GATE_IDS = {
    'id': 0, 'h': 1, 'x': 2, 'y': 3, 'z': 4, 's': 5, 'sdg': 6, 't': 7, 'tdg': 8,
    'rx': 9, 'ry': 10, 'rz': 11,
    'p': 12, 'u1': 12, 'phase': 12,
    'sx': 13,
    'gphase': 14,
    'cx': 20, 'cz': 21, 'cp': 22, 'cphase': 22,
    'cy': 24, 'crz': 25,
}

_TWO_QUBIT_PARAMETRIC_GATES = frozenset(('cp', 'cphase', 'crz'))


def _rx(theta):
    c, s = np.cos(theta / 2), np.sin(theta / 2)
    return _m([[c, -1j * s], [-1j * s, c]])


def _ry(theta):
    c, s = np.cos(theta / 2), np.sin(theta / 2)
    return _m([[c, -s], [s, c]])


def _rz(theta):
    return _m([[np.exp(-0.5j * theta), 0], [0, np.exp(0.5j * theta)]])


def _phase(lam):
    return _m([[1, 0], [0, np.exp(1j * lam)]])


def _u3(theta, phi, lam):
    c, s = np.cos(theta / 2), np.sin(theta / 2)
    return _m([[c, -np.exp(1j * lam) * s], [np.exp(1j * phi) * s, np.exp(1j * (phi + lam)) * c]])


PARAMETRIC_GATES = {
    'rx': _rx,
    'ry': _ry,
    'rz': _rz,
    'cp': lambda lam: np.diag([1, 1, 1, np.exp(1j * lam)]).astype(np.complex128),
    'crz': lambda theta: np.diag([1, 1, np.exp(-0.5j * theta), np.exp(0.5j * theta)]).astype(np.complex128),
    'u3': _u3,
    'u2': lambda phi, lam: INV2 * _m([[1, -np.exp(1j * lam)], [np.exp(1j * phi), np.exp(1j * (phi + lam))]]),
    'u1': _phase,
    'p': _phase,
    'gphase': lambda alpha: np.exp(1j * alpha) * np.eye(2, dtype=np.complex128),
}

__all__ = ['GATES', 'GATE_IDS', 'PARAMETRIC_GATES', 'INV2']
