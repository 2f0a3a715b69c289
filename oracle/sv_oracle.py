"""CPU oracle for the dense statevector path -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its ``cpu_baseline`` leg and its
``--impl reference`` arm) may import it.  The shipped package never imports
it, and it never stands in for a missing CUDA extension.

It restates, in plain NumPy complex128, the algorithm of the reference's CPU
("eager") path of tatopenn-cell/Dense-Evolution v8.3.4:

* gate tables -- ``dense_evolution/circuits/gates.py:33-91``
* transpiler decompositions -- ``dense_evolution/circuits/compiler.py:369-488``
* 1-/2-qubit gate application by tensor contraction, MSB-first qubit order --
  ``dense_evolution/backends/statevector.py:167-203``
* circuit dispatch by gate name -- ``statevector.py:362-410`` (eager loop) and
  the GATE_IDS-only names the compiled path adds (``statevector.py:414-471``,
  ``compiler.py:52-315``)
* Pauli-term application and expectations -- ``dense_evolution/physics/observables.py:38-308``
* the energy function's parameter-injection order -- ``dense_evolution/solvers/autodiff.py:21-169``
* fidelity -- ``dense_evolution/utils/measurement.py:71-94``

Parity of this restatement is pinned against fixtures produced by the
reference itself (``tests/golden/make_golden.py`` imports the reference's own
modules and writes ``tests/golden/*.npz``/``*.json``) and against the
known-answer tests of the reference's test-suite.
"""
from __future__ import annotations

import math
from typing import Dict, List, Sequence, Tuple

import numpy as np

INV2 = 1.0 / math.sqrt(2.0)

# ---------------------------------------------------------------------------
# gate tables (gates.py:33-91)
# ---------------------------------------------------------------------------

_STATIC = {
    'h': INV2 * np.array([[1, 1], [1, -1]], dtype=np.complex128),
    'x': np.array([[0, 1], [1, 0]], dtype=np.complex128),
    'y': np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    'z': np.array([[1, 0], [0, -1]], dtype=np.complex128),
    's': np.array([[1, 0], [0, 1j]], dtype=np.complex128),
    'sdg': np.array([[1, 0], [0, -1j]], dtype=np.complex128),
    't': np.array([[1, 0], [0, np.exp(1j * np.pi / 4)]], dtype=np.complex128),
    'tdg': np.array([[1, 0], [0, np.exp(-1j * np.pi / 4)]], dtype=np.complex128),
    'sx': 0.5 * np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]], dtype=np.complex128),
    'id': np.eye(2, dtype=np.complex128),
    'cx': np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=np.complex128),
    'cz': np.diag([1, 1, 1, -1]).astype(np.complex128),
    'cy': np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, -1j], [0, 0, 1j, 0]], dtype=np.complex128),
    'swap': np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=np.complex128),
    'iswap': np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=np.complex128),
    'ecr': INV2 * np.array([[0, 0, 1, 1j], [0, 0, 1j, 1], [1, -1j, 0, 0], [-1j, 1, 0, 0]],
                           dtype=np.complex128),
}
_CCX = np.eye(8, dtype=np.complex128)
_CCX[[6, 7]] = _CCX[[7, 6]]
_STATIC['ccx'] = _CCX


def _rx(t):
    c, s = math.cos(t / 2), math.sin(t / 2)
    return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)


def _ry(t):
    c, s = math.cos(t / 2), math.sin(t / 2)
    return np.array([[c, -s], [s, c]], dtype=np.complex128)


def _rz(t):
    return np.diag([np.exp(-0.5j * t), np.exp(0.5j * t)]).astype(np.complex128)


def _p(lam):
    return np.diag([1.0, np.exp(1j * lam)]).astype(np.complex128)


def _u3(t, phi, lam):
    c, s = math.cos(t / 2), math.sin(t / 2)
    return np.array([[c, -np.exp(1j * lam) * s],
                     [np.exp(1j * phi) * s, np.exp(1j * (phi + lam)) * c]], dtype=np.complex128)


_PARAM = {
    'rx': _rx, 'ry': _ry, 'rz': _rz,
    'cp': lambda lam: np.diag([1, 1, 1, np.exp(1j * lam)]).astype(np.complex128),
    'crz': lambda t: np.diag([1, 1, np.exp(-0.5j * t), np.exp(0.5j * t)]).astype(np.complex128),
    'u3': _u3,
    'u2': lambda phi, lam: INV2 * np.array([[1.0, -np.exp(1j * lam)],
                                            [np.exp(1j * phi), np.exp(1j * (phi + lam))]]),
    'u1': _p, 'p': _p,
    'gphase': lambda a: np.exp(1j * a) * np.eye(2, dtype=np.complex128),
}

# The compiled path's id table (gates.py:53-63): names it accepts besides the
# eager tables ('phase', 'cphase', 'swap' id 23 never dispatched).
GATE_IDS = {
    'id': 0, 'h': 1, 'x': 2, 'y': 3, 'z': 4, 's': 5, 'sdg': 6, 't': 7, 'tdg': 8,
    'rx': 9, 'ry': 10, 'rz': 11, 'p': 12, 'u1': 12, 'phase': 12, 'sx': 13,
    'gphase': 14, 'cx': 20, 'cz': 21, 'cp': 22, 'cphase': 22, 'cy': 24, 'crz': 25,
}
_TWO_Q_PARAM = ('cp', 'cphase', 'crz')


def gate_matrix(name: str, params: Sequence[float]) -> np.ndarray:
    """Complex128 matrix of a gate by name (qubit order: first qubit = MSB of the index)."""
    name = name.lower()
    if name in _STATIC:
        return _STATIC[name]
    if name == 'phase':
        return _p(*params) if params else np.eye(2, dtype=np.complex128)
    if name == 'cphase':
        return _PARAM['cp'](*params) if params else np.eye(4, dtype=np.complex128)
    if name in _PARAM:
        return _PARAM[name](*params)
    raise ValueError(f"unknown gate '{name}'")


# ---------------------------------------------------------------------------
# transpiler (compiler.py:369-488)
# ---------------------------------------------------------------------------

def transpile(circuit) -> List[Tuple]:
    out: List[Tuple] = []
    for cmd in circuit:
        name = cmd[0].lower()
        a = cmd[1:]
        if name == 'ccx':
            c1, c2, t = a[:3]
            out += [('h', t), ('cx', c2, t), ('tdg', t), ('cx', c1, t), ('t', t), ('cx', c2, t),
                    ('tdg', t), ('cx', c1, t), ('t', c2), ('t', t), ('cx', c1, c2), ('h', t),
                    ('t', c1), ('tdg', c2), ('cx', c1, c2)]
        elif name == 'swap':
            q1, q2 = a[:2]
            out += [('cx', q1, q2), ('cx', q2, q1), ('cx', q1, q2)]
        elif name == 'iswap':
            q1, q2 = a[:2]
            out += [('s', q1), ('h', q1), ('s', q2), ('cx', q1, q2), ('cx', q2, q1), ('h', q2)]
        elif name == 'ecr':
            q1, q2 = a[:2]
            out += [('s', q1), ('sx', q2), ('cx', q1, q2), ('x', q1), ('gphase', q1, -np.pi / 4.0)]
        elif name == 'u3' and len(cmd) >= 5:
            q, th, ph, lam = a[:4]
            out += [('rz', q, lam), ('ry', q, th), ('rz', q, ph), ('gphase', q, (ph + lam) / 2.0)]
        elif name == 'u2' and len(cmd) >= 4:
            q, ph, lam = a[:3]
            th = np.pi / 2.0
            out += [('rz', q, lam), ('ry', q, th), ('rz', q, ph), ('gphase', q, (ph + lam) / 2.0)]
        else:
            out.append(cmd)
    return out


# ---------------------------------------------------------------------------
# gate application (statevector.py:167-203, MSB-first: qubit q = bit n-1-q)
# ---------------------------------------------------------------------------

def apply_1q(sv: np.ndarray, n: int, U: np.ndarray, q: int) -> np.ndarray:
    if not 0 <= q < n:
        raise ValueError(f"Qubit index {q} out of range [0, {n})")
    v = sv.reshape(1 << q, 2, 1 << (n - 1 - q))
    return np.matmul(U.astype(sv.dtype), v).reshape(-1)


def apply_2q(sv: np.ndarray, n: int, U: np.ndarray, q1: int, q2: int) -> np.ndarray:
    if q1 == q2:
        raise ValueError("Control and target qubits must differ")
    if not (0 <= q1 < n and 0 <= q2 < n):
        raise ValueError(f"Qubit indices ({q1},{q2}) out of range [0, {n})")
    t = np.moveaxis(sv.reshape([2] * n), (q1, q2), (0, 1))
    shp = t.shape
    r = (U.astype(sv.dtype) @ t.reshape(4, -1)).reshape(shp)
    return np.moveaxis(r, (0, 1), (q1, q2)).reshape(-1)


def zero_state(n: int, dtype=np.complex128) -> np.ndarray:
    sv = np.zeros(1 << n, dtype=dtype)
    sv[0] = 1.0
    return sv


def run_circuit(sv: np.ndarray, n: int, circuit, do_transpile: bool = True) -> np.ndarray:
    """Run a gate-tuple circuit; names follow the union of the eager tables and GATE_IDS."""
    target = transpile(circuit) if do_transpile else list(circuit)
    for cmd in target:
        name = (cmd[0] if isinstance(cmd[0], str) else str(cmd[0])).lower()
        a = cmd[1:]
        if name in ('cp', 'cphase', 'crz'):
            U = gate_matrix(name, [float(x) for x in a[2:3]])
            sv = apply_2q(sv, n, U, int(a[0]), int(a[1]))
        elif name in ('cx', 'cz', 'cy', 'swap', 'iswap', 'ecr'):
            sv = apply_2q(sv, n, gate_matrix(name, ()), int(a[0]), int(a[1]))
        elif name == 'ccx':
            t = np.moveaxis(sv.reshape([2] * n), (int(a[0]), int(a[1]), int(a[2])), (0, 1, 2))
            shp = t.shape
            r = (_CCX @ t.reshape(8, -1)).reshape(shp)
            sv = np.moveaxis(r, (0, 1, 2), (int(a[0]), int(a[1]), int(a[2]))).reshape(-1)
        elif name in _STATIC or name in _PARAM or name == 'phase':
            sv = apply_1q(sv, n, gate_matrix(name, [float(x) for x in a[1:]]), int(a[0]))
        else:
            raise ValueError(f"unknown gate '{cmd[0]}' (issue #4)")
    return sv


# ---------------------------------------------------------------------------
# Pauli observables (observables.py:38-308)
# ---------------------------------------------------------------------------

def normalize_terms(pauli_terms, n_qubits=None) -> Dict[int, str]:
    if isinstance(pauli_terms, str):
        if n_qubits is not None and len(pauli_terms) != n_qubits:
            raise ValueError("pauli string length mismatch")
        terms = {q: p.upper() for q, p in enumerate(pauli_terms) if p.upper() != 'I'}
    elif isinstance(pauli_terms, dict):
        terms = {int(q): str(p).upper() for q, p in pauli_terms.items() if str(p).upper() != 'I'}
    else:
        terms = {int(q): str(p).upper() for q, p in pauli_terms if str(p).upper() != 'I'}
    for q, p in terms.items():
        if p not in ('X', 'Y', 'Z'):
            raise ValueError(f"unknown Pauli operator {p!r}")
        if q < 0:
            raise ValueError("negative qubit")
    return terms


def apply_pauli_term(sv: np.ndarray, terms: Dict[int, str], n: int) -> np.ndarray:
    """P|psi>[i] = psi[i ^ flip] * prod(+-1, +-i) read from the SOURCE index bits."""
    if not terms:
        return sv
    flip = 0
    for q, p in terms.items():
        if p in ('X', 'Y'):
            flip |= 1 << (n - 1 - q)
    src = np.arange(sv.shape[0], dtype=np.int64) ^ flip
    coeff = np.ones(sv.shape[0], dtype=np.complex128)
    for q, p in terms.items():
        bit = (src >> (n - 1 - q)) & 1
        if p == 'Y':
            coeff *= np.where(bit == 0, 1j, -1j)
        elif p == 'Z':
            coeff *= np.where(bit == 0, 1.0, -1.0)
    return sv[src] * coeff


def _nq(sv):
    d = sv.shape[0]
    n = d.bit_length() - 1
    if 1 << n != d:
        raise ValueError("length is not a power of 2")
    return n


def pauli_expectation(sv, pauli_terms, n_qubits=None) -> float:
    sv = np.asarray(sv)
    n = _nq(sv)
    t = normalize_terms(pauli_terms, n_qubits)
    if t and max(t) >= n:
        raise ValueError("qubit out of range")
    return float(np.real(np.vdot(sv, apply_pauli_term(sv, t, n))))


def pauli_sum_expectation(sv, terms, n_qubits=None) -> float:
    total = 0.0
    for c, p in terms:
        total += c * pauli_expectation(sv, p, n_qubits)
    return total


def pauli_sum_matvec(v, terms, n_qubits=None) -> np.ndarray:
    v = np.asarray(v, dtype=np.complex128)
    n = _nq(v)
    out = np.zeros_like(v)
    for c, p in terms:
        t = normalize_terms(p, n_qubits)
        if t and max(t) >= n:
            raise ValueError("qubit out of range")
        out += c * apply_pauli_term(v, t, n)
    return out


_PM = {'I': np.eye(2), 'X': np.array([[0, 1], [1, 0]]), 'Y': np.array([[0, -1j], [1j, 0]]),
       'Z': np.diag([1, -1])}


def pauli_hamiltonian_to_matrix(terms, n_qubits) -> np.ndarray:
    d = 1 << n_qubits
    H = np.zeros((d, d), dtype=np.complex128)
    for c, p in terms:
        t = normalize_terms(p, n_qubits)
        m = np.array([[1.0 + 0j]])
        for q in range(n_qubits):
            m = np.kron(m, _PM[t.get(q, 'I')])
        H += c * m
    return H


def fidelity(a, b) -> float:
    return float(abs(np.vdot(np.asarray(a), np.asarray(b))) ** 2)


# ---------------------------------------------------------------------------
# energy function (autodiff.py:21-169): theta is injected, in gate order, into
# the parametric gates rx/ry/rz/u1/p/cp/crz; every other gate keeps param 0.
# ---------------------------------------------------------------------------

PARAMETRIC = ('rx', 'ry', 'rz', 'u1', 'p', 'cp', 'crz')
TWO_Q = ('cx', 'cy', 'cz', 'cp', 'crz', 'swap')


def energy_template(ops: List[dict], n: int) -> Tuple[List[Tuple], int]:
    tuples = []
    for op in ops:
        name = str(op['name']).lower().strip()
        qs = [int(q) for q in op.get('qubits', [])]
        if not qs or any(q >= n for q in qs):
            continue
        tuples.append((name, *qs))
    rows = []
    for cmd in transpile(tuples):
        name = cmd[0].lower()
        if name not in GATE_IDS:
            raise ValueError(f"gate '{name}' has no GATE_IDS entry")
        qs = cmd[1:]
        par = name in PARAMETRIC
        if name in TWO_Q and len(qs) >= 2:
            rows.append((name, int(qs[0]), int(qs[1]), par))
        else:
            rows.append((name, int(qs[0]), 0, par))
    n_params = sum(1 for op in ops if str(op['name']).lower().strip() in PARAMETRIC)
    return rows, n_params


def _row_to_tuple(name, q1, q2, p):
    """A template row as a gate tuple, using the compiled path's id semantics."""
    gid = GATE_IDS[name]
    if gid <= 14:
        return (name, q1, p) if name in ('rx', 'ry', 'rz', 'p', 'u1', 'phase', 'gphase') else (name, q1)
    if gid == 22 and q1 == q2:           # 'cphase' row: ctrl == tgt, phase on |1> of q1
        return ('p', q1, p)
    if gid in (22, 25):
        return (name, q1, q2, p)
    return (name, q1, q2)


def template_circuit(rows, theta) -> List[Tuple]:
    out, k = [], 0
    for name, q1, q2, par in rows:
        p = 0.0
        if par:
            p = float(theta[k])
            k += 1
        out.append(_row_to_tuple(name, q1, q2, p))
    return out


def energy(theta, rows, n, terms, sv0=None) -> Tuple[float, np.ndarray]:
    sv = zero_state(n) if sv0 is None else np.asarray(sv0, dtype=np.complex128).copy()
    sv = run_circuit(sv, n, template_circuit(rows, theta), do_transpile=False)
    if callable(terms):
        hv = terms(sv)
    elif isinstance(terms, np.ndarray):
        hv = terms @ sv
    else:
        hv = pauli_sum_matvec(sv, terms)
    return float(np.real(np.vdot(sv, hv))), sv


def fd_gradient(theta, rows, n, terms, h=1e-3, indices=None) -> np.ndarray:
    theta = np.asarray(theta, dtype=np.float64)
    idx = range(theta.size) if indices is None else indices
    g = np.zeros(len(list(idx)) if indices is not None else theta.size)
    for j, i in enumerate(range(theta.size) if indices is None else indices):
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        g[j] = (energy(tp, rows, n, terms)[0] - energy(tm, rows, n, terms)[0]) / (2 * h)
    return g


# ---------------------------------------------------------------------------
# stochastic single-qubit Kraus channels, NumPy branch
# (dense_evolution/noise/kraus_channels.py:104-236 and noise/kraus/*.py)
# ---------------------------------------------------------------------------

NOISE_MODELS = ['ideal', 'depolarizing', 'bitflip', 'phaseflip', 'amplitude_damping', 'combined']


def _noise_pairs(dim: int, q: int):
    """Index pairs of qubit q: bit q of the amplitude index (LSB-first here,
    unlike the simulator's MSB-first order) -- kraus_channels.py:60-80."""
    i = np.arange(dim)
    i0 = i[(i >> q) & 1 == 0]
    return i0, i0 | (1 << q)


def _noise_pauli(v, i0, i1, which):
    a0, a1 = v[i0].copy(), v[i1].copy()
    if which == 'x':
        v[i0], v[i1] = a1, a0
    elif which == 'y':
        v[i0], v[i1] = -1j * a1, 1j * a0
    else:
        v[i1] = -a1


def _noise_depolarizing(v, i0, i1, p, rng):        # kraus/depolarizing.py
    r, ch = rng.random(), rng.random()
    if r < p:
        _noise_pauli(v, i0, i1, 'x' if ch < 1.0 / 3.0 else 'y' if ch < 2.0 / 3.0 else 'z')


def _noise_damping(v, i0, i1, p, rng):             # kraus/amplitude_damping.py
    gamma = float(np.clip(p, 0.0, 1.0))
    r = rng.random()
    a0, a1 = v[i0].copy(), v[i1].copy()
    p1 = float(np.clip(gamma * np.sum(np.abs(a1) ** 2), 0.0, 1.0))
    if r < p1:
        v[i0] = a1 * np.sqrt(gamma) / np.sqrt(max(p1, 1e-15))
        v[i1] = 0.0
    else:
        nn = np.sqrt(max(1.0 - p1, 1e-15))
        v[i0] = a0 / nn
        v[i1] = a1 * np.sqrt(1.0 - gamma) / nn


def noise_apply(sv, n, model, p, rng, qubits=None):
    """NoiseModel.apply_to_sv, NumPy branch: per target qubit one channel step
    with the draws in the reference's order, then division by (norm + 1e-15)."""
    if model == 'ideal' or p <= 0.0:
        return sv
    if model not in NOISE_MODELS:
        raise KeyError(model)
    v = np.array(sv, dtype=np.complex128).copy()
    for q in (list(range(n)) if qubits is None else list(qubits)):
        i0, i1 = _noise_pairs(len(v), q)
        if model == 'depolarizing':
            _noise_depolarizing(v, i0, i1, p, rng)
        elif model == 'bitflip':
            if rng.random() < p:
                _noise_pauli(v, i0, i1, 'x')
        elif model == 'phaseflip':
            if rng.random() < p:
                _noise_pauli(v, i0, i1, 'z')
        elif model == 'amplitude_damping':
            _noise_damping(v, i0, i1, p, rng)
        else:                                     # combined (kraus/combined.py)
            _noise_depolarizing(v, i0, i1, p * 0.5, rng)
            _noise_damping(v, i0, i1, p * 0.333333, rng)
    return v / (np.linalg.norm(v) + 1e-15)


def sample_counts(statevector, n_shots, rng=None):
    """Finite-shot counts (utils/measurement.py:17-68): probabilities |a|^2,
    normalised, sampled with ``rng.choice`` (cumsum + searchsorted of
    ``rng.random(n_shots)``); keys are bitstrings with qubit 0 leftmost."""
    sv = np.asarray(statevector)
    dim = sv.shape[0]
    n = dim.bit_length() - 1
    if 1 << n != dim:
        raise ValueError(f"statevector length {dim} is not a power of 2")
    if n_shots < 1:
        raise ValueError(f"n_shots must be >= 1, got {n_shots}")
    probs = np.abs(sv) ** 2
    total = probs.sum()
    if not np.isfinite(total) or total <= 0:
        raise ValueError("statevector has zero or non-finite total probability")
    rng = np.random.default_rng() if rng is None else rng
    idx = rng.choice(dim, size=n_shots, p=probs / total)
    v, f = np.unique(idx, return_counts=True)
    return {format(int(a), f'0{n}b'): int(b) for a, b in zip(v, f)}


# ---------------------------------------------------------------------------
# interop bit order (interop/qiskit_pennylane.py:115-136, tests/_helpers.py:14-25)
# ---------------------------------------------------------------------------

def bit_reversal_perm(n_qubits: int) -> List[int]:
    """MSB-first <-> little-endian index permutation, as the reference's test
    helper writes it: the index's n-bit binary string reversed."""
    return [int(format(i, f'0{n_qubits}b')[::-1], 2) for i in range(2 ** n_qubits)] if n_qubits else [0]


def to_qiskit_bit_order(probs: np.ndarray, n_qubits: int) -> np.ndarray:
    """probs reindexed into Qiskit's little-endian order (the reference's
    _to_qiskit_bit_order: probs[perm] with perm the bit reversal)."""
    return np.asarray(probs)[bit_reversal_perm(n_qubits)]
