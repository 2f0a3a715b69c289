"""The oracle (oracle/sv_oracle.py) pinned against fixtures produced by the
reference itself (tests/golden/make_golden.py) and the reference test-suite's
known answers."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import sv_oracle as O


def _cases():
    with open(os.path.join(GOLDEN, 'golden_cases.json')) as f:
        return json.load(f)


STATES = np.load(os.path.join(GOLDEN, 'golden_states.npz'))


@pytest.mark.parametrize('case', _cases(), ids=lambda c: c['name'])
def test_oracle_matches_reference_states(case):
    n = case['n']
    circ = [tuple(c) for c in case['circuit']]
    sv = O.run_circuit(O.zero_state(n), n, circ)
    ref = STATES[case['name'] + '__c128']
    assert np.max(np.abs(sv - ref)) < 1e-12
    ref64 = STATES[case['name'] + '__c64']
    assert np.max(np.abs(sv - ref64)) < 1e-5


def test_known_answers():
    # X on qubit 0 of 3 qubits lands on index 4 (MSB-first)
    sv = O.run_circuit(O.zero_state(3), 3, [('x', 0)])
    assert abs(sv[4]) == pytest.approx(1.0)
    # Bell / GHZ
    b = O.run_circuit(O.zero_state(2), 2, [('h', 0), ('cx', 0, 1)])
    assert np.allclose(np.abs(b) ** 2, [0.5, 0, 0, 0.5])
    assert O.pauli_expectation(b, 'ZZ') == pytest.approx(1.0)
    assert O.pauli_expectation(b, 'XX') == pytest.approx(1.0)
    g = O.run_circuit(O.zero_state(3), 3, [('h', 0), ('cx', 0, 1), ('cx', 1, 2)])
    assert O.pauli_expectation(g, 'ZZZ') == pytest.approx(0.0, abs=1e-12)
    # CCX |110> = |111>
    s = O.zero_state(3)
    s = O.run_circuit(s, 3, [('x', 0), ('x', 1), ('ccx', 0, 1, 2)])
    assert abs(s[7]) == pytest.approx(1.0)


def test_oracle_matches_reference_pauli():
    with open(os.path.join(GOLDEN, 'golden_pauli.json')) as f:
        meta = json.load(f)
    d = np.load(os.path.join(GOLDEN, 'golden_pauli.npz'))
    for i, m in enumerate(meta):
        psi = d[f'psi{i}']
        terms = [(c, s) for c, s in m['terms']]
        exp = [O.pauli_expectation(psi, s) for _, s in terms]
        assert np.allclose(exp, d[f'exp{i}'], atol=1e-12)
        assert O.pauli_sum_expectation(psi, terms) == pytest.approx(float(d[f'sum{i}']), abs=1e-12)
        assert np.allclose(O.pauli_sum_matvec(psi, terms), d[f'mv{i}'], atol=1e-12)


def test_oracle_transpile_matches_reference():
    with open(os.path.join(GOLDEN, 'golden_transpile.json')) as f:
        t = json.load(f)
    out = O.transpile([tuple(c) for c in t['in']])
    assert [list(c) for c in out] == t['out']


def test_oracle_energy_and_fd_gradient_match_reference():
    d = np.load(os.path.join(GOLDEN, 'golden_energy.npz'))
    for n, layers in ((4, 2), (6, 3)):
        theta = d[f'theta_n{n}']
        ops = []
        k = 0
        for _ in range(layers):
            for q in range(n):
                ops.append({'name': 'ry', 'qubits': [q], 'params': [theta[k]]})
                ops.append({'name': 'rz', 'qubits': [q], 'params': [theta[k + 1]]})
                k += 2
            for q in range(n - 1):
                ops.append({'name': 'cx', 'qubits': [q, q + 1], 'params': []})
        rows, npar = O.energy_template(ops, n)
        assert npar == theta.size
        terms = [(-1.0, {i: 'Z', i + 1: 'Z'}) for i in range(n - 1)] + [(-1.0, {i: 'X'}) for i in range(n)]
        e, _ = O.energy(theta, rows, n, terms)
        assert e == pytest.approx(float(d[f'energy_n{n}']), abs=1e-12)
        g = O.fd_gradient(theta, rows, n, terms, h=1e-5)
        assert np.allclose(g, d[f'grad_n{n}'], atol=1e-7)


def test_oracle_config1_fingerprint():
    """20 qubits, 20 layers of U3 + brick CZ, complex128 -- the reference's own run."""
    d = np.load(os.path.join(GOLDEN, 'golden_config1.npz'))
    from dense_evolution.workloads import brick_u3_circuit
    n, layers, seed = int(d['n']), int(d['layers']), int(d['seed'])
    sv = O.run_circuit(O.zero_state(n), n, brick_u3_circuit(n, layers, seed))
    assert np.max(np.abs(sv[d['idx']] - d['amp'])) < 1e-12
    p = np.abs(sv) ** 2
    i = np.arange(1 << n)
    z = np.array([np.sum(p * (1 - 2 * ((i >> (n - 1 - q)) & 1))) for q in range(n)])
    assert np.allclose(z, d['z'], atol=1e-12)
