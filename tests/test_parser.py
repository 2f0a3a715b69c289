"""QASM parser against the reference parser's own outputs (golden_parser.json)
and the reference test-suite's behaviours."""
import json
import os

import pytest

from conftest import GOLDEN
from dense_evolution.circuits.parser import QASMParser, QASMCircuit


def _golden():
    with open(os.path.join(GOLDEN, 'golden_parser.json')) as f:
        return json.load(f)


@pytest.mark.parametrize('case', _golden(), ids=lambda c: str(len(c['qasm'])))
def test_matches_reference(case):
    c = QASMParser().parse(case['qasm'])
    assert c.n_qubits == case['n_qubits']
    assert c.n_cbits == case['n_cbits']
    assert len(c.ops) == len(case['ops'])
    for a, b in zip(c.ops, case['ops']):
        assert a['name'] == b['name'] and a['qubits'] == b['qubits']
        assert a['params'] == pytest.approx(b['params'], abs=1e-15)
    for t, ref in zip(c.to_tuples(), case['tuples']):
        assert t[0] == ref[0] and len(t) == len(ref)
        assert list(t[1:]) == pytest.approx(ref[1:], abs=1e-15)
    assert list(QASMParser().validate(c)) == case['valid']


def test_invalid_parameter_raises():
    with pytest.raises(ValueError):
        QASMParser().parse('qreg q[1]; rx(pi * / 2) q[0];')
    with pytest.raises(ValueError):
        QASMParser().parse("qreg q[1]; rx(().__class__) q[0];")


def test_range_and_for_loop():
    c = QASMParser().parse('OPENQASM 3.0; qubit[5] q; h q[1:4]; for int i in [0:3] { cx q[i], q[4]; }')
    assert [op['qubits'] for op in c.ops[:3]] == [[1], [2], [3]]
    assert [op['qubits'] for op in c.ops[3:]] == [[0, 4], [1, 4], [2, 4], [3, 4]]
    # like the reference, an index expression such as q[i+1] is not resolved (only q[<int>])
    c = QASMParser().parse('OPENQASM 3.0; qubit[5] q; for int i in [0:1] { cx q[i], q[i+1]; }')
    assert [op['qubits'] for op in c.ops] == [[0], [1]]


def test_gate_definition_expansion_and_arity_error():
    c = QASMParser().parse('qreg q[2]; gate g(a) x, y { rz(a) x; cx x, y; } g(0.5) q[1], q[0];')
    assert [(o['name'], o['qubits']) for o in c.ops] == [('rz', [1]), ('cx', [1, 0])]
    with pytest.raises(ValueError):
        QASMParser().parse('qreg q[2]; gate g x, y { cx x, y; } g q[0];')


def test_iteration_and_validate():
    c = QASMParser().parse('qreg q[2]; h q[0]; cx q[0], q[1];')
    assert list(c) == [('h', 0), ('cx', 0, 1)]
    assert QASMParser().validate(QASMCircuit(0, 0, [])) == (False, 'n_qubits must be > 0.')
    assert QASMParser().validate(QASMCircuit(1, 0, [])) == (False, 'No gate operations found in circuit.')
    bad = QASMCircuit(1, 0, [{'type': 'gate', 'name': 'x', 'qubits': [3], 'params': []}])
    assert QASMParser().validate(bad)[0] is False


def test_package_transpiler_matches_reference_output():
    """QuantumTranspiler.transpile of the package (not only the oracle) against
    the reference's own transpile output on the same input: same gate tuples in
    the same order, so the theta-slot order of run_batch_jit / energy_fn and
    the global phases agree with the reference's."""
    import json
    import os
    from dense_evolution.circuits.compiler import QuantumTranspiler
    with open(os.path.join(os.path.dirname(__file__), 'golden', 'golden_transpile.json')) as f:
        t = json.load(f)
    out = QuantumTranspiler.transpile([tuple(c) for c in t['in']])
    assert [list(c) for c in out] == t['out']
