"""Qiskit / PennyLane bit-order interop on the GPU against the reference's own
permutation (restated in the oracle from interop/qiskit_pennylane.py:115-136
and tests/_helpers.py:14-25), and run_qiskit_circuit end to end through the
OpenQASM bridge (qiskit is not installed here: its qasm2.dumps is stood in by
a fake that returns the circuit's QASM text)."""
import types

import numpy as np
import pytest
import torch

from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('n', [0, 1, 3, 9, 10, 11, 14, 20])
@pytest.mark.parametrize('dtype', [torch.float64, torch.complex64, torch.complex128])
def test_bit_reversal_matches_reference_permutation(n, dtype):
    from dense_evolution.interop import to_little_endian
    rng = np.random.default_rng(n)
    a = rng.normal(size=1 << n) + (1j * rng.normal(size=1 << n) if dtype != torch.float64 else 0)
    t = torch.from_numpy(np.asarray(a)).to('cuda').to(dtype)
    got = to_little_endian(t).cpu().numpy()
    ref = np.asarray(a).astype(got.dtype)[O.bit_reversal_perm(n)] if n else np.asarray(a).astype(got.dtype)
    assert np.array_equal(got, ref)
    # an involution
    assert torch.equal(to_little_endian(to_little_endian(t)), t)


def test_host_helper_signature():
    from dense_evolution.interop import _to_qiskit_bit_order
    n = 12
    p = np.random.default_rng(1).random(1 << n)
    assert np.array_equal(_to_qiskit_bit_order(p, n), O.to_qiskit_bit_order(p, n))
    with pytest.raises(ValueError):
        _to_qiskit_bit_order(p[:-1], n)


def test_run_qiskit_circuit_through_the_qasm_bridge(monkeypatch):
    from dense_evolution.interop import qiskit_pennylane as Q
    n = 5
    qasm = '\n'.join(['OPENQASM 2.0;', 'include "qelib1.inc";', f'qreg q[{n}];', 'h q[0];', 'cx q[0],q[3];',
                      'ry(0.7) q[1];', 'x q[4];', 'cz q[1],q[2];', 'rz(0.3) q[2];'])
    fake = types.SimpleNamespace(dumps=lambda circuit: circuit)
    monkeypatch.setattr(Q, '_qasm2', fake)
    monkeypatch.setattr(Q, 'HAS_QISKIT', True)
    sim, probs = Q.run_qiskit_circuit(qasm, use_float32=False)
    circ = Q.from_qiskit(qasm).to_tuples()
    sv = O.run_circuit(O.zero_state(n), n, circ)
    p = np.abs(sv) ** 2
    p /= p.sum()
    assert np.allclose(probs, O.to_qiskit_bit_order(p, n), atol=1e-12)
    # asymmetric: qubit 4 flipped -> little-endian index bit 4 set
    assert probs[1 << 4:].sum() == pytest.approx(1.0)


def test_missing_packages_raise_the_reference_messages(monkeypatch):
    from dense_evolution.interop import qiskit_pennylane as Q
    monkeypatch.setattr(Q, 'HAS_QISKIT', False)
    monkeypatch.setattr(Q, 'HAS_PENNYLANE', False)
    with pytest.raises(ImportError, match="requires the 'qiskit' package"):
        Q.from_qiskit(object())
    with pytest.raises(ImportError, match="requires the 'pennylane' package"):
        Q.from_pennylane(object())
