"""Energy functions and the adjoint-method gradient vs the reference's own
energies / finite-difference gradients (golden) and the oracle."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu

VQE_QASM = ('OPENQASM 2.0; include "qelib1.inc"; qreg q[2]; creg c[2]; '
            'ry(0.5) q[0]; rx(0.5) q[1]; cx q[0],q[1]; rz(0.2) q[1]; cx q[0],q[1]; '
            'ry(0.5) q[0]; rx(0.5) q[1]; measure q -> c;')


def _oracle_rows(circ, n):
    ops = circ.ops
    return O.energy_template(ops, n)


def test_reference_vqe_qasm_gradient_matches_fd():
    import torch
    import dense_evolution as de
    circ = de.QASMParser().parse(VQE_QASM)
    energy_fn, n_params = de.circuit_to_energy_fn(circ, circ.n_qubits)
    assert n_params == 5
    rng = np.random.default_rng(7)
    h = np.diag(np.sort(rng.uniform(-2.5, 2.5, 4)))
    theta0 = np.random.default_rng(3).uniform(-np.pi, np.pi, n_params)
    th = torch.tensor(theta0, requires_grad=True)
    e, sv = energy_fn(th, h)
    e.backward()
    rows, _ = _oracle_rows(circ, 2)
    fd = O.fd_gradient(theta0, rows, 2, lambda v: h @ v, h=1e-6)
    assert np.allclose(th.grad.numpy(), fd, atol=1e-6)
    assert float(e) == pytest.approx(O.energy(theta0, rows, 2, lambda v: h @ v)[0], abs=1e-12)


def test_default_initial_state_and_empty_circuit():
    import dense_evolution as de
    circ = de.QASMParser().parse('OPENQASM 2.0; qreg q[2]; creg c[2]; measure q -> c;')
    energy_fn, n_params = de.circuit_to_energy_fn(circ, circ.n_qubits)
    assert n_params == 0
    e, sv = energy_fn(np.array([]), np.diag([1.0, 2.0, 3.0, 4.0]))
    assert float(e) == pytest.approx(1.0, abs=1e-9)
    assert abs(complex(sv[0].item())) == pytest.approx(1.0)


@pytest.mark.parametrize('n', [4, 6])
def test_golden_energy_and_gradient(n):
    import dense_evolution as de
    from dense_evolution.workloads import hea_qasm, tfim_terms
    d = np.load(os.path.join(GOLDEN, 'golden_energy.npz'))
    theta = d[f'theta_n{n}']
    layers = theta.size // (2 * n)
    circ = de.QASMParser().parse(hea_qasm(n, layers, theta))
    energy_fn, npar = de.circuit_to_energy_fn(circ, n)
    op = de.PauliSumOperator(tfim_terms(n), n)
    e, g, _ = energy_fn.program.value_and_grad(theta, op)
    assert e == pytest.approx(float(d[f'energy_n{n}']), abs=1e-10)
    assert np.allclose(g, d[f'grad_n{n}'], atol=1e-7)


@pytest.mark.parametrize('n,f32', [(9, False), (10, False), (12, True), (13, False)])
def test_fused_adjoint_vs_oracle_fd_and_parameter_shift(n, f32):
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, tfim_terms
    layers = 2
    circ = hea_circuit(n, layers) + [('crz', 0, n - 1, 0.0), ('cp', 2, 1, 0.0), ('p', 3, 0.0), ('rx', 4, 0.0)]
    energy_fn, npar = de.circuit_to_energy_fn(circ, n, use_float32=f32)
    rng = np.random.default_rng(n)
    theta = rng.uniform(-np.pi, np.pi, npar)
    terms = tfim_terms(n) + [(0.3, {0: 'Y', n - 1: 'Y'}), (0.2, {1: 'X', 2: 'Y', 7: 'Z'})]
    e, g, psi = energy_fn.program.value_and_grad(theta, terms)
    rows, _ = O.energy_template([{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]}
                                 for c in circ], n)
    e_ref, psi_ref = O.energy(theta, rows, n, terms)
    fd = O.fd_gradient(theta, rows, n, terms, h=1e-5)
    tol_e, tol_g = (1e-6, 1e-5) if f32 else (1e-10, 1e-7)
    assert e == pytest.approx(e_ref, abs=tol_e)
    assert np.allclose(g, fd, atol=tol_g)
    ps = energy_fn.program.parameter_shift_grad(theta, terms)
    assert np.allclose(ps, fd, atol=tol_g if not f32 else 1e-5)


def test_config3_shape_small_against_c128_fd():
    """Config 3 structure (HEA 10 layers, TFIM) at 10 qubits: complex64 adjoint vs
    complex128 central differences (h = 1e-3)."""
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, tfim_terms
    n, layers = 10, 10
    circ = hea_circuit(n, layers)
    f64, npar = de.circuit_to_energy_fn(circ, n)
    f32, _ = de.circuit_to_energy_fn(circ, n, use_float32=True)
    theta = np.random.default_rng(0).uniform(-np.pi, np.pi, npar)
    op = de.PauliSumOperator(tfim_terms(n), n)
    e32, g32, _ = f32.program.value_and_grad(theta, op)
    h = 1e-3
    idx = np.random.default_rng(1).choice(npar, 12, replace=False)
    fd = []
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd.append((float(f64(tp, op)[0]) - float(f64(tm, op)[0])) / (2 * h))
    e64 = float(f64(theta, op)[0])
    assert e32 == pytest.approx(e64, abs=1e-6)
    # central FD at h=1e-3 has O(h^2) truncation error ~1e-7 * |E'''|
    assert np.allclose(g32[idx], fd, atol=2e-5)


def test_torch_autograd_and_unsupported_gates():
    import torch
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, tfim_terms
    n = 9
    fn, npar = de.circuit_to_energy_fn(hea_circuit(n, 1), n)
    th = torch.zeros(npar, dtype=torch.float64, requires_grad=True)
    e, sv = fn(th, de.PauliSumOperator(tfim_terms(n), n))
    (2 * e).backward()
    _, g, _ = fn.program.value_and_grad(np.zeros(npar), de.PauliSumOperator(tfim_terms(n), n))
    assert np.allclose(th.grad.numpy(), 2 * g)
    circ = de.QASMParser().parse('OPENQASM 2.0; qreg q[1]; u3(0.1,0.2,0.3) q[0];')
    with pytest.raises(ValueError):
        de.circuit_to_energy_fn(circ, 1)
    # noise= reads .model / .p / .jax_key / .qubits like the reference's energy_fn
    # (solvers/autodiff.py:159-164), so an object without them fails the same way
    with pytest.raises(AttributeError):
        fn(np.zeros(npar), [(1.0, 'Z' * n)], noise=object())
