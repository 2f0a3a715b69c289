"""Config 5 shape: 32-qubit complex64 adjoint gradient (three 32 GiB states),
checked for consistency; complex64 accuracy at 30 qubits against complex128."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_30q_c64_against_c128():
    """Config 5's structure (HEA of 4 layers, XXX chain) at 30 qubits:
    complex64 against complex128 -- |dE| <= 1e-6 (the complex64 bar), the
    adjoint gradients to 1e-5, and two complex64 gradient entries against
    complex128 central differences (h = 1e-3, truncation error ~1e-7) to 2e-5."""
    import torch
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, xxx_terms
    n, layers = 30, 4
    theta = np.random.default_rng(1).uniform(-np.pi, np.pi, 2 * n * layers)
    op = de.PauliSumOperator(xxx_terms(n), n)
    res = {}
    for f32 in (True, False):
        fn, _ = de.circuit_to_energy_fn(hea_circuit(n, layers), n, use_float32=f32)
        e, g, psi = fn.program.value_and_grad(theta, op)
        res[f32] = (e, g)
        del psi
        torch.cuda.empty_cache()
    assert abs(res[True][0] - res[False][0]) <= 1e-6
    assert np.max(np.abs(res[True][1] - res[False][1])) <= 1e-5
    f64, _ = de.circuit_to_energy_fn(hea_circuit(n, layers), n)
    h = 1e-3
    for i in (3, 2 * n * layers - 5):
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        ep = float(f64(tp, op)[0])
        torch.cuda.empty_cache()
        em = float(f64(tm, op)[0])
        torch.cuda.empty_cache()
        assert abs(res[True][1][i] - (ep - em) / (2 * h)) < 2e-5, i


def test_32q_adjoint_consistency():
    import torch
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, xxx_terms
    n, layers = 32, 1
    if torch.cuda.mem_get_info()[0] < 3.2 * (1 << n) * 8:
        pytest.skip('not enough free HBM for three 32 GiB states')
    fn, npar = de.circuit_to_energy_fn(hea_circuit(n, layers), n, use_float32=True)
    theta = np.random.default_rng(2).uniform(-np.pi, np.pi, npar)
    op = de.PauliSumOperator(xxx_terms(n), n)
    e, g, psi = fn.program.value_and_grad(theta, op)
    assert np.all(np.isfinite(g)) and g.shape == (npar,)
    e2 = de.pauli_sum_expectation(psi, xxx_terms(n))
    assert e == pytest.approx(e2, abs=1e-6)
    sim_norm = torch.linalg.vector_norm(psi.to(torch.complex64)).item()
    assert sim_norm == pytest.approx(1.0, abs=1e-5)
    del psi
    torch.cuda.empty_cache()


def test_config3_full_size_against_c128_fd():
    """Config 3 at its full size: 24 qubits, HEA 10 layers (480 parameters),
    TFIM.  complex64 adjoint gradient against complex128 central differences
    (h = 1e-3) on a seeded subset of 8 parameters; energies c64 vs c128."""
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, tfim_terms
    n, layers = 24, 10
    circ = hea_circuit(n, layers)
    f64, npar = de.circuit_to_energy_fn(circ, n)
    f32, _ = de.circuit_to_energy_fn(circ, n, use_float32=True)
    assert npar == 480
    theta = np.random.default_rng(2024).uniform(-np.pi, np.pi, npar)
    op = de.PauliSumOperator(tfim_terms(n), n)
    e32, g32, _ = f32.program.value_and_grad(theta, op)
    e64 = float(f64(theta, op)[0])
    assert abs(e32 - e64) <= 1e-6
    h = 1e-3
    idx = np.random.default_rng(7).choice(npar, 8, replace=False)
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (float(f64(tp, op)[0]) - float(f64(tm, op)[0])) / (2 * h)
        assert abs(g32[i] - fd) < 2e-5, (i, g32[i], fd)
