"""Config 5 shape: 32-qubit complex64 adjoint gradient (three 32 GiB states),
checked for consistency; complex64 accuracy at 30 qubits against complex128."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_30q_c64_against_c128():
    import torch
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, xxx_terms
    n, layers = 30, 2
    theta = np.random.default_rng(1).uniform(-np.pi, np.pi, 2 * n * layers)
    res = {}
    for f32 in (True, False):
        fn, _ = de.circuit_to_energy_fn(hea_circuit(n, layers), n, use_float32=f32)
        e, g, psi = fn.program.value_and_grad(theta, de.PauliSumOperator(xxx_terms(n), n))
        res[f32] = (e, g)
        del psi
        torch.cuda.empty_cache()
    assert abs(res[True][0] - res[False][0]) <= 1e-5
    assert np.max(np.abs(res[True][1] - res[False][1])) <= 1e-4


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
