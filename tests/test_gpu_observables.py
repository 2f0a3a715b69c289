"""Fused Pauli-sum kernels vs the reference's observables (golden) and the oracle."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu


def test_golden_pauli():
    import dense_evolution as de
    with open(os.path.join(GOLDEN, 'golden_pauli.json')) as f:
        meta = json.load(f)
    d = np.load(os.path.join(GOLDEN, 'golden_pauli.npz'))
    for i, m in enumerate(meta):
        psi = d[f'psi{i}']
        terms = [(c, s) for c, s in m['terms']]
        exp = [de.pauli_expectation(psi, s) for _, s in terms]
        assert np.allclose(exp, d[f'exp{i}'], atol=1e-12)
        assert de.pauli_sum_expectation(psi, terms) == pytest.approx(float(d[f'sum{i}']), abs=1e-12)
        assert np.allclose(de.pauli_sum_matvec(psi, terms), d[f'mv{i}'], atol=1e-12)


def _rand_terms(rng, n, k, maxw=None):
    terms = []
    for _ in range(k):
        w = int(rng.integers(1, (maxw or n) + 1))
        qs = rng.choice(n, w, replace=False)
        terms.append((float(rng.normal()), {int(q): str(rng.choice(list('XYZ'))) for q in qs}))
    return terms


@pytest.mark.parametrize('n', [3, 5, 9, 13, 17])
def test_random_hamiltonians_vs_oracle(n):
    import torch
    import dense_evolution as de
    rng = np.random.default_rng(n)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    terms = _rand_terms(rng, n, 40) + _rand_terms(rng, n, 10, maxw=2)
    e = de.pauli_sum_expectation(psi, terms)
    assert e == pytest.approx(O.pauli_sum_expectation(psi, terms), abs=1e-10)
    mv = de.pauli_sum_matvec(psi, terms)
    assert np.allclose(mv, O.pauli_sum_matvec(psi, terms), atol=1e-10)
    # complex64 device state: FP32 amplitude products, FP64 accumulation
    t = torch.from_numpy(psi.astype(np.complex64)).cuda()
    e32 = de.pauli_sum_expectation(t, terms)
    assert e32 == pytest.approx(O.pauli_sum_expectation(psi.astype(np.complex64).astype(complex), terms), abs=1e-6)
    op = de.PauliSumOperator(terms, n)
    assert np.allclose((op @ t).cpu().numpy(), O.pauli_sum_matvec(psi, terms), atol=1e-5)


def test_wide_terms_use_direct_pass():
    import dense_evolution as de
    from dense_evolution.physics.observables import PauliPlan
    n = 20
    rng = np.random.default_rng(1)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    terms = [(0.7, 'X' * n), (0.2, 'Y' * 10 + 'Z' * 10), (-0.4, {0: 'X', 19: 'Y'})]
    plan = PauliPlan(terms, n, tile_bits=10)
    assert any(int(p['tile_bits']) == 0 for p in plan.passes)
    assert de.pauli_sum_expectation(psi, terms) == pytest.approx(O.pauli_sum_expectation(psi, terms), abs=1e-10)
    assert np.allclose(de.pauli_sum_matvec(psi, terms), O.pauli_sum_matvec(psi, terms), atol=1e-10)


def test_api_edge_cases():
    import dense_evolution as de
    psi = np.array([1.0, 0, 0, 0])
    assert de.pauli_sum_expectation(psi, []) == 0.0
    with pytest.raises(ValueError):
        de.pauli_expectation(psi, 'ZZZ', n_qubits=2)
    with pytest.raises(ValueError):
        de.pauli_expectation(psi, {0: 'Q'})
    with pytest.raises(ValueError):
        de.pauli_expectation(psi, {5: 'Z'})
    with pytest.raises(ValueError):
        de.pauli_expectation(np.ones(3), 'Z')
    sim = de.DenseSVSimulator(3)
    sim.run_circuit([('h', 0), ('cx', 0, 1), ('cx', 1, 2)])
    assert de.pauli_expectation(sim.get_statevector(), 'ZZZ') == pytest.approx(0.0, abs=1e-12)
    assert de.pauli_expectation(sim.sv, 'ZZI') == pytest.approx(1.0, abs=1e-12)
    assert de.multiply_pauli_terms([(1.0, 'X'), (1.0, 'Y')]) == (1j, {0: 'Z'})
    H = de.pauli_hamiltonian_to_matrix([(1.0, 'ZZ'), (0.5, {0: 'X'})], 2)
    assert np.allclose(H, O.pauli_hamiltonian_to_matrix([(1.0, 'ZZ'), (0.5, {0: 'X'})], 2))


def test_expect_passes_on_side_streams_from_two_threads():
    """<H> runs its passes concurrently on the library's side streams: two host
    threads on two streams, each with its own state, get their own energies, and a
    graph capture of the same call (which runs the passes in order) agrees."""
    import threading
    import torch
    from dense_evolution.physics.observables import PauliPlan
    n = 17
    rng = np.random.default_rng(5)
    terms = _rand_terms(rng, n, 40) + _rand_terms(rng, n, 10, maxw=2)
    plan = PauliPlan(terms, n, tile_bits=10)     # complex128 states: 10-bit tiles
    assert plan.npasses > 1
    states, want = [], []
    for _ in range(2):
        v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        v /= np.linalg.norm(v)
        states.append(torch.from_numpy(v).cuda())
        want.append(O.pauli_sum_expectation(v, terms))
    got = [[], []]

    def worker(i):
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            for _ in range(20):
                got[i].append(plan.expect(states[i]))
        s.synchronize()

    th = [threading.Thread(target=worker, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i in range(2):
        for e in got[i]:
            assert float(e[0]) == pytest.approx(want[i], abs=1e-10)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        plan.expect(states[0])           # warm the plan's buffers outside the capture
        with torch.cuda.graph(g, stream=s):
            e = plan.expect(states[0])
    g.replay()
    torch.cuda.synchronize()
    assert float(e[0]) == pytest.approx(want[0], abs=1e-10)
