"""DenseSVSimulator API behaviour (ported from the reference's test_simulator.py)."""
import warnings

import numpy as np
import pytest

from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def de():
    import dense_evolution
    return dense_evolution


def test_init_and_state(de):
    sim = de.DenseSVSimulator(2)
    assert np.allclose(sim.get_statevector(), [1, 0, 0, 0])
    assert np.allclose(sim.get_probabilities(), [1, 0, 0, 0])
    sim.set_initial_state(np.array([1, 1, 0, 0]))
    assert np.allclose(sim.get_statevector(), np.array([1, 1, 0, 0]) / np.sqrt(2))
    with pytest.raises(ValueError):
        sim.set_initial_state(np.zeros(3))
    with pytest.raises(ValueError):
        sim.set_initial_state(np.zeros(4))
    sim.set_initial_state(None)
    assert np.allclose(sim.get_statevector(), [1, 0, 0, 0])
    sim.set_state(np.array([0, 0, 0, 2.0]))
    assert np.allclose(sim.get_statevector(), [0, 0, 0, 1])
    for bad in (0, 35):
        with pytest.raises(ValueError):
            de.DenseSVSimulator(bad)
    assert de.DenseSVSimulator(12).memory_mb() == pytest.approx(4096 * 16 / 1e6)
    assert de.DenseSVSimulator(12, use_float32=True).memory_mb() == pytest.approx(4096 * 8 / 1e6)


def test_msb_first_and_single_gates(de):
    sim = de.DenseSVSimulator(3)
    sim.run_circuit([('x', 0)])
    assert abs(sim.get_statevector()[4]) == pytest.approx(1.0)
    sim = de.DenseSVSimulator(3)
    sim.apply_gate_1q(de.GATES['x'], 0)
    assert abs(sim.get_statevector()[4]) == pytest.approx(1.0)
    sim.apply_cx(0, 2)
    assert abs(sim.get_statevector()[5]) == pytest.approx(1.0)
    sim.apply_cz(0, 2)
    assert sim.get_statevector()[5] == pytest.approx(-1.0)
    sim.apply_gate_2q(de.GATES['swap'], 0, 1)
    assert abs(sim.get_statevector()[3]) == pytest.approx(1.0)
    for q, t in ((0, 0.3), (1, 1.1), (2, -0.4)):
        sim.apply_rx(q, t)
        sim.apply_ry(q, t)
        sim.apply_rz(q, t)
    ref = O.zero_state(3)
    ref = O.apply_1q(ref, 3, O._STATIC['x'], 0)
    ref = O.apply_2q(ref, 3, O._STATIC['cx'], 0, 2)
    ref = O.apply_2q(ref, 3, O._STATIC['cz'], 0, 2)
    ref = O.apply_2q(ref, 3, O._STATIC['swap'], 0, 1)
    for q, t in ((0, 0.3), (1, 1.1), (2, -0.4)):
        ref = O.apply_1q(ref, 3, O._rx(t), q)
        ref = O.apply_1q(ref, 3, O._ry(t), q)
        ref = O.apply_1q(ref, 3, O._rz(t), q)
    assert np.allclose(sim.get_statevector(), ref, atol=1e-12)


def test_validation_errors(de):
    sim = de.DenseSVSimulator(4)
    with pytest.raises(ValueError):
        sim.apply_gate_1q(de.GATES['h'], 4)
    with pytest.raises(ValueError):
        sim.apply_cx(1, 1)
    with pytest.raises(ValueError):
        sim.apply_gate_2q(de.GATES['cz'], 0, 7)
    with pytest.raises(ValueError, match='issue #4'):
        sim.run_circuit([('hh', 0)])
    with pytest.raises(ValueError, match='issue #4'):
        sim.run_circuit_jit([('hh', 0)])
    with pytest.raises(ValueError):
        sim.run_circuit_jit([('h', 9)])
    with pytest.raises(ValueError):
        sim.run_circuit([('cx', 0, 9)])
    with pytest.raises(ValueError, match='issue #6'):
        sim.run_batch_jit([('rx', 0, 0.1), ('ry', 1, 0.2)], np.zeros((3, 1)))
    with pytest.raises(ValueError):
        sim.run_batch_jit([('rx', 5, 0.1)], np.zeros((3, 1)))


def test_jit_paths_and_aliases(de):
    circ = [('h', 0), ('cx', 0, 3), ('ry', 2, 0.3), ('cy', 3, 1), ('crz', 1, 2, 0.7), ('sx', 2), ('tdg', 0),
            ('swap', 0, 2), ('cp', 3, 0, 1.1), ('u3', 1, 0.1, 0.2, 0.3), ('phase', 2, 0.4), ('cphase', 1, 0, 0.5)]
    ref = O.run_circuit(O.zero_state(4), 4, circ)
    for call in ('run_circuit', 'run_circuit_jit', 'run_circuit_with_chunking'):
        sim = de.DenseSVSimulator(4)
        getattr(sim, call)(circ)
        assert np.allclose(sim.get_statevector(), ref, atol=1e-12)
    sim = de.DenseSVSimulator(4)
    with pytest.warns(DeprecationWarning):
        sim.run_circuit_jit_beast_mode(circ)
    assert np.allclose(sim.get_statevector(), ref, atol=1e-12)
    sim = de.DenseSVSimulator(4)
    sim.run_circuit(circ, transpile=False)
    assert np.allclose(sim.get_statevector(), O.run_circuit(O.zero_state(4), 4, circ), atol=1e-12)


def test_run_batch_jit_matches_run_circuit(de):
    rng = np.random.default_rng(0)
    n = 10
    base = [('ry', q, 0.0) for q in range(n)] + [('cx', q, q + 1) for q in range(n - 1)] + \
        [('rz', q, 0.0) for q in range(n)] + [('cp', 0, 5, 0.0), ('crz', 9, 2, 0.0)]
    pb = rng.uniform(-np.pi, np.pi, (5, 2 * n + 2))
    sim = de.DenseSVSimulator(n)
    out = sim.run_batch_jit(base, pb).cpu().numpy()
    for r in range(5):
        k = iter(pb[r])
        circ = [(c[0], *c[1:-1], next(k)) if c[0] in ('ry', 'rz', 'cp', 'crz') else c for c in base]
        ref = O.run_circuit(O.zero_state(n), n, circ)
        assert np.allclose(out[r], ref, atol=1e-12)
    with pytest.warns(DeprecationWarning):
        sim.run_parametric_batch_jit(base, pb)


@pytest.mark.parametrize('n,f32', [(14, False), (14, True), (9, True)])
def test_run_batch_jit_one_launch_rows(de, n, f32):
    """run_batch_jit's rows: resident states (<= 12 qubits, one persistent
    launch) and wider ones (the rows path: every pass over all output rows in
    one launch), both precisions, against the oracle per row."""
    rng = np.random.default_rng(n)
    base = [('h', q) for q in range(n)] + [('ry', q, 0.0) for q in range(n)] + \
        [('cx', q, q + 1) for q in range(n - 1)] + [('rx', q, 0.0) for q in range(0, n, 2)] + \
        [('cp', 1, n - 1, 0.0), ('crz', n - 2, 0, 0.0), ('t', 3), ('rz', n - 1, 0.0)]
    npar = sum(1 for c in base if c[0] in ('ry', 'rx', 'rz', 'cp', 'crz'))
    pb = rng.uniform(-np.pi, np.pi, (7, npar))
    sim = de.DenseSVSimulator(n, use_float32=f32)
    out = sim.run_batch_jit(base, pb).cpu().numpy()
    assert out.shape == (7, 1 << n)
    for r in range(7):
        k = iter(pb[r])
        circ = [(c[0], *c[1:-1], next(k)) if c[0] in ('ry', 'rx', 'rz', 'cp', 'crz') else c for c in base]
        ref = O.run_circuit(O.zero_state(n), n, circ)
        assert np.max(np.abs(out[r] - ref)) <= (1e-5 if f32 else 1e-12)


def test_float32_matches_float64(de):
    n = 12
    circ = de.random_circuit(n, 300, seed=11)
    a = de.DenseSVSimulator(n, use_float32=True)
    b = de.DenseSVSimulator(n)
    a.run_circuit(circ)
    b.run_circuit(circ)
    assert np.allclose(a.get_probabilities(), b.get_probabilities(), atol=1e-6)
    assert a.sv.dtype.__str__() == 'torch.complex64'


def test_measure(de):
    np.random.seed(0)
    sim = de.DenseSVSimulator(2)
    assert sim.measure(0) == 0
    sim = de.DenseSVSimulator(2)
    sim.run_circuit([('x', 0)])
    assert sim.measure(0) == 1
    sim = de.DenseSVSimulator(3)
    sim.run_circuit([('h', 0), ('cx', 0, 1), ('cx', 1, 2)])
    r = sim.measure(1)
    assert r in (0, 1)
    sv = sim.get_statevector()
    assert np.linalg.norm(sv) == pytest.approx(1.0)
    assert abs(sv[7 if r else 0]) == pytest.approx(1.0)
    with pytest.raises(ValueError):
        sim.measure(3)
    with pytest.raises(ValueError):
        sim.measure(0, jax_key=1)
    z = de.DenseSVSimulator(2)
    z.sv.zero_()
    with pytest.raises(RuntimeError):
        z.measure(0)


def test_norm_preserved_and_normalize(de):
    sim = de.DenseSVSimulator(14)
    sim.run_circuit(de.random_circuit(14, 500, seed=2))
    assert np.linalg.norm(sim.get_statevector()) == pytest.approx(1.0, abs=1e-12)
    sim.sv.mul_(3.0)
    sim.normalize()
    assert np.linalg.norm(sim.get_statevector()) == pytest.approx(1.0, abs=1e-12)


def test_fidelity_and_counts(de):
    sim = de.DenseSVSimulator(2)
    sim.run_circuit([('h', 0), ('cx', 0, 1)])
    sv = sim.get_statevector()
    assert de.statevector_fidelity(sv, sv) == pytest.approx(1.0)
    assert de.statevector_fidelity(sim.sv, np.array([1, 0, 0, 0])) == pytest.approx(0.5)
    c = de.sample_counts(sv, 1000, rng=np.random.default_rng(0))
    assert set(c) <= {'00', '11'} and sum(c.values()) == 1000
    with pytest.raises(ValueError):
        de.statevector_fidelity(sv, np.ones(8))


@pytest.mark.parametrize('n,f32', [(10, False), (20, True)])
def test_run_circuit_reuses_the_structure_with_new_angles(de, n, f32):
    """Circuits that differ only in their angles share one compiled plan (the
    angles become parameter slots); each call's state still matches the oracle
    (general fused passes at 10 qubits complex128, rotation passes at 20
    qubits complex64)."""
    from dense_evolution.workloads import brick_u3_circuit
    sim = de.DenseSVSimulator(n, use_float32=f32)
    for seed in (1, 2, 3):
        circ = brick_u3_circuit(n, 3, seed=seed)
        sim.set_initial_state(None)
        sim.run_circuit(circ)
        ref = O.run_circuit(O.zero_state(n), n, circ)
        err = float(np.max(np.abs(sim.get_statevector().astype(np.complex128) - ref)))
        assert err < (1e-5 if f32 else 1e-12), err
    assert len(sim._plans) == 1
