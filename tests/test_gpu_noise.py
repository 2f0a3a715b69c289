"""Stochastic Kraus channels on the GPU against fixtures made by the reference
(tests/golden/make_noise_golden.py), and energy_fn(noise=...) against the
oracle: one noisy shot, and for the Pauli channels the adjoint gradient
against central differences of the same shot."""
import os

import numpy as np
import pytest

from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'golden_noise.npz')


def _cases():
    z = np.load(GOLD)
    for k in range(int(z['ncases'][0])):
        n, p, seed, mi = z[f'c{k}_meta']
        q = [int(x) for x in z[f'c{k}_qubits']] if bool(z[f'c{k}_hasq'][0]) else None
        yield (str(z['models'][int(mi)]), int(n), float(p), int(seed), q, z[f'c{k}_in'], z[f'c{k}_out'])


CASES = list(_cases())


@pytest.mark.parametrize('case', CASES, ids=lambda c: f'{c[0]}-n{c[1]}-p{c[2]}-s{c[3]}')
def test_apply_to_sv_matches_reference(case):
    import torch
    import dense_evolution as de
    model, n, p, seed, q, v, ref = case
    got = de.NoiseModel.apply_to_sv(v.copy(), n, model, p, rng=np.random.default_rng(seed), qubits=q)
    assert isinstance(got, np.ndarray)
    assert np.max(np.abs(got - ref)) < 1e-12
    # a CUDA tensor stays on the device and is not modified
    t = torch.from_numpy(v.copy()).cuda()
    got_t = de.NoiseModel.apply_to_sv(t, n, model, p, rng=np.random.default_rng(seed), qubits=q)
    assert got_t.is_cuda and np.max(np.abs(got_t.cpu().numpy() - ref)) < 1e-12
    assert np.array_equal(t.cpu().numpy(), v)
    # complex64 input keeps its precision
    got32 = de.NoiseModel.apply_to_sv(v.astype(np.complex64), n, model, p, rng=np.random.default_rng(seed),
                                      qubits=q)
    assert got32.dtype == np.complex64 and np.max(np.abs(got32 - ref)) < 1e-5


def test_noise_model_api():
    import dense_evolution as de
    assert de.NoiseModel.MODELS == ['ideal', 'depolarizing', 'bitflip', 'phaseflip', 'amplitude_damping',
                                    'combined']
    assert de.NoiseModel.kraus_description('bitflip')['physical'] == 'Bit flip σ_x with probability p'
    v = np.ones(8, np.complex128) / np.sqrt(8)
    assert de.NoiseModel.apply_to_sv(v, 3, 'ideal', 0.5) is v
    assert de.NoiseModel.apply_to_sv(v, 3, 'bitflip', 0.0) is v
    with pytest.raises(KeyError):
        de.NoiseModel.apply_to_sv(v, 3, 'nonsense', 0.5)


def _problem(n):
    from dense_evolution.workloads import hea_circuit, tfim_terms
    circ = hea_circuit(n, 2)
    ops = [{'name': c[0], 'qubits': [x for x in c[1:] if isinstance(x, int)]} for c in circ]
    rows, npar = O.energy_template(ops, n)
    theta = np.random.default_rng(5).uniform(-np.pi, np.pi, npar)
    return circ, rows, npar, theta, tfim_terms(n)


@pytest.mark.parametrize('model', ['depolarizing', 'bitflip', 'phaseflip', 'amplitude_damping', 'combined'])
def test_energy_fn_noise_matches_oracle(model):
    import dense_evolution as de
    n = 10
    circ, rows, npar, theta, terms = _problem(n)
    fn, _ = de.circuit_to_energy_fn(circ, n)
    spec = de.NoiseSpec(model, 0.4, 11, qubits=[0, 3, 4, 9])
    e, sv = fn(theta, terms, noise=spec)
    _, psi = O.energy(theta, rows, n, terms)
    noisy = O.noise_apply(psi, n, model, 0.4, np.random.default_rng([11]), [0, 3, 4, 9])
    e_ref = float(np.real(np.vdot(noisy, O.pauli_sum_matvec(noisy, terms))))
    assert float(e) == pytest.approx(e_ref, abs=1e-10)
    assert np.max(np.abs(sv.cpu().numpy() - noisy)) < 1e-12


def test_energy_fn_pauli_noise_gradient():
    import torch
    import dense_evolution as de
    n = 10
    circ, rows, npar, theta, terms = _problem(n)
    fn, _ = de.circuit_to_energy_fn(circ, n)
    spec = de.NoiseSpec('depolarizing', 0.6, 4)
    th = torch.tensor(theta, requires_grad=True)
    e, _ = fn(th, terms, noise=spec)
    e.backward()
    g = th.grad.numpy()
    h = 1e-5
    for i in np.random.default_rng(2).choice(npar, 6, replace=False):
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (float(fn(tp, terms, noise=spec)[0]) - float(fn(tm, terms, noise=spec)[0])) / (2 * h)
        assert g[i] == pytest.approx(fd, abs=1e-7)


def test_energy_fn_damping_gradient_refused():
    import torch
    import dense_evolution as de
    n = 9
    circ, rows, npar, theta, terms = _problem(n)
    fn, _ = de.circuit_to_energy_fn(circ, n)
    th = torch.tensor(theta, requires_grad=True)
    e, _ = fn(th, terms, noise=de.NoiseSpec('amplitude_damping', 0.3, 1))
    with pytest.raises(NotImplementedError):
        e.backward()


@pytest.mark.parametrize('model', ['depolarizing', 'bitflip', 'phaseflip'])
def test_noise_rides_in_the_circuit_passes(model):
    """energy_fn(noise=...) without a gradient applies the Pauli shot inside the
    circuit's own passes (the noise template's angles); at 20 qubits complex64
    (rotation passes) it matches the shot applied as passes of their own over a
    copy of the state: |dE| <= 1e-6, amplitudes to 1e-5."""
    import dense_evolution as de
    n = 20
    circ, rows, npar, theta, terms = _problem(n)
    fn, _ = de.circuit_to_energy_fn(circ, n, use_float32=True)
    prog = fn.program
    spec = de.NoiseSpec(model, 0.3, 7, qubits=[0, 5, 13, 19])
    e1, sv1 = fn(theta, terms, noise=spec)
    psi = prog.forward_state(np.asarray(theta))
    noisy, errs = prog.apply_noise(psi, spec)
    _, e2 = prog.apply_h(terms, noisy, need_lambda=False)
    assert errs                      # the seed fires at least one error
    assert float(e1) == pytest.approx(e2, abs=1e-6)
    assert float(np.max(np.abs(sv1.cpu().numpy() - noisy.cpu().numpy()))) < 1e-5
