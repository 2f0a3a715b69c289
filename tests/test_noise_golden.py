"""The oracle's restatement of the stochastic Kraus channels and of finite-shot sampling against fixtures
produced by the reference itself (tests/golden/make_noise_golden.py,
tests/golden/make_sample_golden.py)."""
import os

import numpy as np
import pytest

from oracle import sv_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'golden_noise.npz')


def _cases():
    z = np.load(GOLD)
    for k in range(int(z['ncases'][0])):
        n, p, seed, mi = z[f'c{k}_meta']
        q = list(z[f'c{k}_qubits']) if bool(z[f'c{k}_hasq'][0]) else None
        yield (str(z['models'][int(mi)]), int(n), float(p), int(seed), q, z[f'c{k}_in'], z[f'c{k}_out'])


@pytest.mark.parametrize('case', list(_cases()), ids=lambda c: f'{c[0]}-n{c[1]}-p{c[2]}-s{c[3]}')
def test_oracle_noise_matches_reference(case):
    model, n, p, seed, q, v, ref = case
    got = O.noise_apply(v, n, model, p, np.random.default_rng(seed), q)
    assert np.max(np.abs(np.asarray(got) - ref)) < 1e-12


def _sample_cases():
    import json
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from make_sample_golden import sample_states
    with open(os.path.join(os.path.dirname(__file__), 'golden', 'golden_sample.json')) as f:
        ref = json.load(f)
    return [(c, v) for c, (_, _, _, v) in zip(ref, sample_states())]


@pytest.mark.parametrize('case', _sample_cases(), ids=lambda c: f"n{c[0]['n']}-shots{c[0]['shots']}")
def test_oracle_sample_counts_matches_reference(case):
    c, v = case
    got = O.sample_counts(v, c['shots'], rng=np.random.default_rng(c['seed']))
    assert got == c['counts']


@pytest.mark.parametrize('model', ['depolarizing', 'bitflip', 'phaseflip'])
def test_pauli_noise_template_matches_the_channel(model):
    """The Pauli-channel template appended to the energy circuit (rx / ry / rz
    per noise qubit at angle 0 or pi, one gphase of pi/2 per fired error),
    with the drawn errors as its angles, gives the channel's noisy state
    (before the final normalisation) exactly: checked with the oracle on the
    template's gate list."""
    import torch
    from dense_evolution.noise import kraus_channels as K
    from dense_evolution.solvers.adjoint import AdjointProgram
    from dense_evolution.solvers.autodiff import build_template
    from dense_evolution.workloads import hea_circuit
    n, qubits = 7, [0, 2, 5, 6]
    circ = hea_circuit(n, 2)
    rows, slots, npar = build_template(circ, n)
    prog = AdjointProgram(rows, slots, n, torch.complex128)
    theta = np.random.default_rng(9).uniform(-np.pi, np.pi, npar)
    cc, where, gslot = prog._noise_template(model, qubits)
    for seed in range(6):
        errs = K.draw_pauli_errors(model, 0.6, n, np.random.default_rng(seed), qubits)
        full = np.zeros(gslot + 1)
        full[:npar] = theta
        for q, w in errs:
            full[where[(q, w)]] = np.pi
        full[gslot] = 0.5 * np.pi * len(errs)
        bound = []
        for cmd, sl in zip(cc._target, cc._slots):
            bound.append(tuple(cmd[:-1]) + (float(full[sl]),) if sl >= 0 else tuple(cmd))
        got = O.run_circuit(O.zero_state(n), n, bound, do_transpile=False)
        orows, _ = O.energy_template([{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]}
                                      for c in circ], n)
        _, psi = O.energy(theta, orows, n, [])
        ref = O.noise_apply(psi, n, model, 0.6, np.random.default_rng(seed), qubits)
        got = got / (np.linalg.norm(got) + 1e-15)
        assert np.max(np.abs(got - ref)) < 1e-12, (seed, errs)
