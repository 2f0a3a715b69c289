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
