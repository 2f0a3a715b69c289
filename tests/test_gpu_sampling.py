"""Finite-shot sampling on the GPU (desv_sample_prepare / desv_sample_pick
through sample_counts) against counts made by the reference itself
(tests/golden/make_sample_golden.py)."""
import json
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(__file__)
sys.path.insert(0, os.path.join(HERE, 'golden'))


def _cases():
    from make_sample_golden import sample_states
    with open(os.path.join(HERE, 'golden', 'golden_sample.json')) as f:
        ref = json.load(f)
    return [(c, v) for c, (_, _, _, v) in zip(ref, sample_states())]


@pytest.mark.parametrize('case', _cases(), ids=lambda c: f"n{c[0]['n']}-shots{c[0]['shots']}")
def test_sample_counts_matches_reference(case):
    import torch
    import dense_evolution as de
    c, v = case
    got = de.sample_counts(v, c['shots'], rng=np.random.default_rng(c['seed']))
    assert got == c['counts']
    # a CUDA tensor input gives the same draws
    got_t = de.sample_counts(torch.from_numpy(v).cuda(), c['shots'], rng=np.random.default_rng(c['seed']))
    assert got_t == c['counts']
    # complex64 input: FP64 |a|^2 of the rounded amplitudes -- a few shots may cross a CDF step
    got32 = de.sample_counts(v.astype(np.complex64), c['shots'], rng=np.random.default_rng(c['seed']))
    keys = set(got32) | set(c['counts'])
    diff = sum(abs(got32.get(k, 0) - c['counts'].get(k, 0)) for k in keys)
    assert sum(got32.values()) == c['shots'] and diff <= max(6, c['shots'] // 1000)


def test_sample_counts_errors_and_large_state():
    import torch
    import dense_evolution as de
    with pytest.raises(ValueError):
        de.sample_counts(np.zeros(8, np.complex128), 10)
    with pytest.raises(ValueError):
        de.sample_counts(np.ones(6, np.complex128), 10)
    with pytest.raises(ValueError):
        de.sample_counts(np.ones(8, np.complex128), 0)
    # 26 qubits: qubit 0 in |+>, the rest |0>: two outcomes, about half each
    n = 26
    sim = de.DenseSVSimulator(n, use_float32=True)
    sim.run_circuit([('h', 0)])
    counts = de.sample_counts(sim.sv, 200000, rng=np.random.default_rng(1))
    assert set(counts) <= {'0' * n, '1' + '0' * (n - 1)}
    assert abs(counts['0' * n] - 100000) < 2000
    assert sum(counts.values()) == 200000
