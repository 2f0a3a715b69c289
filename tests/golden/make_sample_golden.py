"""Generate golden_sample.json from the REFERENCE's sample_counts
(dense_evolution/utils/measurement.py:17-68), imported unmodified with the
stubs of make_golden.py.  Each case records a seeded state, the shot count, the
generator seed and the reference's counts dict; the states are rebuilt from
``sample_states()`` (seeded NumPy draws), so only the counts are stored.

    python tests/golden/make_sample_golden.py --reference PATH_OF_REFERENCE_CHECKOUT
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import load_reference  # noqa: E402


CASES = [(3, 1000, 1, False), (6, 5000, 2, False), (10, 20000, 3, False), (13, 50000, 4, True),
         (14, 3000, 5, False), (1, 7, 6, False)]


def sample_states():
    """(n, shots, seed, state) of every case, from one seeded generator."""
    rng0 = np.random.default_rng(99)
    out = []
    for n, shots, seed, sparse in CASES:
        v = rng0.normal(size=1 << n) + 1j * rng0.normal(size=1 << n)
        if sparse:
            v[rng0.random(1 << n) < 0.7] = 0.0          # zero-probability outcomes in between
        v /= np.linalg.norm(v)
        out.append((n, shots, seed, v))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', required=True, help='path of the reference checkout')
    args = ap.parse_args()
    ref = load_reference(args.reference)
    cases = []
    for n, shots, seed, v in sample_states():
        counts = ref.measurement.sample_counts(v, shots, rng=np.random.default_rng(seed))
        cases.append({'n': n, 'shots': shots, 'seed': seed, 'counts': counts})
    with open(os.path.join(HERE, 'golden_sample.json'), 'w') as f:
        json.dump(cases, f)
    print(f'{len(cases)} cases -> golden_sample.json')


if __name__ == '__main__':
    main()
