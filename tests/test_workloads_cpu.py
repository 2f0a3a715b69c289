"""Seeded generators reproduce the reference's circuits (golden_cases.json was
produced by the reference's random_circuit) and its topology helper."""
import json
import os

import pytest

from conftest import GOLDEN
from dense_evolution.random_circuit import random_circuit
from dense_evolution.topology import entangling_layer


def test_random_circuit_seed_parity_with_reference():
    with open(os.path.join(GOLDEN, 'golden_cases.json')) as f:
        cases = json.load(f)
    for c in cases:
        if not c['name'].startswith('random_'):
            continue
        n = c['n']
        seed = int(c['name'].split('_s')[1])
        got = random_circuit(n, 12 * n + 5, seed=seed)
        assert [list(x) for x in got] == c['circuit']


def test_random_circuit_validation():
    with pytest.raises(ValueError):
        random_circuit(0, 3)
    with pytest.raises(ValueError):
        random_circuit(2, -1)
    with pytest.raises(ValueError):
        random_circuit(2, 3, gate_set=['foo'])


def test_entangling_layer_patterns():
    assert entangling_layer(4, 'brick', 'cz') == [('cz', 0, 1), ('cz', 2, 3), ('cz', 1, 2)]
    assert entangling_layer(3, 'circular') == [('cx', 0, 1), ('cx', 1, 2), ('cx', 2, 0)]
    assert entangling_layer(2, 'circular') == [('cx', 0, 1)]
    assert entangling_layer(3, 'star', hub=1) == [('cx', 1, 0), ('cx', 1, 2)]
    assert entangling_layer(3, 'linear', reverse=True) == [('cx', 1, 0), ('cx', 2, 1)]
    with pytest.raises(ValueError):
        entangling_layer(1)
