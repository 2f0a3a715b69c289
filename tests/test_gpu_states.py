"""GPU parity: DenseSVSimulator (fused CUDA passes / single-gate kernels) vs the
reference's own outputs (golden fixtures) and the oracle.

Tolerances: complex128 fidelity >= 1 - 1e-12; complex64
max |d amplitude| <= 1e-5."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu


def _cases():
    with open(os.path.join(GOLDEN, 'golden_cases.json')) as f:
        return json.load(f)


STATES = np.load(os.path.join(GOLDEN, 'golden_states.npz'))


def _fid(a, b):
    return abs(np.vdot(a, b)) ** 2


@pytest.mark.parametrize('case', _cases(), ids=lambda c: c['name'])
@pytest.mark.parametrize('f32', [False, True])
def test_golden_cases(case, f32):
    import dense_evolution as de
    sim = de.DenseSVSimulator(case['n'], use_float32=f32)
    sim.run_circuit([tuple(c) for c in case['circuit']])
    got = sim.get_statevector()
    ref = STATES[case['name'] + '__c128']
    assert got.dtype == (np.complex64 if f32 else np.complex128)
    if f32:
        assert np.max(np.abs(got - ref)) <= 1e-5
    else:
        assert _fid(got, ref) >= 1 - 1e-12
        assert np.max(np.abs(got - ref)) < 1e-12


@pytest.mark.parametrize('n', [9, 10, 12, 14, 16])
@pytest.mark.parametrize('seed', [0, 1])
def test_fused_random_circuits_vs_oracle(n, seed):
    import dense_evolution as de
    circ = de.random_circuit(n, 30 * n, seed=seed)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    for f32 in (False, True):
        sim = de.DenseSVSimulator(n, use_float32=f32)
        sim.run_circuit(circ)
        got = sim.get_statevector()
        if f32:
            assert np.max(np.abs(got - ref)) <= 1e-5
        else:
            assert _fid(got, ref) >= 1 - 1e-12


@pytest.mark.parametrize('tile_bits', [9, 10, 11, 12])
def test_every_tile_size(tile_bits, monkeypatch):
    import torch
    import dense_evolution as de
    from dense_evolution.circuits.compiler import CompiledCircuit
    from dense_evolution.workloads import brick_u3_circuit
    n = 15
    circ = brick_u3_circuit(n, 5, seed=tile_bits)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    for dt in (torch.complex128, torch.complex64):
        if dt == torch.complex128 and tile_bits > 12:
            continue
        plan = CompiledCircuit(de.QuantumTranspiler.transpile(circ), n, dt, tile_bits=tile_bits)
        sv = torch.zeros(1 << n, dtype=dt, device='cuda')
        sv[0] = 1
        plan.run(sv)
        got = sv.cpu().numpy()
        tol = 1e-12 if dt == torch.complex128 else 1e-5
        assert np.max(np.abs(got - ref)) <= tol


def test_config1_full_size_vs_reference_fingerprint():
    """20 qubits, 20 layers, complex128 (config 1)."""
    import dense_evolution as de
    from dense_evolution.workloads import brick_u3_circuit
    d = np.load(os.path.join(GOLDEN, 'golden_config1.npz'))
    n = int(d['n'])
    sim = de.DenseSVSimulator(n)
    sim.run_circuit(brick_u3_circuit(n, int(d['layers']), int(d['seed'])))
    sv = sim.get_statevector()
    assert np.max(np.abs(sv[d['idx']] - d['amp'])) < 1e-12
    assert np.allclose(sim.expectation_z(), d['z'], atol=1e-12)
    ref = O.run_circuit(O.zero_state(n), n, brick_u3_circuit(n, int(d['layers']), int(d['seed'])))
    assert _fid(sv, ref) >= 1 - 1e-12


def test_device_status_clean():
    import dense_evolution as de
    from dense_evolution import _native as N
    sim = de.DenseSVSimulator(12)
    sim.run_circuit(de.random_circuit(12, 200, seed=3))
    N.device_status()
