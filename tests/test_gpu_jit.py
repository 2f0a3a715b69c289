"""Plan-specialised pass kernels (NVRTC-compiled for sm_100a) against the fused
interpreter and the oracle on the same seeded circuits.

The specialised kernel runs the interpreter's op bodies in the same order, so
the two agree to rounding (FMA contraction may differ); both are held to the
oracle at the engine's tolerances (complex128 1e-12, complex64 1e-5)."""
import numpy as np
import pytest

from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu

# every lowering family: controlled on slots / lanes / thread bits, diagonals,
# sign groups, predicated and anti-diagonal ops
MIXED = ['h', 'x', 'y', 'z', 's', 'sdg', 't', 'rx', 'ry', 'rz', 'p', 'u3', 'sx',
         'cx', 'cz', 'cy', 'swap', 'iswap', 'ecr', 'cp', 'crz', 'ccx']


def _run(plan, n, dt, theta=None):
    import torch
    sv = torch.zeros(1 << n, dtype=dt, device='cuda')
    sv[0] = 1
    plan.run(sv, theta)
    torch.cuda.synchronize()
    return sv.cpu().numpy()


def _circuit(n, seed):
    import dense_evolution as de
    rng = np.random.default_rng(seed)
    circ = de.random_circuit(n, 25 * n, seed=seed)
    for _ in range(3 * n):
        a, b, c = (int(x) for x in rng.choice(n, 3, replace=False))
        g = MIXED[rng.integers(len(MIXED))]
        if g == 'ccx':
            circ.append(('ccx', a, b, c))
        elif g in ('cp', 'crz'):
            circ.append((g, a, b, float(rng.choice([np.pi, rng.uniform(-3, 3)]))))
        elif g in ('cx', 'cz', 'cy', 'swap', 'iswap', 'ecr'):
            circ.append((g, a, b))
        elif g == 'u3':
            circ.append(('u3', a, *rng.uniform(0, 2 * np.pi, 3)))
        elif g in ('rx', 'ry', 'rz', 'p'):
            circ.append((g, a, float(rng.uniform(-3, 3))))
        else:
            circ.append((g, a))
    return circ


@pytest.mark.parametrize('n,seed', [(10, 0), (13, 1), (16, 2)])
def test_specialised_passes_match_interpreter_and_oracle(n, seed, monkeypatch):
    import torch
    import dense_evolution as de
    from dense_evolution.circuits.compiler import CompiledCircuit
    circ = _circuit(n, seed)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    for dt, tol in ((torch.complex128, 1e-12), (torch.complex64, 1e-5)):
        plan = CompiledCircuit(de.QuantumTranspiler.transpile(circ), n, dt)
        monkeypatch.setenv('DESV_JIT', '0')
        interp = _run(plan, n, dt)
        monkeypatch.setenv('DESV_JIT', '1')
        spec = _run(plan, n, dt)
        assert np.max(np.abs(spec - interp)) <= (1e-14 if dt == torch.complex128 else 1e-6)
        assert np.max(np.abs(spec - ref)) <= tol


@pytest.mark.parametrize('tile_bits', [10, 11, 12])
def test_specialised_brick_every_tile_and_new_angles(tile_bits, monkeypatch):
    """Kernels compile once per structure; new angles reuse them."""
    import torch
    import dense_evolution as de
    from dense_evolution.circuits.compiler import CompiledCircuit
    from dense_evolution.circuits import jit
    from dense_evolution.workloads import brick_u3_circuit
    n = 17
    monkeypatch.setenv('DESV_JIT', '1')
    for seed in (5, 6):
        circ = brick_u3_circuit(n, 6, seed=seed)
        ref = O.run_circuit(O.zero_state(n), n, circ)
        plan = CompiledCircuit(de.QuantumTranspiler.transpile(circ), n, torch.complex64, tile_bits=tile_bits)
        before = len(jit._cache)
        got = _run(plan, n, torch.complex64)
        assert np.max(np.abs(got - ref)) <= 1e-5
        if seed == 6:
            assert len(jit._cache) == before   # same structure: no new compile


def test_parametric_plan_follows_theta(monkeypatch):
    import torch
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, tfim_terms
    n = 14
    monkeypatch.setenv('DESV_JIT', '1')
    fn, npar = de.circuit_to_energy_fn(hea_circuit(n, 3), n)
    op = de.PauliSumOperator(tfim_terms(n), n)
    rows, _ = O.energy_template([{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]}
                                 for c in hea_circuit(n, 3)], n)
    for s in (0, 1):
        theta = np.random.default_rng(s).uniform(-np.pi, np.pi, npar)
        e, _ = fn(theta, op)
        assert float(e) == pytest.approx(O.energy(theta, rows, n, tfim_terms(n))[0], abs=1e-10)


def test_default_path_at_22_qubits_matches_interpreter(monkeypatch):
    import torch
    import dense_evolution as de
    from dense_evolution.circuits.compiler import CompiledCircuit
    from dense_evolution.circuits import jit
    from dense_evolution.workloads import brick_u3_circuit
    n = 22
    monkeypatch.delenv('DESV_JIT', raising=False)
    assert jit.enabled(n)
    plan = CompiledCircuit(de.QuantumTranspiler.transpile(brick_u3_circuit(n, 12, 3)), n, torch.complex64)
    spec = _run(plan, n, torch.complex64)
    monkeypatch.setenv('DESV_JIT', '0')
    interp = _run(plan, n, torch.complex64)
    assert np.max(np.abs(spec - interp)) <= 1e-6
    de._native.device_status()


@pytest.mark.parametrize('n', [12, 15])
def test_specialised_adjoint_matches_interpreter_and_fd(n, monkeypatch):
    """Backward passes compiled per pass (complex64) against the interpreted
    backward sweep and complex128 central differences."""
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, tfim_terms
    layers = 3
    circ = hea_circuit(n, layers) + [('crz', 0, n - 1, 0.0), ('cp', 2, 1, 0.0), ('p', 3, 0.0)]
    terms = tfim_terms(n) + [(0.3, {0: 'Y', n - 1: 'Y'})]
    theta = np.random.default_rng(n).uniform(-np.pi, np.pi, de.circuit_to_energy_fn(circ, n)[1])
    res = {}
    for flag in ('0', '1'):
        monkeypatch.setenv('DESV_JIT', flag)
        fn, _ = de.circuit_to_energy_fn(circ, n, use_float32=True)
        e, g, _ = fn.program.value_and_grad(theta, terms)
        res[flag] = (e, g)
    assert res['1'][0] == pytest.approx(res['0'][0], abs=1e-7)
    assert np.max(np.abs(res['1'][1] - res['0'][1])) <= 1e-6
    monkeypatch.setenv('DESV_JIT', '0')
    f64, _ = de.circuit_to_energy_fn(circ, n)
    h = 1e-4
    for i in np.random.default_rng(1).choice(theta.size, 6, replace=False):
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (float(f64(tp, terms)[0]) - float(f64(tm, terms)[0])) / (2 * h)
        assert res['1'][1][i] == pytest.approx(fd, abs=2e-5)


@pytest.mark.parametrize('n,dtname', [(12, 'complex128'), (13, 'complex64'), (21, 'complex64')])
def test_specialised_pauli_passes_match_interpreter_and_oracle(n, dtname, monkeypatch):
    """<H> and H|psi> with the tiled Pauli passes compiled per pass against the
    interpreted passes and the oracle; the terms mix flip masks, Y phases,
    sign masks reaching outside the tile and one mask too wide for a tile."""
    import torch
    from dense_evolution.physics.observables import plan_for
    from dense_evolution.workloads import tfim_terms, xxz_terms
    dt = getattr(torch, dtname)
    terms = (tfim_terms(n) + xxz_terms(n, 0.7) + [(0.3, {0: 'Y', n - 1: 'Y'}), (0.2, {1: 'X', 2: 'Y', 7: 'Z'}),
             (-0.4, 'Z' * n), (0.15, {q: 'X' for q in range(0, n, 2)})])
    rng = np.random.default_rng(n)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    psi = torch.from_numpy(v.astype(np.complex64 if dt == torch.complex64 else np.complex128)).cuda()
    got = {}
    for flag in ('0', '1'):
        monkeypatch.setenv('DESV_JIT', flag)
        plan = plan_for(terms, n, dtype=dt)
        e = float(plan.expect(psi)[0])
        out, e2 = plan.matvec(psi, want_expect=True)
        torch.cuda.synchronize()
        got[flag] = (e, out.cpu().numpy(), float(e2[0]))
    e_tol, v_tol = (1e-12, 1e-13) if dt == torch.complex128 else (1e-9, 1e-6)
    # complex64 <H> passes form each amplitude's products Re(conj(a) p) in FP32
    # (sums widened to FP64 once per tile): random rounding of about 6e-8 of
    # each product, which on this unit state of 2^13 amplitudes sums to a few
    # 1e-9 per term; 1e-7 bounds it, ten times under the 1e-6 energy bar
    x_tol = 1e-12 if dt == torch.complex128 else 1e-7
    assert got['1'][0] == pytest.approx(got['0'][0], abs=x_tol)
    assert got['1'][2] == pytest.approx(got['0'][2], abs=e_tol)
    assert np.max(np.abs(got['1'][1] - got['0'][1])) <= v_tol
    if n <= 13:
        ref_v = psi.cpu().numpy().astype(np.complex128)
        assert got['1'][0] == pytest.approx(O.pauli_sum_expectation(ref_v, terms, n), abs=max(x_tol, 1e-9))
        assert np.max(np.abs(got['1'][1] - O.pauli_sum_matvec(ref_v, terms, n))) <= (1e-12 if dt == torch.complex128
                                                                                      else 1e-5)
