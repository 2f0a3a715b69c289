"""Host fusion pass + packer, executed by the NumPy plan emulator (the exact
semantics of the CUDA pass kernels) and checked against the oracle."""
import numpy as np
import pytest

from oracle import sv_oracle as O
from plan_emulator import run_passes
from dense_evolution.circuits import fusion
from dense_evolution.circuits.compiler import QuantumTranspiler
from dense_evolution.random_circuit import random_circuit
from dense_evolution.workloads import brick_u3_circuit, hea_circuit
from dense_evolution.solvers import adjoint, autodiff


def _emulate(circ, n, kmax, theta=None, slots=None, merge=True):
    target = QuantumTranspiler.transpile(circ)
    ir, fops, packed = fusion.build(target, n, kmax, slots, merge)
    mats = packed.materialize(theta, np.complex128)
    got = run_passes(O.zero_state(n), n, packed.passes, packed.ops, mats)
    # the grouped stream the forward kernels run must give the same state
    ops, passes, pool = packed.compact(mats)
    grouped = run_passes(O.zero_state(n), n, passes, ops, pool)
    assert np.max(np.abs(grouped - got)) < 1e-12
    return got, packed


@pytest.mark.parametrize('n,kmax', [(9, 9), (10, 9), (11, 10), (12, 12), (13, 11)])
@pytest.mark.parametrize('seed', [0, 1, 2])
def test_random_circuits(n, kmax, seed):
    circ = random_circuit(n, 40 * n, seed=seed)
    got, packed = _emulate(circ, n, kmax)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(got - ref)) < 1e-12


@pytest.mark.parametrize('n,kmax', [(10, 9), (12, 12), (14, 11)])
def test_brick_u3(n, kmax):
    circ = brick_u3_circuit(n, 6, seed=n)
    got, packed = _emulate(circ, n, kmax)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(got - ref)) < 1e-12
    # fewer passes than layers x tile coverage would need without light-cone packing
    assert len(packed.passes) <= 6 * ((n + kmax - 1) // kmax) + 1


def test_mixed_gates_all_kinds():
    rng = np.random.default_rng(5)
    n = 11
    circ = []
    for _ in range(300):
        a, b, c = (int(x) for x in rng.choice(n, 3, replace=False))
        th = [float(x) for x in rng.uniform(-np.pi, np.pi, 3)]
        k = rng.integers(12)
        circ.append([('u3', a, *th), ('u2', a, th[0], th[1]), ('ccx', a, b, c), ('iswap', a, b), ('ecr', a, b),
                     ('cp', a, b, th[0]), ('crz', a, b, th[1]), ('p', a, th[2]), ('cy', a, b), ('swap', a, b),
                     ('sx', a), ('tdg', b)][k])
    got, _ = _emulate(circ, n, 10)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(got - ref)) < 1e-12


def test_untranspiled_dense_two_qubit_gates():
    n = 10
    circ = [('h', q) for q in range(n)] + [('swap', 0, 9), ('iswap', 3, 7), ('ecr', 8, 2), ('rx', 5, 0.3),
                                           ('iswap', 9, 6)]
    target = list(circ)          # transpile=False path: m2 ops
    ir, fops, packed = fusion.build(target, n, 9)
    mats = packed.materialize(None, np.complex128)
    got = run_passes(O.zero_state(n), n, packed.passes, packed.ops, mats)
    ref = O.run_circuit(O.zero_state(n), n, circ, do_transpile=False)
    assert np.max(np.abs(got - ref)) < 1e-12


@pytest.mark.parametrize('n,split', [(9, 0), (12, 0), (12, 7)])
def test_adjoint_plan_gradient_matches_fd(n, split):
    """split > 0: backward passes (and stages) split to at most `split` gates,
    as the complex64 path does to keep every pass specialised."""
    layers = 2
    rng = np.random.default_rng(n)
    theta = rng.uniform(-np.pi, np.pi, 2 * n * layers)
    circ = hea_circuit(n, layers) + [('crz', 0, n - 1, 0.0), ('cp', 2, 1, 0.0), ('p', 3, 0.0), ('rx', 4, 0.0)]
    rows, slots, npar = autodiff.build_template(circ, n)
    theta = np.concatenate([theta, rng.uniform(-1, 1, npar - theta.size)])
    ir = fusion.lower(rows, n, slots)
    fops = fusion.fuse_1q(ir)
    fwd = fusion.Packed(n, fops, fusion.schedule(fops, n, 10))
    psi = run_passes(O.zero_state(n), n, fwd.passes, fwd.ops, fwd.materialize(theta, np.complex128))
    terms = [(-1.0, {i: 'Z', i + 1: 'Z'}) for i in range(n - 1)] + [(-0.7, {i: 'X'}) for i in range(n)] + \
        [(0.3, {0: 'Y', n - 1: 'Y'})]
    lam = O.pauli_sum_matvec(psi, terms)
    bops = adjoint.backward_ops(ir)
    specs = adjoint._split_params(fusion.schedule(bops, n, 10), bops, 1024)
    if split:
        pieces = adjoint._split_ops(specs, split)
        assert len(pieces) > len(specs)
        assert all(sum(len(ids) for _, ids in ps.stages) <= split for ps in pieces)
        flat = [i for ps in specs for _, ids in ps.stages for i in ids]
        assert [i for ps in pieces for _, ids in ps.stages for i in ids] == flat
        specs = pieces
    back = fusion.Packed(n, bops, specs, adjoint=True)
    grad = np.zeros(npar)
    _, _, grad = run_passes(psi, n, back.passes, back.ops, back.materialize(theta, np.complex128), lam=lam,
                            grad=grad, param_map=back.param_map)
    orows, onp = O.energy_template([{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]}
                                    for c in circ], n)
    fd = O.fd_gradient(theta, orows, n, terms, h=1e-5)
    assert np.allclose(grad, fd, atol=1e-7)


def test_grouped_stream_follows_new_parameters():
    """One parametric plan, two parameter vectors: the grouped stream (its cached
    structure and its per-call values) must follow theta."""
    n, kmax = 11, 10
    rng = np.random.default_rng(3)
    circ = []
    for q in range(n):
        circ += [('ry', q, 0.0), ('rz', q, 0.0)]
    circ += [('cx', q, q + 1) for q in range(n - 1)]
    circ += [('cp', 0, 6, 0.0), ('crz', 9, 2, 0.0), ('rz', 4, 0.0), ('cz', 3, 8), ('p', 7, 0.0)]
    circ += [('h', q) for q in range(n)] + [('t', q) for q in range(0, n, 2)]
    target = QuantumTranspiler.transpile(circ)
    slots, k = [], 0
    for c in target:
        if c[0] in ('ry', 'rz', 'cp', 'crz', 'p'):
            slots.append(k)
            k += 1
        else:
            slots.append(-1)
    _, _, packed = fusion.build(target, n, kmax, slots)
    for trial in range(3):
        theta = rng.uniform(-np.pi, np.pi, k)
        mats = packed.materialize(theta, np.complex128)
        ops, passes, pool = packed.compact(mats)
        got = run_passes(O.zero_state(n), n, passes, ops, pool)
        it = iter(theta)
        ref_circ = [(c[0], *c[1:-1], next(it)) if s >= 0 else c for c, s in zip(target, slots)]
        ref = O.run_circuit(O.zero_state(n), n, ref_circ)
        assert np.max(np.abs(got - ref)) < 1e-12, trial
