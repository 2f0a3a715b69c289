"""Generate the golden fixtures in this folder from the REFERENCE implementation.

Run here (the reference checkout is not present on a GPU box):

    python tests/golden/make_golden.py --reference PATH_OF_REFERENCE_CHECKOUT

It imports the reference's own hot-path modules -- gates.py, compiler.py,
parser.py, backends/statevector.py, physics/observables.py,
circuits/random_circuit.py, circuits/topology.py, utils/measurement.py --
unmodified from the reference checkout.  JAX, matplotlib and the hardware
registry are absent from this image, so three modules are replaced by stubs
before the import: ``dense_evolution.circuits.registry`` (HAS_JAX=False),
``dense_evolution.config`` (no-op ``ensure_x64``) and ``jax``/``jax.numpy``
(aliased to NumPy; only the ``*_jax`` observables touch it).  With
HAS_JAX=False the reference ``DenseSVSimulator`` runs its NumPy eager branch
(``backends/statevector.py:381-410``) in complex128 or complex64.

Outputs (committed, small): ``golden_states.npz``, ``golden_cases.json``,
``golden_pauli.npz``, ``golden_parser.json``, ``golden_energy.npz``,
``golden_config1.npz``.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(root: str):
    """Import the reference's hot-path modules with the three stubs described above."""
    pkg_root = os.path.join(root, 'dense_evolution')
    for name, sub in [('dense_evolution', ''), ('dense_evolution.circuits', 'circuits'),
                      ('dense_evolution.backends', 'backends'), ('dense_evolution.physics', 'physics'),
                      ('dense_evolution.utils', 'utils'), ('dense_evolution.solvers', 'solvers')]:
        m = types.ModuleType(name)
        m.__path__ = [os.path.join(pkg_root, sub) if sub else pkg_root]
        sys.modules[name] = m
    reg = types.ModuleType('dense_evolution.circuits.registry')
    reg.HAS_JAX = False
    reg.NoiseModel = None
    reg.NoiseSpec = None
    sys.modules['dense_evolution.circuits.registry'] = reg
    cfg = types.ModuleType('dense_evolution.config')
    cfg.ensure_x64 = lambda: None
    sys.modules['dense_evolution.config'] = cfg
    jax = types.ModuleType('jax')
    jax.numpy = np
    sys.modules['jax'] = jax
    sys.modules['jax.numpy'] = np
    mods = {}
    for short, full in [('gates', 'dense_evolution.circuits.gates'),
                        ('compiler', 'dense_evolution.circuits.compiler'),
                        ('parser', 'dense_evolution.circuits.parser'),
                        ('statevector', 'dense_evolution.backends.statevector'),
                        ('observables', 'dense_evolution.physics.observables'),
                        ('random_circuit', 'dense_evolution.circuits.random_circuit'),
                        ('topology', 'dense_evolution.circuits.topology'),
                        ('measurement', 'dense_evolution.utils.measurement')]:
        mods[short] = importlib.import_module(full)
    return types.SimpleNamespace(**mods)


def brick_u3_circuit(n, layers, seed):
    """U3 on every qubit with angles U[0,2pi)^3 in gate order, then a brick of CZ:
    (2i,2i+1) on even layers, (2i+1,2i+2) on odd layers."""
    rng = np.random.default_rng(seed)
    ops = []
    for layer in range(layers):
        for q in range(n):
            th, ph, lam = rng.uniform(0.0, 2 * np.pi, 3)
            ops.append(('u3', q, float(th), float(ph), float(lam)))
        start = 0 if layer % 2 == 0 else 1
        for a in range(start, n - 1, 2):
            ops.append(('cz', a, a + 1))
    return ops


def hea_qasm(n, layers, theta):
    """Hardware-efficient ansatz: per layer RY then RZ on every qubit, then CX(i, i+1)."""
    lines = ['OPENQASM 2.0;', 'include "qelib1.inc";', f'qreg q[{n}];']
    k = 0
    for _ in range(layers):
        for q in range(n):
            lines.append(f'ry({float(theta[k])!r}) q[{q}];')
            lines.append(f'rz({float(theta[k + 1])!r}) q[{q}];')
            k += 2
        for q in range(n - 1):
            lines.append(f'cx q[{q}],q[{q + 1}];')
    return '\n'.join(lines)


def tfim_terms(n, h=1.0):
    t = [(-1.0, {i: 'Z', i + 1: 'Z'}) for i in range(n - 1)]
    t += [(-h, {i: 'X'}) for i in range(n)]
    return t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', required=True, help='path of the reference checkout')
    ap.add_argument('--skip-config1', action='store_true')
    args = ap.parse_args()
    ref = load_reference(args.reference)
    Sim = ref.statevector.DenseSVSimulator

    # ---- circuits -> final statevectors (c128 and c64) ----
    cases, states = [], {}

    def add(name, n, circ):
        for f32 in (False, True):
            sim = Sim(n, use_float32=f32)
            sim.run_circuit(circ)
            states[f'{name}__{"c64" if f32 else "c128"}'] = sim.get_statevector()
        cases.append({'name': name, 'n': n, 'circuit': [list(c) for c in circ]})

    for n in range(1, 11):
        for seed in (0, 1):
            add(f'random_n{n}_s{seed}', n, ref.random_circuit.random_circuit(n, 12 * n + 5, seed=seed))
    rng = np.random.default_rng(123)
    mixed = []
    n = 5
    for _ in range(40):
        k = rng.integers(9)
        a, b, c = (int(x) for x in rng.choice(n, 3, replace=False))
        th = [float(x) for x in rng.uniform(-np.pi, np.pi, 3)]
        mixed.append([('u3', a, *th), ('u2', a, th[0], th[1]), ('ccx', a, b, c), ('iswap', a, b),
                      ('ecr', a, b), ('cp', a, b, th[0]), ('crz', a, b, th[1]), ('p', a, th[2]),
                      ('u1', b, th[0])][k])
    add('mixed_n5', n, mixed)
    add('brick_u3_n10_l4', 10, brick_u3_circuit(10, 4, seed=7))
    add('brick_u3_n12_l3', 12, brick_u3_circuit(12, 3, seed=8))
    hea_theta = np.random.default_rng(5).uniform(-np.pi, np.pi, 2 * 8 * 3)
    hea = []
    k = 0
    for _ in range(3):
        for q in range(8):
            hea += [('ry', q, float(hea_theta[k])), ('rz', q, float(hea_theta[k + 1]))]
            k += 2
        hea += [('cx', q, q + 1) for q in range(7)]
    add('hea_n8_l3', 8, hea)
    add('x_on_q0_n3', 3, [('x', 0)])
    add('ghz_n3', 3, [('h', 0), ('cx', 0, 1), ('cx', 1, 2)])
    add('asym_n4', 4, [('h', 0), ('cx', 0, 3), ('ry', 2, 0.3), ('cy', 3, 1), ('crz', 1, 2, 0.7),
                       ('sx', 2), ('tdg', 0), ('swap', 0, 2), ('cp', 3, 0, 1.1)])
    np.savez_compressed(os.path.join(HERE, 'golden_states.npz'), **states)
    with open(os.path.join(HERE, 'golden_cases.json'), 'w') as f:
        json.dump(cases, f)
    # transpile outputs for the mixed case
    with open(os.path.join(HERE, 'golden_transpile.json'), 'w') as f:
        json.dump({'in': [list(c) for c in mixed],
                   'out': [list(c) for c in ref.compiler.QuantumTranspiler.transpile(mixed)]}, f)

    # ---- Pauli expectations and matvec ----
    pauli = {}
    prng = np.random.default_rng(42)
    meta = []
    for i in range(12):
        n = int(prng.integers(3, 9))
        psi = prng.normal(size=1 << n) + 1j * prng.normal(size=1 << n)
        psi /= np.linalg.norm(psi)
        terms = []
        for _ in range(int(prng.integers(1, 9))):
            s = ''.join(prng.choice(list('IXYZ'), n))
            terms.append((float(prng.normal()), s))
        pauli[f'psi{i}'] = psi
        pauli[f'exp{i}'] = np.array([ref.observables.pauli_expectation(psi, s) for _, s in terms])
        pauli[f'sum{i}'] = np.array(ref.observables.pauli_sum_expectation(psi, terms))
        pauli[f'mv{i}'] = ref.observables.pauli_sum_matvec(psi, terms)
        meta.append({'n': n, 'terms': terms})
    np.savez_compressed(os.path.join(HERE, 'golden_pauli.npz'), **pauli)
    with open(os.path.join(HERE, 'golden_pauli.json'), 'w') as f:
        json.dump(meta, f)

    # ---- parser ----
    qasms = [
        'OPENQASM 2.0; include "qelib1.inc"; qreg q[2]; creg c[2]; ry(0.5) q[0]; rx(0.5) q[1]; '
        'cx q[0],q[1]; rz(0.2) q[1]; cx q[0],q[1]; ry(0.5) q[0]; rx(0.5) q[1]; measure q -> c;',
        'OPENQASM 2.0;\nqreg a[2];\nqreg b[3];\nh a[1];\ncx a[1], b[2];\nu3(pi/2, -pi/4, sqrt(2)) b[0];\n'
        'cu1(pi/8) a[0],b[1];\nu1(0.1) b[2];\nbarrier a;\n// comment\n/* block\ncomment */ x b;\n',
        'OPENQASM 3.0;\nqubit[4] q;\nbit[4] c;\nh q[0:3];\nint n = 3;\nfor int i in [0:n-1] { cx q[i], q[i+1]; }\n'
        'if (c[0]) { x q[0]; }\nrz(2*pi/3) q[3];\n',
        'OPENQASM 2.0; qreg q[3]; gate maj(t) a,b,c { cx c,b; cx c,a; ccx a,b,c; rz(t) a; } '
        'maj(0.25) q[0],q[1],q[2]; toffoli q[2],q[1],q[0]; cnot q[0],q[2]; id q[1];',
        'OPENQASM 2.0; qreg q[2]; rx(cos(0.3)+2**2) q[0]; ry(-tau/4) q[1]; p(euler) q[0]; u2(0, pi) q[1];',
    ]
    pres = []
    for s in qasms:
        c = ref.parser.QASMParser().parse(s)
        ok, msg = ref.parser.QASMParser().validate(c)
        pres.append({'qasm': s, 'n_qubits': c.n_qubits, 'n_cbits': c.n_cbits, 'ops': c.ops,
                     'tuples': [list(t) for t in c.to_tuples()], 'valid': [ok, msg]})
    with open(os.path.join(HERE, 'golden_parser.json'), 'w') as f:
        json.dump(pres, f)

    # ---- energy and its finite-difference gradient (HEA + TFIM), via the
    # reference simulator and observables with theta injected in gate order ----
    en = {}
    for n, layers, seed in ((4, 2, 3), (6, 3, 4)):
        theta = np.random.default_rng(seed).uniform(-np.pi, np.pi, 2 * n * layers)
        terms = tfim_terms(n)

        def e_of(th):
            c = ref.parser.QASMParser().parse(hea_qasm(n, layers, th))
            sim = Sim(n)
            sim.run_circuit(c.to_tuples())
            return ref.observables.pauli_sum_expectation(sim.get_statevector(), terms)

        h = 1e-5
        grad = np.array([(e_of(theta + h * np.eye(theta.size)[i]) - e_of(theta - h * np.eye(theta.size)[i]))
                         / (2 * h) for i in range(theta.size)])
        en[f'theta_n{n}'] = theta
        en[f'energy_n{n}'] = np.array(e_of(theta))
        en[f'grad_n{n}'] = grad
    np.savez_compressed(os.path.join(HERE, 'golden_energy.npz'), **en)

    # ---- config 1 at full size: 20 qubits, 20 layers, complex128 ----
    if not args.skip_config1:
        n, layers, seed = 20, 20, 2024
        circ = brick_u3_circuit(n, layers, seed)
        t0 = time.time()
        sim = Sim(n)
        sim.run_circuit(circ)
        dt = time.time() - t0
        sv = sim.get_statevector()
        probs = np.abs(sv) ** 2
        idx = np.arange(1 << n)
        z = np.array([np.sum(probs * (1 - 2 * ((idx >> (n - 1 - q)) & 1))) for q in range(n)])
        pick = np.sort(np.random.default_rng(0).choice(1 << n, 512, replace=False))
        np.savez_compressed(os.path.join(HERE, 'golden_config1.npz'), z=z, idx=pick, amp=sv[pick],
                            norm=np.array(np.linalg.norm(sv)), seconds=np.array(dt),
                            n=np.array(n), layers=np.array(layers), seed=np.array(seed))
        print(f'config1 reference run: {dt:.1f} s')
    print('golden fixtures written to', HERE)


if __name__ == '__main__':
    main()
