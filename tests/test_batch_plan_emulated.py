"""Batched-VQE plans on the CPU: the device recipes (restated here) rebuild
each circuit's matrix pool from theta, the plan emulator runs the forward and
adjoint passes, and the result must match the oracle's energy and gradient."""
import numpy as np
import pytest

from oracle import sv_oracle as O
from plan_emulator import run_passes


def _recipe_pool(plan, theta, cpool):
    pool = cpool.copy()
    for r in plan.recipes:
        kind, off = int(r['kind']), int(r['off'])
        base = kind & 0xFF
        if base == 0:
            pool[off:off + int(r['count'])] = cpool[int(r['src']):int(r['src']) + int(r['count'])]
            continue
        th = float(theta[int(r['param'])]) * (-1.0 if kind & 0x100 else 1.0)
        c, s = np.cos(th / 2), np.sin(th / 2)
        e1 = np.exp(1j * th)
        vals = {1: [c, -1j * s, -1j * s, c], 2: [c, -s, s, c], 3: [c - 1j * s, 0, 0, c + 1j * s], 4: [1, 0, 0, e1],
                5: [c - 1j * s, c + 1j * s, c - 1j * s, c + 1j * s], 6: [1, e1, 1, e1], 7: [1, 1, 1, e1],
                8: [1, c - 1j * s, 1, c + 1j * s], 9: [e1] * 4}[base]
        pool[off:off + 4] = vals
    return pool


@pytest.mark.parametrize('n', [9, 13])
def test_batch_plan_energy_and_gradient(n):
    import torch
    from dense_evolution.batch import _Plan, _term_structure, hea_xxz_batch
    from dense_evolution.solvers.autodiff import build_template
    circ, _, terms = hea_xxz_batch([n], 2, [0.8])[0]
    rows, slots, npar = build_template(circ, n)
    ts, coef = _term_structure(terms, n)
    p = _Plan(rows, slots, n, ts, torch.complex128)
    theta = np.random.default_rng(n).uniform(-np.pi, np.pi, npar)
    pool = _recipe_pool(p, theta, p.cpool.astype(np.complex128))
    psi = run_passes(O.zero_state(n), n, p.fwd.passes, p.fwd.ops, pool)
    lam = O.pauli_sum_matvec(psi, terms)
    grad = np.zeros(npar)
    # adjoint records already carry theta indices (identity map) and pool offsets after the forward pool
    bp = p.bwd.passes.copy()
    bp['map_begin'] = 0
    _, _, grad = run_passes(psi, n, bp, p.bwd.ops, pool, lam=lam, grad=grad, param_map=np.arange(4096))
    orows, _ = O.energy_template([{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]}
                                  for c in circ], n)
    e_ref, psi_ref = O.energy(theta, orows, n, terms)
    assert np.max(np.abs(psi - psi_ref)) < 1e-12
    assert float(np.real(np.vdot(psi, lam))) == pytest.approx(e_ref, abs=1e-12)
    fd = O.fd_gradient(theta, orows, n, terms, h=1e-5)
    assert np.allclose(grad, fd, atol=1e-7)
