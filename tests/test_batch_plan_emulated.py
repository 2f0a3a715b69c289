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


@pytest.mark.parametrize('n,dtype_name', [(13, 'complex64'), (14, 'complex128')])
def test_rows_plan_energy_and_gradient(n, dtype_name):
    """The rows plan of one structure (forward tiles of 12 bits, adjoint tiles
    of the single-circuit width, local gradient slots with a parameter map)
    gives every row its energy and gradient: pools rebuilt from each row's
    theta by the recipes, each row's term table with its own J_z folded into
    the plan's packed term order."""
    import torch
    from dense_evolution.batch import _RowsPlan, hea_xxz_batch
    from dense_evolution.solvers.autodiff import build_template
    items = hea_xxz_batch([n, n], 2, [0.7, 1.3])
    circ = items[0][0]
    rows, slots, npar = build_template(circ, n)
    p = _RowsPlan(rows, slots, n, getattr(torch, dtype_name), 12, terms=items[0][2])
    assert all(int(ps['tile_bits']) == 12 for ps in p.fwd.passes)
    coefs = [[float(c) for c, _ in it[2]] for it in items]
    table = p.term_rows(coefs)
    assert table.shape == (2, len(items[0][2]))
    orows, _ = O.energy_template([{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]}
                                  for c in circ], n)
    for r, (_, _, terms) in enumerate(items):
        theta = np.random.default_rng(100 + r).uniform(-np.pi, np.pi, npar)
        pool = _recipe_pool(p, theta, p.cpool.astype(np.complex128))
        psi = run_passes(O.zero_state(n), n, p.fwd.passes, p.fwd.ops, pool)
        # H psi from the row's packed term table: (P psi)[i] = psi[i ^ x] c (-1)^popcount((i ^ x) & z)
        lam = np.zeros_like(psi)
        idx = np.arange(1 << n)
        for t in table[r]:
            src = idx ^ int(t['xmask'])
            sign = 1 - 2 * (np.array([bin(v).count('1') for v in (src & int(t['zmask']))]) & 1)
            lam += (t['cre'] + 1j * t['cim']) * sign * psi[src]
        assert np.max(np.abs(lam - O.pauli_sum_matvec(psi, terms))) < 1e-12
        grad = np.zeros(npar)
        _, _, grad = run_passes(psi, n, p.bwd.passes, p.bwd.ops, pool, lam=lam, grad=grad,
                                param_map=np.asarray(p.bwd.param_map))
        e_ref, psi_ref = O.energy(theta, orows, n, terms)
        assert np.max(np.abs(psi - psi_ref)) < 1e-12
        assert float(np.real(np.vdot(psi, lam))) == pytest.approx(e_ref, abs=1e-12)
        fd = O.fd_gradient(theta, orows, n, terms, h=1e-5, indices=[0, npar // 2, npar - 1])
        assert np.allclose(grad[[0, npar // 2, npar - 1]], fd, atol=1e-7)


def test_adjoint_tangent_plan_bookkeeping():
    """The tangent variant's host bookkeeping (tangents, running 1/c products,
    probe corrections, pass-end factors) gives the exact gradient when every
    tangent record is read as (1/c) times its gate -- the kernel's arithmetic in
    exact form -- every probe is scaled by its correction and every pass ends by
    scaling both arrays by its end factor."""
    import os
    import torch
    from dense_evolution.solvers.adjoint import AdjointProgram, TangentPlan
    from dense_evolution.solvers.autodiff import build_template
    from dense_evolution.workloads import hea_circuit, tfim_terms
    os.environ['DESV_JIT'] = '1'
    try:
        n = 11
        circ = hea_circuit(n, 3)
        rows, slots, npar = build_template(circ, n)
        prog = AdjointProgram(rows, slots, n, torch.complex64)
    finally:
        del os.environ['DESV_JIT']
    theta = np.random.default_rng(5).uniform(-np.pi, np.pi, npar)
    mats = prog.back.materialize(theta, np.complex128)
    tp = TangentPlan(prog.back, len(mats), prog.back.materialize(0.37 + 0.0137 * np.arange(npar), np.complex128))
    out, flags = tp.transform(mats)
    assert any(flags) and sum(len(t) for t, _ in tp.passes) > npar // 2
    # exact-arithmetic reading of the tangent pool: a tangent record is (1/c) U
    emu = out[:len(mats)].copy()
    for i, (tan, events) in enumerate(tp.passes):
        if not flags[i]:
            continue
        for kind, off, extra in events:
            if kind == 't':
                t = out[off].real
                if extra == 'rot':
                    emu[off:off + 4] = [1.0, -t, t, 1.0]        # [[1, -t], [t, 1]] = [[c, s], [-s, c]] / c
                else:
                    emu[off:off + 4] = [1 + 1j * t, 1 - 1j * t, 1 + 1j * t, 1 - 1j * t]
            elif not extra:
                emu[off:off + 4] = mats[off:off + 4] * out[off].real    # immediate probe: its correction
    terms = tfim_terms(n)
    orows, _ = O.energy_template([{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]}
                                  for c in circ], n)
    _, psi = O.energy(theta, orows, n, terms)
    lam = O.pauli_sum_matvec(psi, terms)
    mu = psi.copy()
    grad = np.zeros(npar)
    for i, ps in enumerate(prog.back.passes):
        one = prog.back.passes[i:i + 1]
        mu, lam, grad = run_passes(mu, n, one, prog.back.ops, emu if flags[i] else mats, lam=lam, grad=grad,
                                   param_map=np.asarray(prog.back.param_map))
        if flags[i]:
            f = out[tp.end_base + i].real
            mu, lam = mu * f, lam * f
    fd = O.fd_gradient(theta, orows, n, terms, h=1e-5, indices=list(range(0, npar, 7)))
    assert np.allclose(grad[list(range(0, npar, 7))], fd, atol=1e-7)
    assert np.max(np.abs(mu - O.zero_state(n))) < 1e-10


def test_rows_tangent_events_reproduce_the_host_transform():
    """The event arrays a rows plan hands the device (kinds 0/1 tangent ry/rz
    records, 2/3 probes with compiled-in / pool-read generators, per pass),
    walked as the device kernel walks them, rewrite a row's pool exactly as the
    host TangentPlan.transform does, pass-end factors included."""
    import torch
    from dense_evolution.batch import _RowsPlan, hea_xxz_batch
    from dense_evolution.solvers.autodiff import build_template
    n = 13
    circ, _, terms = hea_xxz_batch([n], 3, [0.8])[0]
    rows, slots, npar = build_template(circ, n)
    p = _RowsPlan(rows, slots, n, torch.complex64, 12, terms=terms, use_jit=True)
    assert p.tangent is not None
    theta = np.random.default_rng(2).uniform(-np.pi, np.pi, npar)
    pool = _recipe_pool(p, theta, p.cpool.astype(np.complex128)).astype(np.complex64)
    want, flags = p.tangent.transform(pool)
    dev = np.concatenate([pool, np.ones(p.pool_stride - len(pool), np.complex64)])
    for q in range(len(p.bwd.passes)):
        b, e = int(p.ev_begin[q]), int(p.ev_begin[q + 1])
        S, ok, anyt = 1.0, True, False
        for k in range(b, e):
            kind, off = int(p.ev_kind[k]), int(p.ev_off[k])
            if kind <= 1:
                c = float(dev[off].real)
                t = (float(dev[off + 2].real) if kind == 0 else float(dev[off].imag)) / c
                anyt, S = True, S / c
                ok = ok and abs(t) <= p.tangent.TMAX and abs(S) <= p.tangent.TMAX ** 2
        assert (ok and anyt) == flags[q]
        if not (ok and anyt):
            continue
        S = 1.0
        for k in range(b, e):
            kind, off = int(p.ev_kind[k]), int(p.ev_off[k])
            if kind <= 1:
                c = float(dev[off].real)
                t = (float(dev[off + 2].real) if kind == 0 else float(dev[off].imag)) / c
                dev[off] = t
                S /= c
            elif kind == 2:
                dev[off] = 1.0 / (S * S)
            else:
                dev[off:off + 4] = dev[off:off + 4] * (1.0 / (S * S))
        dev[p.tangent.end_base + q] = 1.0 / S
    m = len(want)
    assert np.allclose(dev[:m], want, rtol=1e-6, atol=1e-7)


def test_single_circuit_backward_values_from_recipes():
    """The single-circuit gradient builds its backward passes' values on the
    device: the batched VQE's recipes applied to theta reproduce the host
    materialisation of the backward pool, and the angle-only tangent choice
    (TangentPlan.allowed, with its margin) never admits a pass the full check
    on the matrices would refuse."""
    import os
    import torch
    from dense_evolution.batch import _Plan
    from dense_evolution.solvers.adjoint import AdjointProgram, TangentPlan
    from dense_evolution.solvers.autodiff import build_template
    from dense_evolution.workloads import hea_circuit
    os.environ['DESV_JIT'] = '1'
    try:
        n = 12
        rows, slots, npar = build_template(hea_circuit(n, 3), n)
        prog = AdjointProgram(rows, slots, n, torch.complex64)
    finally:
        del os.environ['DESV_JIT']
    generic = prog.back.materialize(0.37 + 0.0137 * np.arange(npar), np.complex128)
    recipes = _Plan._recipes(prog.back, 0)

    class _P:
        pass
    holder = _P()
    holder.recipes = recipes
    tp = TangentPlan(prog.back, len(generic), generic.astype(np.complex64))
    rng = np.random.default_rng(4)
    for k in range(5):
        theta = rng.uniform(-np.pi, np.pi, npar)
        if k == 4:
            theta[::3] = np.pi - 1e-9          # near pi: tangents out of range
        dev = _recipe_pool(holder, theta, generic)
        host = prog.back.materialize(theta, np.complex128)
        assert np.allclose(dev, host, atol=1e-12)
        _, ok = tp.transform(host.astype(np.complex64))
        al = tp.allowed(theta)
        assert all((not a) or o for a, o in zip(al, ok))
        if k < 4:
            assert all(al)
        else:
            assert not all(al)
