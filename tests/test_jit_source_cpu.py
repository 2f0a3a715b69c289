"""Generated sources of the specialised adjoint passes, checked on the CPU:
every inverse gate is applied to both phi (a) and lambda (b), the probes of
ry / rz / p / cp / crz use the generator-specific forms, a CX becomes a
register swap, and the sources compile with NVRTC (no GPU needed)."""
import ctypes
import re

import numpy as np
import pytest
import torch

from dense_evolution import _native as N
from dense_evolution.circuits import jit
from dense_evolution.solvers import autodiff
from dense_evolution.solvers.adjoint import AdjointProgram
from dense_evolution.workloads import hea_circuit


def _sources(n=12, layers=3):
    circ = hea_circuit(n, layers) + [('crz', 0, n - 1, 0.0), ('cp', 2, 1, 0.0), ('p', 3, 0.0), ('rx', 5, 0.0)]
    rows, slots, npar = autodiff.build_template(circ, n)
    prog = AdjointProgram(rows, slots, n, torch.complex64)
    theta = np.random.default_rng(3).uniform(-np.pi, np.pi, npar)
    mats = prog.back.materialize(theta, np.complex64)
    words = np.ascontiguousarray(mats).view(np.uint32)
    out = []
    for p in prog.back.passes:
        b, e = int(p['op_begin']), int(p['op_end'])
        if 0 < e - b <= jit.MAX_OPS:
            K = int(p['tile_bits'])
            out.append(jit.adjoint_source(prog.back.ops, b, e, K, jit.adjoint_nbuf_for(K, True), True, words, 2))
    return prog, mats, theta, out


def test_every_gate_reaches_both_states():
    _, _, _, srcs = _sources()
    assert srcs
    call = re.compile(r'\b(\w+(?:<[^>]*>)?)\((a|b)(?=[,)])')
    for src in srcs:
        lines = [ln.strip() for ln in src.splitlines()]
        for i, ln in enumerate(lines):
            if 'jit_grad' in ln or 'S::' in ln or 'JitStage' in ln:
                continue
            m = call.search(ln)
            if m and m.group(2) == 'a':
                twin = lines[i + 1] if i + 1 < len(lines) else ''
                assert twin == ln.replace('(a, ', '(b, ').replace('(a);', '(b);'), (ln, twin)


def test_generator_specific_probes_and_swaps():
    _, _, _, srcs = _sources()
    text = '\n'.join(srcs)
    assert 'jit_grad_y<' in text            # ry
    assert 'jit_grad_dim<' in text          # rz, p, cp, crz
    assert 'swap_reg<' in text              # the CX ladder
    assert 'jit_grad_reg<' not in text and 'jit_grad_diag<' not in text


def test_value_key_is_stable_across_angles():
    prog, mats, theta, _ = _sources()
    other = prog.back.materialize(theta + 0.37, np.complex64)
    assert jit.value_key(prog.back.ops, mats) == jit.value_key(prog.back.ops, other)


def test_sources_compile_with_nvrtc():
    _, _, _, srcs = _sources()
    log = ctypes.create_string_buffer(16384)
    r = N.lib().desv_jit_compile_check(srcs[0].encode(), jit.INCLUDE_PATH.encode(), log, 16384)
    if r == N.DESV_EUNSUPPORTED:
        pytest.skip('NVRTC not available: ' + N.last_error())
    assert r == 0, log.value.decode()[-3000:]


def test_tangent_variant_sources():
    """The tangent variant of the backward passes: uncontrolled ry / rz inverses
    on register slots or thread-fixed bits become tan_rot / tan_phase on both
    arrays, every immediate-form probe is scaled by its pool slot, the last stage
    scales both arrays by the pass-end factor, and the sources compile."""
    import os
    from dense_evolution.solvers.adjoint import TangentPlan
    os.environ['DESV_JIT'] = '1'
    try:
        prog, mats, theta, _ = _sources()
    finally:
        del os.environ['DESV_JIT']
    tp = TangentPlan(prog.back, len(mats), mats)
    info = tp.sources_info()
    words = np.ascontiguousarray(mats).view(np.uint32)
    srcs = []
    for p, inf in zip(prog.back.passes, info):
        b, e = int(p['op_begin']), int(p['op_end'])
        if inf is None or not 0 < e - b <= jit.MAX_OPS:
            continue
        K = int(p['tile_bits'])
        srcs.append(jit.adjoint_source(prog.back.ops, b, e, K, jit.adjoint_nbuf_for(K, True), True, words, 2,
                                       tangent=inf))
    assert srcs
    text = '\n'.join(srcs)
    assert 'tan_rot<' in text and 'tan_phase<' in text and 'scale_both(a, b, mats[' in text
    assert '(a, t); tan_rot' in text or 'tan_rot<' in text
    assert all(src.count('scale_both(') == 1 for src in srcs)
    for ln in text.splitlines():
        if 'tan_rot<' in ln or 'tan_phase<' in ln:
            assert '(a, t' in ln and '(b, t' in ln
        if 'jit_grad_y<' in ln or 'jit_grad_dim<' in ln:
            assert 'v *= (double)mats[' in ln
    log = ctypes.create_string_buffer(16384)
    r = N.lib().desv_jit_compile_check(srcs[0].encode(), jit.INCLUDE_PATH.encode(), log, 16384)
    if r == N.DESV_EUNSUPPORTED:
        pytest.skip('NVRTC not available: ' + N.last_error())
    assert r == 0, log.value.decode()[-3000:]


def test_rows_pauli_sources_read_per_row_coefficients():
    """H psi kernels of a rows group: coefficients equal in every row (the XX and
    YY terms of the XXZ chains) are compiled in, the others (each row's J_z)
    are read per row from the symbol table, terms sharing a column fold into one
    class, and the sources compile with NVRTC."""
    from dense_evolution.physics.observables import plan_for
    from dense_evolution.workloads import xxz_terms
    n = 14
    plan = plan_for([(1.0, p) for _, p in xxz_terms(n, 1.0)], n, None, torch.complex64)
    jz = np.array([0.7, 1.3, 0.9])
    co = np.array([[float(c) for c, _ in xxz_terms(n, z)] for z in jz])[:, plan.order]
    syms = [None if np.all(co[:, k] == co[0, k]) else 0 for k in range(co.shape[1])]
    assert syms.count(0) == n - 1
    srcs = []
    for p, mode in zip(plan.passes, jit.pauli_modes(plan.passes, True)):
        b, e = int(p['term_begin']), int(p['term_end'])
        if mode is None or int(p['tile_bits']) < 10:
            continue
        srcs.append(jit.pauli_source(plan.terms[b:e], int(p['tile_bits']), int(p['low_bits']), p['high'], mode, True,
                                     syms=syms[b:e]))
    assert srcs
    text = '\n'.join(srcs)
    assert 'const double C0 = csym[0];' in text and 'RowStrides rs' in text and '* C0)' in text
    log = ctypes.create_string_buffer(16384)
    for src in srcs:
        r = N.lib().desv_jit_compile_check(src.encode(), jit.INCLUDE_PATH.encode(), log, 16384)
        if r == N.DESV_EUNSUPPORTED:
            pytest.skip('NVRTC not available: ' + N.last_error())
        assert r == 0, log.value.decode()[-3000:]


@pytest.mark.parametrize('dtname', ['complex64', 'complex128'])
def test_pauli_sources_of_mixed_terms_compile(dtname):
    """Every specialised Pauli pass (both <H> and H psi modes) of a term set
    mixing flip masks, Y phases, negative and complex coefficients, sign masks
    reaching outside the tile and a wide mask compiles with NVRTC."""
    from dense_evolution.physics.observables import plan_for
    from dense_evolution.workloads import tfim_terms, xxz_terms
    n = 13
    terms = (tfim_terms(n) + xxz_terms(n, 0.7) + [(0.3, {0: 'Y', n - 1: 'Y'}), (0.2, {1: 'X', 2: 'Y', 7: 'Z'}),
             (-0.4, 'Z' * n), (0.15j, {q: 'X' for q in range(0, n, 2)}), (-0.25, {3: 'Y'})])
    dt = getattr(torch, dtname)
    plan = plan_for(terms, n, dtype=dt)
    log = ctypes.create_string_buffer(16384)
    count = 0
    for p, mode in zip(plan.passes, jit.pauli_modes(plan.passes, True)):
        K, L = int(p['tile_bits']), int(p['low_bits'])
        b, e = int(p['term_begin']), int(p['term_end'])
        if mode is None or K < 10 or K - L > 8 or not 0 < e - b <= jit.MAX_PAULI_TERMS:
            continue
        for m in (mode, 0):
            src = jit.pauli_source(plan.terms[b:e], K, L, p['high'], m, dt == torch.complex64)
            r = N.lib().desv_jit_compile_check(src.encode(), jit.INCLUDE_PATH.encode(), log, 16384)
            if r == N.DESV_EUNSUPPORTED:
                pytest.skip('NVRTC not available: ' + N.last_error())
            assert r == 0, log.value.decode()[-3000:]
            count += 1
    assert count >= 2


@pytest.mark.parametrize('K', [11, 12])
@pytest.mark.parametrize('which', ['tfim', 'xxz', 'random'])
def test_pauli_plan_balance_keeps_every_term_in_a_covering_tile(K, which):
    """The planner spreads flip masks that several tiles cover over the passes:
    every term still sits in exactly one pass whose tile holds all its flip bits,
    the packed terms are the caller's (a permutation), and for the TFIM chain no
    pass carries more than one flip mask above an even share."""
    import torch
    from dense_evolution.physics.observables import PauliPlan
    from dense_evolution.workloads import tfim_terms, xxz_terms
    n = 24
    if which == 'tfim':
        terms = tfim_terms(n)
    elif which == 'xxz':
        terms = xxz_terms(n, 1.0)
    else:
        rng = np.random.default_rng(3)
        terms = []
        for _ in range(90):
            w = int(rng.integers(1, 4))
            qs = rng.choice(n, w, replace=False)
            terms.append((float(rng.normal()), {int(q): str(rng.choice(list('XYZ'))) for q in qs}))
    plan = PauliPlan(terms, n, tile_bits=K)
    assert sorted(plan.order.tolist()) == list(range(len(terms)))
    masks_per_pass = []
    for r in plan.passes:
        b, e = int(r['term_begin']), int(r['term_end'])
        assert e - b <= PauliPlan.MAX_TERMS_PER_PASS
        if int(r['tile_bits']) == 0:
            continue
        L = int(r['low_bits'])
        high = [int(h) for h in r['high'][:int(r['tile_bits']) - L]]
        cover = ((1 << L) - 1) | sum(1 << h for h in high)
        xs = plan.terms['xmask'][b:e].astype(np.uint64)
        assert all(int(x) & ~cover == 0 for x in xs)
        masks_per_pass.append(len({int(x) for x in xs if int(x)}))
    if which == 'tfim':
        share = -(-n // len(masks_per_pass))
        assert max(masks_per_pass) <= share + 1, masks_per_pass
