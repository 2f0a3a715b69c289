"""Rotation passes on the CPU: the planner, the value program and the
kernels' index arithmetic (through the tile emulator, which walks tiles,
stages, thread deposits and the padded shared-memory layout exactly as the
generated CUDA does) against the oracle at 1e-12 in FP64; the bank-conflict
rule of the register sets; structure sharing across circuits that differ only
in their angles; and (where nvcc is installed) that the generated sources
compile for sm_100a."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import rotation_emulator as E
from oracle import sv_oracle as O
from dense_evolution.circuits import rotation as R
from dense_evolution.circuits.compiler import QuantumTranspiler
from dense_evolution.workloads import brick_u3_circuit, hea_circuit


def _mixed_circuit(n, count, seed):
    rng = np.random.default_rng(seed)
    names1 = ['h', 'x', 'y', 'z', 's', 'sdg', 't', 'tdg', 'sx', 'rx', 'ry', 'rz', 'p', 'u3', 'u2']
    names2 = ['cx', 'cy', 'cz', 'cp', 'crz', 'swap', 'iswap', 'ecr']
    out = []
    for _ in range(count):
        if rng.random() < 0.6:
            nm = names1[rng.integers(len(names1))]
            q = int(rng.integers(n))
            if nm in ('rx', 'ry', 'rz', 'p'):
                out.append((nm, q, float(rng.uniform(-3, 3))))
            elif nm == 'u3':
                out.append((nm, q, *[float(x) for x in rng.uniform(-3, 3, 3)]))
            elif nm == 'u2':
                out.append((nm, q, *[float(x) for x in rng.uniform(-3, 3, 2)]))
            else:
                out.append((nm, q))
        elif rng.random() < 0.1:
            a, b, c = (int(x) for x in rng.choice(n, 3, replace=False))
            out.append(('ccx', a, b, c))
        else:
            nm = names2[rng.integers(len(names2))]
            a, b = (int(x) for x in rng.choice(n, 2, replace=False))
            out.append((nm, a, b, float(rng.uniform(-3, 3))) if nm in ('cp', 'crz') else (nm, a, b))
    out.append(('gphase', 0, 0.3))
    return out


def _check(circ, n, cap=32, tol=1e-12):
    plan = R.RotationPlan(QuantumTranspiler.transpile(circ), n, 12, max_rots=cap)
    blocks, _ = plan.materialize(None, np.float64)
    sv = np.zeros(1 << n, dtype=np.complex128)
    sv[0] = 1
    E.run(plan, sv, blocks)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(sv - ref)) <= tol
    return plan


@pytest.mark.parametrize('n,layers,cap', [(12, 6, 32), (13, 9, 24), (14, 5, 48), (10, 4, 8)])
def test_brick_circuits_against_oracle(n, layers, cap):
    _check(brick_u3_circuit(n, layers, seed=n), n, cap)


@pytest.mark.parametrize('n', [11, 13])
def test_hea_with_cx_ladder_against_oracle(n):
    theta = np.random.default_rng(n).uniform(-np.pi, np.pi, 2 * n * 3)
    _check(hea_circuit(n, 3, theta), n)


@pytest.mark.parametrize('seed', [1, 2, 3])
def test_every_gate_kind_against_oracle(seed):
    """cx / cy become H.CZ.H around the target, cp / crz mixed diagonals with
    thread-fixed bits, swap / iswap / ecr / ccx through the transpiler, global
    phases into the last pass's end factor."""
    n = 12
    _check(_mixed_circuit(n, 160, seed), n, cap=16)


@pytest.mark.parametrize('circ', [[('gphase', 0, -1.9)], [('id', 3)], [('gphase', 0, 0.4), ('gphase', 2, 0.3)]])
def test_circuits_without_rotations_or_diagonals(circ):
    """A circuit of global phases (or identities) only still gets one pass,
    whose end factor applies the global factor."""
    _check(circ, 12)


def test_gate_free_tail_and_trailing_phases():
    n = 12
    circ = [('h', q) for q in range(n)] + [('rz', q, 0.1 * q) for q in range(n)] + [('cp', 0, 11, 0.7), ('t', 5)]
    _check(circ, n)


def test_structure_shared_across_angles():
    """A plan made from one circuit runs another of the same structure (other
    angles) when the new circuit's IR gates are bound to it."""
    n = 12
    c1 = brick_u3_circuit(n, 5, seed=1)
    c2 = brick_u3_circuit(n, 5, seed=2)
    t1, t2 = QuantumTranspiler.transpile(c1), QuantumTranspiler.transpile(c2)
    ir1, ir2 = R.lowered_gates(t1, n), R.lowered_gates(t2, n)
    assert R.structure_key(ir1, n, 12) == R.structure_key(ir2, n, 12)
    plan = R.RotationPlan(t1, n, 12)
    blocks, _ = plan.materialize(None, np.float64, ir2)
    sv = np.zeros(1 << n, dtype=np.complex128)
    sv[0] = 1
    E.run(plan, sv, blocks)
    assert np.max(np.abs(sv - O.run_circuit(O.zero_state(n), n, c2))) <= 1e-12


def test_parametrised_template_values_per_theta():
    """energy_fn templates: theta slots bound per call (rx/ry/rz/cp values)."""
    from dense_evolution.solvers.autodiff import build_template
    n = 12
    circ = hea_circuit(n, 2)
    rows, slots, npar = build_template(circ, n)
    plan = R.RotationPlan(rows, n, 12, slots=slots)
    theta = np.random.default_rng(3).uniform(-np.pi, np.pi, npar)
    blocks, _ = plan.materialize(theta, np.float64)
    sv = np.zeros(1 << n, dtype=np.complex128)
    sv[0] = 1
    E.run(plan, sv, blocks)
    ref = O.run_circuit(O.zero_state(n), n, hea_circuit(n, 2, theta))
    assert np.max(np.abs(sv - ref)) <= 1e-12


def test_register_sets_are_bank_conflict_free():
    """Every stage's register set gives 16 distinct 8-byte bank pairs for each
    half-warp, in the layout it reads (natural for the first stage, padded
    after) and the padded layout it writes."""
    n = 30
    plan = R.RotationPlan(QuantumTranspiler.transpile(brick_u3_circuit(n, 40, 2024)), n, 12)
    for ps in plan.passes:
        for si, st in enumerate(ps.stages):
            assert R._bank_ok(st.regs, ps.K, padded=True)
            if si == 0:
                assert R._bank_ok(st.regs, ps.K, padded=False)
            if si == len(ps.stages) - 1:
                assert all(b >= 4 for b in st.regs)       # half-warp stores of 128 contiguous bytes
    # the padded layout is injective and fits its slot; slots start on 16-byte
    # boundaries (bulk-copy destinations) and match libdesv's shared-memory size
    for K in (9, 10, 11, 12):
        pos = [R.padded(i) for i in range(1 << K)]
        assert len(set(pos)) == 1 << K and max(pos) < R.slot_elems(K)
        assert (R.slot_elems(K) * 8) % 16 == 0
        assert R.slot_elems(K) == (1 << K) + (1 << (K - 4))


def test_headline_schedule_shape():
    """30 qubits, 40 layers: every rotation is planned, and the pass count is
    well below the general fused path's."""
    n = 30
    plan = R.RotationPlan(QuantumTranspiler.transpile(brick_u3_circuit(n, 40, 2024)), n, 12)
    st = plan.stats()
    assert st['rots'] == sum(1 for p in plan.prims if p.kind == 'rot')
    assert st['passes'] <= 50
    assert all(r <= R.MAX_ROTS_PER_PASS for r, _, _ in st['per_pass'])


@pytest.mark.skipif(shutil.which('nvcc') is None and not os.path.exists('/usr/local/cuda/bin/nvcc'),
                    reason='nvcc not installed')
@pytest.mark.parametrize('nbuf', [1, 2, 3])
def test_generated_sources_compile(tmp_path, nbuf):
    nvcc = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    n = 22
    plan = R.RotationPlan(QuantumTranspiler.transpile(_mixed_circuit(n, 200, 5)), n, 12, max_rots=24)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for i in (0, len(plan.passes) - 1):
        src = tmp_path / f'p{i}.cu'
        src.write_text(R.pass_source(plan, i, nbuf=nbuf))
        r = subprocess.run([nvcc, '-gencode', 'arch=compute_100a,code=sm_100a', '-std=c++17', '-c', str(src),
                            '-o', str(tmp_path / f'p{i}.o'), '-I', os.path.join(root, 'dense-evolution_b200', 'csrc'),
                            '-I', os.path.join(root, 'include')], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]


def test_generated_sources_compile_with_nvrtc():
    """The kernels are compiled at run time by NVRTC, whose headers differ from
    nvcc's: compile the generated sources (normal and DESV_ROT_CHECK builds)
    through libdesv's compile-only entry point, which needs no GPU."""
    import ctypes
    from dense_evolution import _native as N
    from dense_evolution.circuits import jit
    n = 21
    plan = R.RotationPlan(QuantumTranspiler.transpile(_mixed_circuit(n, 150, 8)), n, 12, max_rots=24)
    for check, general in (('0', False), ('0', True), ('1', False), ('1', True)):
        os.environ['DESV_ROT_CHECK'] = check
        try:
            for i in (0, len(plan.passes) - 1):
                log = ctypes.create_string_buffer(16384)
                r = N.lib().desv_jit_compile_check(R.pass_source(plan, i, general=general).encode(),
                                                   jit.INCLUDE_PATH.encode(), log, 16384)
                if r == N.DESV_EUNSUPPORTED:
                    pytest.skip('NVRTC not available: ' + N.last_error())
                assert r == 0, log.value.decode()[-3000:]
        finally:
            os.environ.pop('DESV_ROT_CHECK', None)


def test_pending_scale_limit_splits_the_tangent_form():
    """Rotations near pi have cos(theta / 2) near 0, so their tangent scales
    1 / cos multiply past SCALE_LIMIT inside one pass: the value program then
    takes the general form for the rotations past the limit, keeps every
    pass's tangent scale at or under it, and the state still matches the oracle."""
    n = 12
    rng = np.random.default_rng(8)
    circ = []
    for _ in range(6):
        for q in range(n):
            circ.append(('ry', q, float(np.pi - rng.uniform(1e-4, 1e-3))))
        for q in range(0, n - 1, 2):
            circ.append(('cz', q, q + 1))
    plan = R.RotationPlan(QuantumTranspiler.transpile(circ), n, 12)
    blocks, _ = plan.materialize(None, np.float64)
    vp = plan._prepare_values()
    split = 0
    for pidx, ps in enumerate(plan.passes):
        us, pos = vp['rots'][pidx]
        if not len(us):
            continue
        off = pos - int(vp['offs'][pidx])
        b = blocks[pidx]
        tan = b[off + 3] == 0
        split += int(np.sum(~tan))
        scale = np.prod(1.0 / b[off + 1][tan])
        assert scale <= R.SCALE_LIMIT
        if ps.end_scale_off >= 0:
            o = ps.end_scale_off
            assert abs(complex(b[o], b[o + 1]) * scale) == pytest.approx(1.0, rel=1e-9)
    assert split > 0
    sv = np.zeros(1 << n, dtype=np.complex128)
    sv[0] = 1
    E.run(plan, sv, blocks)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(sv - ref)) <= 1e-9
