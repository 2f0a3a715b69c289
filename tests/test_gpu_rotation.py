"""Rotation passes on the GPU (the default complex64 path from 20 qubits):
states against the oracle (complex128) and against the general fused passes
(DESV_ROT=0), at max |d amplitude| <= 1e-5 -- the complex64 bar -- and the
accuracy of the full 40-layer brick circuit against complex128."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu


def _run(circ, n, dtype=torch.complex64):
    import dense_evolution as de
    from dense_evolution.circuits.compiler import CompiledCircuit
    plan = CompiledCircuit(de.QuantumTranspiler.transpile(circ), n, dtype)
    sv = torch.zeros(1 << n, dtype=dtype, device='cuda')
    sv[0] = 1
    plan.run(sv)
    return plan, sv


def _mixed(n, count, seed):
    import test_rotation_plan_cpu as T
    return T._mixed_circuit(n, count, seed)


@pytest.mark.parametrize('n,layers', [(20, 3), (21, 2)])
def test_brick_against_oracle(n, layers):
    from dense_evolution.workloads import brick_u3_circuit
    circ = brick_u3_circuit(n, layers, seed=n)
    plan, sv = _run(circ, n)
    assert plan.rotation is not None
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(sv.cpu().numpy().astype(np.complex128) - ref)) <= 1e-5
    from dense_evolution import _native as N
    N.device_status()


def test_every_gate_kind_against_oracle():
    n = 20
    circ = _mixed(n, 120, 4)
    plan, sv = _run(circ, n)
    assert plan.rotation is not None
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(sv.cpu().numpy().astype(np.complex128) - ref)) <= 1e-5


@pytest.mark.parametrize('n', [12, 15])
def test_forced_at_small_sizes(monkeypatch, n):
    """DESV_ROT=1 runs the rotation passes below 20 qubits too (one tile at 12
    qubits, eight at 15)."""
    from dense_evolution.workloads import brick_u3_circuit
    monkeypatch.setenv('DESV_ROT', '1')
    circ = brick_u3_circuit(n, 8, seed=3) + _mixed(n, 60, n)
    plan, sv = _run(circ, n)
    assert plan.rotation is not None
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(sv.cpu().numpy().astype(np.complex128) - ref)) <= 1e-5


def test_against_general_passes_at_24_qubits(monkeypatch):
    from dense_evolution.workloads import brick_u3_circuit
    n = 24
    circ = brick_u3_circuit(n, 12, seed=9)
    plan, a = _run(circ, n)
    assert plan.rotation is not None
    monkeypatch.setenv('DESV_ROT', '0')
    plan2, b = _run(circ, n)
    assert plan2.rotation is None
    assert torch.max(torch.abs(a - b)).item() <= 1e-5


def test_headline_structure_accuracy_at_26_qubits():
    """The 40-layer brick circuit (the headline's structure) at 26 qubits:
    complex64 rotation passes against the complex128 general passes."""
    from dense_evolution.workloads import brick_u3_circuit
    n = 26
    circ = brick_u3_circuit(n, 40, seed=2024)
    plan, a = _run(circ, n)
    assert plan.rotation is not None
    _, b = _run(circ, n, torch.complex128)
    a64 = a.to(torch.complex128)
    fid = float(torch.abs(torch.vdot(b, a64)) ** 2)
    assert fid >= 1 - 1e-6
    assert torch.max(torch.abs(a64 - b)).item() <= 1e-5
    assert abs(float(torch.vdot(a64, a64).real) - 1.0) <= 1e-5


def test_new_angles_reuse_the_kernels():
    """Two circuits of one structure share the plan and the compiled kernels;
    the second runs with its own angles."""
    from dense_evolution.workloads import brick_u3_circuit
    n = 20
    c1, c2 = brick_u3_circuit(n, 3, seed=1), brick_u3_circuit(n, 3, seed=2)
    p1, _ = _run(c1, n)
    p2, sv = _run(c2, n)
    assert p1.rotation.prog is p2.rotation.prog
    ref = O.run_circuit(O.zero_state(n), n, c2)
    assert np.max(np.abs(sv.cpu().numpy().astype(np.complex128) - ref)) <= 1e-5


def test_c_abi_rejects_bad_calls():
    """desv_rot_pass checks its handle kind, parameter count and geometry
    before launching."""
    from dense_evolution import _native as N
    from dense_evolution.workloads import brick_u3_circuit
    n = 20
    plan, sv = _run(brick_u3_circuit(n, 2, seed=1), n)
    prog = plan.rotation.prog
    k = prog.compile(torch.cuda.current_device())[0]
    blk = plan.rotation.blocks()[0]
    lib = N.lib()
    row = prog.rows[0:1].copy()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    r = lib.desv_rot_pass(k.handle, ctypes.c_void_p(sv.data_ptr()), n, ctypes.c_void_p(row.ctypes.data),
                          blk.ctypes.data_as(ctypes.c_void_p), len(blk) + 1, st)
    assert r == N.DESV_EINVAL and 'parameter block' in N.last_error()
    bad = row.copy()
    bad['tile_bits'] = 11
    r = lib.desv_rot_pass(k.handle, ctypes.c_void_p(sv.data_ptr()), n, ctypes.c_void_p(bad.ctypes.data),
                          blk.ctypes.data_as(ctypes.c_void_p), len(blk), st)
    assert r == N.DESV_EINVAL and 'geometry' in N.last_error()
    r = lib.desv_rot_pass(k.handle, ctypes.c_void_p(sv.data_ptr() + 8), n, ctypes.c_void_p(row.ctypes.data),
                          blk.ctypes.data_as(ctypes.c_void_p), len(blk), st)
    assert r == N.DESV_EINVAL


def test_general_form_variant():
    """A call whose rotation has cos = 0 (ry(pi) alone on its qubit) runs the pass
    variant with the run-time form choice; a later call of the same structure
    with generic angles runs the tangent-only variant.  Both match the oracle."""
    from dense_evolution.workloads import brick_u3_circuit
    n = 20
    base = brick_u3_circuit(n, 2, seed=5)
    c1 = base + [('ry', 3, float(np.pi)), ('ry', 7, float(np.pi))]
    c2 = base + [('ry', 3, 0.37), ('ry', 7, 1.1)]
    for circ, general in ((c1, True), (c2, False)):
        plan, sv = _run(circ, n)
        prog = plan.rotation.prog
        blocks = plan.rotation.blocks()
        flags = [prog.needs_general(i, b) for i, b in enumerate(blocks)]
        if general:
            assert any(flags)
        ref = O.run_circuit(O.zero_state(n), n, circ)
        assert np.max(np.abs(sv.cpu().numpy().astype(np.complex128) - ref)) <= 1e-5
        if general:
            assert prog.general, 'the general variant was compiled for this call'
        else:
            assert not any(flags)
