"""Split statevectors on one GPU: 2 and 4 chunks, the per-chunk gates on the
engine's fused passes and the half-chunk exchanges by desv_swap_blocks,
against the oracle (complex128, 1e-12) and against the unsplit engine
(complex64, the 1e-5 amplitude bar)."""
import numpy as np
import pytest
import torch

from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu


def _circuit(n, seed, count=120):
    import test_rotation_plan_cpu as T
    return T._mixed_circuit(n, count, seed)


@pytest.mark.parametrize('m', [1, 2])
def test_split_state_against_oracle(m):
    from dense_evolution.backends.sharded import ShardedState
    n = 12
    circ = _circuit(n, 3 + m)
    st = ShardedState(n, m, torch.complex128)
    st.run_circuit(circ)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert st.exchanges > 0
    assert np.max(np.abs(st.logical_state() - ref)) <= 1e-12
    from dense_evolution import _native as N
    N.device_status()


def test_split_state_against_unsplit_engine_complex64():
    import dense_evolution as de
    from dense_evolution.backends.sharded import ShardedState
    from dense_evolution.workloads import brick_u3_circuit
    n, m = 22, 2
    circ = brick_u3_circuit(n, 6, seed=11)
    st = ShardedState(n, m, torch.complex64)
    st.run_circuit(circ)
    sim = de.DenseSVSimulator(n, use_float32=True)
    sim.run_circuit(circ)
    a = st.logical_state()
    b = sim.get_statevector().astype(np.complex128)
    assert np.max(np.abs(a - b)) <= 1e-5


def test_block_swap_rejects_overlap_and_misalignment():
    import ctypes
    from dense_evolution import _native as N
    t = torch.zeros(64, dtype=torch.complex64, device='cuda')
    lib = N.lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.desv_swap_blocks(ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(t.data_ptr() + 64), 128, st) == \
        N.DESV_EINVAL
    assert lib.desv_swap_blocks(ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(t.data_ptr() + 256), 24, st) == \
        N.DESV_EINVAL
    a = torch.arange(32, dtype=torch.float32, device='cuda')
    b = -a
    assert lib.desv_swap_blocks(ctypes.c_void_p(a[:16].data_ptr()), ctypes.c_void_p(b[16:].data_ptr()), 64, st) == 0
    assert torch.equal(a[:16].cpu(), -torch.arange(16, 32, dtype=torch.float32))
