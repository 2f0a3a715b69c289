"""Split statevectors on the CPU: the exchange schedule (which gates trade a
chunk-select qubit for the top local one), the per-chunk specialisation of
diagonal gates on chunk-select qubits, and the half-chunk exchanges -- in one
process with 2, 4 and 8 chunks, and across two gloo ranks.  The per-chunk
gates run through the oracle here (no GPU); on a GPU the engine runs them."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import sv_oracle as O


def oracle_applier(chunk, n_local, gates):
    out = O.run_circuit(chunk.numpy().astype(np.complex128), n_local, gates, do_transpile=False)
    chunk.copy_(torch.from_numpy(out.astype(np.complex128)))


def _circuit(n, seed, count=80):
    import test_rotation_plan_cpu as T
    return T._mixed_circuit(n, count, seed)


@pytest.mark.parametrize('m', [1, 2, 3])
@pytest.mark.parametrize('seed', [1, 2])
def test_split_state_matches_oracle(m, seed):
    from dense_evolution.backends.sharded import ShardedState
    n = 8
    circ = _circuit(n, seed)
    st = ShardedState(n, m, torch.complex128, device='cpu', applier=oracle_applier)
    st.run_circuit(circ)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(st.logical_state() - ref)) <= 1e-12
    assert st.exchanges > 0


def test_diagonal_gates_on_select_qubits_need_no_exchange():
    """rz / p / cz / cp / crz and cx controls on chunk-select qubits run without
    moving data; only non-diagonal action on them exchanges."""
    from dense_evolution.backends.sharded import ShardedState, plan_steps
    n, m = 6, 2
    circ = [('h', q) for q in range(2, n)] + [('rz', 0, 0.3), ('p', 1, 0.2), ('cz', 0, 3), ('cp', 1, 4, 0.7),
                                              ('crz', 0, 5, 0.4), ('crz', 4, 1, 0.9), ('cx', 0, 2), ('cy', 1, 5),
                                              ('t', 0), ('s', 1)]
    steps = plan_steps(circ, n, m)
    assert all(k == 'gates' for k, _ in steps)
    st = ShardedState(n, m, torch.complex128, device='cpu', applier=oracle_applier)
    full = [('h', 0), ('h', 1)] + circ
    st.run_circuit(full)
    trades = [x for k, x in plan_steps(full, n, m) if k == 'trade']
    assert st.exchanges == len(trades) and trades[:2] == [0, 1]
    ref = O.run_circuit(O.zero_state(n), n, [('h', 0), ('h', 1)] + circ)
    assert np.max(np.abs(st.logical_state() - ref)) <= 1e-12


def _rank_main(rank, world, port, out):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    import datetime
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from dense_evolution.backends.sharded import ShardedState
        n, m = 8, 2
        st = ShardedState(n, m, torch.complex128, device='cpu', group=dist.group.WORLD, applier=oracle_applier)
        st.run_circuit(_circuit(n, 5))
        full = st.logical_state()
        out.put((rank, st.owned, st.exchanges, full))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_exchange_halves():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    n = 8
    ref = O.run_circuit(O.zero_state(n), n, _circuit(n, 5))
    owned = sorted(o for _, o, _, _ in got)
    assert owned == [[0, 1], [2, 3]]
    for _, _, ex, full in got:
        assert ex > 0
        assert np.max(np.abs(full - ref)) <= 1e-12


def test_split_state_with_rotation_plans_for_the_chunks():
    """The per-chunk circuits (specialised gates, chunk-local phases, circuits of
    a global phase alone) through the rotation planner and the tile emulator --
    the path the chunks take on a GPU from 20 local qubits on."""
    import rotation_emulator as E
    from dense_evolution.backends.sharded import ShardedState
    from dense_evolution.circuits import rotation as R
    from dense_evolution.workloads import brick_u3_circuit

    def applier(chunk, n_local, gates):
        bp = R.program_for(list(gates), n_local, 12)
        blocks, _ = bp.plan.materialize(None, np.float64, bp.ir)
        sv = chunk.numpy().astype(np.complex128)
        E.run(bp.plan, sv, blocks)
        chunk.copy_(torch.from_numpy(sv))

    n = 14
    circ = brick_u3_circuit(n, 6, seed=11)
    st = ShardedState(n, 2, torch.complex128, device='cpu', applier=applier)
    st.run_circuit(circ)
    ref = O.run_circuit(O.zero_state(n), n, circ)
    assert np.max(np.abs(st.logical_state() - ref)) <= 1e-12
