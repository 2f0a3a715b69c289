"""Several-rank host logic on CPU (gloo, world size 2): the sharded batched VQE
partitions circuits without communicating and gathers every result once.
The per-circuit energy and gradient come from the oracle here (no GPU); on a
GPU box each rank would run BatchVQE on its shard."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from dense_evolution.batch import gather_results, shard_items
from dense_evolution.workloads import hea_circuit, xxz_terms
from oracle import sv_oracle as O

NS = [3, 5, 4, 3, 6, 4, 5]
LAYERS = 2


def _energy_grad(i):
    """Oracle energy + central-FD gradient of circuit i (seeded)."""
    n = NS[i]
    rng = np.random.default_rng([7, i])
    ops = [{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]} for c in hea_circuit(n, LAYERS)]
    rows, npar = O.energy_template(ops, n)
    theta = rng.uniform(-np.pi, np.pi, npar)
    terms = xxz_terms(n, 1.0 + 0.1 * i, 1.0)
    e = O.energy(theta, rows, n, terms)[0]
    g = O.fd_gradient(theta, rows, n, terms, 1e-4)
    return e, g


def _rank_main(rank, world, port, out):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        mine = shard_items(NS, rank, world)
        res = [_energy_grad(i) for i in mine]
        e, g = gather_results(mine, [r[0] for r in res], [r[1] for r in res], len(NS))
        if rank == 0:
            out.put((mine, e, [x.tolist() for x in g]))
        else:
            out.put((mine, None, None))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_partition_is_complete_and_balanced():
    for world in (1, 2, 3, 4):
        parts = [shard_items(NS, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(NS)))
        loads = [sum(1 << NS[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= (1 << max(NS))
    with pytest.raises(ValueError):
        shard_items(NS, 2, 2)


def test_two_gloo_ranks_gather_the_same_results_as_one_process():
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
    shards = sorted(m for m, _, _ in got)
    assert sorted(i for s in shards for i in s) == list(range(len(NS)))
    e, g = next((e, g) for _, e, g in got if e is not None)
    for i in range(len(NS)):
        e_ref, g_ref = _energy_grad(i)
        assert abs(e[i] - e_ref) < 1e-12
        assert np.max(np.abs(np.asarray(g[i]) - g_ref)) < 1e-12
