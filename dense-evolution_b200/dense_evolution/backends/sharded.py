"""Split statevectors: one 2^n state held as 2^m chunks, for states larger than
one GPU's HBM or spread over several GPUs (the reference's ``Chunk`` engine,
``backends/chunk/core.py:310-409`` and ``backends/chunk/kernels.py:188-477``).

**Layout.**  As in the reference, chunk c holds the amplitudes whose top m
index bits equal c -- at the start, the values of qubits 0..m-1 (MSB-first),
so that ``full.reshape(2^m, -1)[c]`` is chunk c -- and a chunk is an ordinary
(n-m)-qubit state of this engine.  Index positions n-m..n-1 are
*chunk-select* positions, 0..n-m-1 *local* positions; a map records which
logical qubit sits at which position.

**Exchange.**  The reference exchanges whole chunk rows with a ``ppermute``
for EVERY gate that touches a chunk-select qubit (``kernels.py:300-330``).
Here a gate that acts on a chunk-select qubit diagonally (rz, p, cz, cp, crz
and the controls of cx / cy) needs no data at all: each chunk knows its own
chunk-select bits, so the gate becomes a phase, a 1-qubit gate on the other
(local) qubit, or nothing.  Only a gate that acts on a chunk-select qubit
NON-diagonally makes the qubit trade places with the qubit at the top local
position n-m-1: chunk c0 (select bit k clear) and its partner c1 = c0 | 1<<k
swap c0's upper half with c1's lower half -- both halves contiguous, half a
chunk each way -- and the position map is updated.  Between exchanges the
gates run per chunk through the engine's fused passes.  On one GPU the halves
swap in place (``desv_swap_blocks``); across ranks each pair exchanges its
halves point to point (``torch.distributed`` isend / irecv: NCCL over NVLink
on GPUs, gloo on the CPU in tests).  No TMA multicast is involved.

Multi-GPU runs are not measured on hardware here (every run of this build has
one GPU); the exchange schedule and the data movement are tested with 2 and 4
chunks on one GPU and with world-size-2 gloo ranks on the CPU.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from ..circuits.gates import GATES, PARAMETRIC_GATES

# single-qubit gates that are diagonal for every parameter value
_DIAG_1Q = ('z', 's', 'sdg', 't', 'tdg', 'rz', 'p', 'u1', 'phase', 'gphase', 'id')
_TWO_Q = ('cx', 'cy', 'cz', 'cp', 'cphase', 'crz')


def _matrix_1q(name: str, params: Sequence[float]) -> np.ndarray:
    if name in GATES:
        return GATES[name]
    if name in ('u1', 'phase'):
        return PARAMETRIC_GATES['p'](*params)
    return PARAMETRIC_GATES[name](*params)


def nondiagonal_qubits(cmd: tuple) -> Tuple[int, ...]:
    """Qubits a transpiled gate acts on non-diagonally (they must sit at local
    positions while it runs)."""
    name = str(cmd[0]).lower()
    if name in _DIAG_1Q or name in ('cz', 'cp', 'cphase', 'crz'):
        return ()
    if name in ('cx', 'cy'):
        return (int(cmd[2]),)
    return (int(cmd[1]),)


class ChunkLayout:
    """Which logical qubit sits at which index position."""

    def __init__(self, n: int, m: int):
        if not 0 < m < n:
            raise ValueError(f'need 0 < m < n for a split state, got n={n}, m={m}')
        self.n, self.m = n, m
        self.pos = [n - 1 - q for q in range(n)]          # logical qubit -> index position
        self.at = {p: q for q, p in enumerate(self.pos)}  # index position -> logical qubit

    @property
    def top_local(self) -> int:
        return self.n - self.m - 1

    def is_select(self, q: int) -> bool:
        return self.pos[q] >= self.n - self.m

    def select_bit(self, q: int) -> int:
        """Chunk-index bit of a qubit at a chunk-select position."""
        return self.pos[q] - (self.n - self.m)

    def local_qubit(self, q: int) -> int:
        """The chunk-local (MSB-first) qubit index of a qubit at a local position."""
        return self.n - self.m - 1 - self.pos[q]

    def trade(self, q: int) -> Tuple[int, int]:
        """q (at a chunk-select position) trades places with the qubit at the top
        local position; returns (chunk-index bit, evicted qubit)."""
        k = self.select_bit(q)
        p_sel, p_loc = self.pos[q], self.top_local
        other = self.at[p_loc]
        self.pos[q], self.pos[other] = p_loc, p_sel
        self.at[p_loc], self.at[p_sel] = q, other
        return k, other


def plan_steps(target: Sequence[tuple], n: int, m: int) -> List[tuple]:
    """('gates', [transpiled gate tuples]) runs and ('trade', qubit) exchanges,
    in order, for a transpiled circuit on a layout that starts as identity."""
    lay = ChunkLayout(n, m)
    steps: List[tuple] = []
    cur: List[tuple] = []
    for cmd in target:
        for q in nondiagonal_qubits(cmd):
            if lay.is_select(q):
                if cur:
                    steps.append(('gates', cur))
                    cur = []
                lay.trade(q)
                steps.append(('trade', q))
        cur.append(tuple(cmd))
    if cur:
        steps.append(('gates', cur))
    return steps


def chunk_circuit(gates: Sequence[tuple], lay: ChunkLayout, c: int) -> List[tuple]:
    """The gates of one run as a circuit on chunk c's n-m local qubits: gates on
    chunk-select qubits are specialised by c's select bits (every such action
    is diagonal by construction of the run)."""
    out: List[tuple] = []

    def bit(q):
        return (c >> lay.select_bit(q)) & 1

    for cmd in gates:
        name = str(cmd[0]).lower()
        if name == 'cphase':
            name = 'cp'
        if name == 'id':
            continue
        if name not in _TWO_Q:
            q = int(cmd[1])
            params = [float(x) for x in cmd[2:]]
            if name == 'gphase':
                out.append(('gphase', 0, params[0] if params else 0.0))
                continue
            if lay.is_select(q):
                d = np.diag(_matrix_1q(name, params))[bit(q)]
                out.append(('gphase', 0, float(np.angle(d))))
            else:
                out.append((name, lay.local_qubit(q), *params))
            continue
        a, b = int(cmd[1]), int(cmd[2])
        th = float(cmd[3]) if len(cmd) > 3 else 0.0
        sa, sb = lay.is_select(a), lay.is_select(b)
        la = None if sa else lay.local_qubit(a)
        lb = None if sb else lay.local_qubit(b)
        if name in ('cx', 'cy'):                  # a control (diagonal), b target (local)
            if sa:
                if bit(a):
                    out.append((name[1], lb))
            else:
                out.append((name, la, lb))
        elif name in ('cz', 'cp'):
            ph = np.pi if name == 'cz' else th
            if sa and sb:
                if bit(a) and bit(b):
                    out.append(('gphase', 0, ph))
            elif sa or sb:
                if bit(a if sa else b):
                    out.append(('z', lb if sa else la) if name == 'cz' else ('p', lb if sa else la, th))
            else:
                out.append((name, la, lb) if name == 'cz' else (name, la, lb, th))
        else:                                     # crz: control a, target b
            if sa and sb:
                if bit(a):
                    out.append(('gphase', 0, (0.5 if bit(b) else -0.5) * th))
            elif sa:
                if bit(a):
                    out.append(('rz', lb, th))
            elif sb:
                out.append(('p', la, (0.5 if bit(b) else -0.5) * th))
            else:
                out.append(('crz', la, lb, th))
    return out


def _gpu_applier():
    """Run a chunk circuit in place on a CUDA chunk through the engine (plans
    cached per specialised circuit)."""
    from ..circuits.compiler import CompiledCircuit
    cache: Dict[tuple, CompiledCircuit] = {}

    def apply(chunk: torch.Tensor, n_local: int, gates: List[tuple]):
        if not gates:
            return
        key = (tuple(gates), n_local, chunk.dtype)
        plan = cache.get(key)
        if plan is None:
            if len(cache) > 256:
                cache.clear()
            plan = CompiledCircuit(list(gates), n_local, chunk.dtype)
            cache[key] = plan
        plan.run(chunk)
    return apply


class ShardedState:
    """A 2^n statevector split into 2^m chunks over this process's ranks.

    ``group``: a torch.distributed process group (None: one process holding
    every chunk).  Ranks own contiguous blocks of chunk ids.  ``applier``
    (chunk tensor, n_local, gate tuples) runs a chunk circuit; the default
    runs it on the GPU through the fused passes.  States start in |0...0>."""

    def __init__(self, n: int, m: int, dtype: torch.dtype = torch.complex64, device=None, group=None,
                 applier: Optional[Callable] = None):
        self.n, self.m = int(n), int(m)
        self.layout = ChunkLayout(self.n, self.m)
        self.dtype = dtype
        self.group = group
        if group is not None:
            import torch.distributed as dist
            self.world, self.rank = dist.get_world_size(group), dist.get_rank(group)
        else:
            self.world, self.rank = 1, 0
        nch = 1 << self.m
        if nch % self.world:
            raise ValueError(f'{nch} chunks do not divide over {self.world} ranks')
        self.per_rank = nch // self.world
        self.owned = list(range(self.rank * self.per_rank, (self.rank + 1) * self.per_rank))
        if device is None:
            device = torch.device('cuda', torch.cuda.current_device()) if applier is None else torch.device('cpu')
        self.device = torch.device(device)
        self.n_local = self.n - self.m
        self.chunks = {c: torch.zeros(1 << self.n_local, dtype=dtype, device=self.device) for c in self.owned}
        if 0 in self.chunks:
            self.chunks[0][0] = 1
        self.applier = applier or _gpu_applier()
        self.exchanges = 0

    # ------------------------------------------------------------ execution
    def run_circuit(self, circuit, transpile: bool = True):
        from ..circuits.compiler import QuantumTranspiler
        target = QuantumTranspiler.transpile(circuit) if transpile else list(circuit)
        lay = self.layout
        for cmd in target:
            for q in nondiagonal_qubits(cmd):
                if not 0 <= q < self.n:
                    raise ValueError(f'Qubit index {q} out of range [0, {self.n})')
        cur: List[tuple] = []
        for cmd in target:
            for q in nondiagonal_qubits(cmd):
                if lay.is_select(q):
                    self._run(cur)
                    cur = []
                    self._trade(q)
            cur.append(tuple(cmd))
        self._run(cur)

    def _run(self, gates: List[tuple]):
        if not gates:
            return
        for c in self.owned:
            self.applier(self.chunks[c], self.n_local, chunk_circuit(gates, self.layout, c))

    def _trade(self, q: int):
        """q's chunk-select position trades places with the top local position:
        every pair (c0, c1 = c0 | 1<<k) swaps c0's upper half with c1's lower half."""
        k, _ = self.layout.trade(q)
        half = 1 << (self.n_local - 1)
        reqs, fixups = [], []
        for c in self.owned:
            partner = c ^ (1 << k)
            mine = self.chunks[c][half:] if not (c >> k) & 1 else self.chunks[c][:half]
            if partner in self.chunks:
                if (c >> k) & 1:
                    continue                      # the pair is swapped once, from c0's side
                theirs = self.chunks[partner][:half]
                self._swap_local(mine, theirs)
                continue
            peer = partner // self.per_rank
            import torch.distributed as dist
            send = mine.contiguous().clone()
            recv = torch.empty_like(send)
            tag = min(c, partner)
            reqs.append(dist.isend(send, peer, group=self.group, tag=tag))
            reqs.append(dist.irecv(recv, peer, group=self.group, tag=tag))
            fixups.append((mine, recv, send))
        for r in reqs:
            r.wait()
        for mine, recv, _ in fixups:
            mine.copy_(recv)
        self.exchanges += 1

    @staticmethod
    def _swap_local(a: torch.Tensor, b: torch.Tensor):
        if a.is_cuda:
            from .. import _native as N
            N.check(N.lib().desv_swap_blocks(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                             a.numel() * a.element_size(), ctypes.c_void_p(N.stream_ptr())),
                    'chunk exchange')
        else:
            t = a.clone()
            a.copy_(b)
            b.copy_(t)

    # ------------------------------------------------------------ read-out
    def physical_chunks(self) -> Dict[int, torch.Tensor]:
        return self.chunks

    def logical_state(self) -> np.ndarray:
        """The whole state in logical MSB-first order as a host array (every
        rank gets it; for states that fit host memory)."""
        full = np.zeros(1 << self.n, dtype=np.complex128)
        local = {c: t.detach().cpu().numpy().astype(np.complex128) for c, t in self.chunks.items()}
        if self.world > 1:
            import torch.distributed as dist
            objs = [None] * self.world
            dist.all_gather_object(objs, local, group=self.group)
            for d in objs:
                local.update(d)
        phys = np.concatenate([local[c] for c in range(1 << self.m)])
        idx = np.arange(1 << self.n, dtype=np.int64)
        logical = np.zeros_like(idx)
        for q in range(self.n):
            logical |= ((idx >> self.layout.pos[q]) & 1) << (self.n - 1 - q)
        full[logical] = phys
        return full
