"""Fusion pass: transpiled gate tuples -> fused tile passes for libdesv.

The reference compiler has no fusion: every gate row of
``circuits/compiler.py:318-355`` is one full read + gather + write of the
state.  This pass rewrites a transpiled circuit into a handful of HBM passes:

1. **Lowering.**  Every gate becomes an IR gate on index bits (qubit q is bit
   n-1-q, MSB-first): a 2x2 matrix on a target bit with optional control
   bits (h, rx, cx, cy, ...), a diagonal on two bits (cz, cp, crz), a dense
   4x4 on two bits (untranspiled swap/iswap/ecr) or a global scalar (gphase).
2. **1-qubit fusion.**  Runs of uncontrolled 1-qubit gates on one bit are
   multiplied into one 2x2 in FP64 (U3 -> Rz.Ry.Rz.GPhase collapses back into
   one matrix).  Diagonal / anti-diagonal / real / phase-only matrices are
   flagged so the kernel uses the cheaper update.
3. **Pass scheduling.**  A pass owns a tile of 2^K amplitudes: the L low index
   bits plus K-L chosen high bits.  Gates are taken greedily in circuit order
   while their NON-DIAGONAL bits fit the tile; diagonal actions (cz, cp, crz,
   controls) never need their bits in the tile.  A gate that cannot run is
   deferred and blocks later gates that do not commute with it (gates commute
   when every shared bit is acted on diagonally by both).
4. **Stage scheduling.**  Inside a pass each register stage owns 4 tile bits
   (>= 5); tile bits 0..4 are warp lanes and are available in every stage.
   The same greedy rule assigns the pass's ops to stages.

The output is packed into the ``desv_pass`` / ``desv_op`` structs of
``include/desv.h`` plus a pool of complex matrices.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .. import _native as N
from .gates import GATES, PARAMETRIC_GATES

LANE_BITS = 5
REG_SLOTS = 4
MIN_FUSED_QUBITS = 9  # 5 lane bits + 4 register bits

_STATIC_1Q = ('h', 'x', 'y', 'z', 's', 'sdg', 't', 'tdg', 'sx')
_PARAM_1Q = ('rx', 'ry', 'rz', 'p', 'u1', 'phase', 'gphase')
# generator G with dU/dtheta = G U for the differentiable gates (adjoint method)
GENERATOR = {'rx': 'x', 'ry': 'y', 'rz': 'z', 'p': 'p1', 'u1': 'p1', 'phase': 'p1', 'cp': 'cp', 'cphase': 'cp',
             'crz': 'crz'}


def _unknown(name):
    return ValueError(
        f"unknown gate '{name}' -- not in GATES or PARAMETRIC_GATES. A typo in a gate name used to be "
        f"silently dropped from the circuit instead of raising (issue #4).")


# grouped op streams by structure (see PackedPlan.compact), oldest dropped first
_STRUCT_CACHE: dict = {}


@dataclass
class IRGate:
    """One gate on index bits.  kind: 'm1' | 'd2' | 'm2' | 'scalar'."""
    kind: str
    name: str
    t: int = -1              # m1 target bit; d2 / m2: bit a (LOW bit of the matrix index)
    t2: int = -1             # d2 / m2: bit b (HIGH bit of the matrix index)
    cbits: Tuple[int, ...] = ()
    cvals: Tuple[int, ...] = ()
    value: float = 0.0       # parameter value
    slot: int = -1           # theta slot (energy functions), -1 = constant
    const: Optional[np.ndarray] = None  # matrix of non-parametric gates

    def matrix(self, theta=None) -> np.ndarray:
        v = self.value if (self.slot < 0 or theta is None) else float(theta[self.slot])
        if self.const is not None:
            return self.const
        return gate_matrix_of(self.kind, self.name, v)


def _is_diag(m: np.ndarray) -> bool:
    return m.shape == (2, 2) and m[0, 1] == 0 and m[1, 0] == 0


def gate_matrix_of(kind: str, name: str, v: float) -> np.ndarray:
    """FP64 matrix of a parametric IR gate (m1: 2x2; d2: 4 diagonal factors)."""
    if kind == 'm1':
        if name in ('p', 'u1', 'phase'):
            return PARAMETRIC_GATES['p'](v)
        if name == 'gphase':
            return PARAMETRIC_GATES['gphase'](v)
        return PARAMETRIC_GATES[name](v)
    if kind == 'd2':
        if name in ('cp', 'cphase'):
            return np.array([1, 1, 1, np.exp(1j * v)], dtype=np.complex128)
        if name == 'crz':  # factor index: bit(control) + 2 * bit(target)
            return np.array([1, np.exp(-0.5j * v), 1, np.exp(0.5j * v)], dtype=np.complex128)
    if kind == 'scalar':
        return np.full(4, np.exp(1j * v), dtype=np.complex128)
    raise ValueError(f'no parametric matrix for {kind} {name}')


def lower(target: Sequence[tuple], n: int, slots: Optional[Sequence[int]] = None) -> List[IRGate]:
    """Transpiled gate tuples -> IR gates.  `slots[i]` (optional) is the theta
    slot of gate i (energy functions) or -1."""
    out: List[IRGate] = []
    for gi, cmd in enumerate(target):
        name = (cmd[0] if isinstance(cmd[0], str) else str(cmd[0])).lower()
        a = cmd[1:]
        slot = -1 if slots is None else int(slots[gi])

        def qbit(q, what='gate'):
            qi = int(q)
            if not 0 <= qi < n:
                raise ValueError(f"Qubit index {qi} out of range [0, {n}) in {what} '{name}'")
            return n - 1 - qi

        def two(with_param: bool):
            if len(a) < 2:
                raise ValueError(f"gate '{name}' needs two qubits")
            c, t = qbit(a[0]), qbit(a[1])
            if c == t:
                raise ValueError('Control and target qubits must differ')
            p = float(a[2]) if with_param and len(a) > 2 else 0.0
            return c, t, p

        if name == 'id':
            if a:
                qbit(a[0])
            continue
        if name in _STATIC_1Q:
            if not a:
                raise ValueError(f"gate '{name}' needs a qubit")
            out.append(IRGate('m1', name, t=qbit(a[0]), const=GATES[name]))
        elif name in _PARAM_1Q:
            if not a:
                raise ValueError(f"gate '{name}' needs a qubit")
            t = qbit(a[0])
            p = float(a[1]) if len(a) > 1 else 0.0
            if name == 'gphase':
                out.append(IRGate('scalar', name, value=p, slot=slot))
            else:
                out.append(IRGate('m1', name, t=t, value=p, slot=slot))
        elif name in ('u3', 'u2'):
            need = 4 if name == 'u3' else 3
            if len(a) < need:
                raise ValueError(f"gate '{name}' needs {need - 1} parameters")
            t = qbit(a[0])
            out.append(IRGate('m1', name, t=t, const=PARAMETRIC_GATES[name](*[float(x) for x in a[1:need]])))
        elif name in ('cx', 'cy'):
            c, t, _ = two(False)
            out.append(IRGate('m1', name, t=t, cbits=(c,), cvals=(1,), const=GATES[name[1]]))
        elif name == 'cz':
            c, t, _ = two(False)
            out.append(IRGate('d2', name, t=c, t2=t, const=np.array([1, 1, 1, -1], dtype=np.complex128)))
        elif name in ('cp', 'cphase', 'crz'):
            c, t, p = two(True)
            out.append(IRGate('d2', name, t=c, t2=t, value=p, slot=slot))
        elif name in ('swap', 'iswap', 'ecr'):
            # exact CX decompositions (same as the transpiler's): keeps every gate of
            # a fused pass a 2x2 / diagonal, whichever bits it touches
            q1, q2 = int(a[0]), int(a[1])
            two(False)
            if name == 'swap':
                sub = [('cx', q1, q2), ('cx', q2, q1), ('cx', q1, q2)]
            elif name == 'iswap':
                sub = [('s', q1), ('h', q1), ('s', q2), ('cx', q1, q2), ('cx', q2, q1), ('h', q2)]
            else:
                sub = [('s', q1), ('sx', q2), ('cx', q1, q2), ('x', q1), ('gphase', q1, -np.pi / 4.0)]
            out.extend(lower(sub, n))
        else:
            raise _unknown(cmd[0])
    return out


# ---------------------------------------------------------------------------
# fused ops
# ---------------------------------------------------------------------------

@dataclass
class FOp:
    kind: str                       # 'm1' | 'd2' | 'm2' | 'scalar'
    t: int = -1
    t2: int = -1
    cbits: Tuple[int, ...] = ()
    cvals: Tuple[int, ...] = ()
    src: List[IRGate] = field(default_factory=list)
    nd: int = 0
    d: int = 0

    def matrix(self, theta=None) -> np.ndarray:
        if self.kind == 'm1':
            m = np.eye(2, dtype=np.complex128)
            for g in self.src:
                if g.kind == 'scalar':
                    m = np.exp(1j * (g.value if g.slot < 0 or theta is None else float(theta[g.slot]))) * m
                else:
                    m = g.matrix(theta) @ m
            return m
        if self.kind in ('d2', 'scalar'):
            v = np.ones(4, dtype=np.complex128)
            for g in self.src:
                v = v * g.matrix(theta)
            return v
        return self.src[0].matrix(theta)


def fuse_1q(gates: Sequence[IRGate], merge: bool = True) -> List[FOp]:
    """Merge runs of uncontrolled 1-qubit gates per bit (and global scalars into
    the next 1-qubit run) into single 2x2 ops; keep everything else in order."""
    out: List[FOp] = []
    pending = {}        # bit -> FOp under construction (not yet in `out`)
    scal: List[IRGate] = []

    def flush(bits_mask: int):
        for b in [b for b in pending if (bits_mask >> b) & 1]:
            out.append(pending.pop(b))

    for g in gates:
        if g.kind == 'scalar':
            if merge and pending:
                next(iter(pending.values())).src.append(g)
            else:
                scal.append(g)
            continue
        if g.kind == 'm1' and not g.cbits and merge:
            op = pending.get(g.t)
            if op is None:
                op = FOp('m1', t=g.t)
                pending[g.t] = op
            op.src.append(g)
            continue
        touched = 0
        for b in (g.t, g.t2, *g.cbits):
            if b >= 0:
                touched |= 1 << b
        flush(touched)
        out.append(FOp(g.kind, t=g.t, t2=g.t2, cbits=g.cbits, cvals=g.cvals, src=[g]))
    flush(~0)
    for s in scal:
        out.append(FOp('scalar', src=[s]))
    for op in out:
        _classify(op)
    if merge:
        out = _merge_diagonals(out)
    return out


def _constant(op: FOp) -> bool:
    return all(g.slot < 0 for g in op.src)


def zyz(u: np.ndarray):
    """u = D_post @ R @ D_pre with R = Ry(b) real and D_pre / D_post diagonal
    (the global phase is folded into D_pre).  Returns (d_pre, r, d_post) or
    None when the factors do not reproduce u to 1e-12."""
    det = u[0, 0] * u[1, 1] - u[0, 1] * u[1, 0]
    if abs(abs(det) - 1.0) > 1e-9:
        return None
    g = np.sqrt(det)
    v = u / g                                   # SU(2): [[e^-ip c, -e^-im s], [e^im s, e^ip c]]
    c, sn = abs(v[0, 0]), abs(v[1, 0])
    b = 2.0 * np.arctan2(sn, c)
    p = np.angle(v[1, 1]) if c > 1e-12 else 0.0          # (a + c') / 2
    m = np.angle(v[1, 0]) if sn > 1e-12 else 0.0         # (a - c') / 2
    a, cc = p + m, p - m
    r = np.array([[np.cos(b / 2), -np.sin(b / 2)], [np.sin(b / 2), np.cos(b / 2)]], dtype=np.complex128)
    d_pre = g * np.diag([np.exp(-0.5j * cc), np.exp(0.5j * cc)])
    d_post = np.diag([np.exp(-0.5j * a), np.exp(0.5j * a)])
    if np.max(np.abs(d_post @ r @ d_pre - u)) > 1e-12:
        return None
    return d_pre, r, d_post


def _split_zyz(ops: List[FOp]) -> List[FOp]:
    """Constant uncontrolled 2x2 ops with a general (complex, non-diagonal)
    matrix become diagonal . real . diagonal.  The real middle factor costs
    half the arithmetic of a general 2x2 on the device, and the diagonals
    commute through cz / cp / controls and merge with their neighbours."""
    out: List[FOp] = []
    for op in ops:
        if op.kind != 'm1' or op.cbits or not _constant(op) or not op.nd:
            out.append(op)
            continue
        u = op.matrix(None)
        if not np.any(u.imag) or (u[0, 0] == 0 and u[1, 1] == 0):
            out.append(op)          # already real, or anti-diagonal (x / y-like)
            continue
        f = zyz(u)
        if f is None:
            out.append(op)
            continue
        for m in f:
            kind_name = 'zyz_r' if m[0, 1] != 0 else 'zyz_d'
            fo = FOp('m1', t=op.t, src=[IRGate('m1', kind_name, t=op.t, const=m)])
            _classify(fo)
            out.append(fo)
    return out


def _merge_diagonals(ops: List[FOp]) -> List[FOp]:
    """Merge every constant uncontrolled 1-bit diagonal into the previous one on
    the same bit when everything in between acts on that bit diagonally (or not
    at all): the later diagonal commutes back past those ops."""
    out: List[FOp] = []
    open_: dict = {}
    for op in ops:
        if op.kind == 'm1' and not op.cbits and not op.nd and _constant(op):
            j = open_.get(op.t)
            if j is not None:
                out[j].src.extend(op.src)
                continue
            open_[op.t] = len(out)
            out.append(op)
            continue
        for b in _bits(op.nd):
            open_.pop(b, None)
        out.append(op)
    return out


def _classify(op: FOp):
    """Bits acted on non-diagonally (`nd`) and diagonally (`d`)."""
    nd = d = 0
    for b in op.cbits:
        d |= 1 << b
    if op.kind == 'm1':
        diag = all(g.kind == 'scalar' or (g.const is not None and _is_diag(g.const)) or
                   (g.const is None and g.name in ('rz', 'p', 'u1', 'phase')) for g in op.src)
        if diag:
            d |= 1 << op.t
        else:
            nd |= 1 << op.t
    elif op.kind == 'd2':
        d |= (1 << op.t) | (1 << op.t2)
    elif op.kind == 'm2':
        nd |= (1 << op.t) | (1 << op.t2)
    op.nd, op.d = nd, d


# ---------------------------------------------------------------------------
# scheduling
# ---------------------------------------------------------------------------

def _bits(mask: int):
    b = 0
    while mask:
        if mask & 1:
            yield b
        mask >>= 1
        b += 1


def _greedy(ids: Sequence[int], ops: Sequence[FOp], fits) -> Tuple[List[int], List[int]]:
    """Take ops in order while `fits(op)` (which may grow the resource set);
    a deferred op blocks every later op that does not commute with it."""
    taken, deferred = [], []
    b_any = b_nd = 0
    for i in ids:
        op = ops[i]
        if ((op.nd | op.d) & b_any) or (op.nd & b_nd) or not fits(op):
            deferred.append(i)
            b_any |= op.nd
            b_nd |= op.d
        else:
            taken.append(i)
    return taken, deferred


@dataclass
class PassSpec:
    K: int
    L: int
    high: List[int]
    stages: List[Tuple[List[int], List[int]]]   # (register tile-local bits[4], op ids)


def schedule(ops: Sequence[FOp], n: int, kmax: int) -> List[PassSpec]:
    K = min(kmax, n)
    remaining = list(range(len(ops)))
    passes: List[PassSpec] = []
    while remaining:
        H = set()

        def fits_pass(op):
            need = {b for b in _bits(op.nd) if b >= LANE_BITS} - H
            if len(H) + len(need) > K - LANE_BITS:
                return False
            H.update(need)
            return True

        taken, remaining = _greedy(remaining, ops, fits_pass)
        if not taken:
            raise RuntimeError('fusion: no schedulable gate (internal error)')
        # widen the low contiguous run while the tile has spare bits
        L = LANE_BITS
        while True:
            high = sorted(h for h in H if h >= L)
            L2 = K - len(high)
            if L2 == L:
                break
            L = L2
        high = sorted(h for h in H if h >= L)
        assert len(high) == K - L
        tl = {b: b for b in range(L)}
        for i, h in enumerate(high):
            tl[h] = L + i
        passes.append(PassSpec(K, L, high, _stages(taken, ops, tl, K)))
    return passes


def _stages(ids: List[int], ops: Sequence[FOp], tl: dict, K: int):
    stages = []
    remaining = list(ids)
    while remaining:
        G: List[int] = []

        def fits_stage(op):
            need = []
            for b in _bits(op.nd):
                p = tl[b]
                if op.kind == 'm2' and p < LANE_BITS:
                    return False          # a dense 4x4 needs both bits in registers
                if p >= LANE_BITS and p not in G and p not in need:
                    need.append(p)
            if op.kind in ('m1', 'g1'):
                creg = [tl[c] for c in op.cbits if c in tl and tl[c] >= LANE_BITS and (tl[c] in G or tl[c] in need)]
                if len(creg) > 1:
                    return False
            if len(G) + len(need) > REG_SLOTS:
                return False
            G.extend(need)
            return True

        taken, remaining = _greedy(remaining, ops, fits_stage)
        if not taken:
            raise RuntimeError('fusion: no schedulable op in a stage (internal error)')
        g = sorted(G)
        for p in range(LANE_BITS, K):
            if len(g) == REG_SLOTS:
                break
            if p not in g:
                g.append(p)
        stages.append((sorted(g), taken))
    return stages


# ---------------------------------------------------------------------------
# packing
# ---------------------------------------------------------------------------

def _m1_flags(m: np.ndarray) -> int:
    f = 0
    if m[0, 1] == 0 and m[1, 0] == 0:
        f |= N.F_DIAG
        if m[0, 0] == 1:
            f |= N.F_PHASE1
    elif m[0, 0] == 0 and m[1, 1] == 0:
        f |= N.F_ANTI
    if not np.any(m.imag):
        f |= N.F_REAL
    return f


def _clean(m: np.ndarray) -> np.ndarray:
    m = np.array(m, dtype=np.complex128)
    scale = max(1.0, float(np.abs(m).max()))
    re, im = m.real.copy(), m.imag.copy()
    re[np.abs(re) < 1e-15 * scale] = 0.0
    im[np.abs(im) < 1e-15 * scale] = 0.0
    return re + 1j * im


class Packed:
    """Packed pass/op/matrix arrays (host) for one fused circuit."""

    def __init__(self, n: int, ops: List[FOp], passes: List[PassSpec], adjoint: bool = False):
        self.n = n
        self.fops = ops
        self.specs = passes
        self.adjoint = adjoint
        recs, pass_rows, self.op_slots = [], [], []   # op_slots: (record index, fop index)
        self.m2_swap = {}
        self.diag1 = {}        # record index -> control value on gb (None: no gb control) for 1-bit diagonals
        self.param_map: List[int] = []                # adjoint: local gradient slot -> theta index
        for ps in passes:
            begin = len(recs)
            map_begin = len(self.param_map)
            local = {}
            tl = {b: b for b in range(ps.L)}
            for i, h in enumerate(ps.high):
                tl[h] = ps.L + i
            for g, ids in ps.stages:
                rec = np.zeros((), dtype=N.OP_DTYPE)
                rec['kind'] = N.OP_STAGE
                rec['g'] = g
                rec['mat'] = len(ids)
                rec['param'] = -1
                recs.append(rec)
                slot_of = {p: s for s, p in enumerate(g)}
                for i in ids:
                    self._pending_diag1 = 'none'
                    rec = self._op_record(ops[i], tl, slot_of)
                    if self._pending_diag1 != 'none':
                        self.diag1[len(recs)] = self._pending_diag1
                    if ops[i].kind in ('g1', 'gd'):
                        th = ops[i].src[0].slot
                        if th not in local:
                            local[th] = len(local)
                            self.param_map.append(th)
                        rec['param'] = local[th]
                    recs.append(rec)
                    self.op_slots.append((len(recs) - 1, i))
                    if ops[i].kind == 'm2':
                        self.m2_swap[len(recs) - 1] = slot_of[tl[ops[i].t]] > slot_of[tl[ops[i].t2]]
            end = len(recs)
            row = np.zeros((), dtype=N.ADJ_PASS_DTYPE if adjoint else N.PASS_DTYPE)
            row['tile_bits'], row['low_bits'], row['op_begin'], row['op_end'] = ps.K, ps.L, begin, end
            h = np.zeros(16, np.uint8)
            h[:len(ps.high)] = ps.high
            row['high'] = h
            if adjoint:
                row['nparams'], row['map_begin'] = len(local), map_begin
            pass_rows.append(row)
        pdt = N.ADJ_PASS_DTYPE if adjoint else N.PASS_DTYPE
        self.ops = np.array(recs, dtype=N.OP_DTYPE) if recs else np.zeros(0, N.OP_DTYPE)
        self.passes = np.array(pass_rows, dtype=pdt) if pass_rows else np.zeros(0, pdt)
        self.nstages = sum(len(p.stages) for p in passes)
        self.max_params = max([int(r['nparams']) for r in pass_rows], default=0) if adjoint else 0

    def _op_record(self, op: FOp, tl: dict, slot_of: dict):
        rec = np.zeros((), dtype=N.OP_DTYPE)
        rec['param'] = -1
        rec['cslot'] = -1
        rec['ga'] = rec['gb'] = 0xFF
        rec['sa'] = rec['sb'] = -1
        cmask = cval = 0
        if op.kind in ('m1', 'g1') and not (op.nd >> op.t) & 1:
            # diagonal on its target: a DIAG record over (target, first control), so the
            # target needs no register slot or lane
            rec['kind'] = N.OP_DIAG if op.kind == 'm1' else N.OP_GRAD
            rec['s1'] = 1 if op.kind == 'g1' else 0
            ctl = None
            rec['ga'] = op.t
            if op.t in tl and tl[op.t] in slot_of:
                rec['sa'] = slot_of[tl[op.t]]
            for i, (c, v) in enumerate(zip(op.cbits, op.cvals)):
                if i == 0:
                    rec['gb'] = c
                    if c in tl and tl[c] in slot_of:
                        rec['sb'] = slot_of[tl[c]]
                    ctl = v
                else:
                    cmask |= 1 << c
                    cval |= v << c
            self._pending_diag1 = ctl
        elif op.kind in ('m1', 'g1'):
            rec['kind'] = N.OP_M1 if op.kind == 'm1' else N.OP_GRAD
            rec['s1'] = 0
            p = tl[op.t]
            rec['s0'] = slot_of[p] if p >= LANE_BITS else 16 + p
            for c, v in zip(op.cbits, op.cvals):
                if c in tl and tl[c] in slot_of:
                    rec['cslot'] = slot_of[tl[c]]
                else:
                    cmask |= 1 << c
                    cval |= v << c
        elif op.kind in ('d2', 'scalar', 'gd'):
            rec['kind'] = N.OP_DIAG if op.kind != 'gd' else N.OP_GRAD
            rec['s1'] = 1 if op.kind == 'gd' else 0
            for key, skey, b in (('ga', 'sa', op.t), ('gb', 'sb', op.t2)):
                if b >= 0:
                    rec[key] = b
                    if b in tl and tl[b] in slot_of:
                        rec[skey] = slot_of[tl[b]]
        elif op.kind == 'm2':
            rec['kind'] = N.OP_M2
            sa, sb = slot_of[tl[op.t]], slot_of[tl[op.t2]]
            rec['s0'], rec['s1'] = min(sa, sb), max(sa, sb)
        rec['cmask'], rec['cval'] = cmask, cval
        return rec

    # ------------------------------------------------------------------ matrices
    def _prepare(self):
        """Vectorised recipe of every record's matrix (built once per plan)."""
        gates, gidx = [], {}

        def gi(g):
            k = id(g)
            if k not in gidx:
                gidx[k] = len(gates)
                gates.append(g)
            return gidx[k]

        R = len(self.op_slots)
        recipes, out, tf, ctl, isgen, gen_m = [], np.zeros(R, np.int8), np.zeros(R, np.int8), \
            np.full(R, -2, np.int8), np.zeros(R, bool), np.zeros((R, 2, 2), np.complex128)
        gen_v = np.zeros((R, 4), np.complex128)
        m2_rec = []
        off = np.zeros(R, np.int64)
        pos = 0
        for r, (rec_i, fi) in enumerate(self.op_slots):
            op = self.fops[fi]
            kind = op.kind
            srcs = [gi(g) for g in op.src]
            recipes.append(srcs)
            bwd = type(op).__name__ == 'BOp'
            if kind in ('g1', 'gd'):
                tf[r] = 2
                isgen[r] = True
                m = op.matrix(None)
                if kind == 'g1':
                    gen_m[r] = m
                else:
                    gen_v[r] = m
            elif bwd:
                tf[r] = 1
            if rec_i in self.diag1:
                out[r] = 1
                c = self.diag1[rec_i]
                ctl[r] = -1 if c is None else int(c)
            elif kind in ('m1', 'g1'):
                out[r] = 0
            elif kind in ('d2', 'scalar', 'gd'):
                out[r] = 2
            else:
                out[r] = 3
                m2_rec.append(r)
            off[r] = pos
            pos += 16 if out[r] == 3 else 4
            self.ops[rec_i]['mat'] = off[r]
        D = max([len(x) for x in recipes], default=1) or 1
        src = np.full((R, D), -1, np.int64)
        for r, x in enumerate(recipes):
            src[r, :len(x)] = x
        G = len(gates)
        code = np.zeros(G, np.int8)
        slot = np.full(G, -1, np.int64)
        value = np.zeros(G)
        cmat = np.tile(np.eye(2, dtype=np.complex128), (G, 1, 1))
        cvec = np.ones((G, 4), np.complex128)
        names = {'rx': 1, 'ry': 2, 'rz': 3, 'p': 4, 'u1': 4, 'phase': 4}
        for i, g in enumerate(gates):
            slot[i], value[i] = g.slot, g.value
            if g.kind == 'scalar':
                code[i] = 5
            elif g.kind == 'm1':
                if g.const is not None:
                    cmat[i] = g.const
                else:
                    code[i] = names[g.name]
            elif g.kind == 'd2':
                if g.const is not None:
                    cvec[i] = g.const
                else:
                    code[i] = 11 if g.name in ('cp', 'cphase') else 12
            else:
                code[i] = 20   # m2: handled per record
        self._vec = dict(R=R, D=D, src=src, out=out, tf=tf, ctl=ctl, isgen=isgen, gen_m=gen_m, gen_v=gen_v,
                         off=off, pool_len=pos, code=code, slot=slot, value=value, cmat=cmat, cvec=cvec,
                         rec_index=np.array([ri for ri, _ in self.op_slots], np.int64), m2_rec=m2_rec,
                         gates=gates)

    def materialize(self, theta=None, dtype=np.complex64):
        """Matrix pool (and per-op flags in self.ops) for the given parameters."""
        if getattr(self, '_vec', None) is None:
            self._prepare()
        V = self._vec
        R = V['R']
        if R == 0:
            return np.zeros(4, dtype=dtype)
        slot, code = V['slot'], V['code']
        v = V['value'].copy()
        if theta is not None:
            th = np.asarray(theta, dtype=np.float64)
            has = slot >= 0
            v[has] = th[slot[has]]
        # every gate as a 2x2 (1-qubit kinds) and as a 4-vector (diagonal kinds)
        mat = V['cmat'].copy()
        vec = V['cvec'].copy()
        c, s = np.cos(v / 2), np.sin(v / 2)
        em, ep, e1 = np.exp(-0.5j * v), np.exp(0.5j * v), np.exp(1j * v)
        k = code == 1
        mat[k] = np.stack([np.stack([c[k], -1j * s[k]], -1), np.stack([-1j * s[k], c[k]], -1)], -2)
        k = code == 2
        mat[k] = np.stack([np.stack([c[k], -s[k]], -1), np.stack([s[k], c[k]], -1)], -2).astype(np.complex128)
        k = code == 3
        mat[k] = 0
        mat[k, 0, 0], mat[k, 1, 1] = em[k], ep[k]
        k = code == 4
        mat[k] = 0
        mat[k, 0, 0], mat[k, 1, 1] = 1.0, e1[k]
        k = code == 5
        mat[k] = 0
        mat[k, 0, 0], mat[k, 1, 1] = e1[k], e1[k]
        vec[k] = e1[k][:, None]
        k = code == 11
        vec[k, 3] = e1[k]
        k = code == 12
        vec[k, 1], vec[k, 3] = em[k], ep[k]
        # record products (in application order: later gates multiply from the left)
        src = V['src']
        M = np.tile(np.eye(2, dtype=np.complex128), (R, 1, 1))
        Vv = np.ones((R, 4), np.complex128)
        for d in range(V['D']):
            sel = src[:, d] >= 0
            if not sel.any():
                continue
            ids = src[sel, d]
            M[sel] = mat[ids] @ M[sel]
            Vv[sel] = Vv[sel] * vec[ids]
        tf = V['tf']
        dag = tf == 1
        M[dag] = np.conj(np.swapaxes(M[dag], -1, -2))
        Vv[dag] = np.conj(Vv[dag])
        gen = tf == 2
        M[gen] = V['gen_m'][gen]
        Vv[gen] = V['gen_v'][gen]
        out = V['out']
        pool = np.zeros(V['pool_len'], np.complex128)
        flags = np.zeros(R, np.uint8)
        # 2x2 records
        k = out == 0
        if k.any():
            m = _clean_batch(M[k].reshape(-1, 4))
            idx = V['off'][k][:, None] + np.arange(4)
            pool[idx] = m
            diag = (m[:, 1] == 0) & (m[:, 2] == 0)
            f = np.where(diag, N.F_DIAG, 0) | np.where(diag & (m[:, 0] == 1), N.F_PHASE1, 0) | \
                np.where(~diag & (m[:, 0] == 0) & (m[:, 3] == 0), N.F_ANTI, 0) | \
                np.where(~np.any(m.imag != 0, axis=1), N.F_REAL, 0)
            flags[k] = np.where(V['isgen'][k], 0, f)
        # 1-bit diagonal tables over (target, first control)
        k = out == 1
        if k.any():
            m = _clean_batch(M[k].reshape(-1, 4))
            d0, d1 = m[:, 0], m[:, 3]
            offv = np.where(V['isgen'][k], 0.0, 1.0).astype(np.complex128)
            ctl = V['ctl'][k]
            tab = np.stack([d0, d1, d0, d1], -1)
            c1 = ctl == 1
            tab[c1] = np.stack([offv[c1], offv[c1], d0[c1], d1[c1]], -1)
            c0 = ctl == 0
            tab[c0] = np.stack([d0[c0], d1[c0], offv[c0], offv[c0]], -1)
            pool[V['off'][k][:, None] + np.arange(4)] = tab
            sign = (~np.any(tab.imag != 0, axis=1)) & np.all(np.abs(tab.real) == 1, axis=1)
            flags[k] = np.where(V['isgen'][k], 0, np.where(sign, N.F_SIGN, 0))
        # diagonal records
        k = out == 2
        if k.any():
            m = _clean_batch(Vv[k])
            pool[V['off'][k][:, None] + np.arange(4)] = m
            sign = (~np.any(m.imag != 0, axis=1)) & np.all(np.abs(m.real) == 1, axis=1)
            flags[k] = np.where(V['isgen'][k], 0, np.where(sign, N.F_SIGN, 0))
        # dense 4x4 records (rare): one by one
        for r in V['m2_rec']:
            rec_i, fi = self.op_slots[r]
            m = _clean(self.fops[fi].matrix(theta))
            if self.m2_swap[rec_i]:
                perm = [0, 2, 1, 3]
                m = m[np.ix_(perm, perm)]
            pool[V['off'][r]:V['off'][r] + 16] = m.reshape(-1)
        self.ops['flags'][V['rec_index']] = flags
        self.ops['code'][V['rec_index']] = self._dispatch_codes(flags)
        return pool.astype(dtype)

    def _dispatch_codes(self, flags: np.ndarray) -> np.ndarray:
        """Per-record dispatch codes of the stage interpreter (include/desv.h, desv_op.code)."""
        recs = self.ops[self._vec['rec_index']]
        kind = recs['kind'].astype(np.int64)
        s0 = recs['s0'].astype(np.int64)
        cs = recs['cslot'].astype(np.int64)
        sa = recs['sa'].astype(np.int64)
        sb = recs['sb'].astype(np.int64)
        pred = recs['cmask'] != 0
        f = flags.astype(np.int64)
        var = np.where(f & N.F_PHASE1, 3, np.where(f & N.F_DIAG, 2, np.where(f & N.F_ANTI, 4,
                                                                        np.where(f & N.F_REAL, 1, 0))))
        code = np.zeros(len(recs), np.int64)
        m1 = kind == N.OP_M1
        lane = m1 & (s0 >= 16)
        reg = m1 & (s0 < 16)
        free_lane = lane & ~pred & (cs < 0)
        code[free_lane] = 53 + var[free_lane]
        code[lane & ~free_lane] = 192
        u = reg & (cs < 0)
        code[u] = 1 + s0[u] * 5 + var[u]
        c = reg & (cs >= 0)
        code[c] = 21 + (s0[c] * 4 + cs[c]) * 2 + (var[c] != 4)
        code[reg & pred] |= 0x8000
        d = kind == N.OP_DIAG
        sign = (f & N.F_SIGN) != 0
        base = np.where(sign, 58, 83)
        code[d] = base[d] + (sa[d] + 1) * 5 + (sb[d] + 1)
        code[d & pred] |= 0x8000
        if np.any(kind == N.OP_M2):
            raise RuntimeError('fusion: dense 4x4 records are not supported by the pass kernels')
        return code.astype(np.uint16)


    # ------------------------------------------------------------ grouping
    def compact(self, pool: np.ndarray):
        """Forward-pass op stream with runs of ops grouped (desv.h grouped codes).

        Inside a stage, a run of uncontrolled general / real 2x2 ops on distinct
        register slots and lane bits becomes one layer op (the gates commute; the
        matrices of an all-real layer are stored as (v, v) pairs), and a run
        of +-1 diagonals becomes one sign group, so the kernel dispatches once
        per run.  Ops are first reordered inside the stage (never across a
        non-commuting pair) to make the runs long.  Call after `materialize`
        (codes and flags are set there).  Returns (ops, passes, pool) for
        desv_apply_passes; the canonical records in self.ops are left untouched.
        """
        codes = self.ops['code']
        c = codes & 0x7FFF
        sg = np.nonzero((c >= 58) & (c <= 82))[0]
        tabs = pool[self.ops['mat'][sg].astype(np.int64)[:, None] + np.arange(4)] if len(sg) else pool[:0]
        key = codes.tobytes() + np.signbit(tabs.real).tobytes()
        cache = getattr(self, '_compact_cache', None)
        if cache is None or cache[0] != key or cache[6] != len(pool) or cache[7] != pool.dtype:
            # plans of the same structure (a circuit re-run with new angles) share the
            # grouping: the records (slots, masks, offsets, codes), the passes and the
            # sign pattern determine it completely
            skey = hashlib.sha1(self.ops.tobytes() + self.passes.tobytes() + key +
                                str((len(pool), pool.dtype.str)).encode()).digest()
            struct = _STRUCT_CACHE.get(skey)
            if struct is None:
                struct = self._compact_structure(pool)
                if len(_STRUCT_CACHE) >= 32:
                    _STRUCT_CACHE.pop(next(iter(_STRUCT_CACHE)))
                _STRUCT_CACHE[skey] = struct
            cache = (key,) + struct + (len(pool), pool.dtype)
            self._compact_cache = cache
        _, ops, passes, (gather, form), words, dv = cache[:6]
        if words is None and not len(gather) and dv is None:
            return ops, passes, pool
        gathered = pool[gather]
        # real layer matrices as (v, v); general register-slot matrices as the
        # packed pairs (re, re), (-im, im): the kernel multiplies them element-wise
        re_ = (form == 1) | (form == 2)
        gathered[re_] = gathered[re_].real * (1 + 1j)
        im_ = form == 3
        gathered[im_] = gathered[im_].imag * (-1 + 1j)
        ext = [pool, gathered]
        wpe = pool.dtype.itemsize // 4
        w = np.zeros(0 if words is None else (len(words) + wpe - 1) // wpe * wpe, np.uint32)
        if words is not None:
            # sign entries: raw uint32 words stored in whole pool elements
            w[:len(words)] = words
        ext.append(np.frombuffer(w.tobytes(), dtype=pool.dtype))
        if dv is not None:
            ext.append(_diag_group_values(dv, pool))
        return ops, passes, np.concatenate(ext)

    def _compact_structure(self, pool):
        recs = self.ops
        wpe = pool.dtype.itemsize // 4
        out, rows, gather, words = [], [], [], []
        base = len(pool)
        nsign_words = 0
        # sign-entry words go after the gathered matrices: offsets are fixed up
        # once the gather length is known
        sign_recs = []
        form = []                     # gathered element: 0 plain, 1 (re, re), 2 (re, re) of packed, 3 (-im, im)
        diag_recs, dvals = [], []     # diagonal groups: pool elements appended after the sign words
        for ps in self.passes:
            begin = len(out)
            k, end = int(ps['op_begin']), int(ps['op_end'])
            while k < end:
                st = recs[k].copy()
                cnt = int(st['mat'])
                body = recs[self._group_order(k + 1, cnt)]
                new = []
                i = 0
                while i < cnt:
                    r = body[i]
                    c = int(r['code'])
                    if _layer_target(r) is not None:
                        run, seen = [i], {_layer_target(r)}
                        j = i + 1
                        while j < cnt:
                            t = _layer_target(body[j])
                            if t is None or t in seen:
                                break
                            run.append(j)
                            seen.add(t)
                            j += 1
                        if len(run) >= 2:
                            by_t = sorted(run, key=lambda x: _layer_target(body[x]))
                            real = all(_layer_real(body[x]) for x in run)
                            mask = sum(1 << t for t in seen if t < 4)
                            lmask = sum(1 << (t - 4) for t in seen if t >= 4)
                            g = r.copy()
                            g['code'] = (176 if real else 160) + mask
                            g['s1'] = lmask
                            g['mat'] = base + len(gather)
                            for x in by_t:
                                m0 = int(body[x]['mat'])
                                if real:
                                    gather.extend(range(m0, m0 + 4))
                                    form.extend([1] * 4)
                                elif _layer_target(body[x]) < 4:
                                    # register slot of a general layer: packed pairs per entry
                                    for e in range(4):
                                        gather.extend([m0 + e, m0 + e])
                                        form.extend([2, 3])
                                else:
                                    gather.extend(range(m0, m0 + 4))
                                    form.extend([0] * 4)
                            new.append(g)
                        else:
                            new.append(r.copy())
                        i = j
                    elif not c & 0x8000 and 58 <= c <= 107:
                        j = i
                        while j < cnt and j - i < 120:
                            cj = int(body[j]['code'])
                            if cj & 0x8000 or not 58 <= cj <= 107:
                                break
                            j += 1
                        run = body[i:j]
                        g = r.copy()
                        sign = (_sign_entries(run, pool)
                                if all(58 <= int(x['code']) <= 82 for x in run) else None)
                        if sign is not None:
                            ents, npairs = sign
                            g['code'] = 152
                            g['s0'] = npairs
                            sign_recs.append((g, nsign_words))
                            words.extend(ents)
                            nsign_words += len(ents)
                            # keep every group's words whole-element aligned
                            pad = (-nsign_words) % wpe
                            words.extend([0] * pad)
                            nsign_words += pad
                        else:
                            ents = _diag_group_plan(run, pool)
                            g['code'] = 154
                            g['s0'] = len(ents) // 5
                            diag_recs.append((g, len(dvals)))
                            gid = len(diag_recs) - 1
                            dvals.extend((e, gid) for e in ents)
                        new.append(g)
                        i = j
                    else:
                        new.append(r.copy())
                        i += 1
                st['mat'] = len(new)
                out.append(st)
                out.extend(new)
                k += 1 + cnt
            row = ps.copy()
            row['op_begin'], row['op_end'] = begin, len(out)
            rows.append(row)
        wbase = base + len(gather)
        for g, w0 in sign_recs:
            g['mat'] = wbase + w0 // wpe
        dbase = wbase + (len(words) + wpe - 1) // wpe
        for g, d0 in diag_recs:
            g['mat'] = dbase + d0
        ops = np.array(out, dtype=N.OP_DTYPE) if out else np.zeros(0, N.OP_DTYPE)
        passes = np.array(rows, dtype=self.passes.dtype) if rows else np.zeros(0, self.passes.dtype)
        dv = None
        if dvals:
            # vectorised recipe of the diagonal-group elements (values come from the pool per call)
            kind = np.array([{'raw': 0, 'fac': 1, 'gph': 2, 'raw1': 3}[e[0]] for e, _ in dvals], np.int8)
            word = np.array([e[1] if e[0] == 'raw' else 0 for e, _ in dvals], np.uint64)
            src = np.array([e[1] + e[2] if e[0] == 'fac' else 0 for e, _ in dvals], np.int64)
            m0 = np.array([e[1] if e[0] == 'fac' else 0 for e, _ in dvals], np.int64)
            norm = np.array([e[0] == 'fac' and e[3] for e, _ in dvals], bool)
            grp = np.array([gid for _, gid in dvals], np.int64)
            raw = np.zeros((len(dvals), pool.dtype.itemsize // 4), np.uint32)
            raw[:, 0] = word.astype(np.uint32)
            dv = dict(kind=kind, raw=np.frombuffer(raw.tobytes(), dtype=pool.dtype).copy(), src=src, m0=m0,
                      norm=norm, grp=grp, ngroups=len(diag_recs))
        gidx = np.array(gather, np.int64)
        return ops, passes, (gidx, np.array(form, np.int8)), (np.array(words, np.uint32) if words else None), dv

    def _group_order(self, first: int, cnt: int) -> np.ndarray:
        """Record indices of one stage, reordered (respecting every non-commuting
        pair) so that mergeable ops sit next to each other: uncontrolled
        general / real 2x2 ops on distinct register slots, and +-1 diagonals."""
        idx = list(range(first, first + cnt))
        if cnt < 3:
            return np.array(idx, np.int64)
        if not hasattr(self, '_fop_of'):
            self._fop_of = {ri: fi for ri, fi in self.op_slots}
        codes = [int(c) for c in self.ops['code'][first:first + cnt]]

        recs = self.ops[first:first + cnt]
        tgt = [_layer_target(r) for r in recs]

        def cls(j):
            if tgt[j] is not None:
                return 'r'
            c = codes[j]
            if not c & 0x8000 and 58 <= c <= 107:
                return 's'
            return 'o'
        kinds = [cls(j) for j in range(cnt)]
        fo = [self.fops[self._fop_of[i]] for i in idx]
        preds = []
        for j in range(cnt):
            pj = set()
            for i in range(j):
                if (fo[i].nd & (fo[j].nd | fo[j].d)) or (fo[i].d & fo[j].nd):
                    pj.add(i)
            preds.append(pj)
        done, order = set(), []
        cur, slots = None, set()
        while len(order) < cnt:
            ready = [j for j in range(cnt) if j not in done and preds[j] <= done]
            pick = None
            if cur == 'r':
                pick = next((j for j in ready if kinds[j] == 'r' and tgt[j] not in slots), None)
            elif cur == 's':
                pick = next((j for j in ready if kinds[j] == 's'), None)
            if pick is None:
                # open the next group with the class that has the most ready ops
                # (ties: diagonals, then layer gates, then the rest)
                slots = set()
                best = None
                for want in ('s', 'r', 'o'):
                    cand = [j for j in ready if kinds[j] == want]
                    if want == 'r':
                        cand = list({tgt[j]: j for j in reversed(cand)}.values())
                    if cand and (best is None or len(cand) > best[0]):
                        best = (len(cand), min(cand))
                pick = best[1]
                cur = kinds[pick]
            if cur == 'r':
                slots.add(tgt[pick])
            done.add(pick)
            order.append(pick)
        return np.array([idx[j] for j in order], np.int64)

DG_SIGN, DG_THREAD, DG_SLOT_A, DG_SLOT_B, DG_TWO = 0, 1, 2, 3, 4


_SLOT_MASKS = (0xAAAA, 0xCCCC, 0xF0F0, 0xFF00)


def _sign_entries(run, pool) -> list:
    """uint32 words of a sign group (dispatch code 152), or None when a mask is
    not affine in the register bits (the caller then emits a diagonal group).

    The group's negation of register amplitude j of a thread is a parity
    (XOR) of terms, each sign diagonal contributing its algebraic normal form
    over the thread-fixed bits it reads.  The record is 64-bit words:
    q[0] the 16-bit mask common to every thread; q[1] the global bits whose
    parity negates all 16 amplitudes; q[2 + S] the global bits whose parity
    negates the amplitudes with register bit S set; then, per distance d of a
    product term, q = d and the mask M of the lower bits i: the parity of
    bit(i) * bit(i + d) over i in M negates all 16.  Returns the words and the
    number of (d, M) pairs."""
    const_mask = 0
    lin = [0] * 5                 # all, slot 0..3
    prod = {}
    j = np.arange(16)
    for r in run:
        m0 = int(r['mat'])
        d = pool[m0:m0 + 4]
        pattern = [bool(d[k].real < 0) for k in range(4)]
        sels = []
        for gkey, skey in (('ga', 'sa'), ('gb', 'sb')):
            sl, gb = int(r[skey]), int(r[gkey])
            sels.append(('slot', sl) if sl >= 0 else ('none', 0) if gb == 0xFF else ('thread', gb))
        tbits = [v for k, v in sels if k == 'thread']
        masks = []
        for idx in range(1 << len(tbits)):
            bits = []
            t = 0
            for k, v in sels:
                if k == 'slot':
                    bits.append((j >> v) & 1)
                elif k == 'thread':
                    bits.append(np.full(16, (idx >> t) & 1))
                    t += 1
                else:
                    bits.append(np.zeros(16, np.int64))
            neg = np.array([pattern[x] for x in (bits[0] + 2 * bits[1])])
            masks.append(int(np.sum(neg.astype(np.int64) << j)))
        const_mask ^= masks[0]
        if len(tbits) >= 1:
            # linear term of the first thread bit (at the second one == 0)
            w = masks[1] ^ masks[0]
            if not _add_linear(lin, tbits[0], w):
                return None
        if len(tbits) == 2:
            w = masks[2] ^ masks[0]
            if not _add_linear(lin, tbits[1], w):
                return None
            w = masks[0] ^ masks[1] ^ masks[2] ^ masks[3]
            if w not in (0, 0xFFFF):
                return None
            if w:
                lo, hi = sorted(tbits)
                if lo == hi:      # bit(i)^2 == bit(i): a linear term
                    lin[0] ^= 1 << lo
                else:
                    prod[hi - lo] = prod.get(hi - lo, 0) ^ (1 << lo)
    q = [const_mask, *lin]
    pairs = [(dd, m) for dd, m in sorted(prod.items()) if m]
    for dd, m in pairs:
        q += [dd, m]
    out = []
    for v in q:
        out += [v & 0xFFFFFFFF, v >> 32]
    return out, len(pairs)


def _add_linear(lin, bit, w) -> bool:
    """Add the linear term bit * w (w a 16-bit mask over the register
    amplitudes) to `lin`; False if w is not affine in the register bits."""
    if w == 0:
        return True
    c = w & 1                     # value at j == 0: the all-amplitudes part
    rest = w ^ (0xFFFF if c else 0)
    if c:
        lin[0] ^= 1 << bit
    for s, sm in enumerate(_SLOT_MASKS):
        if (rest >> (1 << s)) & 1:
            rest ^= sm
            lin[1 + s] ^= 1 << bit
    return rest == 0


def _diag_group_values(dv, pool) -> np.ndarray:
    """Pool elements of every diagonal group for the current pool values."""
    out = dv['raw'].copy()
    fac = dv['kind'] == 1
    vals = pool[dv['src'][fac]].astype(np.complex128)
    d0 = pool[dv['m0'][fac]].astype(np.complex128)
    nrm = dv['norm'][fac]
    vals = np.where(nrm, vals / np.where(nrm, d0, 1.0), vals)
    out[fac] = vals
    # global phase per group: the product of d[0] of its normalised entries (once per entry)
    first = fac.copy()
    first[np.nonzero(fac)[0]] = (dv['src'][fac] == dv['m0'][fac]) & nrm
    gph = np.ones(dv['ngroups'], np.complex128)
    np.multiply.at(gph, dv['grp'][first], pool[dv['m0'][first]].astype(np.complex128))
    g = dv['kind'] == 2
    out[g] = gph[dv['grp'][g]]
    out[dv['kind'] == 3] = 1.0
    return out


def _diag_group_plan(run, pool) -> list:
    """Element specs of a diagonal group (dispatch code 154): 5 pool elements
    per entry, a raw header word (a | b << 8 | kind << 16 | sign pattern << 20)
    then the four factors d[bit(a) + 2 bit(b)].  Entries touching a register
    slot are normalised so that d[0] == 1 (the factor removed is a global phase,
    carried by one extra thread-only entry), which lets the kernel apply them to
    the amplitudes whose slot bits are set only.  Records whose code says +-1
    become sign entries.  The structure depends on the records' codes only; the
    factor values are read from the pool on every call (``_diag_group_values``).

    Specs: ('raw', word) | ('fac', m0, k, normalise) | ('gph',)."""
    def sel(r, gkey, skey):
        sl = int(r[skey])
        if sl >= 0:
            return sl
        g = int(r[gkey])
        return 0xFF if g == 0xFF else 0x40 | g

    out, any_norm = [], False
    for r in run:
        a, b = sel(r, 'ga', 'sa'), sel(r, 'gb', 'sb')
        m0 = int(r['mat'])
        if 58 <= int(r['code']) <= 82:
            d = pool[m0:m0 + 4]
            pattern = sum(1 << k for k in range(4) if d[k].real < 0)
            if pattern:
                out += [('raw', a | b << 8 | DG_SIGN << 16 | pattern << 20)] + [('raw', 0)] * 4
            continue
        ra, rb = a < 4, b < 4
        kind = DG_THREAD if not (ra or rb) else DG_TWO if (ra and rb) else (DG_SLOT_A if ra else DG_SLOT_B)
        norm = kind != DG_THREAD
        any_norm |= norm
        out += [('raw', a | b << 8 | kind << 16)] + [('fac', m0, k, norm) for k in range(4)]
    if any_norm:
        out += [('raw', 0xFF | 0xFF << 8 | DG_THREAD << 16)] + [('gph',)] * 4
    if not out:
        out = [('raw', 0xFF | 0xFF << 8 | DG_THREAD << 16)] + [('raw1',)] * 4
    return out


def _layer_target(r):
    """Target of an op that can join a layer op (uncontrolled general / real
    2x2 without a thread predicate): register slot 0..3, or 4 + lane bit; else None."""
    c = int(r['code'])
    if c & 0x8000:
        return None
    if 1 <= c <= 20 and (c - 1) % 5 in (0, 1):
        return (c - 1) // 5
    if c in (53, 54):
        return 4 + int(r['s0']) - 16
    return None


def _layer_real(r) -> bool:
    c = int(r['code'])
    return c == 54 or (1 <= c <= 20 and (c - 1) % 5 == 1)


def _clean_batch(m: np.ndarray) -> np.ndarray:
    """Zero real / imaginary parts below 1e-15 x max(1, max |entry|) per row."""
    scale = np.maximum(1.0, np.abs(m).max(axis=1, keepdims=True))
    re, im = m.real.copy(), m.imag.copy()
    re[np.abs(re) < 1e-15 * scale] = 0.0
    im[np.abs(im) < 1e-15 * scale] = 0.0
    return re + 1j * im


def build(target: Sequence[tuple], n: int, kmax: int, slots=None, merge_1q: bool = True):
    """Lower + fuse + schedule + pack a transpiled circuit."""
    ir = lower(target, n, slots)
    fops = fuse_1q(ir, merge=merge_1q)
    if n < MIN_FUSED_QUBITS:
        return ir, fops, None
    return ir, fops, Packed(n, fops, schedule(fops, n, kmax))
