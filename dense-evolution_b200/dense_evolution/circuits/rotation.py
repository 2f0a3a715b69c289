"""Rotation passes: the complex64 forward path of the fused circuit engine.

The general fused pass (``fusion.py`` + ``jit.py``) applies every fused
single-qubit matrix as a complex 2x2: eight FP32 multiply-adds per amplitude
and gate, plus warp shuffles for the five lane bits.  At 30 qubits that makes
the pass bound by the FP32 pipe and instruction issue at about a quarter of
the HBM roofline.  This module plans the same circuits in a cheaper form.

**Rewrite.**  Every gate of a transpiled circuit becomes one of three
primitives on index bits (qubit q is bit n-1-q), plus one global factor:

* ``ROT(b)`` -- a real rotation [[c, -s], [s, c]] on bit b: the middle factor
  of the ZYZ form U = e^{ig} Rz(a) Ry(b) Rz(c) of a fused run of
  single-qubit gates.  On the device it runs in tangent form,
  x0 -= t x1, x1 += t x0 with t = s / c, which is ONE packed FP32
  instruction (fma.rn.f32x2) per amplitude; the cosines are collected into
  a per-pass scale that a later multiply applies.  The tangent form keeps
  FP32's relative accuracy for any finite t: each output is one fused
  multiply-add, rounded once, and the pass-end factor 1/prod(1/c) restores
  the scale exactly up to rounding.  Where |t| > TMAX (cos = 0, as in an X
  gate) or the pending scale would pass SCALE_LIMIT, the general form
  c x0 - s x1 (two instructions) is used instead.  That choice is made per
  call from the angles: a pass has a tangent-only kernel for the calls that
  need no general form and a kernel with a run-time form flag per rotation
  for the rest, so new angles never change the plan.
* ``PH(b)`` -- a diagonal diag(1, e^{ia}) on bit b: the outer ZYZ factors
  and every diagonal single-qubit gate.  Phases commute with every other
  diagonal, so the phases of a bit are merged and moved to just before the
  next rotation of that bit, where the bit is a register slot.
* ``D2(a, b)`` -- a two-bit diagonal (cz, cp, crz).  Controlled X and Y
  become H.CZ.H and S.H.CZ.H.Sdg on the target (H = Ry(pi/2) Z), so every
  circuit of the API's gate set lowers to these primitives.

**Passes.**  A pass keeps the tile shape of the fused kernels (2^K
amplitudes: the L low index bits plus K-L chosen high bits, streamed by
bulk copies), but applies all of its gates on register slots: a stage holds
RB = 5 tile bits in registers (32 amplitudes per thread, 128 threads per
4096-amplitude tile), and EVERY tile bit, the five lowest included, can be a
register slot of some stage -- no warp shuffles.  Between stages the tile
sits in shared memory in a padded layout (one spare amplitude per 16) that
keeps the 64-bit accesses free of bank conflicts for the register sets the
stage scheduler allows.  Inside a stage, the diagonals between two layers of
rotations form one *diagonal group*: one complex multiply per amplitude by a
table over the register slots (phases, register-register cz/cp, the pending
tangent scale), plus sign flips for cz with thread-fixed bits.

The pass scheduler picks the tile's high bits greedily to maximise the
rotations a pass can take (the dependency closure of the circuit order); the
stage scheduler picks each stage's register set the same way among the sets
whose shared-memory accesses are conflict-free.  Kernels are generated per
pass as CUDA source with every structural field a constant and compiled by
NVRTC for sm_100a (``desv_rot_load``); the per-call values (tangents, tables,
scales) travel as the kernel's by-value parameter block, so they sit in the
constant bank and are read without load instructions.
"""
from __future__ import annotations

import hashlib
import itertools
import os
import threading
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import fusion
from .gates import GATES

# register bits per stage: 5 (32 amplitudes per thread, 128 threads per 4096-amplitude tile) or 6
# (64 amplitudes, 64 threads); DESV_ROT_RB overrides the default (tuning)
RB = int(os.environ.get('DESV_ROT_RB', '5'))
if RB not in (5, 6):
    raise ValueError('DESV_ROT_RB must be 5 or 6')
LOW_FIXED = 5          # index bits 0..LOW_FIXED-1 are in every tile (contiguous bulk-copy runs)
TMAX = 2.0 ** 20       # tangent form while |tan| <= TMAX (FP32 keeps its relative accuracy; see materialize)
# pending tangent scale above which rotations switch to the general form.  Every tangent rotation
# scales ALL amplitudes by the same 1/c, and a pass starts from |amp| <= 1, so inside a pass
# |amp| <= SCALE_LIMIT and each fma result is at most TMAX * SCALE_LIMIT = 2^120 < FP32's 2^128.
# The product of up to MAX_ROTS_PER_PASS random 1/|cos| is heavy-tailed: at 2^60 about one pass in
# a few dozen of a random-angle circuit needed the general kernel; at 2^100 that is rare.
SCALE_LIMIT = 2.0 ** 100
MAX_ROTS_PER_PASS = 32  # measured on the 30-qubit, 40-layer brick circuit: 24 -> 246 ms, 32 -> 233, 48 -> 236
PAD_SHIFT = 4          # padded stage layout: physical = i + (i >> 4)
# ring slots per CTA, measured on the 30-qubit, 40-layer brick circuit: 1 -> four CTAs (16 warps)
# per SM, 207 ms (the next tile loads while the last stage computes and stores); 2 -> three CTAs,
# 233 ms; 3 -> two CTAs, 274 ms
NBUF = 1
# register bound of the kernel per ring depth (shared memory allows as many); with 6 register
# slots a CTA is half as wide and holds twice the amplitudes per thread
CTAS_PER_SM = {1: 4, 2: 3, 3: 2} if RB == 5 else {1: 5, 2: 4, 3: 3}


def tuning() -> Tuple[int, int]:
    """(rotations per pass at most, ring slots): MAX_ROTS_PER_PASS and NBUF,
    overridden by DESV_ROT_MAX_ROTS / DESV_ROT_NBUF (for tuning sweeps)."""
    cap = int(os.environ.get('DESV_ROT_MAX_ROTS', MAX_ROTS_PER_PASS))
    nb = int(os.environ.get('DESV_ROT_NBUF', NBUF))
    if cap < 1 or nb not in (1, 2, 3):
        raise ValueError('DESV_ROT_MAX_ROTS must be >= 1 and DESV_ROT_NBUF 1, 2 or 3')
    return cap, nb

_H = GATES['h']
_S = GATES['s']
_SDG = GATES['sdg']
_CZ = np.array([1, 1, 1, -1], dtype=np.complex128)


# ---------------------------------------------------------------------------
# lowering to primitives
# ---------------------------------------------------------------------------

@dataclass
class UOp:
    """A fused run of uncontrolled single-qubit gates on one bit."""
    b: int
    gates: List[fusion.IRGate] = field(default_factory=list)
    diag: bool = True            # every gate of the run is diagonal (structurally)


@dataclass
class Prim:
    """A primitive of the rotation program.

    kind 'rot': ROT on bit b, values from UOp u.
    kind 'ph' : PH on bit b, the product of phase factors `factors`
                ((u, 'pre' | 'post' | 'diag') references).
    kind 'd2' : D2 on bits (b, b2) with factor index bit(b) + 2 bit(b2); `gate`
                is the IR gate (values), sign=True for a structural cz.
    """
    kind: str
    b: int
    b2: int = -1
    u: int = -1
    factors: List[Tuple[int, str]] = field(default_factory=list)
    gate: Optional[fusion.IRGate] = None
    sign: bool = False


def _is_const_diag(g: fusion.IRGate) -> bool:
    if g.kind == 'scalar':
        return True
    if g.const is not None:
        m = g.const
        return m.shape == (2, 2) and m[0, 1] == 0 and m[1, 0] == 0
    return g.name in ('rz', 'p', 'u1', 'phase', 'gphase')


def _rewrite_controls(ir: Sequence[fusion.IRGate]) -> Optional[List[fusion.IRGate]]:
    """cx / cy as single-qubit gates around a cz; None when a controlled gate of
    another kind (or with several controls) is present."""
    out: List[fusion.IRGate] = []
    for g in ir:
        if g.kind == 'm1' and g.cbits:
            if len(g.cbits) != 1 or g.cvals[0] != 1 or g.const is None or g.name not in ('cx', 'cy'):
                return None
            c, t = g.cbits[0], g.t
            h = fusion.IRGate('m1', 'h', t=t, const=_H)
            cz = fusion.IRGate('d2', 'cz', t=c, t2=t, const=_CZ)
            if g.name == 'cx':
                out += [h, cz, fusion.IRGate('m1', 'h', t=t, const=_H)]
            else:   # CY = S . CX . Sdg (Sdg applied first)
                out += [fusion.IRGate('m1', 'sdg', t=t, const=_SDG), h, cz,
                        fusion.IRGate('m1', 'h', t=t, const=_H), fusion.IRGate('m1', 's', t=t, const=_S)]
        elif g.kind == 'm2':
            return None
        else:
            out.append(g)
    return out


def lowered_gates(target: Sequence[tuple], n: int, slots=None) -> Optional[List[fusion.IRGate]]:
    """IR gates of a transpiled circuit with cx / cy rewritten around cz, or
    None when the circuit holds a gate this path does not lower."""
    ir = fusion.lower(target, n, slots)
    return _rewrite_controls(ir)


def lower_program(target: Sequence[tuple], n: int, slots=None, ir=None):
    """(uops, prims, scalars, order) of a transpiled circuit, or None when it
    holds a gate this path does not lower (the general fused path runs it
    then).  order[i] says where IR gate i went: ('u', run, position),
    ('d', prim index) or ('s', scalar index), so that a circuit of the same
    structure can be bound to the plan gate by gate."""
    if ir is None:
        ir = lowered_gates(target, n, slots)
    if ir is None:
        return None
    uops: List[UOp] = []
    seq: List[Tuple[str, object]] = []     # ('u', uop index) | ('d2', IRGate), in circuit order
    open_: Dict[int, int] = {}             # bit -> index of the run under construction
    scalars: List[fusion.IRGate] = []
    order: List[tuple] = []
    d2_pos: List[int] = []                 # IR position of every d2, in order
    for gi_, g in enumerate(ir):
        if g.kind == 'scalar':
            order.append(('s', len(scalars)))
            scalars.append(g)
            continue
        if g.kind == 'm1':
            u = open_.get(g.t)
            if u is None:
                u = len(uops)
                uops.append(UOp(g.t))
                open_[g.t] = u
                seq.append(('u', u))
            order.append(('u', u, len(uops[u].gates)))
            uops[u].gates.append(g)
            uops[u].diag &= _is_const_diag(g)
            continue
        # d2: ends the open runs on both of its bits
        for b in (g.t, g.t2):
            open_.pop(b, None)
        order.append(None)           # filled below with the prim index
        d2_pos.append(gi_)
        seq.append(('d2', g))
    # phases move forward to the next rotation of their bit (they commute with
    # every diagonal on the way); a rotation's own pre-phase joins them
    prims: List[Prim] = []
    pending: Dict[int, List[Tuple[int, str]]] = {}
    nd2 = 0
    for kind, x in seq:
        if kind == 'd2':
            g = x
            order[d2_pos[nd2]] = ('d', len(prims))
            nd2 += 1
            prims.append(Prim('d2', g.t, g.t2, gate=g, sign=(g.const is not None and np.array_equal(g.const, _CZ))))
            continue
        u = uops[x]
        if u.diag:
            pending.setdefault(u.b, []).append((x, 'diag'))
            continue
        f = pending.pop(u.b, []) + [(x, 'pre')]
        prims.append(Prim('ph', u.b, factors=f))
        prims.append(Prim('rot', u.b, u=x))
        pending[u.b] = [(x, 'post')]
    for b in sorted(pending):
        prims.append(Prim('ph', b, factors=pending[b]))
    return uops, prims, scalars, order


# ---------------------------------------------------------------------------
# scheduling
# ---------------------------------------------------------------------------

@dataclass
class Unit:
    """A scheduling unit: a rotation with its pre-phase (nd = its bit), or a
    lone diagonal (a d2 or a trailing phase; d = its bits)."""
    rot: int            # prim index of the rotation, -1 for a diagonal unit
    ph: int             # prim index of the phase before the rotation / the lone phase, -1 if none
    d2: int             # prim index of the d2, -1 if none
    nd: int
    d: int
    bit: int = -1


def make_units(prims: List[Prim]) -> List[Unit]:
    units: List[Unit] = []
    i = 0
    while i < len(prims):
        p = prims[i]
        if p.kind == 'ph' and i + 1 < len(prims) and prims[i + 1].kind == 'rot' and prims[i + 1].b == p.b:
            units.append(Unit(i + 1, i, -1, 1 << p.b, 0, p.b))
            i += 2
            continue
        if p.kind == 'rot':
            units.append(Unit(i, -1, -1, 1 << p.b, 0, p.b))
        elif p.kind == 'ph':
            units.append(Unit(-1, i, -1, 0, 1 << p.b))
        else:
            units.append(Unit(-1, -1, i, 0, (1 << p.b) | (1 << p.b2)))
        i += 1
    return units


def _closure(units: Sequence[Unit], ids: Sequence[int], allowed: int, cap: int, count_only: bool = False):
    """Greedy closure in circuit order: a rotation unit is taken when its bit is
    in `allowed` (and fewer than `cap` rotations were taken), a diagonal unit
    always; a unit that is not taken blocks every later unit that does not
    commute with it.  Returns (taken rotations, taken ids, remaining ids)."""
    b_any = b_d = 0
    nrot = 0
    taken, rest = [], []
    full = allowed
    for k, i in enumerate(ids):
        u = units[i]
        if ((u.nd | u.d) & b_any) or (u.nd & b_d) or (u.nd and (not (u.nd & allowed) or nrot >= cap)):
            rest.append(i)
            b_any |= u.nd
            b_d |= u.d
            if count_only and (nrot >= cap or (b_any & full) == full):
                return nrot, None, None
            continue
        taken.append(i)
        if u.nd:
            nrot += 1
    return nrot, taken, rest


@dataclass
class Group:
    """A diagonal group of a stage: the prims it applies and how each one is
    applied against the stage's register slots.

    table_items: (prim, slot a, slot b or -1) factors over register slots,
                 multiplied into one table of 2^|reg_mask| complex entries;
    signs_reg:   cz between two slots without a table (compile-time negations);
    signs_mixed: cz between slot s and the thread-fixed global bit x;
    signs_thread: cz between two thread-fixed global bits;
    f_items:     per-thread factors: ('ph', prim, x, off) -> x ? e : 1,
                 ('d2', prim, x, y, off) -> d[x + 2 y];
    mixed_items: (prim, slot, x, off): a non-sign two-bit diagonal between slot
                 s and thread-fixed bit x: amplitudes get f[x][bit s] (4 values).
    """
    prims: List[int]
    reg_mask: int = 0
    table_items: List[Tuple[int, int, int]] = field(default_factory=list)
    t_off: int = -1
    signs_reg: List[Tuple[int, int]] = field(default_factory=list)
    signs_mixed: List[Tuple[int, int]] = field(default_factory=list)
    signs_thread: List[Tuple[int, int]] = field(default_factory=list)
    f_items: List[tuple] = field(default_factory=list)
    mixed_items: List[Tuple[int, int, int, int]] = field(default_factory=list)

    @property
    def has_table(self) -> bool:
        return bool(self.table_items)

    @property
    def absorbs(self) -> bool:
        """Groups leave the pending tangent scale to the pass-end factor, so a
        table entry for register index 0 is always 1 and only the amplitudes
        with a non-zero index into the table are multiplied."""
        return False


@dataclass
class Stage:
    regs: Tuple[int, ...]                        # tile-local bits of register slots 0..RB-1 (ascending)
    items: List[Tuple[str, object]] = field(default_factory=list)   # ('rot', (prim, slot, off)) | ('grp', Group)


@dataclass
class RotPass:
    K: int
    L: int
    high: List[int]
    stages: List[Stage]
    n_floats: int = 0
    end_scale_off: int = -1      # parameter offset of the pass-end scale (2 floats: re, im), -1 if none
    end_complex: bool = False    # the end factor carries the circuit's global phase (last pass)
    rot_offs: List[Tuple[int, int]] = field(default_factory=list)   # (prim, offset) in program order
    order: List[Tuple[str, object]] = field(default_factory=list)   # program order of rots / groups / end


def _bank_ok(regs: Sequence[int], K: int, padded: bool) -> bool:
    """No bank conflict for the 64-bit shared-memory accesses of a stage: the 16
    lanes of a half-warp (the 4 lowest non-register tile bits) hit 16 distinct
    8-byte bank pairs."""
    lanes = [b for b in range(K) if b not in regs][:4]
    res = []
    for b in lanes:
        if b < 4:
            res.append(1 << b)
        elif padded and b < 8:
            res.append(1 << (b - 4))
        else:
            res.append(0)
    return sorted(res) == [1, 2, 4, 8]


def _candidate_regs(K: int, first: bool, last: bool) -> List[Tuple[int, ...]]:
    """Register sets a stage may use: conflict-free loads and stores (the first
    stage reads the bulk-copied natural layout, later stages the padded one), and
    for the last stage a store whose half-warps write 128 contiguous bytes."""
    out = []
    for regs in itertools.combinations(range(K), RB):
        if (first or last) and any(b < 4 for b in regs):
            continue
        if not _bank_ok(regs, K, padded=True):
            continue
        if first and not _bank_ok(regs, K, padded=False):
            continue
        out.append(regs)
    return out


class RotationPlan:
    """Passes, stages and groups of one circuit structure, plus the value program."""

    def __init__(self, target: Sequence[tuple], n: int, kmax: int = 12, slots=None,
                 max_rots: Optional[int] = None, low_fixed: int = LOW_FIXED):
        low = lower_program(target, n, slots)
        if low is None:
            raise ValueError('rotation passes: the circuit holds a gate this path does not lower')
        self.n = n
        self.uops, self.prims, self.scalars, self.order = low
        self.units = make_units(self.prims)
        self.K = min(kmax, n)
        if self.K < RB + 4 or n < self.K:
            raise ValueError('rotation passes need at least 9 qubits')
        cap, self.nbuf = tuning()
        self.max_rots = cap if max_rots is None else max_rots
        self.low_fixed = min(low_fixed, self.K)
        self.passes: List[RotPass] = []
        self._schedule()
        self._layout()

    # ------------------------------------------------------------ passes
    def _schedule(self):
        n, K = self.n, self.K
        remaining = list(range(len(self.units)))
        fixed = (1 << self.low_fixed) - 1
        while remaining:
            tile = fixed
            free = K - self.low_fixed
            # bits of rotations that are still to come, in the order they first appear
            want = []
            seen = 0
            for i in remaining:
                u = self.units[i]
                if u.nd and not (u.nd & (seen | tile)):
                    want.append(u.bit)
                    seen |= u.nd
            for _ in range(free):
                best, best_b = -1, None
                for b in want:
                    if (tile >> b) & 1:
                        continue
                    c, _, _ = _closure(self.units, remaining, tile | (1 << b), self.max_rots, count_only=True)
                    if c > best:
                        best, best_b = c, b
                if best_b is None:
                    break
                tile |= 1 << best_b
            # fill up to K bits (the tile always has exactly K bits)
            b = 0
            while bin(tile).count('1') < K:
                if not (tile >> b) & 1:
                    tile |= 1 << b
                b += 1
            nrot, taken, rest = _closure(self.units, remaining, tile, self.max_rots)
            if not taken:
                raise RuntimeError('rotation passes: no schedulable unit (internal error)')
            remaining = rest
            L = 0
            while (tile >> L) & 1:
                L += 1
            high = [b for b in range(L, n) if (tile >> b) & 1]
            self.passes.append(self._stages(K, L, high, taken))
        if not self.passes:
            # no primitive at all (global phases or identities only): one pass
            # whose end factor applies the circuit's global factor
            L = K
            self.passes.append(RotPass(K, L, [], [Stage(tuple(_candidate_regs(K, True, True)[0]))]))

    def _stages(self, K: int, L: int, high: List[int], ids: List[int]) -> RotPass:
        tl = {b: b for b in range(L)}
        for i, h in enumerate(high):
            tl[h] = L + i
        remaining = list(ids)
        stages: List[Stage] = []
        first = True
        while remaining:
            nrot_left = sum(1 for i in remaining if self.units[i].nd)
            best = None
            finishing = None     # a non-final register set that would take everything
            for last in ((True, False) if nrot_left else (True,)):
                for regs in _candidate_regs(K, first, last):
                    allowed = 0
                    for p in regs:
                        allowed |= 1 << self._global_of(p, L, high)
                    c, taken, rest = _closure(self.units, remaining, allowed, 1 << 30)
                    if last and rest:
                        continue
                    if not last and not rest:
                        # it would end the pass with a register set the final
                        # (global-store) stage may not use
                        if finishing is None:
                            finishing = (regs, taken)
                        continue
                    key = (c, last)
                    if best is None or key > best[0]:
                        best = (key, regs, taken, rest)
                if best is not None and best[0][1]:
                    break        # one stage finishes the pass
            if finishing is not None and (best is None or best[0][0] == 0):
                # finish with that set, then an item-free final stage for the store
                regs, taken = finishing
                stages.append(self._stage_items(regs, taken, L, high))
                stages.append(Stage(tuple(_candidate_regs(K, False, True)[0])))
                break
            if best is None:
                raise RuntimeError('rotation passes: no register set for a stage (internal error)')
            _, regs, taken, rest = best
            if not taken and first:
                # the pass's next rotations are all on tile bits 0..3, which the
                # first stage cannot hold (its loads read the natural layout):
                # a stage without items moves the tile into the padded layout
                stages.append(Stage(tuple(_candidate_regs(K, True, False)[0])))
                first = False
                continue
            if not taken:
                raise RuntimeError('rotation passes: empty stage (internal error)')
            stages.append(self._stage_items(regs, taken, L, high))
            remaining = rest
            first = False
        return RotPass(K, L, high, stages)

    @staticmethod
    def _global_of(p: int, L: int, high: List[int]) -> int:
        return p if p < L else high[p - L]

    def _stage_items(self, regs, ids, L, high) -> Stage:
        """ASAP layering of a stage: [group][rotations][group][rotations]..."""
        slot_of = {self._global_of(p, L, high): s for s, p in enumerate(regs)}
        st = Stage(tuple(regs))
        # prims of the stage in circuit order, with their bit masks
        seq = []
        for i in ids:
            u = self.units[i]
            if u.ph >= 0:
                seq.append(u.ph)
            if u.rot >= 0:
                seq.append(u.rot)
            if u.d2 >= 0:
                seq.append(u.d2)
        done = [False] * len(seq)
        while not all(done):
            # ready diagonals: no earlier pending rotation on one of their bits
            blocked = 0
            grp = []
            for k, pi in enumerate(seq):
                if done[k]:
                    continue
                p = self.prims[pi]
                bits = (1 << p.b) | ((1 << p.b2) if p.kind == 'd2' else 0)
                if p.kind == 'rot':
                    blocked |= bits
                    continue
                if bits & blocked:
                    blocked |= bits
                    continue
                grp.append(pi)
                done[k] = True
            if grp:
                st.items.append(('grp', Group(grp)))
            blocked = 0
            rots = []
            for k, pi in enumerate(seq):
                if done[k]:
                    continue
                p = self.prims[pi]
                bits = (1 << p.b) | ((1 << p.b2) if p.kind == 'd2' else 0)
                if p.kind != 'rot' or bits & blocked:
                    blocked |= bits
                    continue
                rots.append(pi)
                done[k] = True
                blocked |= bits
            for pi in rots:
                st.items.append(('rot', (pi, slot_of[self.prims[pi].b], -1)))
            if not grp and not rots:
                raise RuntimeError('rotation passes: stage layering stalled (internal error)')
        # classify every group's factors against this stage's register slots
        for kind, x in st.items:
            if kind == 'grp':
                self._classify_group(x, slot_of)
        return st

    def _classify_group(self, g: Group, slot_of: Dict[int, int]):
        for pi in g.prims:
            p = self.prims[pi]
            if p.kind == 'ph':
                if p.b in slot_of:
                    g.table_items.append((pi, slot_of[p.b], -1))
                else:
                    g.f_items.append(('ph', pi, p.b, -1))
                continue
            a, b = p.b, p.b2
            ra, rb = a in slot_of, b in slot_of
            if p.sign:
                if ra and rb:
                    g.signs_reg.append((slot_of[a], slot_of[b]))
                elif ra:
                    g.signs_mixed.append((slot_of[a], b))
                elif rb:
                    g.signs_mixed.append((slot_of[b], a))
                else:
                    g.signs_thread.append((a, b))
                continue
            if ra and rb:
                g.table_items.append((pi, slot_of[a], slot_of[b]))
            elif ra or rb:
                g.mixed_items.append((pi, slot_of[a] if ra else slot_of[b], b if ra else a, -1))
            else:
                g.f_items.append(('d2', pi, a, b, -1))
        if g.table_items:
            # register-register signs fold into the table
            for sa, sb in g.signs_reg:
                g.table_items.append((-1, sa, sb))
            g.signs_reg = []
            for _, sa, sb in g.table_items:
                g.reg_mask |= 1 << sa
                if sb >= 0:
                    g.reg_mask |= 1 << sb

    # ------------------------------------------------------------ parameter layout
    def _layout(self):
        for pi_, ps in enumerate(self.passes):
            off = 0
            order = []
            last_table = -1
            for si, st in enumerate(ps.stages):
                for k, (kind, x) in enumerate(st.items):
                    if kind == 'rot':
                        pi, s, _ = x
                        st.items[k] = ('rot', (pi, s, off))
                        ps.rot_offs.append((pi, off))
                        order.append(('rot', (pi, off)))
                        off += 4
                    else:
                        g = x
                        if g.has_table:
                            g.t_off = off
                            off += 2 << bin(g.reg_mask).count('1')
                            last_table = len(order)
                        fi = []
                        for it in g.f_items:
                            fi.append(it[:-1] + (off,))
                            off += 2 if it[0] == 'ph' else 8
                        g.f_items = fi
                        mi = []
                        for (pi, s_, gb, _) in g.mixed_items:
                            mi.append((pi, s_, gb, off))
                            off += 8
                        g.mixed_items = mi
                        order.append(('grp', g))
            is_last = pi_ == len(self.passes) - 1
            if any(k == 'rot' for k, _ in order) or is_last:
                ps.end_scale_off = off
                ps.end_complex = is_last
                off += 2
                order.append(('end', ps.end_scale_off))
            ps.order = order
            ps.n_floats = max(off, 4)

    # ------------------------------------------------------------ statistics
    def stats(self) -> dict:
        st = [len(p.stages) for p in self.passes]
        rots = [sum(1 for k, _ in p.order if k == 'rot') for p in self.passes]
        grps = [sum(1 for k, _ in p.order if k == 'grp') for p in self.passes]
        return {'passes': len(self.passes), 'stages': sum(st), 'rots': sum(rots), 'groups': sum(grps),
                'per_pass': list(zip(rots, st, grps))}

    # ------------------------------------------------------------ values
    def bind(self, ir: Sequence[fusion.IRGate]):
        """(run gate lists, d2 gates by prim, scalars) of the IR gates of a
        circuit with this plan's structure (same gates and qubits, other
        values), placed by the plan's gate order."""
        if len(ir) != len(self.order):
            raise ValueError('rotation plan: the circuit does not have the plan\'s structure')
        runs_ = [[None] * len(u.gates) for u in self.uops]
        d2g: Dict[int, fusion.IRGate] = {}
        sc: List[fusion.IRGate] = [None] * len(self.scalars)
        for g, o in zip(ir, self.order):
            if o[0] == 'u':
                runs_[o[1]][o[2]] = g
            elif o[0] == 'd':
                d2g[o[1]] = g
            else:
                sc[o[1]] = g
        return runs_, d2g, sc

    _KIND = {'rx': 1, 'ry': 2, 'rz': 3, 'p': 4, 'u1': 4, 'phase': 4}

    def gate_table(self, runs_=None) -> dict:
        """Per-gate arrays of the fused runs (kind, theta slot, fixed value,
        constant matrices), built once per bound circuit so that a call only
        gathers theta."""
        runs_ = [u.gates for u in self.uops] if runs_ is None else runs_
        lens = np.array([len(r) for r in runs_], np.int64)
        flat = [g for r in runs_ for g in r]
        G = len(flat)
        kind = np.zeros(G, np.int8)
        slot = np.full(G, -1, np.int64)
        sval = np.zeros(G)
        cidx, cmats = [], []
        for i, g in enumerate(flat):
            if g.const is not None:
                cidx.append(i)
                cmats.append(np.asarray(g.const, dtype=np.complex128))
            else:
                kind[i] = self._KIND[g.name]
                slot[i] = g.slot
                sval[i] = g.value if g.value is not None else 0.0
        return dict(R=len(runs_), lens=lens, kind=kind, slot=slot, sval=sval, cidx=np.array(cidx, np.int64),
                    cmats=np.array(cmats).reshape(-1, 2, 2), start=np.concatenate([[0], np.cumsum(lens)[:-1]]))

    def uop_matrices(self, theta=None, runs_=None, gtab=None) -> np.ndarray:
        """FP64 2x2 matrix of every fused run for these parameters (vectorised:
        every gate's matrix at once by kind, then the products along the runs
        position by position)."""
        if gtab is None:
            if runs_ is None:
                if getattr(self, '_gtab', None) is None:
                    self._gtab = self.gate_table()
                gtab = self._gtab
            else:
                gtab = self.gate_table(runs_)
        R_ = gtab['R']
        M = np.tile(np.eye(2, dtype=np.complex128), (R_, 1, 1))
        if R_ == 0:
            return M
        lens, kind = gtab['lens'], gtab['kind']
        G = len(kind)
        mats = np.tile(np.eye(2, dtype=np.complex128), (G, 1, 1))
        if len(gtab['cidx']):
            mats[gtab['cidx']] = gtab['cmats']
        val = gtab['sval'].copy()
        if theta is not None:
            th = np.asarray(theta, dtype=np.float64)
            m = gtab['slot'] >= 0
            val[m] = th[gtab['slot'][m]]
        c, s_ = np.cos(val / 2), np.sin(val / 2)
        if 'by_kind' not in gtab:
            gtab['by_kind'] = [np.nonzero(kind == q)[0] for q in range(5)]
        k = gtab['by_kind'][1]          # rx
        mats[k, 0, 0] = mats[k, 1, 1] = c[k]
        mats[k, 0, 1] = mats[k, 1, 0] = -1j * s_[k]
        k = gtab['by_kind'][2]          # ry
        mats[k, 0, 0] = mats[k, 1, 1] = c[k]
        mats[k, 0, 1], mats[k, 1, 0] = -s_[k], s_[k]
        k = gtab['by_kind'][3]          # rz
        mats[k, 0, 0], mats[k, 1, 1] = np.exp(-0.5j * val[k]), np.exp(0.5j * val[k])
        k = gtab['by_kind'][4]          # phase
        mats[k, 1, 1] = np.exp(1j * val[k])
        start = gtab['start']
        for pos in range(int(lens.max())):
            sel = np.nonzero(lens > pos)[0]
            M[sel] = mats[start[sel] + pos] @ M[sel]
        return M

    # ------------------------------------------------------------ value program
    def _prepare_values(self):
        """Index arrays of the value program (once per plan): every table entry,
        phase and two-bit diagonal value is a unit-modulus factor, so a call
        only sums angles (np.bincount) and takes one complex exponential."""
        if getattr(self, '_vp', None) is not None:
            return self._vp
        ph_idx = {pi: i for i, pi in enumerate(pi for pi, pr in enumerate(self.prims) if pr.kind == 'ph')}
        d2_idx = {pi: i for i, pi in enumerate(pi for pi, pr in enumerate(self.prims) if pr.kind == 'd2')}
        nph, nd2 = len(ph_idx), len(d2_idx)
        fr_ph, fr_u, fr_k = [], [], []
        for pi, i in ph_idx.items():
            for u, kind in self.prims[pi].factors:
                fr_ph.append(i)
                fr_u.append(u)
                fr_k.append({'pre': 0, 'post': 1, 'diag': 2}[kind])
        SIGN = nph + 4 * nd2                    # angle source index of a -1 (pi)
        offs = np.cumsum([0] + [ps.n_floats for ps in self.passes])
        tab_ent, tab_src, ent_pos = [], [], []  # table entries: flat entry, angle source; entry -> float position
        cval_src, cval_pos = [], []             # other unit values written as (re, im): source, float position
        nent = 0
        for pidx, ps in enumerate(self.passes):
            base = int(offs[pidx])
            for kind, x in ps.order:
                if kind != 'grp':
                    continue
                g = x
                if g.has_table:
                    slots = [q for q in range(RB) if (g.reg_mask >> q) & 1]
                    idx = {q: k for k, q in enumerate(slots)}
                    ks = np.arange(1 << len(slots))
                    for pi, sa, sb in g.table_items:
                        ba = (ks >> idx[sa]) & 1
                        if pi < 0:
                            sel = ks[(ba & ((ks >> idx[sb]) & 1)) == 1]
                            tab_ent += list(nent + sel)
                            tab_src += [SIGN] * len(sel)
                        elif sb < 0:
                            sel = ks[ba == 1]
                            tab_ent += list(nent + sel)
                            tab_src += [ph_idx[pi]] * len(sel)
                        else:
                            e = ba + 2 * ((ks >> idx[sb]) & 1)
                            tab_ent += list(nent + ks)
                            tab_src += list(nph + 4 * d2_idx[pi] + e)
                    ent_pos += list(base + g.t_off + 2 * ks)
                    nent += len(ks)
                for it in g.f_items:
                    if it[0] == 'ph':
                        cval_src.append(ph_idx[it[1]])
                        cval_pos.append(base + it[3])
                    else:
                        for e in range(4):
                            cval_src.append(nph + 4 * d2_idx[it[1]] + e)
                            cval_pos.append(base + it[4] + 2 * e)
                for pi, s_, x_, off in g.mixed_items:
                    pr = self.prims[pi]
                    # (x, y) -> d[y + 2 x] when the thread-fixed bit is the d2's second
                    # bit, d[x + 2 y] when it is the first
                    order = [0, 2, 1, 3] if pr.b == x_ else [0, 1, 2, 3]
                    for e, dj in enumerate(order):
                        cval_src.append(nph + 4 * d2_idx[pi] + dj)
                        cval_pos.append(base + off + 2 * e)
        rots = []                               # per pass: (uop indices, float positions) in program order
        for pidx, ps in enumerate(self.passes):
            base = int(offs[pidx])
            us = [self.prims[pi].u for k, (pi, off) in ((k, x) for k, x in ps.order if k == 'rot')]
            pos = [base + off for k, (pi, off) in ((k, x) for k, x in ps.order if k == 'rot')]
            rots.append((np.array(us, np.int64), np.array(pos, np.int64)))
        self._vp = dict(ph_idx=ph_idx, d2_idx=d2_idx, nph=nph, nd2=nd2, fr_ph=np.array(fr_ph, np.int64),
                        fr_u=np.array(fr_u, np.int64), fr_k=np.array(fr_k, np.int64),
                        tab_ent=np.array(tab_ent, np.int64), tab_src=np.array(tab_src, np.int64),
                        ent_pos=np.array(ent_pos, np.int64), nent=nent, cval_src=np.array(cval_src, np.int64),
                        cval_pos=np.array(cval_pos, np.int64), offs=offs, rots=rots,
                        rot_u=np.array(sorted({pr.u for pr in self.prims if pr.kind == 'rot'}), np.int64),
                        diag_u=np.array([i for i, u in enumerate(self.uops) if u.diag], np.int64))
        return self._vp

    def bound(self, ir: Sequence[fusion.IRGate]):
        """bind(ir) and the gate table of its runs: what materialize needs of a
        circuit of this structure, computed once per circuit."""
        runs_, d2g, scalars = self.bind(ir)
        return runs_, d2g, scalars, self.gate_table(runs_)

    def materialize(self, theta=None, dtype=np.float32, ir=None, bound=None) -> Tuple[List[np.ndarray], complex]:
        """Per-pass parameter blocks (float32 for the kernels; float64 for exact
        emulation in tests) for these parameters, and the circuit's global
        factor (applied by the last pass's end factor).  bound: the result of
        bound(ir), when the caller keeps it across calls."""
        vp = self._prepare_values()
        if ir is not None and bound is None:
            bound = self.bound(ir)
        if bound is not None:
            runs_, d2g, scalars, gtab = bound
        else:
            runs_, d2g, scalars, gtab = None, {pi: pr.gate for pi, pr in enumerate(self.prims) if pr.kind == 'd2'}, \
                self.scalars, None
        M = self.uop_matrices(theta, runs_, gtab)
        det = M[:, 0, 0] * M[:, 1, 1] - M[:, 0, 1] * M[:, 1, 0]
        g = np.sqrt(det)
        V = M / np.where(g == 0, 1, g)[:, None, None]
        c = np.abs(V[:, 0, 0])
        s = np.abs(V[:, 1, 0])
        p = np.where(c > 1e-300, np.angle(V[:, 1, 1]), 0.0)
        m = np.where(s > 1e-300, np.angle(V[:, 1, 0]), 0.0)
        d0 = M[:, 0, 0]
        # factor angles: pre e^{i(p-m)}, post e^{i(p+m)}, diagonal runs d1 / d0
        fang = np.stack([p - m, p + m, np.angle(M[:, 1, 1]) - np.angle(d0)], 0)
        ph_ang = np.bincount(vp['fr_ph'], weights=fang[vp['fr_k'], vp['fr_u']], minlength=vp['nph']) \
            if vp['nph'] else np.zeros(0)
        # global factor (every piece has modulus 1): rotation runs g e^{-ip}, diagonal runs d0, scalars, d2 d[0]
        gang = float(np.sum(np.angle(g[vp['rot_u']]) - p[vp['rot_u']]) + np.sum(np.angle(d0[vp['diag_u']])))
        for sg in scalars:
            gang += sg.value if sg.slot < 0 or theta is None else float(theta[sg.slot])
        # constant two-bit diagonals (cz, the cx / cy rewrites) have the same
        # angles in every circuit of this structure: computed once per plan
        if vp.get('d2_const') is None:
            const = np.zeros((vp['nd2'], 4))
            cmask = np.zeros(vp['nd2'], bool)
            for pi, i in vp['d2_idx'].items():
                gt = d2g[pi]
                if gt.const is not None:
                    const[i] = np.angle(np.asarray(gt.const, dtype=np.complex128))
                    cmask[i] = True
            vp['d2_const'] = const
            vp['d2_param'] = [(pi, i) for pi, i in vp['d2_idx'].items() if not cmask[i]]
        d2_ang = vp['d2_const'].copy()
        for pi, i in vp['d2_param']:
            gt = d2g[pi]
            val = gt.value if gt.slot < 0 or theta is None else float(theta[gt.slot])
            d2_ang[i] = np.angle(np.asarray(fusion.gate_matrix_of('d2', gt.name, val), dtype=np.complex128))
        if len(d2_ang):
            gang += float(d2_ang[:, 0].sum())
            d2_ang = d2_ang - d2_ang[:, :1]
        src = np.concatenate([ph_ang, d2_ang.reshape(-1), [np.pi]])
        glob = complex(np.exp(1j * gang))
        flat = np.zeros(int(vp['offs'][-1]), dtype=np.float64)
        if vp['nent']:
            T = np.exp(1j * np.bincount(vp['tab_ent'], weights=src[vp['tab_src']], minlength=vp['nent']))
            flat[vp['ent_pos']] = T.real
            flat[vp['ent_pos'] + 1] = T.imag
        if len(vp['cval_src']):
            cv = np.exp(1j * src[vp['cval_src']])
            flat[vp['cval_pos']] = cv.real
            flat[vp['cval_pos'] + 1] = cv.imag
        # every pass's rotations at once: tangents, forms and the pending scale
        ra = vp.get('rot_all')
        if ra is None:
            lens = np.array([len(us) for us, _ in vp['rots']], np.int64)
            live = np.nonzero(lens)[0]
            ra = dict(us=np.concatenate([us for us, _ in vp['rots']] + [np.zeros(0, np.int64)]),
                      pos=np.concatenate([pos for _, pos in vp['rots']] + [np.zeros(0, np.int64)]),
                      lens=lens, live=live, starts=np.concatenate([[0], np.cumsum(lens)[:-1]])[live],
                      pid=np.repeat(np.arange(len(lens)), lens))
            vp['rot_all'] = ra
        scales = np.ones(len(self.passes))
        if len(ra['us']):
            ci, si = c[ra['us']], s[ra['us']]
            with np.errstate(divide='ignore'):
                t = np.where(ci > 0, si / np.where(ci > 0, ci, 1.0), np.inf)
            tan = np.abs(t) <= TMAX
            inv = np.where(tan, 1.0 / np.where(tan, ci, 1.0), 1.0)
            scales[ra['live']] = np.multiply.reduceat(inv, ra['starts'])
            # the pending scale inside each pass, from logs; a pass that may pass
            # SCALE_LIMIT (rare) is redone exactly, rotation by rotation
            lg = np.log(inv)
            cs = np.cumsum(lg)
            within = cs - np.repeat((cs - lg)[ra['starts']], ra['lens'][ra['live']])
            over = within > np.log(SCALE_LIMIT) - 1e-6
            if over.any():
                for pidx in np.unique(ra['pid'][over]):
                    a = int(np.searchsorted(ra['pid'], pidx))
                    sc = 1.0
                    for k in range(a, a + int(ra['lens'][pidx])):
                        if tan[k] and sc / ci[k] <= SCALE_LIMIT:
                            sc /= ci[k]
                        else:
                            tan[k] = False
                    scales[pidx] = sc
            pos = ra['pos']
            flat[pos] = np.where(tan, t, 0.0)
            flat[pos + 1] = ci
            flat[pos + 2] = si
            flat[pos + 3] = np.where(tan, 0.0, 1.0)
        for pidx, ps in enumerate(self.passes):
            if ps.end_scale_off >= 0:
                f = complex(1.0 / scales[pidx]) * (glob if ps.end_complex else 1.0)
                o = int(vp['offs'][pidx]) + ps.end_scale_off
                flat[o], flat[o + 1] = f.real, f.imag
        blocks = [flat[vp['offs'][i]:vp['offs'][i + 1]].astype(dtype) for i in range(len(self.passes))]
        return blocks, glob


# ---------------------------------------------------------------------------
# index maps shared by the code generator and the tests' tile emulator
# ---------------------------------------------------------------------------

def nonreg_bits(K: int, regs: Sequence[int]) -> List[int]:
    """Tile bits that are not register slots, ascending: thread bit k of a
    stage is tile bit nonreg_bits[k]."""
    return [b for b in range(K) if b not in regs]


def runs(src_to_dst: Sequence[int]) -> List[Tuple[int, int, int]]:
    """Maximal runs (src, dst, length) of a map from consecutive source bits
    to destination bits where the destinations are consecutive too."""
    out = []
    k = 0
    while k < len(src_to_dst):
        j = k
        while j + 1 < len(src_to_dst) and src_to_dst[j + 1] == src_to_dst[j] + 1:
            j += 1
        out.append((k, src_to_dst[k], j - k + 1))
        k = j + 1
    return out


def reg_offset(j: int, positions: Sequence[int]) -> int:
    """Offset of register index j when slot k stands for bit positions[k]."""
    o = 0
    for k, p in enumerate(positions):
        if (j >> k) & 1:
            o |= 1 << p
    return o


def padded(i: int) -> int:
    """Shared-memory position of tile-local index i in the padded stage layout
    (one spare amplitude after every 16): linear over disjoint bit sets."""
    return i + (i >> PAD_SHIFT)


def slot_elems(K: int) -> int:
    """Amplitudes per ring slot: room for the padded layout of a 2^K tile
    (positions up to padded(2^K - 1)), rounded so that every slot starts on a
    16-byte boundary as the bulk copies into it require.  libdesv sizes the
    kernel's shared memory with the same value (desv_jit.cu, rot_slot_elems)."""
    return (1 << K) + (1 << (K - PAD_SHIFT))


# ---------------------------------------------------------------------------
# code generation
# ---------------------------------------------------------------------------

def _dep_expr(rs: List[Tuple[int, int, int]], var: str, wide: bool) -> str:
    terms = []
    for s, d, ln in rs:
        m = (1 << ln) - 1
        x = f'(({var} >> {s}) & {m}u)' if s else f'({var} & {m}u)'
        if wide:
            x = f'((uint64_t){x})'
        terms.append(f'({x} << {d})' if d else x)
    return ' | '.join(terms) if terms else ('0ull' if wide else '0u')


def _f(x: float) -> str:
    return repr(float(x)) + 'f'


def pass_source(plan: 'RotationPlan', pidx: int, nbuf: Optional[int] = None, general: bool = False) -> str:
    """CUDA source of one rotation pass (entry point desv_rot_kernel).  With
    general=False every rotation is compiled in tangent form only (the variant
    for calls whose rotations all take it); with general=True each rotation
    picks its form from its form flag at run time.  Both read the same
    parameter block."""
    ps = plan.passes[pidx]
    nbuf = nbuf or plan.nbuf
    K, L, high = ps.K, ps.L, ps.high
    NA = 1 << RB
    nthreads = 1 << (K - RB)
    gmap = [b if b < L else high[b - L] for b in range(K)]
    check = os.environ.get('DESV_ROT_CHECK', '') == '1'
    lines = ([f'#define DESV_ROT_CHECK 1', f'#define ROT_SLOT_ELEMS {slot_elems(K)}u'] if check else []) + \
            ['#include "rot_pass.cuh"', 'using namespace desv;',
             f'struct RotParams {{ float v[{ps.n_floats}]; }};',
             f'extern "C" __global__ void __launch_bounds__({nthreads}, {CTAS_PER_SM[nbuf]})',
             'desv_rot_kernel(float2 *__restrict__ sv, const TileGeom g, const RotParams P) {',
             '    extern __shared__ __align__(128) unsigned char smem[];',
             '    const uint32_t t = threadIdx.x;',
             f'    RotRing<{K}, {nbuf}, {slot_elems(K)}u> ring;',
             '    ring.init(g, sv, smem);',
             '    uint32_t i = 0;',
             '    for (; i < ring.cnt; ++i) {',
             '        uint64_t tb;',
             '        if (!ring.begin(i, tb)) break;',
             '        float2 *s = ring.slot(i);',
             f'        float2 a[{NA}];']
    nst = len(ps.stages)
    for si, st in enumerate(ps.stages):
        first, last = si == 0, si == nst - 1
        regs = list(st.regs)
        nr = nonreg_bits(K, regs)
        loc = _dep_expr(runs(nr), 't', False)
        glob = _dep_expr(runs([gmap[b] for b in nr]), 't', True)
        offs = [reg_offset(j, regs) for j in range(NA)]
        goffs = [reg_offset(j, [gmap[p] for p in regs]) for j in range(NA)]
        need_gi = last or any(k == 'grp' and (x.signs_mixed or x.signs_thread or x.f_items or x.mixed_items)
                              for k, x in st.items)
        lines.append(f'        {{  // stage {si}: register slots at tile bits {regs}')
        lines.append(f'            const uint32_t lb = {loc};')
        if first:
            lines += [f'            ROT_SLD(a[{j}], s, lb + {offs[j]}u);' for j in range(NA)]
        else:
            lines.append('            const uint32_t pb = lb + (lb >> 4);')
            lines += [f'            ROT_SLD(a[{j}], s, pb + {padded(offs[j])}u);' for j in range(NA)]
        if last and nbuf == 1:
            lines.append('            __syncthreads();  // the slot is read: the next tile may load into it')
            lines.append('            ring.release(i);')
        if need_gi:
            lines.append(f'            const uint64_t gi = tb | {glob};')
        for kind, x in st.items:
            if kind == 'rot':
                pi, slot, off = x
                if general:
                    lines.append(f'            rot<{slot}>(a, pv[{off}], pv[{off + 1}], pv[{off + 2}], pv[{off + 3}]);')
                else:
                    lines.append(f'            rot_t<{slot}>(a, pv[{off}]);')
            else:
                lines += ['            ' + ln for ln in _group_code(x)]
        if last:
            if ps.end_scale_off >= 0:
                o = ps.end_scale_off
                if ps.end_complex:
                    lines.append(f'            scale_all_c(a, pv[{o}], pv[{o + 1}]);')
                else:
                    lines.append(f'            scale_all(a, pv[{o}]);')
            lines += [f'            ROT_GST(sv, gi + {goffs[j]}ull, a[{j}]);' for j in range(NA)]
        else:
            if first:
                lines.append('            __syncthreads();  // every natural-layout read is done')
                lines.append('            const uint32_t pb = lb + (lb >> 4);')
            lines += [f'            ROT_SST(s, pb + {padded(offs[j])}u, a[{j}]);' for j in range(NA)]
            lines.append('            fence_proxy_async_smem();')
            lines.append('            __syncthreads();')
        lines.append('        }')
    if nbuf > 1:
        lines.append('        __syncthreads();  // the slot is free for the load NBUF-1 tiles ahead')
    lines += ['    }',
              '    if (i < ring.cnt) ring.drain(i);',
              '}', '']
    src = '\n'.join(lines)
    return src.replace('pv[', 'P.v[')


def _group_code(g: Group) -> List[str]:
    NA = 1 << RB
    out = ['{']
    words = {}
    for s_, x in g.signs_mixed:
        if ('b', x) not in words:
            words[('b', x)] = f'w{len(words)}'
            out.append(f'    const uint32_t {words[("b", x)]} = (uint32_t)((gi >> {x}) & 1ull) << 31;')
    for x, y in g.signs_thread:
        key = ('p', min(x, y), max(x, y))
        if key not in words:
            words[key] = f'w{len(words)}'
            out.append(f'    const uint32_t {words[key]} = (uint32_t)((gi >> {x}) & (gi >> {y}) & 1ull) << 31;')
    has_f = bool(g.f_items)
    if has_f:
        out.append('    float2 F = make_float2(1.f, 0.f);')
        for it in g.f_items:
            if it[0] == 'ph':
                _, pi, x, off = it
                out.append(f'    if ((gi >> {x}) & 1ull) F = cmulc(F, pv[{off}], pv[{off + 1}]);')
            else:
                _, pi, xa, xb, off = it
                out.append(f'    {{ const uint32_t k = (uint32_t)(((gi >> {xa}) & 1ull) | (((gi >> {xb}) & 1ull) << 1));'
                           f' F = cmulc(F, pv[{off} + 2 * k], pv[{off + 1} + 2 * k]); }}')
    slots = [q for q in range(RB) if (g.reg_mask >> q) & 1]
    if g.has_table or has_f:
        for j in range(NA):
            k = 0
            for i, q in enumerate(slots):
                if (j >> q) & 1:
                    k |= 1 << i
            if g.has_table:
                o = g.t_off + 2 * k
                if k == 0 and not has_f:
                    continue          # table entry 0 is 1: the pass-end factor carries the scale
                if k == 0:
                    out.append(f'    a[{j}] = cmulc(a[{j}], F.x, F.y);')
                    continue
                if has_f:
                    out.append(f'    a[{j}] = cmulc(cmulc(a[{j}], pv[{o}], pv[{o + 1}]), F.x, F.y);')
                else:
                    out.append(f'    a[{j}] = cmulc(a[{j}], pv[{o}], pv[{o + 1}]);')
            else:
                out.append(f'    a[{j}] = cmulc(a[{j}], F.x, F.y);')
    for pi, s_, x, off in g.mixed_items:
        out.append(f'    {{ const uint32_t X = (uint32_t)((gi >> {x}) & 1ull);')
        out.append(f'      const float f0r = X ? pv[{off + 4}] : pv[{off}], f0i = X ? pv[{off + 5}] : pv[{off + 1}];')
        out.append(f'      const float f1r = X ? pv[{off + 6}] : pv[{off + 2}], f1i = X ? pv[{off + 7}] : pv[{off + 3}];')
        for j in range(NA):
            if (j >> s_) & 1:
                out.append(f'      a[{j}] = cmulc(a[{j}], f1r, f1i);')
            else:
                out.append(f'      a[{j}] = cmulc(a[{j}], f0r, f0i);')
        out.append('    }')
    # signs: per amplitude the XOR of the words that apply to it
    for j in range(NA):
        ws = []
        for s_, x in g.signs_mixed:
            if (j >> s_) & 1:
                ws.append(words[('b', x)])
        for x, y in g.signs_thread:
            ws.append(words[('p', min(x, y), max(x, y))])
        neg = sum(1 for sa, sb in g.signs_reg if (j >> sa) & 1 and (j >> sb) & 1) & 1
        # XOR of identical words cancels
        cnt = {}
        for w in ws:
            cnt[w] = cnt.get(w, 0) ^ 1
        ws = [w for w, c in cnt.items() if c]
        if neg:
            ws.append('0x80000000u')
        if ws:
            out.append(f'    flip(a[{j}], {" ^ ".join(ws)});')
    out.append('}')
    return out


# ---------------------------------------------------------------------------
# kernels and execution
# ---------------------------------------------------------------------------

# below this many qubits the general passes are used (compile time does not pay off)
MIN_QUBITS = 20
_kcache: Dict[tuple, object] = {}
_kcache_lock = threading.Lock()


class _RotKernel:
    __slots__ = ('handle', 'n_floats')

    def __init__(self, handle, n_floats):
        self.handle = handle
        self.n_floats = n_floats

    def __del__(self):
        try:
            from .. import _native as N
            N.lib().desv_jit_free(self.handle)
        except Exception:
            pass


def enabled(n: int, complex64: bool) -> bool:
    """Rotation passes for an n-qubit complex64 plan: DESV_ROT=1 / 0 forces the
    choice; by default from MIN_QUBITS qubits on, where NVRTC is available."""
    if not complex64:
        return False
    v = os.environ.get('DESV_ROT', '')
    if v in ('0', '1'):
        return v == '1'
    from . import jit
    return n >= MIN_QUBITS and jit.available()


def _load(src: str, K: int, nbuf: int, n_floats: int, device: int) -> _RotKernel:
    import ctypes
    from .. import _native as N
    from . import jit
    key = (hashlib.sha1(src.encode()).hexdigest(), device)
    with _kcache_lock:
        k = _kcache.get(key)
    if k is not None:
        return k
    h = ctypes.c_void_p()
    log = ctypes.create_string_buffer(8192)
    N.check(N.lib().desv_rot_load(src.encode(), jit.INCLUDE_PATH.encode(), K, nbuf, n_floats, device,
                                  ctypes.byref(h), log, 8192), 'desv_rot_load')
    k = _RotKernel(h, n_floats)
    with _kcache_lock:
        _kcache.setdefault(key, k)
        return _kcache[key]


class RotationProgram:
    """A rotation plan with its compiled kernels, run on CUDA statevectors.

    Every pass has two kernels over the same parameter block: the tangent-only
    variant, compiled up front, and the variant that picks each rotation's form
    at run time, compiled the first time a call needs the general form in that
    pass (a rotation with cos = 0, as in an X gate, or a pending scale past
    SCALE_LIMIT)."""

    def __init__(self, plan: RotationPlan):
        self.plan = plan
        self.sources = [pass_source(plan, i) for i in range(len(plan.passes))]
        self.kernels: Dict[int, list] = {}
        self.general: Dict[Tuple[int, int], _RotKernel] = {}
        vp = plan._prepare_values()
        self.form_idx = [pos - int(vp['offs'][i]) + 3 for i, (_, pos) in enumerate(vp['rots'])]
        rows = []
        from .. import _native as N
        for ps in plan.passes:
            row = np.zeros((), dtype=N.PASS_DTYPE)
            row['tile_bits'], row['low_bits'] = ps.K, ps.L
            h = np.zeros(16, np.uint8)
            h[:len(ps.high)] = ps.high
            row['high'] = h
            rows.append(row)
        self.rows = np.array(rows, dtype=N.PASS_DTYPE)

    def compile(self, device: int, workers: int = 0) -> list:
        if device not in self.kernels:
            from concurrent.futures import ThreadPoolExecutor
            jobs = [(src, ps.K, ps.n_floats) for src, ps in zip(self.sources, self.plan.passes)]
            workers = workers or min(32, os.cpu_count() or 1, max(1, len(jobs)))
            nb = self.plan.nbuf
            with ThreadPoolExecutor(max_workers=workers) as ex:
                self.kernels[device] = list(ex.map(lambda j: _load(j[0], j[1], nb, j[2], device), jobs))
        return self.kernels[device]

    def needs_general(self, i: int, block: np.ndarray) -> bool:
        """Whether pass i's parameter block sets the general form for a rotation."""
        fi = self.form_idx[i]
        return bool(len(fi)) and bool(np.any(block[fi] != 0))

    def pass_kernels(self, device: int, blocks: list) -> list:
        """The kernel of every pass for these parameter blocks."""
        kernels = list(self.compile(device))
        for i, b in enumerate(blocks):
            if self.needs_general(i, b):
                key = (device, i)
                if key not in self.general:
                    ps = self.plan.passes[i]
                    self.general[key] = _load(pass_source(self.plan, i, general=True), ps.K, self.plan.nbuf,
                                              ps.n_floats, device)
                kernels[i] = self.general[key]
        return kernels

    def run_blocks(self, sv_ptr: int, device: int, stream: int, blocks: list):
        """Every pass over the complex64 state at sv_ptr with these parameter blocks."""
        import ctypes
        from .. import _native as N
        kernels = self.pass_kernels(device, blocks)
        lib = N.lib()
        st = ctypes.c_void_p(stream)
        base = self.rows.ctypes.data
        for i, (k, b) in enumerate(zip(kernels, blocks)):
            N.check(lib.desv_rot_pass(k.handle, ctypes.c_void_p(sv_ptr), self.plan.n,
                                      ctypes.c_void_p(base + i * self.rows.itemsize), b.ctypes.data_as(ctypes.c_void_p),
                                      len(b), st), 'desv_rot_pass')


_STRUCT_CACHE: Dict[str, RotationProgram] = {}
_STRUCT_LOCK = threading.Lock()


def structure_key(ir: Sequence[fusion.IRGate], n: int, kmax: int) -> str:
    """Structure of a lowered circuit without its parameter values: gate kind,
    name, bits, theta slot, and for constant gates whether the matrix is
    diagonal (it decides the run's kind).  Plans and kernels depend on it only."""
    h = hashlib.sha1()
    h.update(f'{n}:{kmax}:{tuning()}:{LOW_FIXED}:{RB}|'.encode())
    for g in ir:
        cz = g.kind == 'd2' and g.const is not None and np.array_equal(g.const, _CZ)
        h.update(repr((g.kind, g.name, g.t, g.t2, g.cbits, g.slot, _is_const_diag(g) if g.kind == 'm1' else cz))
                 .encode())
    return h.hexdigest()


class BoundProgram:
    """A structure-shared RotationProgram with one circuit's IR gates bound."""

    def __init__(self, prog: RotationProgram, ir: List[fusion.IRGate]):
        self.prog = prog
        self.ir = ir
        self._key = None
        self._blocks = None
        self._bound = None

    @property
    def plan(self) -> RotationPlan:
        return self.prog.plan

    def blocks(self, theta=None) -> list:
        key = None if theta is None else np.asarray(theta, dtype=np.float64).tobytes()
        if self._blocks is None or key != self._key:
            if self._bound is None:
                self._bound = self.prog.plan.bound(self.ir)
            self._blocks = [np.ascontiguousarray(b, dtype=np.float32)
                            for b in self.prog.plan.materialize(theta, np.float32, bound=self._bound)[0]]
            self._key = key
        return self._blocks

    def run(self, sv_ptr: int, device: int, stream: int, theta=None):
        self.prog.run_blocks(sv_ptr, device, stream, self.blocks(theta))


def program_for(target: Sequence[tuple], n: int, kmax: int, slots=None) -> Optional[BoundProgram]:
    """The structure-cached program bound to this circuit's values, or None
    when the circuit holds a gate the rotation path does not lower."""
    ir = lowered_gates(target, n, slots)
    if ir is None:
        return None
    key = structure_key(ir, n, kmax)
    with _STRUCT_LOCK:
        prog = _STRUCT_CACHE.get(key)
    if prog is None:
        plan = RotationPlan(target, n, kmax, slots)
        prog = RotationProgram(plan)
        with _STRUCT_LOCK:
            if len(_STRUCT_CACHE) > 64:
                _STRUCT_CACHE.pop(next(iter(_STRUCT_CACHE)))
            prog = _STRUCT_CACHE.setdefault(key, prog)
    return BoundProgram(prog, ir)
