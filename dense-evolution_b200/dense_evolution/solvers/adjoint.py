"""Adjoint-method gradients of E(theta) = Re<psi(theta)|H|psi(theta)>.

Three device statevectors (the reference's JAX path keeps one residual per
gate instead, ``solvers/autodiff.py:136-166``):

* psi -- the forward state, returned to the caller untouched;
* lambda -- H psi, un-applied gate by gate in reverse;
* mu -- a working copy of psi, un-applied alongside lambda.

For each parametric gate U(theta_k) = exp(theta_k G_k)-style with
dU/dtheta = G U, dE/dtheta_k = 2 Re<lambda|G|mu> evaluated right before U is
un-applied from mu and lambda.  On states of >= 9 qubits the reversed circuit
(GRAD probes + inverse gates) is fused into tile passes that read and write
mu and lambda once per pass (``desv_adjoint_passes``); smaller states walk
gate by gate and materialise G mu in a scratch state.

Generators: rx -> -i/2 X, ry -> -i/2 Y, rz -> -i/2 Z, p/u1/phase -> i|1><1|,
cp -> i|11><11|, crz -> -i/2 |1><1| (x) Z.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from .. import _native as N
from ..circuits import fusion, jit
from ..circuits.compiler import CompiledCircuit, apply_fop
from ..physics.observables import PauliPlan, PauliSumOperator, plan_for

_HALF_I = -0.5j
_GEN_1Q = {
    'rx': np.array([[0, _HALF_I], [_HALF_I, 0]], dtype=np.complex128),
    'ry': np.array([[0, -0.5], [0.5, 0]], dtype=np.complex128),
    'rz': np.array([[_HALF_I, 0], [0, 0.5j]], dtype=np.complex128),
    'p': np.array([[0, 0], [0, 1j]], dtype=np.complex128),
}
_GEN_1Q['u1'] = _GEN_1Q['phase'] = _GEN_1Q['p']
# diagonal generators over (control bit, target bit): index bit(c) + 2 bit(t)
_GEN_D2 = {
    'cp': np.array([0, 0, 0, 1j], dtype=np.complex128),
    'crz': np.array([0, _HALF_I, 0, 0.5j], dtype=np.complex128),
}
_GEN_D2['cphase'] = _GEN_D2['cp']


class BOp(fusion.FOp):
    """A backward op: an inverse gate ('m1' / 'd2' / 'm2' / 'scalar') or a
    gradient probe ('g1' 2x2 generator, 'gd' diagonal generator)."""

    def matrix(self, theta=None) -> np.ndarray:
        g = self.src[0]
        if self.kind == 'g1':
            return _GEN_1Q[g.name]
        if self.kind == 'gd':
            return _GEN_D2[g.name]
        m = g.matrix(theta)
        if self.kind == 'scalar':
            v = np.exp(1j * (g.value if g.slot < 0 or theta is None else float(theta[g.slot])))
            return np.full(4, np.conj(v), dtype=np.complex128)
        if self.kind == 'd2':
            return np.conj(m)
        return np.conj(m).T


def backward_ops(ir: List[fusion.IRGate]) -> List[BOp]:
    ops: List[BOp] = []
    for g in reversed(ir):
        if g.slot >= 0 and g.kind == 'm1' and g.name in _GEN_1Q:
            ops.append(BOp('g1', t=g.t, cbits=g.cbits, cvals=g.cvals, src=[g]))
        elif g.slot >= 0 and g.kind == 'd2' and g.name in _GEN_D2:
            ops.append(BOp('gd', t=g.t, t2=g.t2, src=[g]))
        ops.append(BOp(g.kind, t=g.t, t2=g.t2, cbits=g.cbits, cvals=g.cvals, src=[g]))
    for op in ops:
        _classify_backward(op)
    return ops


def _classify_backward(op: BOp):
    g = op.src[0]
    nd = d = 0
    for b in op.cbits:
        d |= 1 << b
    if op.kind == 'g1':
        if g.name in ('rx', 'ry'):
            nd |= 1 << op.t
        else:
            d |= 1 << op.t
    elif op.kind in ('gd', 'd2'):
        d |= (1 << op.t) | (1 << op.t2)
    elif op.kind == 'm1':
        diag = (g.const is not None and fusion._is_diag(g.const)) or (g.const is None and g.name in
                                                                       ('rz', 'p', 'u1', 'phase'))
        if diag:
            d |= 1 << op.t
        else:
            nd |= 1 << op.t
    elif op.kind == 'm2':
        nd |= (1 << op.t) | (1 << op.t2)
    op.nd, op.d = nd, d


class TangentPlan:
    """The tangent variant of a program's backward passes (complex64,
    specialised kernels).  Uncontrolled ry inverses on register slots become
    x0 -= t x1, x1 += t x0 and uncontrolled rz inverses x += i t x / x -= i t x
    (jit_pass.cuh: tan_rot, tan_phase): half the FP32 work of the general
    forms, each 1/c times the exact gate.  Per call and pass the host forms
    t = s / c and the running product S of the 1/c; a gradient probe is
    multiplied by 1/S^2 (both arrays carry S), and the pass ends by scaling
    both arrays by 1/S.  A pass whose |t| leaves [0, TMAX] or whose S leaves
    [0, TMAX^2] runs in the general form (its matrices untouched) -- the tangent
    blows up near theta = pi.  S scales every amplitude alike, so FP32 keeps its
    relative accuracy; S^2 <= 2^80 keeps the probes' products far inside the
    FP32 range."""

    TMAX = 2.0 ** 20

    def __init__(self, back: fusion.Packed, pool_len: int, generic_pool: np.ndarray):
        words = np.ascontiguousarray(generic_pool).view(np.uint32)
        wpe = generic_pool.dtype.itemsize // 4
        name_of = {rec: back.fops[fi].src[0].name for rec, fi in back.op_slots}
        kind_of = {rec: back.fops[fi].kind for rec, fi in back.op_slots}
        slot_of = {rec: back.fops[fi].src[0].slot for rec, fi in back.op_slots}
        self.off_slot = {}    # pool offset of a tangent record -> its theta slot
        ops = back.ops
        self.end_base = pool_len
        self.passes = []      # per pass: (records in tangent form {rec: 'rot' | 'phase'}, events)
        for ps in back.passes:
            tan, events = {}, []
            if int(ps['op_end']) - int(ps['op_begin']) > jit.MAX_OPS:
                self.passes.append((tan, events))     # no specialised kernel: the interpreter runs it
                continue
            for q in range(int(ps['op_begin']), int(ps['op_end'])):
                o = ops[q]
                k = int(o['kind'])
                if k == N.OP_STAGE:
                    continue
                off = int(o['mat'])
                if k == N.OP_GRAD:
                    events.append(('g', off, jit.grad_reads_pool(o, words, wpe)))
                    continue
                code = int(o['code'])
                if code & 0x8000 or kind_of.get(q) != 'm1':
                    continue
                nm = name_of.get(q)
                if nm == 'ry' and 1 <= code <= 20 and (code - 1) % 5 == 1 and int(o['cslot']) < 0:
                    tan[q] = 'rot'
                elif nm == 'rz' and 83 <= code <= 107 and (code - 83) % 5 == 0 and int(o['gb']) == 0xFF:
                    tan[q] = 'phase'
                else:
                    continue
                events.append(('t', off, tan[q]))
                self.off_slot[off] = int(slot_of.get(q, -1))
            self.passes.append((tan, events))

    def sources_info(self) -> list:
        """Per pass the tangent argument of jit.adjoint_source (None: no record
        in tangent form, the general kernel serves it)."""
        return [(tan, self.end_base + i) if tan else None for i, (tan, _) in enumerate(self.passes)]

    def allowed(self, theta: np.ndarray) -> np.ndarray:
        """Per pass whether it runs in tangent form, from the angles alone and
        with a margin of 2 on both bounds (|t| <= TMAX / 2, S <= TMAX^2 / 4):
        the tangent of a ry / rz inverse is +-tan(theta / 2) and every 1/c is
        1 / cos(theta / 2), so the check needs no matrices (the device then
        rewrites the allowed passes without checking again)."""
        ps, kind, off = self._flat()
        npass = len(self.passes)
        out = np.zeros(npass, bool)
        if ps.size == 0:
            return out
        tanm = kind <= 1
        slots = np.array([self.off_slot.get(int(o), -1) for o in off[tanm]], np.int64) \
            if not hasattr(self, '_tan_slots') else self._tan_slots
        self._tan_slots = slots
        if np.any(slots < 0):
            return out
        half = 0.5 * np.asarray(theta, dtype=np.float64)[slots]
        c = np.abs(np.cos(half))
        with np.errstate(divide='ignore'):
            t = np.abs(np.sin(half)) / c
            lg = -np.log(c)
        tp = ps[tanm]
        ok_t = np.ones(npass, bool)
        np.logical_and.at(ok_t, tp, t <= 0.5 * self.TMAX)
        logs = np.zeros(npass)
        np.add.at(logs, tp, lg)
        has = np.zeros(npass, bool)
        has[tp] = True
        return has & ok_t & (logs <= np.log(0.25 * self.TMAX * self.TMAX))

    def _flat(self):
        """Flat event arrays (pass, kind 0 rot / 1 phase / 2 probe with compiled-in
        generator / 3 probe reading its generator, pool offset), built once."""
        if getattr(self, '_flat_ev', None) is None:
            ps, kind, off = [], [], []
            for i, (tan, events) in enumerate(self.passes):
                if not tan:
                    continue
                for k, o, x in events:
                    ps.append(i)
                    kind.append((0 if x == 'rot' else 1) if k == 't' else (3 if x else 2))
                    off.append(o)
            self._flat_ev = (np.array(ps, np.int64), np.array(kind, np.int8), np.array(off, np.int64))
        return self._flat_ev

    def transform(self, mats: np.ndarray):
        """(pool extended by one pass-end factor per pass, with every pass that
        can run in tangent form rewritten for it; per-pass flags).  Vectorised
        over the events: the running product S of a pass is a cumulative
        product of its tangent records' 1/c."""
        npass = len(self.passes)
        out = np.concatenate([mats, np.ones(npass, mats.dtype)])
        ps, kind, off = self._flat()
        flags = np.zeros(npass, bool)
        if ps.size == 0:
            return out, list(flags)
        tanm = kind <= 1
        c = np.ones(ps.size)
        t = np.zeros(ps.size)
        with np.errstate(divide='ignore', invalid='ignore'):
            c[tanm] = mats[off[tanm]].real
            num = np.where(kind == 0, mats[np.minimum(off + 2, len(mats) - 1)].real, mats[off].imag)
            t[tanm] = (num / c)[tanm]
            f = 1.0 / c                                   # 1 at probes
        # S after every event, per pass (cumulative product restarted at each pass)
        S = np.empty(ps.size)
        starts = np.flatnonzero(np.r_[True, ps[1:] != ps[:-1]])
        ends = np.r_[starts[1:], ps.size]
        ok_pass = np.zeros(npass, bool)
        for a, b in zip(starts, ends):
            S[a:b] = np.cumprod(f[a:b])
            seg_ok = (np.all(np.abs(t[a:b][tanm[a:b]]) <= self.TMAX) and
                      np.all(np.abs(S[a:b]) <= self.TMAX * self.TMAX) and np.any(tanm[a:b]))
            ok_pass[ps[a]] = bool(seg_ok)
        flags = ok_pass
        use = flags[ps]
        # tangent records: t; immediate probes: 1/S^2; probes reading their
        # generator: the generator times 1/S^2 (S at a probe: its factor is 1)
        sel = use & tanm
        out[off[sel]] = t[sel]
        corr = 1.0 / (S * S)
        sel = use & (kind == 2)
        out[off[sel]] = corr[sel]
        sel = np.flatnonzero(use & (kind == 3))
        for q in range(4):
            out[off[sel] + q] = mats[off[sel] + q] * corr[sel]
        # pass-end factors 1/S of the last event of every pass in tangent form
        last = ends - 1
        for a, l in zip(starts, last):
            if flags[ps[a]]:
                out[self.end_base + ps[a]] = 1.0 / S[l]
        return out, list(flags)


def _adjoint_tile_bits(n: int, dtype) -> int:
    return min(11 if dtype == torch.complex64 else 10, n)


class AdjointProgram:
    """Forward + adjoint plans of one parametrised circuit at one precision."""

    def __init__(self, rows, slots, n: int, dtype=torch.complex128):
        self.n = int(n)
        self.dtype = dtype
        self.rows, self.slots = rows, slots
        self.forward = CompiledCircuit(rows, self.n, dtype, slots=slots)
        self.ir = self.forward.ir
        self.bops = backward_ops(self.ir)
        self.nparams = 1 + max([s for s in slots if s >= 0], default=-1)
        if self.n >= fusion.MIN_FUSED_QUBITS:
            kb = _adjoint_tile_bits(self.n, dtype)
            specs = fusion.schedule(self.bops, self.n, kb)
            specs = _split_params(specs, self.bops, 1024)
            if dtype == torch.complex64 and jit.enabled(self.n):
                specs = _split_ops(specs, ops_per_pass())
            self.back = fusion.Packed(self.n, self.bops, specs, adjoint=True)
        else:
            self.back = None
        self._back_dev = None
        self._map_dev = None
        self._stage: dict = {}
        self._scratch = None
        self._tangent = None          # TangentPlan, built with the first specialised gradient
        self._dv = None               # device-built backward values (recipes + tangent form), or False
        import os
        self._use_tangent = (self.back is not None and dtype == torch.complex64 and jit.enabled(self.n)
                             and os.environ.get('DESV_ADJ_TANGENT', '1') != '0')

    # ------------------------------------------------------------ helpers
    def _device(self):
        return N.require_cuda()

    def initial_state(self, stato_zero=None) -> torch.Tensor:
        dev = self._device()
        if stato_zero is None:
            sv = torch.empty(1 << self.n, dtype=self.dtype, device=dev)
            N.check(N.lib().desv_init_basis(ctypes.c_void_p(sv.data_ptr()), self.n, N.dtype_code(sv), 0,
                                            ctypes.c_void_p(N.stream_ptr())), 'init')
            return sv
        if isinstance(stato_zero, torch.Tensor):
            return stato_zero.detach().to(device=dev, dtype=self.dtype).reshape(-1).clone()
        return torch.from_numpy(np.asarray(stato_zero).astype(np.complex128).reshape(-1)).to(dev).to(self.dtype)

    def forward_state(self, theta: np.ndarray, stato_zero=None) -> torch.Tensor:
        psi = self.initial_state(stato_zero)
        self.forward.run(psi, theta=theta)
        return psi

    def norm_ratio(self, psi: torch.Tensor, stato_zero=None) -> float:
        """<psi0|psi0> / <psi|psi> in FP64 for a complex64 program, 1 otherwise.

        The circuit is unitary, so in exact arithmetic the ratio is 1; in
        complex64 the rounding of the gate passes drifts the norm by about
        1e-7.  Multiplying E = <psi|H|psi> and its gradient by the ratio
        removes the first-order effect of that drift on both (the reference's
        energy is the unnormalised <psi|H|psi> of a state whose norm is the
        initial state's, so the ratio keeps unnormalised initial states
        exact too)."""
        if self.dtype != torch.complex64:
            return 1.0
        n0 = self._initial_norm2(stato_zero)
        nn = float(self._norm_device(psi)[0].item())
        return n0 / nn if nn > 0 else 1.0

    @staticmethod
    def _initial_norm2(stato_zero) -> float:
        if stato_zero is None:
            return 1.0
        if isinstance(stato_zero, torch.Tensor):
            return float(torch.linalg.vector_norm(stato_zero.detach().to(torch.complex128)).item()) ** 2
        a = np.asarray(stato_zero).astype(np.complex128).reshape(-1)
        return float(np.vdot(a, a).real)

    def _norm_device(self, psi: torch.Tensor) -> torch.Tensor:
        """<psi|psi> in FP64 as a device tensor (element 0), queued only."""
        out = torch.empty(2, dtype=torch.float64, device=psi.device)
        sc = N.scratch(self.n, psi.device)
        N.check(N.lib().desv_norm2(ctypes.c_void_p(psi.data_ptr()), self.n, N.dtype_code(psi),
                                   ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8,
                                   ctypes.c_void_p(N.stream_ptr())), 'norm')
        return out

    def hamiltonian(self, h):
        """('pauli', PauliPlan) or ('dense', tensor)."""
        if isinstance(h, PauliSumOperator):
            return 'pauli', plan_for(h.terms, self.n, h.n_qubits, self.dtype)
        if isinstance(h, PauliPlan):
            return 'pauli', h
        if isinstance(h, (list, tuple)):
            return 'pauli', plan_for(list(h), self.n, None, self.dtype)
        t = h if isinstance(h, torch.Tensor) else torch.from_numpy(np.asarray(h))
        return 'dense', t.to(device=self._device(), dtype=self.dtype)

    def apply_h(self, h, psi: torch.Tensor, need_lambda: bool):
        """(lambda or None, energy float)."""
        kind, H = self.hamiltonian(h)
        if kind == 'pauli':
            if need_lambda:
                lam, e = H.matvec(psi, want_expect=True)
                return lam, float(e[0].item())
            return None, float(H.expect(psi)[0].item())
        lam = H @ psi
        e = float(torch.vdot(psi.to(torch.complex128), lam.to(torch.complex128)).real.item())
        return (lam if need_lambda else None), e

    # ------------------------------------------------------------ gradient
    def gradient(self, theta: np.ndarray, psi: torch.Tensor, lam: torch.Tensor) -> np.ndarray:
        """dE/dtheta by the adjoint method; psi is not modified, lam is consumed."""
        return self._gradient_device(theta, psi, lam)[:self.nparams].cpu().numpy()

    def _gradient_device(self, theta: np.ndarray, psi: torch.Tensor, lam: torch.Tensor) -> torch.Tensor:
        """The gradient as a float64 device tensor (launches only, no host read)."""
        mu = psi.clone()
        grad = torch.zeros(max(self.nparams, 1), dtype=torch.float64, device=psi.device)
        if self.back is None:
            self._gradient_per_gate(theta, mu, lam, grad)
        else:
            self._gradient_fused(theta, mu, lam, grad)
        return grad

    def _staged(self, name: str, data: np.ndarray, dev) -> torch.Tensor:
        """data's bytes in a device buffer, copied from a pinned host buffer
        without blocking the host (stream-ordered after the work already
        queued); the pinned buffer is reused once its last copy has ended."""
        raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
        nb = max(int(raw.size), 1)
        ent = self._stage.get(name)
        if ent is None or ent[0].numel() < nb or ent[1].device != dev:
            cap = max(nb, 4096)
            ent = (torch.empty(cap, dtype=torch.uint8, pin_memory=True), torch.empty(cap, dtype=torch.uint8,
                                                                                      device=dev),
                   torch.cuda.Event())
            self._stage[name] = ent
        host, devbuf, ev = ent
        ev.synchronize()
        host[:raw.size].numpy()[:] = raw
        devbuf[:raw.size].copy_(host[:raw.size], non_blocking=True)
        ev.record()
        return devbuf

    def _device_values(self, dev):
        """Recipes, constants and event tables that build the backward passes'
        values on the device from theta (complex64 tangent-form programs):
        the host then uploads only theta and one byte per pass.  False when a
        record has no recipe (a controlled parametric diagonal, a dense 4x4)."""
        if self._dv is not None:
            return self._dv
        self._dv = False
        if not self._use_tangent:
            return False
        from ..batch import _Plan
        cdt = np.complex64
        generic = self.back.materialize(0.37 + 0.0137 * np.arange(max(self.nparams, 1)), cdt)
        try:
            recipes = _Plan._recipes(self.back, 0)
        except (RuntimeError, KeyError):
            return False
        if self._tangent is None:
            self._tangent = TangentPlan(self.back, len(generic), generic)
        tp = self._tangent
        begin, kinds, offs = [0], [], []
        for tan, events in tp.passes:
            if tan:
                for kind, off, x in events:
                    kinds.append((0 if x == 'rot' else 1) if kind == 't' else (3 if x else 2))
                    offs.append(off)
            begin.append(len(kinds))

        def up(a):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)

        npass = len(self.back.passes)
        self._dv = dict(
            generic=generic, recipes=up(recipes), nrec=len(recipes),
            cpool=torch.from_numpy(generic.view(np.float32).copy()).to(dev),
            pool=torch.empty(len(generic) + npass, dtype=torch.complex64, device=dev),
            ev_begin=up(np.array(begin, np.int32)), ev_kind=up(np.array(kinds or [0], np.uint8)),
            ev_off=up(np.array(offs or [0], np.uint32)), flags=torch.empty(npass, dtype=torch.uint8, device=dev))
        return self._dv

    def _upload_backward_device(self, theta, dev, dv):
        key = np.asarray(theta, dtype=np.float64).tobytes()
        if self._back_dev is not None and self._back_dev[0] == key:
            return self._back_dev
        th = np.zeros(max(self.nparams, 1))
        t = np.asarray(theta, dtype=np.float64).reshape(-1)[:th.size]
        th[:t.size] = t
        allowed = self._tangent.allowed(th)
        ops_t = self._staged('ops', self.back.ops, dev)
        th_t = self._staged('theta', th, dev)
        al_t = self._staged('allowed', allowed.astype(np.uint8), dev)
        vp = ctypes.c_void_p
        st = vp(N.stream_ptr())
        pool = dv['pool']
        N.check(N.lib().desv_rows_prepare(None, self.n, N.DESV_C64, 1, vp(dv['recipes'].data_ptr()), dv['nrec'],
                                          vp(th_t.data_ptr()), th.size, vp(dv['cpool'].data_ptr()),
                                          vp(pool.data_ptr()), pool.numel(), st), 'backward values')
        N.check(N.lib().desv_rows_tangent_prepare(vp(pool.data_ptr()), N.DESV_C64, 1, pool.numel(),
                                                  len(self.back.passes), vp(dv['ev_begin'].data_ptr()),
                                                  vp(dv['ev_kind'].data_ptr()), vp(dv['ev_off'].data_ptr()),
                                                  self._tangent.end_base, TangentPlan.TMAX, vp(al_t.data_ptr()),
                                                  vp(dv['flags'].data_ptr()), st), 'backward tangent form')
        if self._map_dev is None or self._map_dev.device != dev:
            self._map_dev = torch.tensor(self.back.param_map or [0], dtype=torch.int32, device=dev)
        self._back_dev = (key, ops_t, pool, self._map_dev, dv['generic'], [bool(x) for x in allowed])
        return self._back_dev

    def _upload_backward(self, theta, dev):
        dv = self._device_values(dev) if self._use_tangent else False
        if dv:
            return self._upload_backward_device(theta, dev, dv)
        return self._upload_backward_host(theta, dev)

    def _upload_backward_host(self, theta, dev):
        """(key, ops, mats, map, host mats) of the backward passes for theta;
        the host work and the uploads do not wait for the device, so they
        overlap forward passes already queued."""
        key = np.asarray(theta, dtype=np.float64).tobytes()
        if self._back_dev is not None and self._back_dev[0] == key:
            return self._back_dev
        cdt = np.complex64 if self.dtype == torch.complex64 else np.complex128
        mats = self.back.materialize(theta, cdt)
        ops_t = self._staged('ops', self.back.ops, dev)
        flags = None
        up = mats
        if self._use_tangent:
            if self._tangent is None:
                self._tangent = TangentPlan(self.back, len(mats),
                                            self.back.materialize(0.37 + 0.0137 * np.arange(max(self.nparams, 1)),
                                                                  cdt))
            up, flags = self._tangent.transform(mats)
        mats_t = self._staged('mats', up, dev)
        if self._map_dev is None or self._map_dev.device != dev:
            self._map_dev = torch.tensor(self.back.param_map or [0], dtype=torch.int32, device=dev)
        self._back_dev = (key, ops_t, mats_t, self._map_dev, mats, flags)
        return self._back_dev

    def _gradient_fused(self, theta, mu, lam, grad):
        dev = mu.device
        _, ops_t, mats_t, map_t, mats, flags = self._upload_backward(theta, dev)
        need = int(N.lib().desv_adjoint_scratch_bytes(max(self.back.max_params, 1)))
        if self._scratch is None or self._scratch.numel() * 8 < need:
            self._scratch = torch.empty((need + 7) // 8, dtype=torch.float64, device=dev)
        p = self.back.passes
        if jit.enabled(self.n) and self.dtype == torch.complex64:
            # plan-specialised backward passes (complex64: the complex128 pair of
            # register tiles does not fit the register file); sources, and so
            # kernels, change only with the records' dispatch codes
            # the sources (and so the kernels) depend on the op records and on the
            # pool values of generator and X records (jit.value_key), none of which
            # change with the angles: reuse them while those stay the same
            import hashlib
            okey = (hashlib.sha1(self.back.ops.tobytes()).hexdigest(), jit.value_key(self.back.ops, mats), dev.index)
            dix = dev.index if dev.index is not None else torch.cuda.current_device()
            if getattr(self, '_adj_kernels', None) is None or self._adj_kernels[0] != okey:
                kt = None
                if flags is not None:
                    info = self._tangent.sources_info()
                    kt = jit.compile_adjoint(self.back.ops, p, mats, True, dix, tangents=info)
                    kt = [k if inf is not None else None for k, inf in zip(kt, info)]
                # the general kernels of every pass as well: a pass whose angles
                # leave the tangent range (near theta = pi) runs in the general form,
                # and which passes do changes with every theta
                kg = jit.compile_adjoint(self.back.ops, p, mats, self.dtype == torch.complex64, dix)
                self._adj_kernels = (okey, kg, kt)
            _, kg, kt = self._adj_kernels
            kernels = list(kg)
            if kt is not None:
                for i, (use, k) in enumerate(zip(flags, kt)):
                    if use and k is not None:
                        kernels[i] = k
            jit.run_adjoint(kernels, mu.data_ptr(), lam.data_ptr(), self.n, N.dtype_code(mu), p, ops_t.data_ptr(),
                            mats_t.data_ptr(), map_t.data_ptr(), grad.data_ptr(), self._scratch.data_ptr(),
                            self._scratch.numel() * 8, N.stream_ptr())
            return
        N.check(N.lib().desv_adjoint_passes(
            ctypes.c_void_p(mu.data_ptr()), ctypes.c_void_p(lam.data_ptr()), self.n, N.dtype_code(mu),
            ctypes.c_void_p(p.ctypes.data), len(p), ctypes.c_void_p(ops_t.data_ptr()),
            ctypes.c_void_p(mats_t.data_ptr()), ctypes.c_void_p(map_t.data_ptr()), ctypes.c_void_p(grad.data_ptr()),
            ctypes.c_void_p(self._scratch.data_ptr()), self._scratch.numel() * 8,
            ctypes.c_void_p(N.stream_ptr())), 'adjoint passes')

    def _gradient_per_gate(self, theta, mu, lam, grad):
        st = ctypes.c_void_p(N.stream_ptr())
        tmp = torch.empty_like(mu)
        inner = torch.empty((len(self.bops), 2), dtype=torch.float64, device=mu.device)
        sc = N.scratch(self.n, mu.device)
        probes = []
        for i, op in enumerate(self.bops):
            if op.kind in ('g1', 'gd'):
                tmp.copy_(mu)
                m = op.matrix(theta)
                if op.kind == 'g1':
                    bits, full = [op.t], m
                else:
                    bits, full = [op.t, op.t2], np.diag(m)     # row = bit(t) + 2 bit(t2)
                mat = np.ascontiguousarray(np.asarray(full, dtype=np.complex128).reshape(-1)).view(np.float64)
                tb = (ctypes.c_int * len(bits))(*bits)
                N.check(N.lib().desv_apply_gate(ctypes.c_void_p(tmp.data_ptr()), self.n, N.dtype_code(tmp),
                                                len(bits), tb, 0, 0, ctypes.c_void_p(mat.ctypes.data), st),
                        'apply generator')
                row = inner[i]
                N.check(N.lib().desv_inner(ctypes.c_void_p(lam.data_ptr()), ctypes.c_void_p(tmp.data_ptr()), self.n,
                                           N.dtype_code(mu), ctypes.c_void_p(row.data_ptr()),
                                           ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8, st), 'inner')
                probes.append((op.src[0].slot, i))
            else:
                apply_fop(mu, self.n, op, theta, st)
                apply_fop(lam, self.n, op, theta, st)
        if probes:
            vals = inner[:, 0].cpu().numpy()
            acc = np.zeros(grad.numel())
            for s_, i in probes:
                acc[s_] += 2.0 * vals[i]
            grad += torch.from_numpy(acc).to(grad.device)

    # ------------------------------------------------------------ public
    def energy(self, theta, h, stato_zero=None, noise=None):
        """(E as a float64 tensor -- differentiable when theta requires grad, psi).

        ``noise`` (a NoiseSpec-like object: model, p, jax_key, qubits) applies one
        stochastic Kraus shot to the circuit's output state before the energy,
        as the reference's energy_fn does (solvers/autodiff.py:159-164).  For the
        Pauli channels the shot is a fixed Pauli string P, so E = <psi|P H P|psi>
        and the adjoint gradient runs with lambda = P H P psi; the damping
        channels are not differentiable here."""
        if isinstance(theta, torch.Tensor) and theta.requires_grad:
            box = {}
            e = _EnergyFunction.apply(theta, self, h, stato_zero, box, noise)
            return e, box['sv']
        th = _as_theta(theta)
        if noise is not None and self._fused_noise_applies(noise):
            psi = self._noisy_state(th, stato_zero, noise)
            _, e = self.apply_h(h, psi, need_lambda=False)
            return torch.tensor(e, dtype=torch.float64), psi
        psi = self.forward_state(th, stato_zero)
        if noise is not None:
            psi, _ = self.apply_noise(psi, noise)
            ratio = 1.0        # the noisy state is normalised in FP64 already
        else:
            ratio = self.norm_ratio(psi, stato_zero)
        _, e = self.apply_h(h, psi, need_lambda=False)
        return torch.tensor(e * ratio, dtype=torch.float64), psi

    # ------------------------------------------------------------ noise in the circuit's passes
    @staticmethod
    def _fused_noise_applies(noise) -> bool:
        from ..noise import kraus_channels as K
        return noise.model in K.PAULI_MODELS and float(noise.p) > 0.0

    def _noise_template(self, model: str, bits):
        """(CompiledCircuit, slot of every (bit, letter), gphase slot): the
        circuit followed by a parametric Pauli template on the noise qubits --
        per noise qubit rx / ry / rz (depolarizing), rx (bitflip) or rz
        (phaseflip), then one gphase -- compiled once per (model, qubits), so
        the template's gates ride in the circuit's own passes.  A fired error w
        on bit q sets its gate's angle to pi (X = i Rx(pi), Y = i Ry(pi),
        Z = i Rz(pi)) and adds pi/2 to the gphase angle; every other angle is 0."""
        key = (model, tuple(bits))
        cache = self.__dict__.setdefault('_noise_tpl', {})
        got = cache.get(key)
        if got is not None:
            return got
        letters = 'xyz' if model == 'depolarizing' else ('x' if model == 'bitflip' else 'z')
        rows, slots = list(self.rows), list(self.slots)
        k = max(self.nparams, 1 + max(slots, default=-1))
        where = {}
        for q in bits:
            for w in letters:
                rows.append((f'r{w}', self.n - 1 - int(q), 0.0))
                slots.append(k)
                where[(int(q), w)] = k
                k += 1
        rows.append(('gphase', 0, 0.0))
        slots.append(k)
        got = (CompiledCircuit(rows, self.n, self.dtype, slots=slots), where, k)
        cache[key] = got
        return got

    def _noisy_state(self, th: np.ndarray, stato_zero, noise) -> torch.Tensor:
        """The circuit's output under one Pauli-channel shot, normalised as the
        reference does (division by norm + 1e-15): the drawn errors are the
        angles of the noise template, so they are applied inside the circuit's
        passes instead of as passes of their own over a copy."""
        from ..noise import kraus_channels as K
        rng = K.resolve_rng(getattr(noise, 'rng', None), getattr(noise, 'jax_key', None))
        qubits = list(noise.qubits) if getattr(noise, 'qubits', None) is not None else list(range(self.n))
        errs = K.draw_pauli_errors(noise.model, float(noise.p), self.n, rng, qubits)
        cc, where, gslot = self._noise_template(noise.model, qubits)
        full = np.zeros(gslot + 1)
        full[:min(th.size, gslot + 1)] = th[:gslot + 1]
        for q, w in errs:
            full[where[(int(q), w)]] = np.pi
        full[gslot] = 0.5 * np.pi * len(errs)
        psi = self.initial_state(stato_zero)
        cc.run(psi, theta=full)
        K.normalize_plus_eps(psi)
        return psi

    def apply_noise(self, psi: torch.Tensor, noise):
        """(noisy normalised copy of psi, Pauli errors or None for damping channels)."""
        from ..noise import kraus_channels as K
        model, p = noise.model, float(noise.p)
        out = psi.clone()
        if model == 'ideal' or p <= 0.0:
            return out, []
        if model not in K.MODELS:
            raise KeyError(model)
        rng = K.resolve_rng(getattr(noise, 'rng', None), getattr(noise, 'jax_key', None))
        qubits = list(noise.qubits) if getattr(noise, 'qubits', None) is not None else None
        if model in K.PAULI_MODELS:
            errs = K.draw_pauli_errors(model, p, self.n, rng, qubits)
            K.apply_pauli_errors(out, self.n, errs)
            K.normalize_plus_eps(out)
            return out, errs
        K.apply_channel(out, self.n, model, p, rng, qubits)
        K.normalize_plus_eps(out)
        return out, None

    def value_and_grad(self, theta, h, stato_zero=None):
        """(E, dE/dtheta as NumPy float64, psi) without autograd bookkeeping.

        Everything is queued before the host reads anything: the forward
        passes, then (on the host, while they run) the backward passes' values
        and their upload, then <psi|psi>, lambda = H psi with E, and the backward
        sweep; one read at the end brings E, the norm and the gradient back."""
        th = _as_theta(theta)
        if self.back is None:
            psi = self.forward_state(th, stato_zero)
            ratio = self.norm_ratio(psi, stato_zero)
            lam, e = self.apply_h(h, psi, need_lambda=True)
            return e * ratio, self.gradient(th, psi, lam) * ratio, psi
        psi = self.forward_state(th, stato_zero)
        self._upload_backward(th, psi.device)
        nrm = self._norm_device(psi) if self.dtype == torch.complex64 else None
        kind, H = self.hamiltonian(h)
        if kind == 'pauli':
            lam, e_dev = H.matvec(psi, want_expect=True)
        else:
            lam = H @ psi
            e_dev = torch.vdot(psi.to(torch.complex128), lam.to(torch.complex128)).real.reshape(1)
        grad = self._gradient_device(th, psi, lam)
        parts = [e_dev.reshape(-1)[:1].to(torch.float64),
                 nrm[:1] if nrm is not None else torch.ones(1, dtype=torch.float64, device=psi.device),
                 grad[:self.nparams]]
        vals = torch.cat(parts).cpu().numpy()
        ratio = 1.0
        if nrm is not None:
            n0 = self._initial_norm2(stato_zero)
            ratio = n0 / vals[1] if vals[1] > 0 else 1.0
        return float(vals[0]) * ratio, vals[2:] * ratio, psi

    def parameter_shift_grad(self, theta, h, stato_zero=None) -> np.ndarray:
        """Parameter-shift gradient on the same kernels: two forward runs + <H> per
        parameter (+-pi/2 for rx/ry/rz/p/u1/cp; four-term rule for crz)."""
        th = _as_theta(theta)
        kinds = {}
        for g in self.ir:
            if g.slot >= 0:
                kinds[g.slot] = g.name

        def f(t):
            psi = self.forward_state(t, stato_zero)
            return self.apply_h(h, psi, need_lambda=False)[1] * self.norm_ratio(psi, stato_zero)

        grad = np.zeros(self.nparams)
        for k in range(self.nparams):
            e = np.zeros(self.nparams)
            e[k] = 1.0
            if kinds.get(k) == 'crz':
                c1 = (np.sqrt(2) + 1) / (4 * np.sqrt(2))
                c2 = (np.sqrt(2) - 1) / (4 * np.sqrt(2))
                grad[k] = c1 * (f(th + np.pi / 2 * e) - f(th - np.pi / 2 * e)) - \
                    c2 * (f(th + 3 * np.pi / 2 * e) - f(th - 3 * np.pi / 2 * e))
            else:
                grad[k] = 0.5 * (f(th + np.pi / 2 * e) - f(th - np.pi / 2 * e))
        return grad


def _as_theta(theta) -> np.ndarray:
    if isinstance(theta, torch.Tensor):
        return theta.detach().cpu().numpy().astype(np.float64).reshape(-1)
    return np.asarray(theta, dtype=np.float64).reshape(-1)


def _split_params(specs, ops, cap):
    """Keep every pass at <= cap distinct gradient slots (split stage lists)."""
    out = []
    for ps in specs:
        cur, seen = [], set()
        for g, ids in ps.stages:
            slots = {ops[i].src[0].slot for i in ids if ops[i].kind in ('g1', 'gd')}
            if cur and len(seen | slots) > cap:
                out.append(fusion.PassSpec(ps.K, ps.L, ps.high, cur))
                cur, seen = [], set()
            cur.append((g, ids))
            seen |= slots
        out.append(fusion.PassSpec(ps.K, ps.L, ps.high, cur))
    return out


# Backward passes with more op records than the code generator takes
# (jit.MAX_OPS) would run on the interpreter.  Splitting them into passes of
# at most this many gates keeps every pass specialised: measured on the
# 24-qubit, 10-layer ansatz, the first backward pass (330 records, the last
# layers of the circuit) took 15.8 ms interpreted, and the gradient went from
# 30.0 ms to 19.4 ms (cap 60) and 17.5 ms (cap 40).
SPECIALISED_OPS_PER_PASS = 40


def ops_per_pass() -> int:
    """SPECIALISED_OPS_PER_PASS, or DESV_ADJ_OPS_PER_PASS (tuning sweeps)."""
    import os
    v = int(os.environ.get('DESV_ADJ_OPS_PER_PASS', SPECIALISED_OPS_PER_PASS))
    if not 8 <= v <= 90:
        raise ValueError('DESV_ADJ_OPS_PER_PASS must be in [8, 90]')
    return v


def _split_ops(specs, cap):
    """Split passes (and, where needed, their stages, keeping the gate order)
    so that every pass holds at most cap gates; each piece keeps its pass's
    tile geometry, so it is a valid pass of its own."""
    out = []
    for ps in specs:
        cur, cnt = [], 0
        for g, ids in ps.stages:
            ids = list(ids)
            while ids:
                if cnt >= cap:
                    out.append(fusion.PassSpec(ps.K, ps.L, ps.high, cur))
                    cur, cnt = [], 0
                take = ids[:cap - cnt]
                cur.append((g, take))
                cnt += len(take)
                ids = ids[len(take):]
        if cur:
            out.append(fusion.PassSpec(ps.K, ps.L, ps.high, cur))
    return out


class _EnergyFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta_t, prog: AdjointProgram, h, stato_zero, box, noise=None):
        from ..noise import kraus_channels as K
        th = _as_theta(theta_t)
        psi = prog.forward_state(th, stato_zero)
        ctx.differentiable = True
        ctx.ratio = 1.0
        if noise is None:
            lam, e = prog.apply_h(h, psi, need_lambda=True)
            ctx.ratio = prog.norm_ratio(psi, stato_zero)
            e *= ctx.ratio
            box['sv'] = psi
        else:
            noisy, errs = prog.apply_noise(psi, noise)
            lam, e = prog.apply_h(h, noisy, need_lambda=True)
            box['sv'] = noisy
            if errs is None:
                ctx.differentiable = False
            else:
                # E = <psi|P H P|psi> (up to the (1 + 1e-15)^-2 of the final
                # normalisation): lambda = P H (P psi); P is Hermitian
                K.apply_pauli_errors(lam, prog.n, errs)
        ctx.prog, ctx.th, ctx.psi, ctx.lam = prog, th, psi, lam
        ctx.tdev, ctx.tdtype = theta_t.device, theta_t.dtype
        return torch.tensor(e, dtype=torch.float64, device=theta_t.device)

    @staticmethod
    def backward(ctx, g):
        if not ctx.differentiable:
            raise NotImplementedError('the gradient through an amplitude-damping channel (amplitude_damping, '
                                      'combined) is not supported; the Pauli channels are')
        grad = ctx.prog.gradient(ctx.th, ctx.psi, ctx.lam) * ctx.ratio
        gt = torch.from_numpy(grad).to(device=ctx.tdev, dtype=ctx.tdtype)
        return g * gt, None, None, None, None, None
