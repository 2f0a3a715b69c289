"""Batched VQE: energy and adjoint gradient of many independent circuits of
uneven qubit count in one persistent GPU launch (``desv_batch_vqe``), optionally
replayed from a captured CUDA graph.

The reference evaluates one parameter row of one circuit shape at a time
(``run_batch_jit`` vmaps a single structure at a single qubit count,
``backends/statevector.py:496-584``; gradients come from ``jax.grad`` per
circuit, ``solvers/autodiff.py:92-169``).  Here:

* circuits sharing a structure (gate list + Pauli term structure) share one
  plan -- forward fused passes and adjoint fused passes from the same fusion
  pass as single circuits (1-qubit gates unmerged so that every op's matrix
  can be rebuilt from theta on the device);
* each circuit brings its theta and its real term coefficients (e.g. its own
  J_z of an XXZ chain);
* circuits of <= 12 qubits are ordered by decreasing cost and pulled from an
  atomic queue, one per CTA, in one persistent launch; their states never
  leave shared memory;
* wider circuits run as rows: all circuits of one structure form one set of
  full-width states back to back, and every pass (forward, H psi with the
  energy, adjoint with the gradient) covers all of them in one launch over
  all SMs, with each row's own matrix pool (built from its theta on the
  device) and its own term coefficients.

Parameters are injected like the energy functions: into rx/ry/rz/u1/p/cp/crz
in gate order (``solvers/autodiff.py:21,150-157``).
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from . import _native as N
from .circuits import fusion
from .physics.observables import _normalize_terms
from .solvers import adjoint
from .solvers.autodiff import build_template

RESIDENT_BITS = 12

RCP = dict(CONST=0, RX=1, RY=2, RZ=3, P=4, RZ_TAB=5, P_TAB=6, CP_VEC=7, CRZ_VEC=8, PHASE_VEC=9)
RCP_INVERSE = 0x100

RECIPE_DTYPE = np.dtype([('off', '<u4'), ('param', '<i4'), ('kind', '<u2'), ('count', '<u2'), ('src', '<u4')])
PLAN_DTYPE = np.dtype([(k, '<i4') for k in ('n', 'fwd_begin', 'fwd_end', 'bwd_begin', 'bwd_end', 'rec_begin',
                                            'rec_end', 'term_begin', 'term_end', 'nparams', 'pool_len', 'pad')])
CIRC_DTYPE = np.dtype([('plan', '<i4'), ('out_index', '<i4'), ('theta_off', '<i8'), ('coef_off', '<i8'),
                       ('grad_off', '<i8'), ('state_off', '<i8')])
assert RECIPE_DTYPE.itemsize == 16 and PLAN_DTYPE.itemsize == 48 and CIRC_DTYPE.itemsize == 40


class BatchArgs(ctypes.Structure):
    """ctypes mirror of desv_batch_args (include/desv.h)."""
    _fields_ = [('ncirc', ctypes.c_int32), ('pad', ctypes.c_int32), ('circuits', ctypes.c_void_p),
                ('plans', ctypes.c_void_p), ('passes', ctypes.c_void_p), ('ops', ctypes.c_void_p),
                ('recipes', ctypes.c_void_p), ('cpool', ctypes.c_void_p), ('theta', ctypes.c_void_p),
                ('coef', ctypes.c_void_p), ('terms', ctypes.c_void_p), ('energy', ctypes.c_void_p),
                ('grad', ctypes.c_void_p), ('workspace', ctypes.c_void_p), ('ws_amps', ctypes.c_uint64),
                ('pool_ws', ctypes.c_void_p), ('pool_stride_bytes', ctypes.c_uint64), ('states', ctypes.c_void_p)]


def _term_structure(terms, n):
    """[(xmask, zmask, i^nY)] and real coefficients of a Pauli term list."""
    st, coef = [], []
    for c, p in terms:
        t = _normalize_terms(p, None)
        if t and max(t) >= n:
            raise ValueError(f"term references qubit {max(t)}, but the circuit has {n} qubits")
        x = z = ny = 0
        for q, l in t.items():
            b = 1 << (n - 1 - q)
            if l in ('X', 'Y'):
                x |= b
            if l in ('Y', 'Z'):
                z |= b
            ny += l == 'Y'
        ph = 1j ** ny
        if complex(c).imag != 0:
            raise ValueError('batched VQE takes real term coefficients')
        st.append((x, z, ph.real, ph.imag))
        coef.append(float(np.real(c)))
    return tuple(st), coef


class _Plan:
    """Forward + adjoint passes and matrix recipes of one circuit structure."""

    def __init__(self, rows, slots, n, term_struct, dtype, tile_bits=None, forward_only: bool = False):
        if n < fusion.MIN_FUSED_QUBITS:
            raise ValueError(f'batched VQE needs at least {fusion.MIN_FUSED_QUBITS} qubits per circuit')
        self.n = n
        self.nparams = 1 + max([s for s in slots if s >= 0], default=-1)
        # a resident state (<= 12 qubits) is one tile; wider states stream tiles of
        # the tuned width
        K = n if n <= RESIDENT_BITS else min(n, tile_bits or RESIDENT_BITS)
        self.K = K
        ir = fusion.lower(rows, n, slots)
        fops = fusion.fuse_1q(ir, merge=False)
        self.fwd = fusion.Packed(n, fops, fusion.schedule(fops, n, K))
        bops = [] if forward_only else adjoint.backward_ops(ir)
        self.bwd = fusion.Packed(n, bops, adjoint._split_params(fusion.schedule(bops, n, K), bops, 4096)
                                 if bops else [], adjoint=True)
        for p in list(self.fwd.passes) + list(self.bwd.passes):
            if int(p['tile_bits']) != (n if n <= RESIDENT_BITS else K):
                raise RuntimeError('batched plan: unexpected tile geometry')
        cdt = np.complex64 if dtype == torch.complex64 else np.complex128
        th0 = 0.37 + 0.0137 * np.arange(max(self.nparams, 1))   # generic angles: flags valid for every theta
        fpool = self.fwd.materialize(th0, cdt)
        bpool = self.bwd.materialize(th0, cdt)
        self.fwd_len = len(fpool)
        self.pool_len = len(fpool) + len(bpool)
        self.cpool = np.concatenate([fpool, bpool])
        # adjoint records: GRAD param -> theta index, matrices after the forward pool
        bops_arr = self.bwd.ops
        for ps in self.bwd.passes:
            for r in range(int(ps['op_begin']), int(ps['op_end'])):
                if bops_arr[r]['kind'] == N.OP_GRAD:
                    bops_arr[r]['param'] = self.bwd.param_map[int(ps['map_begin']) + int(bops_arr[r]['param'])]
        is_rec = bops_arr['kind'] != N.OP_STAGE
        bops_arr['mat'][is_rec] += self.fwd_len
        self.recipes = np.concatenate([self._recipes(self.fwd, 0), self._recipes(self.bwd, self.fwd_len)])
        self.term_struct = term_struct

    @staticmethod
    def _recipes(packed, base):
        V = packed._vec
        out = np.zeros(V['R'], RECIPE_DTYPE)
        for r, (rec_i, fi) in enumerate(packed.op_slots):
            op = packed.fops[fi]
            g = op.src[0]
            kind_out, tf = int(V['out'][r]), int(V['tf'][r])
            off = int(V['off'][r])
            count = 16 if kind_out == 3 else 4
            out[r]['off'] = base + off
            out[r]['src'] = base + off
            out[r]['count'] = count
            out[r]['param'] = -1
            if tf == 2 or g.slot < 0 or len(op.src) != 1:
                out[r]['kind'] = RCP['CONST']
                continue
            name = g.name
            if kind_out == 0:
                k = {'rx': 'RX', 'ry': 'RY', 'rz': 'RZ', 'p': 'P', 'u1': 'P', 'phase': 'P'}[name]
            elif kind_out == 1:
                if int(V['ctl'][r]) != -1:
                    raise RuntimeError('batched plan: controlled parametric diagonal')
                k = {'rz': 'RZ_TAB', 'p': 'P_TAB', 'u1': 'P_TAB', 'phase': 'P_TAB'}[name]
            elif kind_out == 2:
                k = {'cp': 'CP_VEC', 'cphase': 'CP_VEC', 'crz': 'CRZ_VEC', 'gphase': 'PHASE_VEC'}[name]
            else:
                raise RuntimeError('batched plan: parametric dense 4x4')
            out[r]['kind'] = RCP[k] | (RCP_INVERSE if tf == 1 else 0)
            out[r]['param'] = g.slot
        return out

    @property
    def cost(self):
        return (1 << self.n) * (len(self.fwd.ops) + 2 * len(self.bwd.ops))


class _RowsPlan:
    """One circuit structure planned for the rows path: every row (parameter
    set) of the structure is a full-width state of its own, and each pass runs
    over all rows in one launch over all SMs (``desv_apply_passes_rows``,
    ``desv_pauli_matvec_rows``, ``desv_adjoint_passes_rows``).  Forward passes
    use tiles of ``tile_bits``; adjoint passes the single-circuit adjoint tile
    width; matrices come from theta on the device (recipes), one pool per row."""

    def __init__(self, rows, slots, n, dtype, tile_bits, terms=None, forward_only: bool = False, use_jit=None):
        import os
        from .circuits import jit
        if use_jit is None:
            use_jit = os.environ.get('DESV_JIT', '') != '0' and jit.available()
        self.use_jit = bool(use_jit)
        self._kernels = {}
        n = int(n)
        if n < fusion.MIN_FUSED_QUBITS:
            raise ValueError(f'rows path needs at least {fusion.MIN_FUSED_QUBITS} qubits per circuit')
        self.n = n
        self.dtype = dtype
        self.nparams = 1 + max([s for s in slots if s >= 0], default=-1)
        K = min(n, int(tile_bits))
        ir = fusion.lower(rows, n, slots)
        fops = fusion.fuse_1q(ir, merge=False)
        self.fwd = fusion.Packed(n, fops, fusion.schedule(fops, n, K))
        if forward_only:
            self.bwd = None
        else:
            bops = adjoint.backward_ops(ir)
            kb = adjoint._adjoint_tile_bits(n, dtype)
            specs = adjoint._split_params(fusion.schedule(bops, n, kb), bops, 1024) if bops else []
            if self.use_jit and dtype == torch.complex64:
                # every backward pass short enough for a specialised kernel
                specs = adjoint._split_ops(specs, adjoint.ops_per_pass())
            self.bwd = fusion.Packed(n, bops, specs, adjoint=True)
        cdt = np.complex64 if dtype == torch.complex64 else np.complex128
        th0 = 0.37 + 0.0137 * np.arange(max(self.nparams, 1))   # generic angles: flags valid for every theta
        fpool = self.fwd.materialize(th0, cdt)
        self.fwd_len = len(fpool)
        recs = [_Plan._recipes(self.fwd, 0)]
        pools = [fpool]
        if self.bwd is not None:
            bpool = self.bwd.materialize(th0, cdt)
            bops_arr = self.bwd.ops
            is_rec = bops_arr['kind'] != N.OP_STAGE
            bops_arr['mat'][is_rec] += self.fwd_len
            recs.append(_Plan._recipes(self.bwd, self.fwd_len))
            pools.append(bpool)
        self.cpool = np.concatenate(pools)
        self.recipes = np.concatenate(recs)
        # tangent form of the backward passes (complex64, specialised kernels):
        # the events the device walks per pass and row, and one pass-end factor
        # per backward pass after the pool
        self.tangent = None
        extra = 0
        if self.use_jit and dtype == torch.complex64 and self.bwd is not None and len(self.bwd.passes) and \
                os.environ.get('DESV_ADJ_TANGENT', '1') != '0':
            tp = adjoint.TangentPlan(self.bwd, len(self.cpool), self.cpool.astype(np.complex64))
            if any(t for t, _ in tp.passes):
                self.tangent = tp
                extra = len(self.bwd.passes)
                begin, kinds, offs = [0], [], []
                for tan, events in tp.passes:
                    if tan:
                        for kind, off, x in events:
                            kinds.append((0 if x == 'rot' else 1) if kind == 't' else (3 if x else 2))
                            offs.append(off)
                    begin.append(len(kinds))
                self.ev_begin = np.array(begin, np.int32)
                self.ev_kind = np.array(kinds or [0], np.uint8)
                self.ev_off = np.array(offs or [0], np.uint32)
        # every row's pool starts on a 256-byte boundary
        per = 256 // (8 if dtype == torch.complex64 else 16)
        self.pool_stride = max(per, (len(self.cpool) + extra + per - 1) // per * per)
        self.pauli = None
        if terms is not None and not forward_only:
            from .physics.observables import plan_for
            self.pauli = plan_for([(1.0, p) for _, p in terms], n, None, dtype, wide_tiles=self.use_jit)

    def kernels(self, device: int):
        """(forward, backward) lists of specialised kernels per pass (None: that
        pass runs on the interpreter), compiled once per device.  The sources
        read only pool values that no angle changes (generator and constant
        records), so one set serves every row.  complex128 backward passes stay
        on the interpreter (two double2 register tiles exceed the register file)."""
        if not self.use_jit:
            return None, None, None
        got = self._kernels.get(device)
        if got is None:
            from .circuits import jit
            c64 = self.dtype == torch.complex64
            kf = jit.compile_passes(self.fwd.ops, self.fwd.passes, self.cpool, c64, device)
            kb = jit.compile_adjoint(self.bwd.ops, self.bwd.passes, self.cpool, c64, device) \
                if (self.bwd is not None and c64) else None
            kt = None
            if self.tangent is not None:
                info = self.tangent.sources_info()
                kt = jit.compile_adjoint(self.bwd.ops, self.bwd.passes, self.cpool, True, device, tangents=info)
                kt = [k if inf is not None else None for k, inf in zip(kt, info)]
            got = (kf, kb, kt)
            self._kernels[device] = got
        return got

    def term_rows(self, coefs: Sequence[Sequence[float]]) -> np.ndarray:
        """(rows x terms) table of Pauli term records with every row's real
        coefficients folded in, in the plan's packed term order."""
        base = self.pauli.terms
        co = np.asarray(coefs, dtype=np.float64)[:, self.pauli.order]     # (rows, terms)
        out = np.zeros((co.shape[0], max(len(base), 1)), N.TERM_DTYPE)
        if len(base):
            out['xmask'][:, :len(base)] = base['xmask']
            out['zmask'][:, :len(base)] = base['zmask']
            out['cre'][:, :len(base)] = base['cre'] * co
            out['cim'][:, :len(base)] = base['cim'] * co
        return out


def rows_forward(kernels, states: torch.Tensor, n: int, code: int, rows: int, passes: np.ndarray, d_ops: torch.Tensor,
                 pools: torch.Tensor, pool_stride: int, st):
    """Every forward pass over all rows: the specialised kernel of a pass where
    there is one, the interpreter otherwise."""
    lib, vp = N.lib(), ctypes.c_void_p
    for i in range(len(passes)):
        pp = vp(passes.ctypes.data + i * passes.itemsize)
        k = kernels[i] if kernels is not None else None
        if k is None:
            N.check(lib.desv_apply_passes_rows(vp(states.data_ptr()), n, code, rows, pp, 1, vp(d_ops.data_ptr()),
                                               vp(pools.data_ptr()), pool_stride, st), 'rows forward pass')
        else:
            N.check(lib.desv_jit_pass_rows(k.handle, vp(states.data_ptr()), n, code, rows, pp, vp(pools.data_ptr()),
                                           pool_stride, st), 'rows forward pass (jit)')


class _RowsGroup:
    """Device buffers and launches of one structure's rows: psi and lambda
    (rows x 2^n each), the per-row pools, term tables, <psi|H|psi> and
    <psi|psi>; theta and the gradient are rows of ``nparams`` at ``theta_base``
    in the batch's theta / gradient buffers.  Everything is allocated here, so
    ``launch`` only queues work (capturable in a CUDA graph)."""

    def __init__(self, plan: _RowsPlan, coefs, theta_base: int, dev, code: int):
        self.plan = plan
        self.B = B = len(coefs)
        self.code = code
        self.theta_base = theta_base
        self.P = max(plan.nparams, 1)
        n = plan.n
        rdt = np.float32 if plan.dtype == torch.complex64 else np.float64
        cdt = np.complex64 if plan.dtype == torch.complex64 else np.complex128

        def up(a):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)

        self.psi = torch.empty((B, 1 << n), dtype=plan.dtype, device=dev)
        self.lam = torch.empty((B, 1 << n), dtype=plan.dtype, device=dev)
        self.pools = torch.empty((B, plan.pool_stride), dtype=plan.dtype, device=dev)
        self.d_cpool = torch.from_numpy(plan.cpool.astype(cdt).view(rdt).copy()).to(dev)
        self.d_recipes = up(plan.recipes)
        self.fwd_passes = np.ascontiguousarray(plan.fwd.passes)
        self.d_fwd_ops = up(plan.fwd.ops if len(plan.fwd.ops) else np.zeros(1, N.OP_DTYPE))
        self.bwd_passes = np.ascontiguousarray(plan.bwd.passes)
        self.d_bwd_ops = up(plan.bwd.ops if len(plan.bwd.ops) else np.zeros(1, N.OP_DTYPE))
        self.d_map = torch.tensor(plan.bwd.param_map or [0], dtype=torch.int32, device=dev)
        tr = plan.term_rows(coefs)
        self.term_stride = tr.shape[1]
        self.d_terms = up(tr.reshape(-1))
        self.ppasses = np.ascontiguousarray(plan.pauli.passes)
        # specialised H psi kernels: a coefficient column equal in every row is
        # compiled in, the others become per-row symbols (equal columns share one)
        self.pk = None
        if plan.use_jit and len(plan.pauli.terms):
            from .circuits import jit
            co = np.asarray(coefs, dtype=np.float64)[:, plan.pauli.order]          # (rows, terms)
            terms = plan.pauli.terms.copy()
            syms, cols = [], {}
            for k in range(co.shape[1]):
                col = co[:, k]
                if np.all(col == col[0]):
                    terms['cre'][k] *= col[0]
                    terms['cim'][k] *= col[0]
                    syms.append(None)
                else:
                    syms.append(cols.setdefault(col.tobytes(), len(cols)))
            csym = np.zeros((B, max(len(cols), 1)))
            for key, i in cols.items():
                csym[:, i] = np.frombuffer(key, dtype=np.float64)
            ks = jit.compile_pauli_rows(terms, self.ppasses, syms, plan.dtype == torch.complex64,
                                        dev.index if dev.index is not None else torch.cuda.current_device())
            if any(k is not None for k in ks):
                self.pk = (ks, (ctypes.c_void_p * len(ks))(*[k.handle.value if k is not None else None for k in ks]))
                self.d_csym = torch.from_numpy(csym.reshape(-1)).to(dev)
                self.nsym = csym.shape[1]
        self.expect = torch.zeros((B, 2), dtype=torch.float64, device=dev)
        self.norm = torch.ones(B, dtype=torch.float64, device=dev)
        sb = int(N.lib().desv_rows_scratch_bytes(B, max(plan.bwd.max_params, 1), max(len(self.ppasses), 1)))
        self.scratch = torch.empty((sb + 7) // 8, dtype=torch.float64, device=dev)
        self.kf, self.kb, self.kt = plan.kernels(dev.index if dev.index is not None else torch.cuda.current_device())
        if plan.tangent is not None and self.kt is not None:
            self.d_ev_begin = torch.from_numpy(plan.ev_begin).to(dev)
            self.d_ev_kind = torch.from_numpy(plan.ev_kind).to(dev)
            self.d_ev_off = torch.from_numpy(plan.ev_off.view(np.int32)).to(dev)
            self.d_flags = torch.zeros(len(self.bwd_passes) * B, dtype=torch.uint8, device=dev)
        else:
            self.kt = None

    def launch(self, d_theta: torch.Tensor, d_grad: torch.Tensor, stream):
        p, n, B, st = self.plan, self.plan.n, self.B, ctypes.c_void_p(N.stream_ptr(stream))
        vp = ctypes.c_void_p
        theta = vp(d_theta.data_ptr() + 8 * self.theta_base)
        grad = d_grad[self.theta_base:self.theta_base + B * self.P]
        N.check(N.lib().desv_rows_prepare(vp(self.psi.data_ptr()), n, self.code, B, vp(self.d_recipes.data_ptr()),
                                          len(p.recipes), theta, self.P, vp(self.d_cpool.data_ptr()),
                                          vp(self.pools.data_ptr()), p.pool_stride, st), 'rows prepare')
        if self.kt is not None:
            N.check(N.lib().desv_rows_tangent_prepare(vp(self.pools.data_ptr()), self.code, B, p.pool_stride,
                                                      len(self.bwd_passes), vp(self.d_ev_begin.data_ptr()),
                                                      vp(self.d_ev_kind.data_ptr()), vp(self.d_ev_off.data_ptr()),
                                                      p.tangent.end_base, adjoint.TangentPlan.TMAX, None,
                                                      vp(self.d_flags.data_ptr()), st), 'rows tangent form')
        rows_forward(self.kf, self.psi, n, self.code, B, self.fwd_passes, self.d_fwd_ops, self.pools, p.pool_stride,
                     st)
        want_norm = p.dtype == torch.complex64
        args = (vp(self.psi.data_ptr()), vp(self.lam.data_ptr()), n, self.code, B, vp(self.ppasses.ctypes.data),
                len(self.ppasses), vp(self.d_terms.data_ptr()), self.term_stride, vp(self.expect.data_ptr()),
                vp(self.norm.data_ptr()) if want_norm else None, vp(self.scratch.data_ptr()),
                self.scratch.numel() * 8, st)
        if self.pk is not None:
            N.check(N.lib().desv_jit_pauli_matvec_rows(self.pk[1], vp(self.d_csym.data_ptr()), self.nsym, *args),
                    'rows H psi (jit)')
        else:
            N.check(N.lib().desv_pauli_matvec_rows(*args), 'rows H psi')
        with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
            grad.zero_()
        lib, sc, nsc = N.lib(), vp(self.scratch.data_ptr()), self.scratch.numel() * 8
        for i in range(len(self.bwd_passes)):
            pp = vp(self.bwd_passes.ctypes.data + i * self.bwd_passes.itemsize)
            k = self.kb[i] if self.kb is not None else None
            kt = self.kt[i] if self.kt is not None else None
            if kt is not None and k is not None:
                N.check(lib.desv_jit_adjoint_rows_split(kt.handle, k.handle, vp(self.d_flags.data_ptr() + i * B),
                                                        vp(self.psi.data_ptr()), vp(self.lam.data_ptr()), n, self.code,
                                                        B, pp, vp(self.d_bwd_ops.data_ptr()),
                                                        vp(self.pools.data_ptr()), p.pool_stride,
                                                        vp(self.d_map.data_ptr()), vp(grad.data_ptr()), self.P, sc, nsc,
                                                        st), 'rows adjoint pass (jit, per-row form)')
                continue
            if k is None:
                N.check(lib.desv_adjoint_passes_rows(vp(self.psi.data_ptr()), vp(self.lam.data_ptr()), n, self.code,
                                                     B, pp, 1, vp(self.d_bwd_ops.data_ptr()),
                                                     vp(self.pools.data_ptr()), p.pool_stride,
                                                     vp(self.d_map.data_ptr()), vp(grad.data_ptr()), self.P, sc, nsc,
                                                     st), 'rows adjoint pass')
            else:
                N.check(lib.desv_jit_adjoint_rows(k.handle, vp(self.psi.data_ptr()), vp(self.lam.data_ptr()), n,
                                                  self.code, B, pp, vp(self.d_bwd_ops.data_ptr()),
                                                  vp(self.pools.data_ptr()), p.pool_stride, vp(self.d_map.data_ptr()),
                                                  vp(grad.data_ptr()), self.P, sc, nsc, st), 'rows adjoint pass (jit)')


class BatchVQE:
    """Energies and adjoint gradients of many circuits in one launch.

    items: sequence of (circuit, n_qubits, terms) -- circuit as gate tuples or
    a QASMCircuit (parameters are ignored; theta is injected in gate order),
    terms as (real coefficient, Pauli term) pairs.  Circuits whose gate list
    and term structure coincide share a plan.

    Circuits of up to ``rows_from - 1`` qubits (default: those whose state fits
    one CTA's shared memory, 12 qubits) run in the persistent launch, one CTA
    each.  Wider ones run as rows: all circuits of one structure form one set
    of full-width states, and each pass runs over all of them in one launch
    over all SMs.  ``DESV_BATCH_ROWS_FROM`` overrides the default.  Rows passes
    run on plan-specialised kernels (compiled once per structure) unless
    ``rows_jit`` is False or ``DESV_JIT=0``."""

    def __init__(self, items: Sequence[Tuple], use_float32: bool = True, tile_bits=None, rows_from=None,
                 rows_jit=None):
        import os
        self.dtype = torch.complex64 if use_float32 else torch.complex128
        self.device = N.require_cuda()
        N.lib()
        if tile_bits is None:
            from . import autotune
            tile_bits = autotune.batch_tile_bits(self.dtype)
        self.tile_bits = int(tile_bits)
        if rows_from is None:
            rows_from = int(os.environ.get('DESV_BATCH_ROWS_FROM', RESIDENT_BITS + 1))
        self.rows_from = max(int(rows_from), fusion.MIN_FUSED_QUBITS)
        plans: Dict[tuple, int] = {}
        rplans: Dict[tuple, int] = {}
        self.plans: List[_Plan] = []
        self.rplans: List[list] = []     # [_RowsPlan, circuit indices, coefficient rows, nparams]
        self.circ = []          # (plan index or -1, coefficients, nparams); rows circuits: -1
        self.row_of = {}        # circuit index -> (rows group, row)
        for i, (circuit, n, terms) in enumerate(items):
            n = int(n)
            rows, slots, n_params = build_template(circuit, n)
            ts, coef = _term_structure(terms, n)
            key = (tuple(rows), tuple(slots), n, ts)
            if n >= self.rows_from:
                if key not in rplans:
                    rplans[key] = len(self.rplans)
                    self.rplans.append([_RowsPlan(rows, slots, n, self.dtype, tile_bits, terms, use_jit=rows_jit),
                                        [], [], n_params])
                g = self.rplans[rplans[key]]
                self.row_of[i] = (rplans[key], len(g[1]))
                g[1].append(i)
                g[2].append(coef)
                self.circ.append((-1, coef, n_params))
                continue
            if key not in plans:
                plans[key] = len(self.plans)
                self.plans.append(_Plan(rows, slots, n, ts, self.dtype, tile_bits))
            self.circ.append((plans[key], coef, n_params))
        self._pack()

    def _pack(self):
        pass_rows, op_rows, rec_rows, term_rows, plan_rows, cpools = [], [], [], [], [], []
        nops = npass = nrec = nterm = ncp = 0
        for p in self.plans:
            prow = np.zeros((), PLAN_DTYPE)
            prow['n'] = p.n
            fwd = p.fwd.passes.copy()
            bwd = np.zeros(len(p.bwd.passes), N.PASS_DTYPE)
            for f in ('tile_bits', 'low_bits', 'op_begin', 'op_end', 'high'):
                bwd[f] = p.bwd.passes[f]
            fwd['op_begin'] += nops
            fwd['op_end'] += nops
            nf = len(p.fwd.ops)
            bwd['op_begin'] += nops + nf
            bwd['op_end'] += nops + nf
            prow['fwd_begin'], prow['fwd_end'] = npass, npass + len(fwd)
            prow['bwd_begin'], prow['bwd_end'] = npass + len(fwd), npass + len(fwd) + len(bwd)
            pass_rows += [fwd, bwd]
            npass += len(fwd) + len(bwd)
            op_rows += [p.fwd.ops, p.bwd.ops]
            nops += nf + len(p.bwd.ops)
            rec = p.recipes.copy()
            rec['src'] += ncp
            rec_rows.append(rec)
            prow['rec_begin'], prow['rec_end'] = nrec, nrec + len(rec)
            nrec += len(rec)
            cpools.append(p.cpool)
            ncp += len(p.cpool)
            prow['term_begin'], prow['term_end'] = nterm, nterm + len(p.term_struct)
            term_rows += list(p.term_struct)
            nterm += len(p.term_struct)
            prow['nparams'], prow['pool_len'] = p.nparams, p.pool_len
            plan_rows.append(prow)
        dev = self.device
        rdt = np.float32 if self.dtype == torch.complex64 else np.float64
        cdt = np.complex64 if self.dtype == torch.complex64 else np.complex128
        code = N.DESV_C64 if self.dtype == torch.complex64 else N.DESV_C128
        self.code = code
        self.graph = None

        def up(a):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)

        # parameters: the persistent launch's circuits first, then every rows
        # group as (rows x nparams) at its base
        pers = [i for i, c in enumerate(self.circ) if c[0] >= 0]
        theta_off = np.zeros(len(self.circ), np.int64)
        coef_off = np.zeros(len(self.circ), np.int64)
        t = c = 0
        for i in pers:
            pi, coef, npar = self.circ[i]
            theta_off[i], coef_off[i] = t, c
            t += max(npar, self.plans[pi].nparams, 1)
            c += max(len(coef), 1)
        self.groups: List[_RowsGroup] = []
        group_base = []
        for plan, idx, coefs, npar in self.rplans:
            P = max(npar, plan.nparams, 1)
            group_base.append(t)
            for r, i in enumerate(idx):
                theta_off[i] = t + r * P
            t += P * len(idx)
        self.theta_off = theta_off
        self.ntheta = t
        self.d_theta = torch.zeros(max(t, 1), dtype=torch.float64, device=dev)
        self.d_grad = torch.zeros(max(t, 1), dtype=torch.float64, device=dev)
        self.d_energy = torch.zeros(max(len(self.circ), 1), dtype=torch.float64, device=dev)
        for (plan, idx, coefs, npar), base in zip(self.rplans, group_base):
            g = _RowsGroup(plan, coefs, base, dev, code)
            g.P = max(npar, plan.nparams, 1)
            self.groups.append(g)
        self.npersistent = len(pers)
        if not pers:
            self.args = None
            self.max_n, self.max_pool = 9, 0
            return
        self.d_passes = up(np.concatenate(pass_rows))
        self.d_ops = up(np.concatenate(op_rows))
        self.d_recipes = up(np.concatenate(rec_rows))
        self.d_cpool = torch.from_numpy(np.concatenate(cpools).astype(cdt).view(rdt).copy()).to(dev)
        terms = np.zeros(max(len(term_rows), 1), N.TERM_DTYPE)
        for i, (x, z, cr, ci) in enumerate(term_rows):
            terms[i] = (x, z, cr, ci)
        self.d_terms = up(terms)
        self.d_plans = up(np.array(plan_rows, PLAN_DTYPE))
        # circuits in decreasing cost; outputs stay in the caller's order
        order = sorted(pers, key=lambda i: -self.plans[self.circ[i][0]].cost)
        crow = np.zeros(len(pers), CIRC_DTYPE)
        coefs = np.zeros(max(c, 1))
        for i in pers:
            coef = self.circ[i][1]
            coefs[coef_off[i]:coef_off[i] + len(coef)] = coef
        for k, i in enumerate(order):
            pi = self.circ[i][0]
            crow[k] = (pi, i, theta_off[i], coef_off[i], theta_off[i], -1)
        self.d_circ = up(crow)
        self.d_coef = torch.from_numpy(coefs).to(dev)
        self.max_n = max(p.n for p in self.plans)
        self.max_pool = max(p.pool_len for p in self.plans)
        wsb = int(N.lib().desv_batch_workspace_bytes(code, max(self.max_n, 9), self.max_pool))
        self.d_ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        a = BatchArgs()
        a.ncirc = len(pers)
        for f, t_ in (('circuits', self.d_circ), ('plans', self.d_plans), ('passes', self.d_passes),
                      ('ops', self.d_ops), ('recipes', self.d_recipes), ('cpool', self.d_cpool),
                      ('theta', self.d_theta), ('coef', self.d_coef), ('terms', self.d_terms),
                      ('energy', self.d_energy), ('grad', self.d_grad)):
            setattr(a, f, t_.data_ptr())
        self.args = a

    # ------------------------------------------------------------------ run
    def nparams_list(self) -> List[int]:
        """Parameter count of every circuit, in item order."""
        return [c[2] for c in self.circ]

    def set_theta(self, thetas: Sequence[np.ndarray]):
        """Copy every circuit's parameters (gate order) into the device buffer."""
        host = np.zeros(self.ntheta)
        for i, th in enumerate(thetas):
            th = np.asarray(th, dtype=np.float64).reshape(-1)
            host[self.theta_off[i]:self.theta_off[i] + th.size] = th
        self.d_theta.copy_(torch.from_numpy(host))

    # streams the independent parts of a batch are spread over
    LANES = 4

    def launch(self, stream=None):
        """Queue the whole batch: the persistent launch over the narrow circuits
        and every rows group (prepare, forward passes, H psi with E and the
        norm, adjoint passes).  The parts are independent, so they run on up to
        LANES streams forked from `stream` and joined back into it (largest
        parts first, each to the least loaded lane): small groups and the tails
        of large passes fill the SMs that a single part leaves idle.  The
        fork and join are events, so a CUDA graph captures them too."""
        main = stream if stream is not None else torch.cuda.current_stream()
        parts = [(float(self.rows_algorithmic_bytes(g)), k) for k, g in enumerate(self.groups)]
        if self.args is not None:
            parts.append((0.0, -1))
        nl = min(self.LANES, len(parts))
        if nl <= 1:
            self.launch_persistent(main)
            for g in self.groups:
                g.launch(self.d_theta, self.d_grad, main)
            return
        side = getattr(self, '_lanes', None)
        if side is None or len(side) < nl - 1 or side[0].device != main.device:
            side = [torch.cuda.Stream(device=main.device) for _ in range(self.LANES - 1)]
            self._lanes = side
        lanes = [main] + side[:nl - 1]
        fork = torch.cuda.Event()
        fork.record(main)
        for s in lanes[1:]:
            s.wait_event(fork)
        load = [0.0] * nl
        for cost, k in sorted(parts, key=lambda x: -x[0]):
            li = min(range(nl), key=lambda i: (load[i], i))
            load[li] += cost
            if k < 0:
                self.launch_persistent(lanes[li])
            else:
                self.groups[k].launch(self.d_theta, self.d_grad, lanes[li])
        for s in lanes[1:]:
            join = torch.cuda.Event()
            join.record(s)
            main.wait_event(join)

    def launch_persistent(self, stream=None):
        """Queue the persistent launch over the narrow circuits (if any)."""
        if self.args is None:
            return
        st = ctypes.c_void_p(N.stream_ptr(stream))
        N.check(N.lib().desv_batch_vqe(self.code, max(self.max_n, 9), self.max_pool, ctypes.byref(self.args),
                                       ctypes.c_void_p(self.d_ws.data_ptr()), self.d_ws.numel(), st),
                'batched VQE')

    def rows_algorithmic_bytes(self, group: '_RowsGroup') -> float:
        """HBM bytes a rows group must move: |0...0> written once, every forward
        pass reads and writes psi, the first Pauli pass reads psi and writes
        lambda and later ones also read lambda, the norm reads psi (complex64),
        every adjoint pass reads and writes psi and lambda."""
        p = group.plan
        es = 8 if p.dtype == torch.complex64 else 16
        nf = int(np.sum(group.fwd_passes['op_end'] > group.fwd_passes['op_begin']))
        npl = int(np.sum(group.ppasses['term_end'] > group.ppasses['term_begin']))
        nb = int(np.sum(group.bwd_passes['op_end'] > group.bwd_passes['op_begin']))
        per = 1 + 2 * nf + (2 + 3 * (npl - 1) if npl else 1) + (1 if p.dtype == torch.complex64 else 0) + 4 * nb
        return float(group.B) * float(1 << p.n) * es * per

    def launches_per_batch(self) -> int:
        """Kernel launches of one batch (the persistent launch, and per rows
        group: prepare, forward passes, Pauli passes and their reductions,
        gradient zeroing, adjoint passes and their reductions)."""
        k = 1 if self.args is not None else 0
        for g in self.groups:
            nf = int(np.sum(g.fwd_passes['op_end'] > g.fwd_passes['op_begin']))
            npl = int(np.sum(g.ppasses['term_end'] > g.ppasses['term_begin']))
            nb = int(np.sum(g.bwd_passes['op_end'] > g.bwd_passes['op_begin']))
            nbr = int(np.sum((g.bwd_passes['op_end'] > g.bwd_passes['op_begin']) & (g.bwd_passes['nparams'] > 0)))
            k += 1 + nf + npl + 1 + (2 if g.plan.dtype == torch.complex64 else 0) + 1 + nb + nbr
            if g.kt is not None:     # the tangent prepare, and a second launch per tangent pass
                k += 1 + sum(1 for kt in g.kt if kt is not None)
        return k

    def capture(self):
        """Capture the launch in a CUDA graph (after one eager warm-up launch)."""
        self.launch()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.launch(stream=s)
        torch.cuda.current_stream().wait_stream(s)
        self.graph = g
        return g

    def run(self, thetas, use_graph: bool = False):
        """(energies [ncirc], list of gradients) for the given parameters."""
        self.set_theta(thetas)
        if use_graph:
            if self.graph is None:
                self.capture()
            self.graph.replay()
        else:
            self.launch()
        e = self.d_energy.cpu().numpy()[:len(self.circ)].copy()
        g = self.d_grad.cpu().numpy()
        for grp, (plan, idx, _, _) in zip(self.groups, self.rplans):
            ex = grp.expect.cpu().numpy()
            # complex64: divide out the FP64 norm drift (<psi|psi> is 1 in exact
            # arithmetic), as the persistent launch does
            ratio = 1.0 / grp.norm.cpu().numpy() if plan.dtype == torch.complex64 else np.ones(len(idx))
            for r, i in enumerate(idx):
                e[i] = ex[r, 0] * ratio[r]
                o = self.theta_off[i]
                g[o:o + grp.P] *= ratio[r]
        grads = [g[self.theta_off[i]:self.theta_off[i] + self.circ[i][2]].copy() for i in range(len(self.circ))]
        return e, grads


def hea_xxz_batch(ns: Sequence[int], layers: int, jz: Sequence[float], jxy: float = 1.0):
    """Items for BatchVQE: hardware-efficient ansatz (RY, RZ per qubit + CX ladder)
    with an open-chain XXZ Hamiltonian per circuit."""
    from .workloads import hea_circuit, xxz_terms
    return [(hea_circuit(n, layers), n, xxz_terms(n, z, jxy)) for n, z in zip(ns, jz)]


# ---------------------------------------------------------------------------
# several GPUs: circuits are independent, so a batch shards by circuit
# ---------------------------------------------------------------------------

def shard_items(qubits: Sequence[int], rank: int, world: int) -> List[int]:
    """Indices of the circuits that `rank` of `world` runs.  Circuits are dealt
    by decreasing cost (2^n amplitudes) to the rank with the least work so far,
    ties to the lowest rank, so every rank computes the same partition without
    communicating."""
    if not 0 <= rank < world:
        raise ValueError(f'rank {rank} not in [0, {world})')
    order = sorted(range(len(qubits)), key=lambda i: (-(1 << int(qubits[i])), i))
    load = [0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += 1 << int(qubits[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def gather_results(indices: Sequence[int], energies: Sequence[float], grads: Sequence[np.ndarray], total: int,
                   group=None):
    """Collect every rank's (index, energy, gradient) on all ranks through
    torch.distributed (any backend with object collectives: gloo, nccl) and
    return (energies, grads) in circuit order.  The only exchange of a sharded
    batch: one gather of results after the launch."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, (list(indices), [float(e) for e in energies], [np.asarray(g) for g in grads]),
                           group=group)
    e_all = np.zeros(total)
    g_all: List[np.ndarray] = [None] * total
    for idx, es, gs in parts:
        for i, e, g in zip(idx, es, gs):
            e_all[i] = e
            g_all[i] = g
    if any(g is None for g in g_all):
        raise RuntimeError('gather_results: some circuits were run by no rank')
    return e_all, g_all


class BatchForward:
    """run_batch_jit's rows: one circuit structure, one parameter row per
    circuit, every row's final state written to its row of a (B, 2^n) tensor,
    each row's matrices built from its theta on the device.  Replaces the
    reference's vmap over one circuit shape (backends/statevector.py:496-584).

    States of <= 12 qubits run in ONE persistent launch (the batched VQE
    kernel's forward-only mode; each state stays in one CTA's shared memory
    until written out).  Wider states run as rows: the output rows are evolved
    in place, every fused pass over all rows in one launch over all SMs."""

    def __init__(self, rows, slots, n: int, dtype=torch.complex64, tile_bits=None):
        self.dtype = dtype
        self.device = N.require_cuda()
        self.n = int(n)
        if tile_bits is None:
            from . import autotune
            tile_bits = autotune.batch_tile_bits(dtype)
        if self.n > RESIDENT_BITS:
            self.rplan = _RowsPlan(rows, slots, self.n, dtype, int(tile_bits), forward_only=True)
            self.plan = None
            self.nparams = self.rplan.nparams
            return
        self.rplan = None
        self.plan = _Plan(rows, slots, self.n, (), dtype, int(tile_bits), forward_only=True)
        self.nparams = self.plan.nparams

    def _run_rows(self, pb: np.ndarray) -> torch.Tensor:
        p, dev, B = self.rplan, self.device, pb.shape[0]
        rdt = np.float32 if self.dtype == torch.complex64 else np.float64
        cdt = np.complex64 if self.dtype == torch.complex64 else np.complex128
        npar = max(p.nparams, 1)
        theta = np.zeros((B, npar))
        theta[:, :pb.shape[1]] = pb
        code = N.DESV_C64 if self.dtype == torch.complex64 else N.DESV_C128
        out = torch.empty((B, 1 << p.n), dtype=self.dtype, device=dev)
        pools = torch.empty((B, p.pool_stride), dtype=self.dtype, device=dev)
        bufs = dict(recipes=torch.from_numpy(p.recipes.view(np.uint8).copy()).to(dev),
                    cpool=torch.from_numpy(p.cpool.astype(cdt).view(rdt).copy()).to(dev),
                    theta=torch.from_numpy(theta.reshape(-1)).to(dev),
                    ops=torch.from_numpy((p.fwd.ops if len(p.fwd.ops) else np.zeros(1, N.OP_DTYPE))
                                         .view(np.uint8).copy()).to(dev))
        passes = np.ascontiguousarray(p.fwd.passes)
        vp = ctypes.c_void_p
        st = vp(N.stream_ptr())
        N.check(N.lib().desv_rows_prepare(vp(out.data_ptr()), p.n, code, B, vp(bufs['recipes'].data_ptr()),
                                          len(p.recipes), vp(bufs['theta'].data_ptr()), npar,
                                          vp(bufs['cpool'].data_ptr()), vp(pools.data_ptr()), p.pool_stride, st),
                'rows prepare')
        kf, _, _ = p.kernels(dev.index if dev.index is not None else torch.cuda.current_device())
        rows_forward(kf, out, p.n, code, B, passes, bufs['ops'], pools, p.pool_stride, st)
        self._keep = (bufs, pools)     # alive until the stream has run the launches
        return out

    def run(self, parameter_batch: np.ndarray) -> torch.Tensor:
        pb = np.asarray(parameter_batch, dtype=np.float64)
        if self.rplan is not None:
            return self._run_rows(pb)
        B = pb.shape[0]
        p = self.plan
        dev = self.device
        rdt = np.float32 if self.dtype == torch.complex64 else np.float64
        cdt = np.complex64 if self.dtype == torch.complex64 else np.complex128

        def up(a):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)

        prow = np.zeros(1, PLAN_DTYPE)
        prow['n'] = p.n
        prow['fwd_begin'], prow['fwd_end'] = 0, len(p.fwd.passes)
        prow['bwd_begin'] = prow['bwd_end'] = len(p.fwd.passes)
        prow['rec_begin'], prow['rec_end'] = 0, len(p.recipes)
        prow['nparams'], prow['pool_len'] = p.nparams, p.pool_len
        npar = max(p.nparams, 1)
        theta = np.zeros((B, npar))
        theta[:, :pb.shape[1]] = pb
        crow = np.zeros(B, CIRC_DTYPE)
        crow['plan'] = 0
        crow['out_index'] = np.arange(B)
        crow['theta_off'] = np.arange(B) * npar
        crow['state_off'] = np.arange(B, dtype=np.int64) << p.n
        out = torch.empty((B, 1 << p.n), dtype=self.dtype, device=dev)
        bufs = dict(plans=up(prow), passes=up(p.fwd.passes), ops=up(p.fwd.ops), recipes=up(p.recipes),
                    cpool=torch.from_numpy(p.cpool.astype(cdt).view(rdt).copy()).to(dev),
                    theta=torch.from_numpy(theta.reshape(-1)).to(dev), circuits=up(crow),
                    coef=torch.zeros(1, dtype=torch.float64, device=dev),
                    terms=up(np.zeros(1, N.TERM_DTYPE)),
                    energy=torch.zeros(B, dtype=torch.float64, device=dev),
                    grad=torch.zeros(1, dtype=torch.float64, device=dev))
        code = N.DESV_C64 if self.dtype == torch.complex64 else N.DESV_C128
        wsb = int(N.lib().desv_batch_workspace_bytes(code, 9, p.pool_len))   # pools only: states are the rows
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        a = BatchArgs()
        a.ncirc = B
        for f, t_ in bufs.items():
            setattr(a, f, t_.data_ptr())
        a.states = out.data_ptr()
        N.check(N.lib().desv_batch_vqe(code, 9, p.pool_len, ctypes.byref(a), ctypes.c_void_p(ws.data_ptr()),
                                       ws.numel(), ctypes.c_void_p(N.stream_ptr())), 'batched forward')
        self._keep = (bufs, ws)        # alive until the stream has run the launch
        return out
