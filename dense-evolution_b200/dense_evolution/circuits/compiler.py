"""Transpiler (same decompositions as the reference) and the compiled-circuit
executor that replaces the reference's JAX scan kernel.

``QuantumTranspiler`` mirrors ``dense_evolution/circuits/compiler.py:362-488``
of the reference: CCX -> 15 gates, SWAP -> 3 CX, iSWAP -> {S,H,CX},
ECR -> {S,SX,X,CX,GPhase}, U3/U2 -> Rz.Ry.Rz.GPhase, everything else passes
through (tuples without parameters pass through untouched, so structural
callers keep working).

``CompiledCircuit`` lowers a transpiled circuit through the fusion pass
(:mod:`.fusion`) and runs it on a torch-owned CUDA statevector through
``desv_apply_passes`` (fused tile passes, states of >= 9 qubits) or
``desv_apply_gate`` (one launch per fused op, smaller states).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _native as N
from . import fusion, jit, rotation


class QuantumTranspiler:
    """Gate-level transpiler: exact decompositions of non-native gates."""

    @staticmethod
    def decompose_toffoli(c1: int, c2: int, t: int) -> List[Tuple]:
        """CCX as 6 CX + 9 single-qubit gates (H/T/Tdg), exact."""
        return [('h', t), ('cx', c2, t), ('tdg', t), ('cx', c1, t), ('t', t), ('cx', c2, t), ('tdg', t),
                ('cx', c1, t), ('t', c2), ('t', t), ('cx', c1, c2), ('h', t), ('t', c1), ('tdg', c2),
                ('cx', c1, c2)]

    @staticmethod
    def decompose_swap(q1: int, q2: int) -> List[Tuple]:
        return [('cx', q1, q2), ('cx', q2, q1), ('cx', q1, q2)]

    @staticmethod
    def decompose_iswap(q1: int, q2: int) -> List[Tuple]:
        return [('s', q1), ('h', q1), ('s', q2), ('cx', q1, q2), ('cx', q2, q1), ('h', q2)]

    @staticmethod
    def decompose_ecr(q1: int, q2: int) -> List[Tuple]:
        return [('s', q1), ('sx', q2), ('cx', q1, q2), ('x', q1), ('gphase', q1, -np.pi / 4.0)]

    @staticmethod
    def decompose_u3(q, theta, phi, lam) -> List[Tuple]:
        """U3(t,p,l) = e^{i(p+l)/2} Rz(p) Ry(t) Rz(l), exact; applied Rz(l) first."""
        return [('rz', q, lam), ('ry', q, theta), ('rz', q, phi), ('gphase', q, (phi + lam) / 2.0)]

    @staticmethod
    def decompose_u2(q, phi, lam) -> List[Tuple]:
        return QuantumTranspiler.decompose_u3(q, np.pi / 2.0, phi, lam)

    @classmethod
    def transpile(cls, circuit) -> List[Tuple]:
        out: List[Tuple] = []
        for cmd in circuit:
            name = cmd[0].lower()
            if name == 'ccx':
                out.extend(cls.decompose_toffoli(*cmd[1:4]))
            elif name == 'swap':
                out.extend(cls.decompose_swap(*cmd[1:3]))
            elif name == 'iswap':
                out.extend(cls.decompose_iswap(*cmd[1:3]))
            elif name == 'ecr':
                out.extend(cls.decompose_ecr(*cmd[1:3]))
            elif name == 'u3' and len(cmd) >= 5:
                out.extend(cls.decompose_u3(*cmd[1:5]))
            elif name == 'u2' and len(cmd) >= 4:
                out.extend(cls.decompose_u2(*cmd[1:4]))
            else:
                out.append(cmd)
        return out


def default_tile_bits(n: int, dtype: torch.dtype) -> int:
    """Largest supported tile (complex64: 2^12 amplitudes = 32 KB, complex128: 2^11)."""
    from .. import autotune
    return autotune.tile_bits(n, dtype)


class CompiledCircuit:
    """A circuit lowered, fused and packed for one qubit count and precision.

    complex64 circuits of >= rotation.MIN_QUBITS qubits run as rotation passes
    (``rotation.py``: real rotations in tangent form, diagonal groups, every
    tile bit a register slot); the general fused passes (``fusion.py``) are
    built lazily, for everything else."""

    def __init__(self, target: Sequence[tuple], n: int, dtype: torch.dtype = torch.complex128,
                 slots: Optional[Sequence[int]] = None, tile_bits: Optional[int] = None, merge_1q: bool = True):
        self.n = int(n)
        self.dtype = dtype
        self.tile_bits = tile_bits or default_tile_bits(self.n, dtype)
        self._target, self._slots, self._merge_1q = list(target), slots, merge_1q
        self.ir = fusion.lower(self._target, self.n, slots)
        self._fops = self._packed = None
        self._built = False
        self._rot = None
        self._dev_cache = None
        self._dev_theta_key = None
        self._host_arrays = None
        self._jit_kernels = None

    def _build(self):
        if not self._built:
            _, self._fops, self._packed = fusion.build(self._target, self.n, self.tile_bits, self._slots,
                                                       self._merge_1q)
            self._built = True

    @property
    def fops(self):
        self._build()
        return self._fops

    @property
    def packed(self):
        self._build()
        return self._packed

    @property
    def rotation(self):
        """The bound rotation program of this circuit, or None when the general
        fused passes run it (complex128, fewer than rotation.MIN_QUBITS qubits,
        DESV_ROT=0, no NVRTC, or a gate the rotation path does not lower)."""
        if self._rot is None:
            self._rot = False
            if self.dtype == torch.complex64 and self.n >= fusion.MIN_FUSED_QUBITS and \
                    rotation.enabled(self.n, True):
                self._rot = rotation.program_for(self._target, self.n, min(12, self.n), self._slots) or False
        return self._rot or None

    # ------------------------------------------------------------ stats
    @property
    def npasses(self) -> int:
        if self.rotation is not None:
            return len(self.rotation.plan.passes)
        return len(self.packed.passes) if self.packed is not None else len(self.fops)

    @property
    def fused(self) -> bool:
        return self.packed is not None

    # ------------------------------------------------------------ execution
    def _np_dtype(self):
        return np.complex64 if self.dtype == torch.complex64 else np.complex128

    @property
    def device_passes(self):
        """desv_pass rows of the grouped op stream that device_arrays() uploaded."""
        return self._passes

    def device_arrays(self, device, theta=None):
        """(ops, mats) device tensors for `theta` (cached for constant circuits)."""
        key = None if theta is None else np.asarray(theta, dtype=np.float64).tobytes()
        if self._dev_cache is not None and self._dev_cache[0] == device and self._dev_theta_key == key:
            return self._dev_cache[1], self._dev_cache[2]
        mats = self.packed.materialize(theta, self._np_dtype())
        ops, self._passes, mats = self.packed.compact(mats)
        self._host_arrays = (ops, mats)
        self._jit_kernels = None
        ops_t = torch.from_numpy(ops.view(np.uint8).copy()).to(device)
        rdt = np.float32 if self.dtype == torch.complex64 else np.float64
        mats_t = torch.from_numpy(mats.view(rdt).copy()).to(device)
        self._dev_cache = (device, ops_t, mats_t)
        self._dev_theta_key = key
        return ops_t, mats_t

    def run(self, sv: torch.Tensor, theta=None, stream=None):
        """Apply the circuit in place to the CUDA statevector `sv`."""
        if sv.dtype != self.dtype or sv.numel() != (1 << self.n) or not sv.is_cuda:
            raise ValueError('statevector does not match the compiled circuit')
        lib = N.lib()
        st = ctypes.c_void_p(N.stream_ptr(stream))
        code = N.dtype_code(sv)
        rot = self.rotation
        if rot is not None:
            dev = sv.device.index if sv.device.index is not None else torch.cuda.current_device()
            rot.run(sv.data_ptr(), dev, st.value or 0, theta)
            return sv
        if self.packed is None:
            for op in self.fops:
                apply_fop(sv, self.n, op, theta, st)
            return sv
        if len(self.packed.passes) == 0:
            return sv
        ops_t, mats_t = self.device_arrays(sv.device, theta)
        passes = self._passes
        if jit.enabled(self.n):
            jit.run_passes(self.specialised_kernels(sv.device), sv.data_ptr(), self.n, code, passes,
                           ops_t.data_ptr(), mats_t.data_ptr(), st.value)
            return sv
        N.check(lib.desv_apply_passes(ctypes.c_void_p(sv.data_ptr()), self.n, code,
                                      ctypes.c_void_p(passes.ctypes.data), len(passes),
                                      ctypes.c_void_p(ops_t.data_ptr()), ctypes.c_void_p(mats_t.data_ptr()), st),
                'apply fused passes')
        return sv


    def specialised_kernels(self, device):
        """Plan-specialised kernels (one per pass) of the op stream that
        device_arrays() uploaded last; compiled once per structure."""
        if self._jit_kernels is None:
            ops, mats = self._host_arrays
            dev = device.index if device.index is not None else torch.cuda.current_device()
            self._jit_kernels = jit.compile_passes(ops, self._passes, mats, self.dtype == torch.complex64, dev)
        return self._jit_kernels


def apply_fop(sv: torch.Tensor, n: int, op: 'fusion.FOp', theta, st):
    """One fused op through the single-gate kernel."""
    lib = N.lib()
    code = N.dtype_code(sv)
    m = op.matrix(theta)
    if op.kind == 'scalar':
        v = complex(m[0])
        N.check(lib.desv_scale(ctypes.c_void_p(sv.data_ptr()), n, code, v.real, v.imag, st), 'scale')
        return
    if op.kind == 'm1':
        tb = (ctypes.c_int * 1)(op.t)
        cm = cv = 0
        for c, v in zip(op.cbits, op.cvals):
            cm |= 1 << c
            cv |= v << c
        mat = np.ascontiguousarray(m.reshape(-1)).view(np.float64)
        N.check(lib.desv_apply_gate(ctypes.c_void_p(sv.data_ptr()), n, code, 1, tb, cm, cv,
                                    ctypes.c_void_p(mat.ctypes.data), st), 'apply gate')
        return
    if op.kind == 'd2':
        full = np.diag(m).astype(np.complex128)
    else:
        full = np.asarray(m, dtype=np.complex128)
    tb = (ctypes.c_int * 2)(op.t, op.t2)
    mat = np.ascontiguousarray(full.reshape(-1)).view(np.float64)
    N.check(lib.desv_apply_gate(ctypes.c_void_p(sv.data_ptr()), n, code, 2, tb, 0, 0,
                                ctypes.c_void_p(mat.ctypes.data), st), 'apply gate')
