"""DenseSVSimulator: the reference's dense statevector API
(``dense_evolution/backends/statevector.py:70-616``) on a torch-owned CUDA
statevector driven by libdesv.

Qubit ordering is MSB-first (qubit q = index bit n-1-q).  ``self.sv`` is a
CUDA ``torch.Tensor`` (complex64 when ``use_float32`` else complex128);
``get_statevector`` / ``get_probabilities`` return NumPy arrays like the
reference.  Circuits are transpiled, fused into tile passes and executed by
the CUDA kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import warnings
from collections import OrderedDict
from typing import List, Optional, Tuple

import numpy as np
import torch

from .. import _native as N
from .. import config
from ..circuits.compiler import CompiledCircuit, QuantumTranspiler
from ..circuits.gates import GATE_IDS

_PARAM_SLOT_GATES = ('rx', 'ry', 'rz', 'p', 'u1', 'phase', 'cp', 'crz', 'cphase')


def _freeze(circuit) -> tuple:
    out = []
    for cmd in circuit:
        out.append(tuple(float(x) if isinstance(x, (np.floating,)) else
                         (int(x) if isinstance(x, np.integer) else x) for x in cmd))
    return tuple(out)


_SLOT_1Q = frozenset(('rx', 'ry', 'rz', 'p', 'u1', 'phase', 'gphase'))
_SLOT_2Q = frozenset(('cp', 'cphase', 'crz'))


def _structure(circuit):
    """(structure key, slots, angles) of a transpiled gate list: the angle of
    every one-angle gate (rx/ry/rz/p/u1/phase/gphase with one qubit, cp/cphase/
    crz with two) becomes a parameter slot, so circuits that differ only in
    those angles share a key; every other gate enters the key whole."""
    key, slots, angles = [], [], []
    for cmd in circuit:
        name = cmd[0].lower() if isinstance(cmd[0], str) else str(cmd[0]).lower()
        if name in _SLOT_1Q and len(cmd) == 3:
            key.append((name, int(cmd[1])))
        elif name in _SLOT_2Q and len(cmd) == 4:
            key.append((name, int(cmd[1]), int(cmd[2])))
        else:
            key.append(tuple(float(x) if isinstance(x, np.floating) else
                             (int(x) if isinstance(x, np.integer) else x) for x in cmd))
            slots.append(-1)
            continue
        slots.append(len(angles))
        angles.append(float(cmd[-1]))
    return tuple(key), slots, np.asarray(angles, dtype=np.float64)


class BoundCircuit:
    """A compiled circuit structure together with one call's angles: run(sv)
    applies it; every other attribute is the CompiledCircuit's."""
    __slots__ = ('plan', 'theta')

    def __init__(self, plan: CompiledCircuit, theta):
        self.plan, self.theta = plan, theta

    def run(self, sv, stream=None):
        return self.plan.run(sv, theta=self.theta, stream=stream)

    def device_arrays(self, device):
        return self.plan.device_arrays(device, self.theta)

    def __getattr__(self, name):
        return getattr(self.plan, name)


def _unknown_jit(name):
    return ValueError(
        f"unknown gate '{name}' -- not in GATE_IDS. A typo in a gate name used to be silently dropped "
        f"from the circuit instead of raising (issue #4).")


class DenseSVSimulator:
    """Dense statevector simulator on one B200.

    Parameters
    ----------
    n_qubits    : number of qubits, 1..34
    use_float32 : complex64 amplitudes (FP32 gate math, FP64 reductions) instead of complex128;
                  None (the default): complex128 unless ``config.set_precision(False)`` was called
    """

    _PLAN_CACHE_SIZE = 32

    def __init__(self, n_qubits: int, use_float32: Optional[bool] = None):
        if n_qubits < 1 or n_qubits > 34:
            raise ValueError(f"n_qubits must be in [1, 34], got {n_qubits}")
        self.n = int(n_qubits)
        self.dim = 1 << self.n
        self.use_float32 = config.default_use_float32(use_float32)
        self.dtype = np.complex64 if self.use_float32 else np.complex128
        self.tdtype = torch.complex64 if self.use_float32 else torch.complex128
        self.device = N.require_cuda()
        N.lib()
        self._plans: "OrderedDict[tuple, CompiledCircuit]" = OrderedDict()
        self.sv = torch.empty(self.dim, dtype=self.tdtype, device=self.device)
        self._reset_sv()

    # ------------------------------------------------------------------ helpers
    def _st(self):
        return ctypes.c_void_p(N.stream_ptr())

    def _code(self):
        return N.DESV_C64 if self.use_float32 else N.DESV_C128

    def _ptr(self, t=None):
        return ctypes.c_void_p((self.sv if t is None else t).data_ptr())

    def _bit(self, q: int) -> int:
        return self.n - 1 - int(q)

    # ------------------------------------------------------------------ state
    def _reset_sv(self):
        """|0...0>."""
        if self.sv is None or self.sv.numel() != self.dim:
            self.sv = torch.empty(self.dim, dtype=self.tdtype, device=self.device)
        N.check(N.lib().desv_init_basis(self._ptr(), self.n, self._code(), 0, self._st()), 'init')

    def set_initial_state(self, state: Optional[np.ndarray] = None):
        """Reset to |0...0> (state=None) or to `state` normalised; raises on a wrong
        length or a zero-norm state (statevector.py:109-133)."""
        if state is None:
            self._reset_sv()
            return
        if isinstance(state, torch.Tensor):
            t = state.detach().to(device=self.device, dtype=self.tdtype).reshape(-1)
            if t.numel() != self.dim:
                raise ValueError(f"State vector length {t.numel()} != 2**{self.n} = {self.dim}")
            self.sv = t.clone()
        else:
            arr = np.asarray(state, dtype=self.dtype)
            if arr.shape != (self.dim,):
                raise ValueError(f"State vector length {len(arr)} != 2**{self.n} = {self.dim}")
            self.sv = torch.from_numpy(arr.copy()).to(self.device)
        norm = self._norm()
        if norm < 1e-12:
            raise ValueError("Cannot set a zero-norm state vector")
        self._scale(1.0 / norm)

    def set_state(self, state: np.ndarray):
        self.set_initial_state(state)

    def _norm(self) -> float:
        out = torch.empty(2, dtype=torch.float64, device=self.device)
        sc = N.scratch(self.n, self.device)
        N.check(N.lib().desv_norm2(self._ptr(), self.n, self._code(), ctypes.c_void_p(out.data_ptr()),
                                   ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8, self._st()), 'norm')
        return float(np.sqrt(max(out[0].item(), 0.0)))

    def _scale(self, re: float, im: float = 0.0):
        N.check(N.lib().desv_scale(self._ptr(), self.n, self._code(), float(re), float(im), self._st()), 'scale')

    def normalize(self):
        norm = self._norm()
        if norm > 1e-12:
            self._scale(1.0 / norm)

    def _check_qubit_range(self, qubit: float, context: str) -> None:
        qi = int(qubit)
        if not 0 <= qi < self.n:
            raise ValueError(f"Qubit index {qi} out of range [0, {self.n}) in {context}")

    # ------------------------------------------------------------------ gates
    def _apply(self, bits, mat: np.ndarray, cmask: int = 0, cval: int = 0):
        m = np.ascontiguousarray(np.asarray(mat, dtype=np.complex128).reshape(-1)).view(np.float64)
        tb = (ctypes.c_int * len(bits))(*bits)
        N.check(N.lib().desv_apply_gate(self._ptr(), self.n, self._code(), len(bits), tb, cmask, cval,
                                        ctypes.c_void_p(m.ctypes.data), self._st()), 'apply gate')

    def apply_gate_1q(self, gate: np.ndarray, qubit: int):
        """Arbitrary 2x2 on `qubit` (statevector.py:167-184)."""
        if not 0 <= qubit < self.n:
            raise ValueError(f"Qubit index {qubit} out of range [0, {self.n})")
        g = _as_np(gate)
        if g.shape != (2, 2):
            raise ValueError('apply_gate_1q expects a 2x2 matrix')
        self._apply([self._bit(qubit)], g.astype(self.dtype).astype(np.complex128))

    def apply_gate_2q(self, gate: np.ndarray, q1: int, q2: int):
        """Arbitrary 4x4 on (q1, q2), q1 the most significant bit of the row index
        (statevector.py:188-203)."""
        if q1 == q2:
            raise ValueError("Control and target qubits must differ")
        if not (0 <= q1 < self.n and 0 <= q2 < self.n):
            raise ValueError(f"Qubit indices ({q1},{q2}) out of range [0, {self.n})")
        g = _as_np(gate).reshape(4, 4)
        # kernel row index = 2*bit(targets[1]) + bit(targets[0])
        self._apply([self._bit(q2), self._bit(q1)], g.astype(self.dtype).astype(np.complex128))

    def apply_cx(self, ctrl: int, tgt: int):
        if ctrl == tgt:
            raise ValueError("Control and target qubits must differ")
        if not (0 <= ctrl < self.n and 0 <= tgt < self.n):
            raise ValueError(f"Qubit indices ({ctrl},{tgt}) out of range [0, {self.n})")
        cb = self._bit(ctrl)
        self._apply([self._bit(tgt)], np.array([[0, 1], [1, 0]]), 1 << cb, 1 << cb)

    def apply_cz(self, ctrl: int, tgt: int):
        if ctrl == tgt:
            raise ValueError("Control and target qubits must differ")
        if not (0 <= ctrl < self.n and 0 <= tgt < self.n):
            raise ValueError(f"Qubit indices ({ctrl},{tgt}) out of range [0, {self.n})")
        cb = self._bit(ctrl)
        self._apply([self._bit(tgt)], np.diag([1, -1]), 1 << cb, 1 << cb)

    def apply_rx(self, qubit: int, theta: float):
        c, s = np.cos(theta / 2), np.sin(theta / 2)
        self.apply_gate_1q(np.array([[c, -1j * s], [-1j * s, c]]), qubit)

    def apply_ry(self, qubit: int, theta: float):
        c, s = np.cos(theta / 2), np.sin(theta / 2)
        self.apply_gate_1q(np.array([[c, -s], [s, c]]), qubit)

    def apply_rz(self, qubit: int, theta: float):
        self.apply_gate_1q(np.diag([np.exp(-0.5j * theta), np.exp(0.5j * theta)]), qubit)

    # ------------------------------------------------------------------ measurement
    def _marginals(self) -> np.ndarray:
        out = torch.empty(self.n + 1, dtype=torch.float64, device=self.device)
        sc = N.scratch(self.n, self.device)
        N.check(N.lib().desv_bit_marginals(self._ptr(), self.n, self._code(), ctypes.c_void_p(out.data_ptr()),
                                           ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8, self._st()),
                'marginals')
        return out.cpu().numpy()

    def measure(self, qubit_idx: int, jax_key=None) -> int:
        """Projective measurement of one qubit: returns 0/1 and collapses the
        state (statevector.py:272-358).  The outcome is drawn with NumPy's
        global RNG like the reference's default path."""
        if not 0 <= qubit_idx < self.n:
            raise ValueError(f"Qubit {qubit_idx} out of range [0, {self.n})")
        if jax_key is not None:
            raise ValueError("measure(jax_key=...) requires JAX to be installed.")
        bit = self._bit(qubit_idx)
        marg = self._marginals()
        total = float(marg[self.n])
        p1 = float(marg[bit])
        p0 = total - p1
        if total < 1e-12:
            raise RuntimeError("Statevector norm is zero — cannot measure")
        p0, p1 = max(p0, 0.0) / total, max(p1, 0.0) / total
        result = int(np.random.choice([0, 1], p=[p0, p1]))
        kept = (p1 if result else p0) * total
        scale = 1.0 / np.sqrt(kept) if kept > 1e-300 else 0.0
        N.check(N.lib().desv_collapse(self._ptr(), self.n, self._code(), bit, result, float(scale), self._st()),
                'collapse')
        self.normalize()
        return result

    def expectation_z(self) -> np.ndarray:
        """<Z_q> for every qubit q (one FP64 reduction pass)."""
        marg = self._marginals()
        total = marg[self.n]
        return np.array([total - 2.0 * marg[self._bit(q)] for q in range(self.n)])

    # ------------------------------------------------------------------ circuits
    def compile(self, circuit, transpile: bool = True) -> BoundCircuit:
        """The circuit's compiled structure with its angles.  Plans are cached by
        structure (gate names, qubits and the fixed parameters), so a circuit
        run again with new angles -- a variational loop -- reuses its lowering,
        fusion plan and kernels and only recomputes the per-call values."""
        target = QuantumTranspiler.transpile(circuit) if transpile else list(circuit)
        skey, slots, angles = _structure(target)
        key = (skey, self.n, self.use_float32)
        plan = self._plans.get(key)
        if plan is None:
            plan = CompiledCircuit(target, self.n, self.tdtype, slots=slots if len(angles) else None)
            self._plans[key] = plan
            if len(self._plans) > self._PLAN_CACHE_SIZE:
                self._plans.popitem(last=False)
        else:
            self._plans.move_to_end(key)
        return BoundCircuit(plan, angles if len(angles) else None)

    def run_circuit(self, circuit: List[Tuple], transpile: bool = True):
        """Transpile, fuse and run `circuit` in place (statevector.py:362-410).
        Unknown gate names raise ValueError (issue #4)."""
        self.compile(circuit, transpile).run(self.sv)

    def run_circuit_jit(self, circuit: List):
        """Compiled-path entry (statevector.py:414-471): only GATE_IDS names after transpile."""
        target = QuantumTranspiler.transpile(circuit)
        for cmd in target:
            name = cmd[0].lower() if isinstance(cmd[0], str) else str(cmd[0]).lower()
            if name not in GATE_IDS:
                raise _unknown_jit(cmd[0])
        if target:
            self.compile(target, transpile=False).run(self.sv)

    def run_circuit_jit_beast_mode(self, circuit: List):
        warnings.warn("run_circuit_jit_beast_mode is deprecated, use run_circuit_jit instead "
                      "(same behavior, shorter name). This alias will be removed in a future release.",
                      DeprecationWarning, stacklevel=2)
        return self.run_circuit_jit(circuit)

    def run_circuit_with_chunking(self, circuit: List, chunk_size: int = 500):
        target = QuantumTranspiler.transpile(circuit)
        for i in range(0, len(target), chunk_size):
            self.run_circuit_jit(target[i:i + chunk_size])

    def run_batch_jit(self, base_circuit: List, parameter_batch: np.ndarray) -> torch.Tensor:
        """Same circuit for every row of `parameter_batch`: one column per parametric
        gate (rx/ry/rz/p/u1/phase/cp/crz/cphase) in gate order after transpile
        (statevector.py:496-584).  Returns a (B, 2^n) CUDA tensor; every row
        starts from |0...0>."""
        target = QuantumTranspiler.transpile(base_circuit)
        slots, k = [], 0
        for cmd in target:
            name = cmd[0].lower() if isinstance(cmd[0], str) else str(cmd[0]).lower()
            if name not in GATE_IDS:
                raise _unknown_jit(cmd[0])
            if name in ('cp', 'crz', 'cphase', 'cx', 'cz', 'swap', 'cy'):
                self._check_qubit_range(cmd[1], f"gate '{name}' (control)")
                self._check_qubit_range(cmd[2] if len(cmd) > 2 else 0, f"gate '{name}' (target)")
            else:
                self._check_qubit_range(cmd[1] if len(cmd) > 1 else 0, f"gate '{name}'")
            if name in _PARAM_SLOT_GATES:
                slots.append(k)
                k += 1
            else:
                slots.append(-1)
        pb = np.asarray(parameter_batch, dtype=np.float64)
        if pb.ndim != 2 or pb.shape[1] != k:
            raise ValueError(
                f"parameter_batch has {pb.shape[-1] if pb.ndim else 0} column(s) but base_circuit has {k} "
                f"parametric gate(s) (rx/ry/rz/p/u1/phase/cp/crz/cphase) -- one column per parametric gate, "
                f"in gate-appearance order. A literal float passed for one of these gates is NOT exempt: it "
                f"still consumes a positional column. A mismatch here used to be clipped silently by JAX's "
                f"default out-of-bounds indexing instead of raising (issue #6).")
        # rows whose slot is bound get a parameter position for lowering; like the
        # reference's batch template, gphase rows carry parameter 0
        norm_target = []
        for cmd, s in zip(target, slots):
            if cmd[0].lower() == 'gphase':
                norm_target.append(('gphase', cmd[1], 0.0))
            elif s >= 0:
                name = cmd[0].lower()
                if name in ('cp', 'crz', 'cphase'):
                    norm_target.append((name, cmd[1], cmd[2], 0.0))
                else:
                    norm_target.append((name, cmd[1], 0.0))
            else:
                norm_target.append(cmd)
        if self.n >= 9 and pb.shape[0] > 0:
            # every row in one persistent launch (the batched kernel's forward-only
            # mode); structures it cannot build fall back to one plan run per row
            key = ('batch_forward', _freeze(norm_target), tuple(slots), self.n, self.use_float32)
            bf = self._plans.get(key)
            if bf is None:
                from ..batch import BatchForward
                try:
                    bf = BatchForward(norm_target, slots, self.n, self.tdtype)
                except (RuntimeError, ValueError, KeyError):
                    bf = False
                self._plans[key] = bf
            if bf:
                return bf.run(pb)
        plan = CompiledCircuit(norm_target, self.n, self.tdtype, slots=slots)
        out = torch.empty((pb.shape[0], self.dim), dtype=self.tdtype, device=self.device)
        for r in range(pb.shape[0]):
            row = out[r]
            N.check(N.lib().desv_init_basis(ctypes.c_void_p(row.data_ptr()), self.n, self._code(), 0, self._st()),
                    'init')
            plan.run(row, theta=pb[r])
        return out

    def run_parametric_batch_jit(self, base_circuit: List, parameter_batch: np.ndarray) -> torch.Tensor:
        warnings.warn("run_parametric_batch_jit is deprecated, use run_batch_jit instead "
                      "(same behavior, shorter name). This alias will be removed in a future release.",
                      DeprecationWarning, stacklevel=2)
        return self.run_batch_jit(base_circuit, parameter_batch)

    # ------------------------------------------------------------------ read-out
    def get_probabilities(self) -> np.ndarray:
        """|a|^2 as float64, clipped to [0, 1] and renormalised (statevector.py:599-607)."""
        out = torch.empty(self.dim, dtype=torch.float64, device=self.device)
        N.check(N.lib().desv_probabilities(self._ptr(), self.n, self._code(), ctypes.c_void_p(out.data_ptr()),
                                           self._st()), 'probabilities')
        probs = np.clip(out.cpu().numpy(), 0.0, 1.0)
        total = probs.sum()
        if total > 1e-12:
            probs /= total
        return probs

    def probabilities_tensor(self) -> torch.Tensor:
        """get_probabilities() as an FP64 CUDA tensor (|a|^2, clipped to [0, 1],
        renormalised), left on the device."""
        out = torch.empty(self.dim, dtype=torch.float64, device=self.device)
        N.check(N.lib().desv_probabilities(self._ptr(), self.n, self._code(), ctypes.c_void_p(out.data_ptr()),
                                           self._st()), 'probabilities')
        out.clamp_(0.0, 1.0)
        total = float(out.sum().item())
        if total > 1e-12:
            out /= total
        return out

    def get_statevector(self) -> np.ndarray:
        return self.sv.detach().cpu().numpy().astype(self.dtype, copy=False)

    def memory_mb(self) -> float:
        return self.dim * (8 if self.use_float32 else 16) / 1_000_000


def _as_np(gate) -> np.ndarray:
    if isinstance(gate, torch.Tensor):
        return gate.detach().cpu().numpy()
    return np.asarray(gate)
