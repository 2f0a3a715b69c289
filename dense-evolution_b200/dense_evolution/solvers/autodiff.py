"""Differentiable energy functions: the reference's ``circuit_to_energy_fn``
(``dense_evolution/solvers/autodiff.py:92-169``) on the GPU engine.

``energy_fn(theta, h_matrix, stato_zero=None, noise=None) -> (energy, sv)``
injects theta, in gate order, into the parametric gates rx/ry/rz/u1/p/cp/crz
of the circuit (every other gate keeps parameter 0, as in the reference's
template), runs the fused forward passes, and evaluates E = Re<psi|H|psi>.
The energy is a torch scalar; when theta is a tensor that requires grad,
``E.backward()`` runs the adjoint method (see :mod:`.adjoint`).
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np
import torch

from .. import _native as N
from .. import config
from ..circuits.compiler import QuantumTranspiler
from ..circuits.gates import GATE_IDS
from ..circuits.parser import QASMCircuit
from . import adjoint

_PARAMETRIC_GATES = ('rx', 'ry', 'rz', 'u1', 'p', 'cp', 'crz')
_TWO_QUBIT_GATES = ('cx', 'cy', 'cz', 'cp', 'crz', 'swap')


def build_template(circuit, n_qubits: int):
    """(gate tuples with placeholder parameters, theta slot per gate, n_params).

    Mirrors the reference's ``_build_template`` (autodiff.py:33-89): ops with
    no qubits or a qubit >= n_qubits are skipped, the structural tuples are
    transpiled, unknown names raise, and n_params counts the parametric ops of
    the ORIGINAL circuit."""
    ops = circuit.ops if isinstance(circuit, QASMCircuit) else [
        {'name': c[0], 'qubits': [int(q) for q in c[1:] if isinstance(q, (int, np.integer))]} for c in circuit]
    tuples = []
    for op in ops:
        name = str(op['name']).lower().strip()
        qubits = [int(q) for q in op.get('qubits', [])]
        if not qubits or any(q >= n_qubits for q in qubits):
            continue
        tuples.append((name, *qubits))
    target = QuantumTranspiler.transpile(tuples)
    rows, slots, k = [], [], 0
    for cmd in target:
        name = cmd[0].lower()
        if name not in GATE_IDS:
            raise ValueError(
                f"circuit_to_energy_fn: gate '{name}' has no GATE_IDS entry, so it can't be represented in this "
                f"template and would otherwise be silently dropped. Multi-parameter gates like 'u2'/'u3' aren't "
                f"supported here (one parameter per row) -- decompose them into rx/ry/rz/cx first, or use "
                f"DenseSVSimulator.run_circuit instead.")
        qs = [int(q) for q in cmd[1:] if isinstance(q, (int, np.integer))]
        par = name in _PARAMETRIC_GATES
        if name in _TWO_QUBIT_GATES and len(qs) >= 2:
            rows.append((name, qs[0], qs[1], 0.0) if name in ('cp', 'crz') else (name, qs[0], qs[1]))
        elif name == 'cphase':
            # the reference's row [22, q, 0, 0.0] is a phase of 0: the identity
            rows.append(('id', qs[0]))
        elif name in ('rx', 'ry', 'rz', 'u1', 'p', 'phase', 'gphase'):
            rows.append((name, qs[0], 0.0))
        else:
            rows.append((name, qs[0]))
        slots.append(k if par else -1)
        k += par
    n_params = sum(1 for op in ops if str(op['name']).lower().strip() in _PARAMETRIC_GATES)
    return rows, slots, n_params


def circuit_to_energy_fn(circuit, n_qubits: int, use_float32: Optional[bool] = None) -> Tuple[Callable, int]:
    """(energy_fn, n_params) for a QASMCircuit (or gate-tuple list).

    ``use_float32`` runs the state in complex64 with FP64 reductions; the
    default (None) is complex128 like the reference, or complex64 after an
    explicit ``config.set_precision(False)``."""
    rows, slots, n_params = build_template(circuit, n_qubits)
    f32 = config.default_use_float32(use_float32)
    prog = adjoint.AdjointProgram(rows, slots, n_qubits, torch.complex64 if f32 else torch.complex128)

    def energy_fn(theta, h_matrix, stato_zero=None, noise=None):
        return prog.energy(theta, h_matrix, stato_zero, noise)

    energy_fn.program = prog
    energy_fn.n_params = n_params
    return energy_fn, n_params
