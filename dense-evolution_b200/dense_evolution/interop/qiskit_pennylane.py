"""Qiskit / PennyLane interop of the dense path (reference
``dense_evolution/interop/qiskit_pennylane.py:115-230``).

This engine, like the reference, keeps amplitudes MSB-first: qubit 0 is the
most significant index bit.  Qiskit and PennyLane number qubits
little-endian, so their probabilities and statevectors are the bit-reversal
permutation of ours.  The permutation runs on the GPU (``desv_bit_reverse``:
a tiled transpose, one HBM read and write); ``_to_qiskit_bit_order`` keeps
the reference's host-array signature on top of it.

``from_qiskit`` / ``from_pennylane`` convert through OpenQASM 2.0 and this
package's ``QASMParser`` exactly as the reference does; they need the
``qiskit`` / ``pennylane`` packages, and raise the reference's ImportError
messages when those are absent.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np
import torch

from .. import _native as N
from ..backends.statevector import DenseSVSimulator
from ..circuits.parser import QASMCircuit, QASMParser

try:  # optional dependencies, as in the reference
    from qiskit import qasm2 as _qasm2
    HAS_QISKIT = True
except Exception:  # pragma: no cover - depends on the environment
    _qasm2 = None
    HAS_QISKIT = False
try:
    import pennylane as qml
    HAS_PENNYLANE = True
except Exception:  # pragma: no cover
    qml = None
    HAS_PENNYLANE = False

_ELEM = {torch.float64: N.DESV_ELEM_F64, torch.complex64: N.DESV_ELEM_C64, torch.complex128: N.DESV_ELEM_C128}


def _require_qiskit():
    if not HAS_QISKIT:
        raise ImportError("Qiskit interop requires the 'qiskit' package. "
                          "Install it with: pip install dense-evolution[qiskit]")


def _require_pennylane():
    if not HAS_PENNYLANE:
        raise ImportError("PennyLane interop requires the 'pennylane' package. "
                          "Install it with: pip install dense-evolution[pennylane]")


def to_little_endian(x: torch.Tensor, n_qubits: Optional[int] = None) -> torch.Tensor:
    """The bit-reversal permutation of a CUDA tensor of 2^n probabilities (FP64)
    or amplitudes (complex64 / complex128), as a new tensor: MSB-first <->
    little-endian (the permutation is its own inverse)."""
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise ValueError('to_little_endian needs a CUDA tensor')
    x = x.reshape(-1)
    n = int(x.numel()).bit_length() - 1
    if x.numel() != 1 << n or (n_qubits is not None and n != int(n_qubits)):
        raise ValueError(f'array length {x.numel()} is not 2**n_qubits')
    if x.dtype not in _ELEM:
        x = x.to(torch.float64)
    x = x.contiguous()
    out = torch.empty_like(x)
    N.check(N.lib().desv_bit_reverse(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), n, _ELEM[x.dtype],
                                     ctypes.c_void_p(N.stream_ptr())), 'bit reversal')
    return out


def _to_qiskit_bit_order(probs, n_qubits: int) -> np.ndarray:
    """Probabilities (or amplitudes) in Qiskit's little-endian order, as a NumPy
    array, from this engine's MSB-first order (the reference helper's
    signature; the permutation itself runs on the GPU)."""
    a = np.asarray(probs)
    if a.shape != (1 << n_qubits,):
        raise ValueError(f'expected {1 << n_qubits} entries, got shape {a.shape}')
    t = torch.from_numpy(np.ascontiguousarray(a)).to(N.require_cuda())
    out = to_little_endian(t, n_qubits).cpu().numpy()
    return out.astype(a.dtype, copy=False)


def from_qiskit(circuit) -> QASMCircuit:
    """A Qiskit QuantumCircuit as a QASMCircuit, through OpenQASM 2.0
    (qiskit.qasm2.dumps) and QASMParser."""
    _require_qiskit()
    return QASMParser().parse(_qasm2.dumps(circuit))


def from_pennylane(circuit, *args, **kwargs) -> QASMCircuit:
    """A PennyLane QNode or tape as a QASMCircuit, through OpenQASM 2.0 with the
    true wire order forced into the export (the reference's rules: a tape's
    own wires sorted ascending, a QNode's device wires)."""
    _require_pennylane()
    if isinstance(circuit, qml.tape.QuantumScript):
        try:
            wires = sorted(circuit.wires)
        except TypeError:
            wires = list(circuit.wires)
        if hasattr(circuit, 'to_openqasm'):
            qasm = circuit.to_openqasm(wires=wires, measure_all=False)
        else:
            qasm = qml.to_openqasm(circuit, wires=wires, measure_all=False)
    else:
        device = getattr(circuit, 'device', None)
        wires = device.wires if device is not None else None
        res = qml.to_openqasm(circuit, wires=wires, measure_all=False)
        qasm = res if isinstance(res, str) else res(*args, **kwargs)
    return QASMParser().parse(qasm)


def run_qiskit_circuit(circuit, use_float32: bool = True,
                       sim: Optional[DenseSVSimulator] = None) -> Tuple[DenseSVSimulator, np.ndarray]:
    """Run a Qiskit QuantumCircuit on DenseSVSimulator: (sim, probabilities in
    Qiskit's little-endian order), comparable to
    Statevector(circuit).probabilities().  The probabilities are formed and
    permuted on the GPU; only the permuted array is copied to the host."""
    circ = from_qiskit(circuit)
    if sim is None:
        sim = DenseSVSimulator(n_qubits=circ.n_qubits, use_float32=use_float32)
    sim.run_circuit(circ.to_tuples())
    probs = sim.probabilities_tensor()
    return sim, to_little_endian(probs, circ.n_qubits).cpu().numpy()
