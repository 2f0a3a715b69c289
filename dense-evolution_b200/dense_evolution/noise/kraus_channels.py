"""Stochastic single-qubit Kraus channels applied to a GPU statevector.

Drop-in for ``NoiseModel`` of ``dense_evolution/noise/kraus_channels.py``
(reference lines 45-236, one module per channel under ``noise/kraus/``): per
target qubit and call, ONE fire / no-fire decision applied to the whole
statevector, qubit q being index bit q (least significant first -- the
channels' own convention, which differs from the simulator's MSB-first gate
order), then division by (norm + 1e-15).

* depolarizing: two draws (fire, then which Pauli at thresholds 1/3, 2/3);
* bitflip / phaseflip: one draw;
* amplitude_damping: one draw against P(K1) = gamma * P(bit q = 1) of the
  current state, then K1 / sqrt(P(K1)) or K0 / sqrt(1 - P(K1));
* combined: depolarizing(p / 2) then amplitude_damping(p * 0.333333).

The random decisions are drawn on the host from a ``numpy.random.Generator``
in exactly the reference's order, so a seeded Generator gives the reference's
NumPy-branch result.  Pauli decisions are applied as one fused circuit
(a few HBM passes for any number of errors); a damping step needs the bit
marginal of the current state (one FP64 reduction) and one 2x2 pass.
The reference's JAX branch draws from ``jax.random`` instead; JAX is not part
of this engine, so a ``jax_key`` here seeds a NumPy Generator (same channel
semantics, a different random stream).
"""
from __future__ import annotations

import ctypes
import os
import time
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _native as N

MODELS = ['ideal', 'depolarizing', 'bitflip', 'phaseflip', 'amplitude_damping', 'combined']
PAULI_MODELS = ('depolarizing', 'bitflip', 'phaseflip')
_THIRD = 1.0 / 3.0
_PAULI = {'x': np.array([[0, 1], [1, 0]], np.complex128), 'y': np.array([[0, -1j], [1j, 0]], np.complex128),
          'z': np.array([[1, 0], [0, -1]], np.complex128)}


def resolve_rng(rng=None, jax_key=None) -> np.random.Generator:
    """The Generator the channels draw from: `rng` if given, else one seeded
    from `jax_key` (an int, a Generator, or an array of ints such as a JAX
    PRNG key's data), else one seeded from OS entropy and a clock."""
    if rng is not None:
        return rng
    if jax_key is not None:
        if isinstance(jax_key, np.random.Generator):
            return jax_key
        return np.random.default_rng(np.asarray(jax_key, dtype=np.uint64).reshape(-1).tolist())
    seed = int.from_bytes(os.urandom(8), 'big') ^ (time.perf_counter_ns() & 0xFFFFFFFFFFFFFFFF)
    return np.random.default_rng(seed)


def draw_pauli_errors(model: str, p: float, n: int, rng: np.random.Generator,
                      qubits: Optional[Sequence[int]] = None) -> List[Tuple[int, str]]:
    """(index bit, 'x' | 'y' | 'z') of every error a Pauli channel fires in one
    call, drawing from `rng` exactly as apply_to_sv does."""
    out = []
    for q in (range(n) if qubits is None else qubits):
        if model == 'depolarizing':
            r, ch = rng.random(), rng.random()
            if r < p:
                out.append((int(q), 'x' if ch < _THIRD else 'y' if ch < 2.0 * _THIRD else 'z'))
        elif model == 'bitflip':
            if rng.random() < p:
                out.append((int(q), 'x'))
        elif model == 'phaseflip':
            if rng.random() < p:
                out.append((int(q), 'z'))
        else:
            raise ValueError(f'{model!r} is not a Pauli channel')
    return out


def apply_pauli_errors(psi: torch.Tensor, n: int, errors: Sequence[Tuple[int, str]]):
    """Apply the Pauli errors (index bits) in place, as one fused circuit."""
    if not errors:
        return psi
    from ..circuits.compiler import CompiledCircuit
    # circuit qubit j is index bit n-1-j
    CompiledCircuit([(w, n - 1 - q) for q, w in errors], n, psi.dtype).run(psi)
    return psi


def _gate(psi: torch.Tensor, n: int, bit: int, m: np.ndarray):
    mm = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(-1)).view(np.float64)
    tb = (ctypes.c_int * 1)(bit)
    N.check(N.lib().desv_apply_gate(ctypes.c_void_p(psi.data_ptr()), n, N.dtype_code(psi), 1, tb, 0, 0,
                                    ctypes.c_void_p(mm.ctypes.data), ctypes.c_void_p(N.stream_ptr())), 'noise gate')


def _damp(psi: torch.Tensor, n: int, bit: int, p: float, rng: np.random.Generator):
    gamma = float(np.clip(p, 0.0, 1.0))
    r = rng.random()
    out = torch.empty(n + 1, dtype=torch.float64, device=psi.device)
    sc = N.scratch(n, psi.device)
    N.check(N.lib().desv_bit_marginals(ctypes.c_void_p(psi.data_ptr()), n, N.dtype_code(psi),
                                       ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(sc.data_ptr()),
                                       sc.numel() * 8, ctypes.c_void_p(N.stream_ptr())), 'noise marginal')
    p1 = float(np.clip(gamma * float(out[bit].item()), 0.0, 1.0))
    if r < p1:
        k = np.array([[0.0, np.sqrt(gamma) / np.sqrt(max(p1, 1e-15))], [0.0, 0.0]])
    else:
        nn = np.sqrt(max(1.0 - p1, 1e-15))
        k = np.array([[1.0 / nn, 0.0], [0.0, np.sqrt(1.0 - gamma) / nn]])
    _gate(psi, n, bit, k)


def apply_channel(psi: torch.Tensor, n: int, model: str, p: float, rng: np.random.Generator,
                  qubits: Optional[Sequence[int]] = None) -> torch.Tensor:
    """One call of the channel on `psi` in place, without the final normalisation."""
    if model in PAULI_MODELS:
        return apply_pauli_errors(psi, n, draw_pauli_errors(model, p, n, rng, qubits))
    for q in (range(n) if qubits is None else qubits):
        if model == 'combined':
            apply_pauli_errors(psi, n, draw_pauli_errors('depolarizing', p * 0.5, n, rng, [q]))
            _damp(psi, n, int(q), p * 0.333333, rng)
        else:
            _damp(psi, n, int(q), p, rng)
    return psi


def normalize_plus_eps(psi: torch.Tensor) -> torch.Tensor:
    """psi / (norm + 1e-15), the channels' final step (FP64 norm on the device)."""
    n = int(psi.numel()).bit_length() - 1
    out = torch.empty(2, dtype=torch.float64, device=psi.device)
    sc = N.scratch(n, psi.device)
    N.check(N.lib().desv_norm2(ctypes.c_void_p(psi.data_ptr()), n, N.dtype_code(psi), ctypes.c_void_p(out.data_ptr()),
                               ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8, ctypes.c_void_p(N.stream_ptr())),
            'norm')
    s = 1.0 / (float(np.sqrt(max(out[0].item(), 0.0))) + 1e-15)
    N.check(N.lib().desv_scale(ctypes.c_void_p(psi.data_ptr()), n, N.dtype_code(psi), s, 0.0,
                               ctypes.c_void_p(N.stream_ptr())), 'scale')
    return psi


class NoiseModel:
    """Stochastic single-qubit Kraus channels applied directly to a statevector
    (``apply_to_sv``); see the module docstring for the exact semantics."""

    MODELS = list(MODELS)

    @staticmethod
    def apply_to_sv(sv, n: int, model: str, p: float, rng: Optional[np.random.Generator] = None,
                    qubits: Optional[List[int]] = None, jax_key=None):
        """One noisy shot: a normalised copy of `sv` (a CUDA tensor stays on the
        device; a NumPy array is processed on the GPU and returned as NumPy).
        The caller's array is never modified."""
        if model == 'ideal':
            return sv
        if p <= 0.0:
            return sv
        if model not in MODELS:
            raise KeyError(model)
        gen = resolve_rng(rng, jax_key)
        if isinstance(sv, torch.Tensor):
            psi = sv.detach().clone().reshape(-1)
            if not psi.is_cuda:
                psi = psi.to(N.require_cuda())
        else:
            a = np.asarray(sv)
            dt = torch.complex64 if a.dtype == np.complex64 else torch.complex128
            psi = torch.from_numpy(np.ascontiguousarray(a.astype(np.complex64 if dt == torch.complex64
                                                                 else np.complex128)).reshape(-1)).to(
                N.require_cuda())
        if psi.numel() != (1 << n):
            raise ValueError(f'statevector length {psi.numel()} != 2**{n}')
        apply_channel(psi, n, model, float(p), gen, qubits)
        normalize_plus_eps(psi)
        if isinstance(sv, torch.Tensor):
            return psi if sv.is_cuda else psi.cpu()
        return psi.cpu().numpy()

    @staticmethod
    def kraus_description(model: str) -> dict:
        """Kraus operators and physical meaning of one of MODELS (unknown names
        describe 'ideal')."""
        desc = {
            'ideal': {'kraus': 1, 'formula': 'K₀ = I', 'physical': 'No noise'},
            'depolarizing': {'kraus': 4, 'formula': 'K₀=√(1-p)I  K₁=√(p/3)X  K₂=√(p/3)Y  K₃=√(p/3)Z',
                             'physical': 'Isotropic Pauli error — equiprobable X, Y, Z'},
            'bitflip': {'kraus': 2, 'formula': 'K₀=√(1-p)I  K₁=√p·X', 'physical': 'Bit flip σ_x with probability p'},
            'phaseflip': {'kraus': 2, 'formula': 'K₀=√(1-p)I  K₁=√p·Z',
                          'physical': 'Pure dephasing σ_z with probability p'},
            'amplitude_damping': {'kraus': 2, 'formula': 'K₀=diag(1,√(1-γ))  K₁=[[0,√γ],[0,0]]',
                                  'physical': 'T₁ energy relaxation |1⟩→|0⟩ with rate γ'},
            'combined': {'kraus': 6, 'formula': 'Depolarizing(p/2) ∘ AmplitudeDamping(p/3)',
                         'physical': 'Worst-case NISQ: dephasing + relaxation'},
        }
        return desc.get(model, desc['ideal'])
