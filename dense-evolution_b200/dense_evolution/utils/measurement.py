"""Measurement helpers (the reference's ``utils/measurement.py:17-94``)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .. import _native as N

__all__ = ['sample_counts', 'statevector_fidelity']


def _as_state(x):
    if isinstance(x, torch.Tensor):
        t = x.reshape(-1)
        return t if t.is_cuda else t.to(N.require_cuda())
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x)).astype(np.complex128).reshape(-1)).to(
        N.require_cuda())


def statevector_fidelity(statevector_a, statevector_b) -> float:
    """|<a|b>|^2 with an FP64-accumulated inner product on the GPU."""
    a, b = _as_state(statevector_a), _as_state(statevector_b)
    if a.shape != b.shape:
        raise ValueError(f"statevector shapes differ: {tuple(a.shape)} vs {tuple(b.shape)}")
    dim = a.shape[0]
    n = dim.bit_length() - 1
    if 1 << n != dim:
        raise ValueError(f"statevector length {dim} is not a power of 2")
    if a.dtype != b.dtype:
        a, b = a.to(torch.complex128), b.to(torch.complex128)
    out = torch.empty(2, dtype=torch.float64, device=a.device)
    sc = N.scratch(n, a.device)
    N.check(N.lib().desv_inner(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), n, N.dtype_code(a),
                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8,
                               ctypes.c_void_p(N.stream_ptr())), 'inner product')
    re, im = out.cpu().numpy()
    return float(re * re + im * im)


def sample_counts(statevector, n_shots, rng=None):
    """Finite-shot counts {'bitstring': count} (qubit 0 = leftmost character)."""
    a = _as_state(statevector)
    dim = a.shape[0]
    n = dim.bit_length() - 1
    if 1 << n != dim:
        raise ValueError(f"statevector length {dim} is not a power of 2")
    if n_shots < 1:
        raise ValueError(f"n_shots must be >= 1, got {n_shots}")
    probs = torch.empty(dim, dtype=torch.float64, device=a.device)
    if a.dtype not in (torch.complex64, torch.complex128):
        a = a.to(torch.complex128)
    N.check(N.lib().desv_probabilities(ctypes.c_void_p(a.data_ptr()), n, N.dtype_code(a),
                                       ctypes.c_void_p(probs.data_ptr()), ctypes.c_void_p(N.stream_ptr())),
            'probabilities')
    p = probs.cpu().numpy()
    total = p.sum()
    if not np.isfinite(total) or total <= 0:
        raise ValueError("statevector has zero or non-finite total probability")
    p = p / total
    rng = np.random.default_rng() if rng is None else rng
    outcomes = rng.choice(dim, size=n_shots, p=p)
    values, freqs = np.unique(outcomes, return_counts=True)
    return {format(int(v), f'0{n}b'): int(f) for v, f in zip(values, freqs)}
