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
    """Finite-shot counts {'bitstring': count} (qubit 0 = leftmost character)
    of n_shots projective measurements in the computational basis
    (utils/measurement.py:17-68 of the reference).

    The distribution stays on the GPU: FP64 block sums and their prefix form
    the CDF, and one warp per shot searches it.  The uniforms are drawn on the
    host as ``rng.random(n_shots)`` -- the draws ``rng.choice`` makes -- so a
    seeded generator gives the reference's samples."""
    a = _as_state(statevector)
    dim = a.shape[0]
    n = dim.bit_length() - 1
    if 1 << n != dim:
        raise ValueError(f"statevector length {dim} is not a power of 2")
    if n_shots < 1:
        raise ValueError(f"n_shots must be >= 1, got {n_shots}")
    if a.dtype not in (torch.complex64, torch.complex128):
        a = a.to(torch.complex128)
    lib, st = N.lib(), ctypes.c_void_p(N.stream_ptr())
    nbytes = int(lib.desv_sample_scratch_bytes(n))
    scratch = torch.empty((nbytes + 7) // 8, dtype=torch.float64, device=a.device)
    total = torch.empty(1, dtype=torch.float64, device=a.device)
    N.check(lib.desv_sample_prepare(ctypes.c_void_p(a.data_ptr()), n, N.dtype_code(a),
                                    ctypes.c_void_p(scratch.data_ptr()), scratch.numel() * 8,
                                    ctypes.c_void_p(total.data_ptr()), st), 'sample prepare')
    t = float(total.item())
    if not np.isfinite(t) or t <= 0:
        raise ValueError("statevector has zero or non-finite total probability")
    rng = np.random.default_rng() if rng is None else rng
    u = torch.from_numpy(rng.random(int(n_shots))).to(a.device)
    idx = torch.empty(int(n_shots), dtype=torch.int64, device=a.device)
    N.check(lib.desv_sample_pick(ctypes.c_void_p(a.data_ptr()), n, N.dtype_code(a),
                                 ctypes.c_void_p(scratch.data_ptr()), scratch.numel() * 8,
                                 ctypes.c_void_p(u.data_ptr()), int(n_shots), ctypes.c_void_p(idx.data_ptr()), st),
            'sample pick')
    values, freqs = torch.unique(idx, return_counts=True)
    return {format(int(v), f'0{n}b'): int(f) for v, f in zip(values.cpu().numpy(), freqs.cpu().numpy())}
