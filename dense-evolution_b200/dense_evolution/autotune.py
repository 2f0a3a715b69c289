"""Tile-size autotuner for the fused passes.

A fused pass's tile is 2^K amplitudes (K register+lane bits).  Larger tiles
fit more gates per HBM round trip but hold fewer pipeline slots per SM.  The
tuner times each supported K on a synthetic brick-wall layer at the requested
qubit count and stores the winner per (GPU name, qubits, precision) in a JSON
cache (``$DESV_TUNE_CACHE`` or ``~/.cache/desv_tune.json``).  Without a cached
entry the defaults below apply; ``DESV_TILE_BITS`` overrides both.
"""
from __future__ import annotations

import json
import os
import threading

import torch

_lock = threading.Lock()
_cache = None
SUPPORTED = {torch.complex64: (9, 10, 11, 12, 13), torch.complex128: (9, 10, 11, 12)}
DEFAULT = {torch.complex64: 12, torch.complex128: 11}


def _path() -> str:
    return os.environ.get('DESV_TUNE_CACHE', os.path.join(os.path.expanduser('~'), '.cache', 'desv_tune.json'))


def _load():
    global _cache
    if _cache is None:
        try:
            with open(_path()) as f:
                _cache = json.load(f)
        except (OSError, ValueError):
            _cache = {}
    return _cache


def _key(n, dtype):
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else 'cpu'
    return f'{name}|{n}|{"c64" if dtype == torch.complex64 else "c128"}'


def tile_bits(n: int, dtype: torch.dtype) -> int:
    env = os.environ.get('DESV_TILE_BITS')
    if env:
        return min(int(env), n)
    with _lock:
        c = _load()
        k = c.get(_key(n, dtype)) if torch.cuda.is_available() else None
    return min(int(k) if k else DEFAULT[dtype], n)


def record(n: int, dtype: torch.dtype, k: int):
    with _lock:
        c = _load()
        c[_key(n, dtype)] = int(k)
        try:
            os.makedirs(os.path.dirname(_path()), exist_ok=True)
            with open(_path(), 'w') as f:
                json.dump(c, f, indent=1)
        except OSError:
            pass


def tune(n: int, dtype: torch.dtype, layers: int = 4, reps: int = 3, seed: int = 0) -> dict:
    """Time every supported tile size on a random U3 + brick-CZ circuit of `layers`
    layers at n qubits; record and return {K: ms per pass}."""
    import numpy as np
    from .circuits.compiler import CompiledCircuit, QuantumTranspiler
    from .workloads import brick_u3_circuit
    circ = QuantumTranspiler.transpile(brick_u3_circuit(n, layers, seed))
    sv = torch.zeros(1 << n, dtype=dtype, device='cuda')
    sv[0] = 1
    res = {}
    for k in SUPPORTED[dtype]:
        if k > n:
            continue
        plan = CompiledCircuit(circ, n, dtype, tile_bits=k)
        plan.run(sv)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            plan.run(sv)
        e1.record()
        torch.cuda.synchronize()
        res[k] = e0.elapsed_time(e1) / reps
    best = min(res, key=res.get)
    record(n, dtype, best)
    return res


# ---------------------------------------------------------------------------
# batched VQE: tile width of the HBM-resident circuits (n > 12)
# ---------------------------------------------------------------------------

BATCH_SUPPORTED = (10, 11, 12)
BATCH_DEFAULT = 12


def _batch_key(dtype):
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else 'cpu'
    return f'{name}|batch|{"c64" if dtype == torch.complex64 else "c128"}'


def batch_tile_bits(dtype: torch.dtype) -> int:
    """Tile bits of the batched-VQE plans: ``DESV_BATCH_TILE_BITS``, else the
    tuned value cached for this GPU, else 12."""
    env = os.environ.get('DESV_BATCH_TILE_BITS')
    if env:
        return int(env)
    with _lock:
        c = _load()
        k = c.get(_batch_key(dtype)) if torch.cuda.is_available() else None
    return int(k) if k else BATCH_DEFAULT


def tune_batch(items, use_float32: bool = True, reps: int = 2, seed: int = 0) -> dict:
    """Time one launch of BatchVQE over `items` at every supported tile width,
    record the fastest for this GPU and return {K: ms per launch}."""
    import numpy as np
    from .batch import BatchVQE
    dtype = torch.complex64 if use_float32 else torch.complex128
    rng = np.random.default_rng(seed)
    res = {}
    for k in BATCH_SUPPORTED:
        # the interpreter's passes stand in for the specialised ones here, so that
        # tuning compiles nothing
        b = BatchVQE(items, use_float32=use_float32, tile_bits=k, rows_jit=False)
        b.set_theta([rng.uniform(-np.pi, np.pi, n) for n in b.nparams_list()])
        b.launch()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            b.launch()
        e1.record()
        torch.cuda.synchronize()
        res[k] = e0.elapsed_time(e1) / reps
        del b
    best = min(res, key=res.get)
    with _lock:
        c = _load()
        c[_batch_key(dtype)] = int(best)
        try:
            os.makedirs(os.path.dirname(_path()), exist_ok=True)
            with open(_path(), 'w') as f:
                json.dump(c, f, indent=1)
        except OSError:
            pass
    return res
