"""ctypes binding of libdesv.so (the C ABI declared in include/desv.h).

The library is built in-tree by ``dense-evolution_b200/build.py`` (or
``__graft_entry__.build()``).  There is no CPU fallback: when the library or a
CUDA device is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, '_lib', 'libdesv.so')

DESV_C64, DESV_C128 = 0, 1
DESV_ELEM_F64, DESV_ELEM_C64, DESV_ELEM_C128 = 0, 1, 2
DESV_OK, DESV_EINVAL, DESV_ENOMEM, DESV_ETIMEOUT, DESV_ECUDA, DESV_EUNSUPPORTED = 0, -1, -2, -3, -4, -5
OP_STAGE, OP_M1, OP_M2, OP_DIAG, OP_GRAD = 0, 1, 2, 3, 4
F_REAL, F_DIAG, F_PHASE1, F_ANTI, F_SIGN, F_PARAM = 1, 2, 4, 8, 16, 32

# numpy mirrors of the packed C structs (little-endian, no implicit padding)
OP_DTYPE = np.dtype([
    ('kind', 'u1'), ('flags', 'u1'), ('s0', 'i1'), ('s1', 'i1'), ('cslot', 'i1'),
    ('ga', 'u1'), ('gb', 'u1'), ('sa', 'i1'), ('sb', 'i1'), ('g', 'u1', (4,)), ('code', '<u2'), ('pad0', 'u1'),
    ('mat', '<u4'), ('param', '<i4'), ('cmask', '<u8'), ('cval', '<u8')])
assert OP_DTYPE.itemsize == 40
PASS_DTYPE = np.dtype([('tile_bits', '<i4'), ('low_bits', '<i4'), ('op_begin', '<i4'), ('op_end', '<i4'),
                       ('high', 'u1', (16,))])
assert PASS_DTYPE.itemsize == 32
ADJ_PASS_DTYPE = np.dtype([('tile_bits', '<i4'), ('low_bits', '<i4'), ('op_begin', '<i4'), ('op_end', '<i4'),
                           ('high', 'u1', (16,)), ('nparams', '<i4'), ('map_begin', '<i4'), ('pad', '<i4', (2,))])
assert ADJ_PASS_DTYPE.itemsize == 48
TERM_DTYPE = np.dtype([('xmask', '<u8'), ('zmask', '<u8'), ('cre', '<f8'), ('cim', '<f8')])
PPASS_DTYPE = np.dtype([('tile_bits', '<i4'), ('low_bits', '<i4'), ('term_begin', '<i4'), ('term_end', '<i4'),
                        ('high', 'u1', (16,))])

_lib = None
_lock = threading.Lock()

_vp, _i, _u64, _d, _sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_double, ctypes.c_size_t
_SIGS = {
    'desv_abi_version': ([], _i),
    'desv_last_error': ([ctypes.c_char_p, _sz], _i),
    'desv_device_status': ([_vp], _i),
    'desv_scratch_bytes': ([_i, _i], _sz),
    'desv_init_basis': ([_vp, _i, _i, _u64, _vp], _i),
    'desv_scale': ([_vp, _i, _i, _d, _d, _vp], _i),
    'desv_apply_gate': ([_vp, _i, _i, _i, _vp, _u64, _u64, _vp, _vp], _i),
    'desv_apply_passes': ([_vp, _i, _i, _vp, _i, _vp, _vp, _vp], _i),
    'desv_norm2': ([_vp, _i, _i, _vp, _vp, _sz, _vp], _i),
    'desv_inner': ([_vp, _vp, _i, _i, _vp, _vp, _sz, _vp], _i),
    'desv_bit_marginals': ([_vp, _i, _i, _vp, _vp, _sz, _vp], _i),
    'desv_probabilities': ([_vp, _i, _i, _vp, _vp], _i),
    'desv_collapse': ([_vp, _i, _i, _i, _i, _d, _vp], _i),
    'desv_pauli_expect': ([_vp, _i, _i, _vp, _i, _vp, _vp, _vp, _sz, _vp], _i),
    'desv_pauli_matvec': ([_vp, _vp, _i, _i, _vp, _i, _vp, _vp, _vp, _sz, _vp], _i),
    'desv_pauli_expect_noalloc': ([_vp, _i, _i, _vp, _i, _vp, _vp, _vp], _i),
    'desv_adjoint_scratch_bytes': ([_i], _sz),
    'desv_batch_workspace_bytes': ([_i, _i, _i], _sz),
    'desv_batch_vqe': ([_i, _i, _i, _vp, _vp, _sz, _vp], _i),
    'desv_adjoint_passes': ([_vp, _vp, _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _sz, _vp], _i),
    'desv_sample_scratch_bytes': ([_i], _sz),
    'desv_sample_prepare': ([_vp, _i, _i, _vp, _sz, _vp, _vp], _i),
    'desv_sample_pick': ([_vp, _i, _i, _vp, _sz, _vp, ctypes.c_int64, _vp, _vp], _i),
    'desv_jit_available': ([ctypes.c_char_p, _sz], _i),
    'desv_jit_load': ([ctypes.c_char_p, ctypes.c_char_p, _i, _i, _i, _i, _i, ctypes.POINTER(_vp),
                       ctypes.c_char_p, _sz], _i),
    'desv_jit_pauli': ([_vp, _vp, _vp, _i, _i, _vp, _i, _vp, _vp, _vp, _sz, _i, _vp], _i),
    'desv_jit_adjoint': ([_vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp], _i),
    'desv_jit_free': ([_vp], _i),
    'desv_jit_pass': ([_vp, _vp, _i, _i, _vp, _vp, _vp], _i),
    'desv_rot_load': ([ctypes.c_char_p, ctypes.c_char_p, _i, _i, _i, _i, ctypes.POINTER(_vp), ctypes.c_char_p, _sz],
                      _i),
    'desv_rot_pass': ([_vp, _vp, _i, _vp, _vp, _i, _vp], _i),
    'desv_bit_reverse': ([_vp, _vp, _i, _i, _vp], _i),
    'desv_jit_compile_check': ([ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _sz], _i),
    'desv_swap_blocks': ([_vp, _vp, _sz, _vp], _i),
    'desv_rows_scratch_bytes': ([_i, _i, _i], _sz),
    'desv_rows_prepare': ([_vp, _i, _i, _i, _vp, _i, _vp, ctypes.c_int64, _vp, _vp, ctypes.c_int64, _vp], _i),
    'desv_apply_passes_rows': ([_vp, _i, _i, _i, _vp, _i, _vp, _vp, ctypes.c_int64, _vp], _i),
    'desv_pauli_matvec_rows': ([_vp, _vp, _i, _i, _i, _vp, _i, _vp, ctypes.c_int64, _vp, _vp, _vp, _sz, _vp], _i),
    'desv_adjoint_passes_rows': ([_vp, _vp, _i, _i, _i, _vp, _i, _vp, _vp, ctypes.c_int64, _vp, _vp,
                                  ctypes.c_int64, _vp, _sz, _vp], _i),
    'desv_jit_pass_rows': ([_vp, _vp, _i, _i, _i, _vp, _vp, ctypes.c_int64, _vp], _i),
    'desv_rows_tangent_prepare': ([_vp, _i, _i, ctypes.c_int64, _i, _vp, _vp, _vp, ctypes.c_int64, _d, _vp, _vp,
                                   _vp], _i),
    'desv_jit_adjoint_rows_split': ([_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, ctypes.c_int64, _vp, _vp,
                                     ctypes.c_int64, _vp, _sz, _vp], _i),
    'desv_jit_pauli_matvec_rows': ([_vp, _vp, _i, _vp, _vp, _i, _i, _i, _vp, _i, _vp, ctypes.c_int64, _vp, _vp, _vp,
                                    _sz, _vp], _i),
    'desv_jit_adjoint_rows': ([_vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, ctypes.c_int64, _vp, _vp, ctypes.c_int64,
                               _vp, _sz, _vp], _i),
}
OPTIONAL = set()


def load_library(path: str = LIB_PATH):
    """Load libdesv.so and declare every exported signature (no CUDA call is made)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(f'libdesv.so not built ({path}); run dense-evolution_b200/build.py')
        lib = ctypes.CDLL(path)
        for name, (args, res) in _SIGS.items():
            if not hasattr(lib, name):
                if name in OPTIONAL:
                    continue
                raise RuntimeError(f'libdesv.so does not export {name}')
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
        if lib.desv_abi_version() != 1:
            raise RuntimeError('libdesv.so ABI version mismatch')
        _lib = lib
        return lib


def lib():
    return _lib if _lib is not None else load_library()


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError('dense_evolution (B200 engine) needs a CUDA device; there is no CPU fallback')
    return torch.device('cuda', torch.cuda.current_device())


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().desv_last_error(buf, 1024)
    return buf.value.decode(errors='replace')


def check(code: int, what: str):
    if code != DESV_OK:
        msg = last_error()
        if code == DESV_EINVAL:
            raise ValueError(f'{what}: {msg}')
        raise RuntimeError(f'{what} failed ({code}): {msg}')


def stream_ptr(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.complex64:
        return DESV_C64
    if t.dtype == torch.complex128:
        return DESV_C128
    raise TypeError(f'statevector dtype must be complex64 or complex128, got {t.dtype}')


_scratch = {}


def scratch(n: int, device: torch.device, stream=None) -> torch.Tensor:
    """Reduction scratch per device and stream, grown on demand and reused by every
    call on that stream (calls on one stream are ordered; two streams never share)."""
    need = int(lib().desv_scratch_bytes(n, 0))
    key = (device.index if device.index is not None else torch.cuda.current_device(), stream_ptr(stream))
    buf = _scratch.get(key)
    if buf is None or buf.numel() * 8 < need:
        buf = torch.empty((need + 7) // 8, dtype=torch.float64, device=device)
        _scratch[key] = buf
    return buf


def device_status():
    check(lib().desv_device_status(ctypes.c_void_p(stream_ptr())), 'device status')
