"""The C-ABI library loads and exports every entry point include/desv.h declares
(no CUDA call is made)."""
import ctypes
import os
import re

from conftest import ROOT


def test_library_exports_header_symbols():
    from dense_evolution import _native as N
    lib = N.load_library()
    with open(os.path.join(ROOT, 'include', 'desv.h')) as f:
        hdr = f.read()
    names = sorted(set(re.findall(r'^\s*(?:int|size_t)\s+(desv_\w+)\s*\(', hdr, re.M)))
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert lib.desv_abi_version() == 1
    assert lib.desv_scratch_bytes(30, 0) > 0


def test_struct_layouts_match_header():
    from dense_evolution import _native as N
    assert N.OP_DTYPE.itemsize == 40 and N.PASS_DTYPE.itemsize == 32 and N.ADJ_PASS_DTYPE.itemsize == 48
    assert N.TERM_DTYPE.itemsize == 32 and N.PPASS_DTYPE.itemsize == 32


def test_invalid_arguments_are_rejected_without_a_gpu():
    from dense_evolution import _native as N
    lib = N.load_library()
    # null statevector: validated on the host before any CUDA call
    r = lib.desv_init_basis(None, 4, 0, 0, None)
    assert r == N.DESV_EINVAL
    assert 'null' in N.last_error()
    r = lib.desv_scale(ctypes.c_void_p(16), 40, 0, 1.0, 0.0, None)
    assert r == N.DESV_EINVAL
