"""desv_pauli_expect_noalloc: the Pauli-sum expectation for callers that can't
allocate device memory -- e.g. a host whose caching allocator already holds
nearly all of HBM, or a plugin that may only allocate at load time.  It takes
no scratch buffer; its partial sums live in a fixed device array inside the
library.  Checked through the C ABI against the allocating entry point
(desv_pauli_expect) on two calls in a row, so the second call also proves
that the shared array's leftover contents from the first call do not leak
into the result.  Collected last (file name) so a failure here cannot hide
any other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _terms(n):
    t = [(-1.0, {i: 'Z', i + 1: 'Z'}) for i in range(n - 1)] + [(-0.8, {i: 'X'}) for i in range(n)]
    t += [(0.3, {i: 'X', i + 1: 'X'}) for i in range(0, n - 1, 3)] + [(0.2, {i: 'Y', i + 2: 'Y'}) for i in range(n - 2)]
    t += [(0.05, 'X' * n), (-0.07, 'YZ' * (n // 2))]       # wider than any tile: direct passes
    return t


@pytest.mark.parametrize('dtype', ['c64', 'c128'])
def test_noalloc_matches_allocating_entry_point(dtype):
    import torch
    from dense_evolution import _native as N
    from dense_evolution.physics.observables import PauliPlan
    lib = N.lib()
    n = 18
    tdt = torch.complex64 if dtype == 'c64' else torch.complex128
    rng = np.random.default_rng(7)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    t = torch.from_numpy(psi).to('cuda').to(tdt)
    plan = PauliPlan(_terms(n), n, tile_bits=11 if dtype == 'c64' else 10)
    terms_dev = plan.terms_dev(t.device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    code = N.dtype_code(t)
    passes = ctypes.c_void_p(plan.passes.ctypes.data)

    ref = torch.zeros(2, dtype=torch.float64, device='cuda')
    sc = torch.empty(int(lib.desv_scratch_bytes(n, code)) // 8 + 1, dtype=torch.float64, device='cuda')
    N.check(lib.desv_pauli_expect(ctypes.c_void_p(t.data_ptr()), n, code, passes, len(plan.passes),
                                  ctypes.c_void_p(terms_dev.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                  ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8, st), 'expect')
    outs = []
    for _ in range(2):
        out = torch.full((2,), float('nan'), dtype=torch.float64, device='cuda')
        N.check(lib.desv_pauli_expect_noalloc(ctypes.c_void_p(t.data_ptr()), n, code, passes, len(plan.passes),
                                              ctypes.c_void_p(terms_dev.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                              st), 'noalloc expect')
        outs.append(out.cpu().numpy())
    r = ref.cpu().numpy()
    tol = 1e-12
    for o in outs:
        assert np.all(np.isfinite(o))
        assert np.allclose(o, r, rtol=0, atol=tol)
    N.device_status()


def test_noalloc_rejects_more_passes_than_the_fixed_array_holds():
    import torch
    from dense_evolution import _native as N
    from dense_evolution.physics.observables import PauliPlan
    lib = N.lib()
    n = 12
    t = torch.zeros(1 << n, dtype=torch.complex128, device='cuda')
    t[0] = 1
    plan = PauliPlan([(1.0, {0: 'X'})], n, tile_bits=10)
    many = np.repeat(plan.passes, 64)           # 64 passes with terms: beyond the fixed partial-sum rows
    out = torch.zeros(2, dtype=torch.float64, device='cuda')
    r = lib.desv_pauli_expect_noalloc(ctypes.c_void_p(t.data_ptr()), n, N.DESV_C128, ctypes.c_void_p(many.ctypes.data),
                                      len(many), ctypes.c_void_p(plan.terms_dev(t.device).data_ptr()),
                                      ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(0))
    assert r == N.DESV_EINVAL
    assert 'partial rows' in N.last_error()


def test_noalloc_with_no_terms_writes_zero():
    """A call whose passes all have empty term ranges launches no pass and
    must still overwrite the caller's output with (0, 0)."""
    import torch
    from dense_evolution import _native as N
    from dense_evolution.physics.observables import PauliPlan
    lib = N.lib()
    n = 12
    t = torch.zeros(1 << n, dtype=torch.complex64, device='cuda')
    t[0] = 1
    plan = PauliPlan([(1.0, {0: 'X'})], n, tile_bits=10)
    empty = plan.passes.copy()
    empty['term_end'] = empty['term_begin']
    out = torch.full((2,), float('nan'), dtype=torch.float64, device='cuda')
    N.check(lib.desv_pauli_expect_noalloc(ctypes.c_void_p(t.data_ptr()), n, N.DESV_C64,
                                          ctypes.c_void_p(empty.ctypes.data), len(empty),
                                          ctypes.c_void_p(plan.terms_dev(t.device).data_ptr()),
                                          ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(0)), 'noalloc expect')
    assert out.cpu().tolist() == [0.0, 0.0]


def test_noalloc_on_a_user_stream():
    """The call is ordered on the caller's stream: run it on a freshly created
    torch stream right after the state is written there, and compare with the
    allocating entry point on the default stream."""
    import torch
    from dense_evolution import _native as N
    from dense_evolution.physics.observables import PauliPlan
    lib = N.lib()
    n = 16
    rng = np.random.default_rng(11)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    plan = PauliPlan(_terms(n), n, tile_bits=11)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        t = torch.from_numpy(psi).to('cuda').to(torch.complex64)
        terms_dev = plan.terms_dev(t.device)
        out = torch.full((2,), float('nan'), dtype=torch.float64, device='cuda')
        N.check(lib.desv_pauli_expect_noalloc(ctypes.c_void_p(t.data_ptr()), n, N.DESV_C64,
                                              ctypes.c_void_p(plan.passes.ctypes.data), len(plan.passes),
                                              ctypes.c_void_p(terms_dev.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                              ctypes.c_void_p(s.cuda_stream)), 'noalloc expect')
    s.synchronize()
    ref = torch.zeros(2, dtype=torch.float64, device='cuda')
    sc = torch.empty(int(lib.desv_scratch_bytes(n, N.DESV_C64)) // 8 + 1, dtype=torch.float64, device='cuda')
    N.check(lib.desv_pauli_expect(ctypes.c_void_p(t.data_ptr()), n, N.DESV_C64, ctypes.c_void_p(plan.passes.ctypes.data),
                                  len(plan.passes), ctypes.c_void_p(terms_dev.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                  ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8,
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), 'expect')
    assert np.allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=0, atol=1e-12)
    N.device_status()
