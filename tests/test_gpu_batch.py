"""Batched VQE (one persistent launch over circuits of different qubit counts)
against the single-circuit adjoint path and the oracle."""
import numpy as np
import pytest

from oracle import sv_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('f32', [False, True])
def test_batch_matches_single_circuit_adjoint(f32):
    import dense_evolution as de
    from dense_evolution.batch import BatchVQE, hea_xxz_batch
    rng = np.random.default_rng(3)
    ns = [9, 14, 10, 12, 13, 9, 11]
    jz = rng.uniform(0.5, 1.5, len(ns))
    items = hea_xxz_batch(ns, 2, jz)
    b = BatchVQE(items, use_float32=f32)
    thetas = [rng.uniform(-np.pi, np.pi, 2 * n * 2) for n in ns]
    e, g = b.run(thetas)
    for i, (circ, n, terms) in enumerate(items):
        fn, npar = de.circuit_to_energy_fn(circ, n, use_float32=f32)
        e1, g1, _ = fn.program.value_and_grad(thetas[i], terms)
        # energies to the complex64 bar |dE| <= 1e-6 (both paths divide by the
        # FP64 norm); gradients to 1e-5
        assert e[i] == pytest.approx(e1, abs=1e-6 if f32 else 1e-10)
        assert np.allclose(g[i], g1, atol=1e-5 if f32 else 1e-10)
    # oracle for the two smallest
    for i in (0, 5):
        circ, n, terms = items[i]
        rows, _ = O.energy_template([{'name': c[0], 'qubits': [q for q in c[1:] if isinstance(q, int)]}
                                     for c in circ], n)
        e_ref, _ = O.energy(thetas[i], rows, n, terms)
        assert e[i] == pytest.approx(e_ref, abs=1e-6 if f32 else 1e-10)
        fd = O.fd_gradient(thetas[i], rows, n, terms, h=1e-5, indices=[0, 7, 20])
        assert np.allclose(g[i][[0, 7, 20]], fd, atol=1e-4 if f32 else 1e-7)
    from dense_evolution import _native as N
    N.device_status()


def test_batch_cuda_graph_replay():
    from dense_evolution.batch import BatchVQE, hea_xxz_batch
    rng = np.random.default_rng(5)
    ns = [10, 13, 12, 9]
    b = BatchVQE(hea_xxz_batch(ns, 3, rng.uniform(0.5, 1.5, len(ns))))
    th = [rng.uniform(-np.pi, np.pi, 6 * n) for n in ns]
    e0, g0 = b.run(th)
    e1, g1 = b.run(th, use_graph=True)
    th2 = [t + 0.1 for t in th]
    e2, g2 = b.run(th2, use_graph=True)
    e3, g3 = b.run(th2)
    assert np.allclose(e0, e1) and all(np.allclose(x, y) for x, y in zip(g0, g1))
    assert np.allclose(e2, e3) and all(np.allclose(x, y) for x, y in zip(g2, g3))
    assert not np.allclose(e0, e2)


@pytest.mark.parametrize('k', [10, 11])
def test_batch_tile_widths_agree(k):
    """Every tile width the autotuner may pick gives the same energies and
    gradients (streamed circuits of 13-15 qubits; resident ones keep one tile)."""
    from dense_evolution import _native as N
    from dense_evolution.batch import BatchVQE, hea_xxz_batch
    rng = np.random.default_rng(11)
    ns = [13, 9, 15, 12, 14]
    items = hea_xxz_batch(ns, 2, rng.uniform(0.5, 1.5, len(ns)))
    th = [rng.uniform(-np.pi, np.pi, 4 * n) for n in ns]
    e_ref, g_ref = BatchVQE(items, use_float32=False, tile_bits=12).run(th)
    e, g = BatchVQE(items, use_float32=False, tile_bits=k).run(th)
    assert np.allclose(e, e_ref, atol=1e-10)
    assert all(np.allclose(x, y, atol=1e-10) for x, y in zip(g, g_ref))
    assert N.device_status() in (None, 0)


@pytest.mark.parametrize('f32', [False, True])
def test_rows_groups_match_persistent_launch(f32):
    """Circuits wider than 12 qubits run as rows (one launch per pass over all
    circuits of a structure); forcing them into the persistent launch (one CTA
    per circuit) must give the same energies and gradients: complex128 to
    1e-10, complex64 energies to the 1e-6 bar and gradients to 1e-5."""
    from dense_evolution import _native as N
    from dense_evolution.batch import BatchVQE, hea_xxz_batch
    rng = np.random.default_rng(21)
    ns = [13, 16, 13, 9, 14, 16, 13, 12, 14]
    items = hea_xxz_batch(ns, 3, rng.uniform(0.5, 1.5, len(ns)))
    th = [rng.uniform(-np.pi, np.pi, 6 * n) for n in ns]
    rows = BatchVQE(items, use_float32=f32)
    assert len(rows.groups) == 3 and [len(g[1]) for g in rows.rplans] == [3, 2, 2]
    pers = BatchVQE(items, use_float32=f32, rows_from=99)
    assert not pers.groups
    e_r, g_r = rows.run(th)
    e_p, g_p = pers.run(th)
    assert np.allclose(e_r, e_p, atol=1e-6 if f32 else 1e-10)
    assert all(np.allclose(x, y, atol=1e-5 if f32 else 1e-10) for x, y in zip(g_r, g_p))
    # graph replay of the rows launches with new angles
    th2 = [t - 0.2 for t in th]
    e_g, g_g = rows.run(th2, use_graph=True)
    e_e, g_e = pers.run(th2)
    assert np.allclose(e_g, e_e, atol=1e-6 if f32 else 1e-10)
    assert all(np.allclose(x, y, atol=1e-5 if f32 else 1e-10) for x, y in zip(g_g, g_e))
    assert N.device_status() in (None, 0)

