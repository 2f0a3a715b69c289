"""Pauli-string observables on the GPU: the reference's
``dense_evolution/physics/observables.py:38-523`` API.

Every term P = prod_q sigma_q acts as (P psi)[i] = psi[i ^ x] * i^{#Y} *
(-1)^popcount((i ^ x) & z) with x = the X/Y bits and z = the Y/Z bits (qubit q
is index bit n-1-q).  Terms are compiled into tile passes (``desv_pauli_pass``):
every term whose flip mask x lies in a pass's tile bits is evaluated from the
tile in shared memory, so a whole Hamiltonian costs a few reads of psi instead
of the reference's >= 4 passes per term.  Expectations are accumulated in FP64.

Statevectors may be NumPy arrays (uploaded as complex128, like the reference's
implicit upcast) or CUDA tensors (used in place, in their own precision).
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from .. import _native as N

__all__ = ['pauli_expectation', 'pauli_sum_expectation', 'pauli_hamiltonian_to_matrix', 'pauli_sum_matvec',
           'multiply_pauli_terms', 'pauli_sum_matvec_jax', 'pauli_sum_expectation_jax', 'PauliSumOperator',
           'PauliPlan']

_PAULI_MATRICES = {
    'I': np.eye(2, dtype=np.complex128),
    'X': np.array([[0, 1], [1, 0]], dtype=np.complex128),
    'Y': np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    'Z': np.array([[1, 0], [0, -1]], dtype=np.complex128),
}


def _normalize_terms(pauli_terms, n_qubits=None) -> Dict[int, str]:
    """String ('IXYZ', qubit 0 first), dict {qubit: letter} or (qubit, letter)
    pairs -> {qubit: 'X'|'Y'|'Z'} with identities dropped (observables.py:38-60)."""
    if isinstance(pauli_terms, str):
        if n_qubits is not None and len(pauli_terms) != n_qubits:
            raise ValueError(f"pauli_terms string has length {len(pauli_terms)}, but n_qubits={n_qubits}")
        terms = {q: p.upper() for q, p in enumerate(pauli_terms) if p.upper() != 'I'}
    elif isinstance(pauli_terms, dict):
        terms = {int(q): str(p).upper() for q, p in pauli_terms.items() if str(p).upper() != 'I'}
    else:
        terms = {int(q): str(p).upper() for q, p in pauli_terms if str(p).upper() != 'I'}
    for q, p in terms.items():
        if p not in ('X', 'Y', 'Z'):
            raise ValueError(f"unknown Pauli operator {p!r} for qubit {q}, expected one of X, Y, Z, I")
        if q < 0:
            raise ValueError(f"qubit index {q} must be >= 0")
    return terms


def _n_of(dim: int, what: str) -> int:
    n = int(dim).bit_length() - 1
    if 1 << n != dim:
        raise ValueError(f"{what} length {dim} is not a power of 2")
    return n


# ---------------------------------------------------------------------------
# term compilation
# ---------------------------------------------------------------------------

class PauliPlan:
    """Terms of a Pauli sum packed into tile passes for one qubit count."""

    MAX_TERMS_PER_PASS = 512

    def __init__(self, terms, n: int, n_qubits_check=None, tile_bits: int = 11):
        self.n = n
        rows = []
        self.all_real = True
        for coeff, pt in terms:
            t = _normalize_terms(pt, n_qubits_check)
            if t and max(t) >= n:
                raise ValueError(f"pauli_terms references qubit {max(t)}, but the statevector only spans {n} qubits")
            x = z = 0
            ny = 0
            for q, p in t.items():
                b = 1 << (n - 1 - q)
                if p in ('X', 'Y'):
                    x |= b
                if p in ('Y', 'Z'):
                    z |= b
                ny += p == 'Y'
            c = complex(coeff) * (1j ** ny)
            if complex(coeff).imag != 0:
                self.all_real = False
            rows.append((x, z, c, len(rows)))
        self.nterms = len(rows)
        K = min(tile_bits, n)
        lane = min(5, K)
        groups: Dict[int, list] = {}
        for x, z, c, i in rows:
            groups.setdefault(x, []).append((x, z, c, i))
        # greedy first-fit of flip masks into tiles (high bits >= lane)
        bins: List[Tuple[set, list]] = []
        direct: List[int] = []        # flip masks wider than a tile
        for x in sorted(groups, key=lambda v: (v.bit_length(), v)):
            need = {b for b in range(n) if (x >> b) & 1 and b >= lane}
            if len(need) > K - lane:
                direct.append(x)
                continue
            placed = False
            for H, members in bins:
                if len(H | need) <= K - lane and sum(len(groups[m]) for m in members) + len(groups[x]) <= \
                        self.MAX_TERMS_PER_PASS:
                    H |= need
                    members.append(x)
                    placed = True
                    break
            if not placed:
                bins.append((set(need), [x]))
        geoms = [self._geometry(H, K, lane) for H, _ in bins]
        self._balance(bins, geoms, groups)
        term_rows, pass_rows = [], []
        order = []          # packed term row -> index of the term in the caller's list
        for (H, members), (L, high) in zip(bins, geoms):
            begin = len(term_rows)
            for x in sorted(members):
                for (xx, z, c, i) in groups[x]:
                    term_rows.append((xx, z, c.real, c.imag))
                    order.append(i)
            r = np.zeros((), dtype=N.PPASS_DTYPE)
            r['tile_bits'], r['low_bits'], r['term_begin'], r['term_end'] = K, L, begin, len(term_rows)
            hb = np.zeros(16, np.uint8)
            hb[:len(high)] = high
            r['high'] = hb
            pass_rows.append(r)
        for i in range(0, len(direct), 64):
            begin = len(term_rows)
            for x in direct[i:i + 64]:
                for (xx, z, c, k) in groups[x]:
                    term_rows.append((xx, z, c.real, c.imag))
                    order.append(k)
            r = np.zeros((), dtype=N.PPASS_DTYPE)
            r['tile_bits'], r['low_bits'], r['term_begin'], r['term_end'] = 0, 0, begin, len(term_rows)
            pass_rows.append(r)
        self.terms = np.array(term_rows, dtype=N.TERM_DTYPE) if term_rows else np.zeros(0, N.TERM_DTYPE)
        self.order = np.array(order, dtype=np.int64)
        self.passes = np.array(pass_rows, dtype=N.PPASS_DTYPE) if pass_rows else np.zeros(0, N.PPASS_DTYPE)
        self._dev = {}
        self._jit = {}

    @staticmethod
    def _geometry(H, K: int, lane: int):
        """(low bits L, sorted high bits) of a tile over the high bits H: the
        contiguous low run grows while fewer than K - L high bits are needed."""
        L = lane
        while True:
            high = sorted(h for h in H if h >= L)
            L2 = K - len(high)
            if L2 == L:
                break
            L = L2
        return L, sorted(h for h in H if h >= L)

    def _balance(self, bins, geoms, groups):
        """Spread the flip masks that more than one tile covers (those on the low
        bits are in every tile) over the passes.  A pass's time grows with its
        flip masks (one partner read and product per mask and amplitude), and the
        first fit puts every low-bit mask into the first pass, which made that
        pass the longest (68 us against 46 and 36 us for the 24-qubit TFIM chain).
        Tile geometries do not change; the term cap per pass still holds."""
        if len(bins) < 2:
            return
        covers = [((1 << L) - 1) | sum(1 << h for h in high) for L, high in geoms]

        def cost(x):
            return (1.0 if x else 0.25) + 0.05 * len(groups[x])

        before = [list(m) for _, m in bins]
        load, nterm = [0.0] * len(bins), [0] * len(bins)
        flexible = []
        for bi, (_, members) in enumerate(bins):
            keep = []
            for x in members:
                cands = [bj for bj, cv in enumerate(covers) if x & ~cv == 0]
                if len(cands) > 1:
                    flexible.append((x, cands))
                else:
                    keep.append(x)
                    load[bi] += cost(x)
                    nterm[bi] += len(groups[x])
            members[:] = keep
        for x, cands in sorted(flexible, key=lambda e: (-cost(e[0]), e[0])):
            ok = [b for b in cands if nterm[b] + len(groups[x]) <= self.MAX_TERMS_PER_PASS]
            if not ok:      # no room under the cap: keep the first fit
                for (_, members), old in zip(bins, before):
                    members[:] = old
                return
            b = min(ok, key=lambda b: (load[b], b))
            bins[b][1].append(x)
            load[b] += cost(x)
            nterm[b] += len(groups[x])

    @property
    def npasses(self) -> int:
        return len(self.passes)

    def specialised(self, device, dtype, matvec: bool):
        """ctypes array of one specialised kernel handle (or NULL) per pass for
        desv_jit_pauli, or None when the interpreter runs every pass."""
        from ..circuits import jit
        if not jit.enabled(self.n):
            return None
        dev = device.index if device.index is not None else torch.cuda.current_device()
        key = (dev, dtype, matvec)
        h = self._jit.get(key)
        if h is None:
            ks = jit.compile_pauli(self.terms, self.passes, matvec, dtype == torch.complex64, dev)
            arr = (ctypes.c_void_p * max(1, len(ks)))(*[k.handle.value if k is not None else None for k in ks])
            h = (arr, ks)                       # the kernels stay referenced with their handles
            self._jit[key] = h
        return h[0]

    def terms_dev(self, device) -> torch.Tensor:
        key = (device.type, device.index)
        t = self._dev.get(key)
        if t is None:
            t = torch.from_numpy(self.terms.view(np.uint8).copy()).to(device)
            self._dev[key] = t
        return t

    def expect(self, psi: torch.Tensor, stream=None) -> torch.Tensor:
        """Device tensor [re, im] of sum_k c_k <psi|P_k|psi> (not synchronised)."""
        out = torch.zeros(2, dtype=torch.float64, device=psi.device)
        if self.nterms == 0:
            return out
        sc = N.scratch(self.n, psi.device, stream)
        tdev = self.terms_dev(psi.device)
        hs = self.specialised(psi.device, psi.dtype, False)
        if hs is not None:
            N.check(N.lib().desv_jit_pauli(hs, ctypes.c_void_p(psi.data_ptr()), None, self.n, N.dtype_code(psi),
                                           ctypes.c_void_p(self.passes.ctypes.data), len(self.passes),
                                           ctypes.c_void_p(tdev.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                           ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8, 0,
                                           ctypes.c_void_p(N.stream_ptr(stream))), 'pauli expectation')
            return out
        N.check(N.lib().desv_pauli_expect(ctypes.c_void_p(psi.data_ptr()), self.n, N.dtype_code(psi),
                                          ctypes.c_void_p(self.passes.ctypes.data), len(self.passes),
                                          ctypes.c_void_p(tdev.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8,
                                          ctypes.c_void_p(N.stream_ptr(stream))), 'pauli expectation')
        return out

    def matvec(self, psi: torch.Tensor, out: torch.Tensor = None, want_expect: bool = False, stream=None):
        """out = H psi (new tensor unless given); optionally also returns <psi|H|psi> as a device tensor."""
        if out is None:
            out = torch.empty_like(psi)
        e = torch.zeros(2, dtype=torch.float64, device=psi.device) if want_expect else None
        if self.nterms == 0:
            out.zero_()
            return (out, e) if want_expect else out
        sc = N.scratch(self.n, psi.device, stream)
        tdev = self.terms_dev(psi.device)
        hs = self.specialised(psi.device, psi.dtype, True)
        if hs is not None:
            N.check(N.lib().desv_jit_pauli(hs, ctypes.c_void_p(psi.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                           self.n, N.dtype_code(psi), ctypes.c_void_p(self.passes.ctypes.data),
                                           len(self.passes), ctypes.c_void_p(tdev.data_ptr()),
                                           ctypes.c_void_p(e.data_ptr()) if e is not None else None,
                                           ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8, 1,
                                           ctypes.c_void_p(N.stream_ptr(stream))), 'pauli matvec')
            return (out, e) if want_expect else out
        N.check(N.lib().desv_pauli_matvec(ctypes.c_void_p(psi.data_ptr()), ctypes.c_void_p(out.data_ptr()), self.n,
                                          N.dtype_code(psi), ctypes.c_void_p(self.passes.ctypes.data),
                                          len(self.passes), ctypes.c_void_p(tdev.data_ptr()),
                                          ctypes.c_void_p(e.data_ptr()) if e is not None else None,
                                          ctypes.c_void_p(sc.data_ptr()), sc.numel() * 8,
                                          ctypes.c_void_p(N.stream_ptr(stream))), 'pauli matvec')
        return (out, e) if want_expect else out


_plan_cache: Dict[tuple, PauliPlan] = {}


def _terms_key(terms, n, nq):
    try:
        key = (n, nq, tuple((complex(c), p if isinstance(p, str) else
                             tuple(sorted(p.items())) if isinstance(p, dict) else tuple(map(tuple, p)))
                            for c, p in terms))
        hash(key)
        return key
    except TypeError:
        return None


def _plan(terms, n, n_qubits, dtype, wide_tiles) -> PauliPlan:
    """The Pauli plan of a term list: 11-bit tiles for complex64 (10 for
    complex128, the interpreter's bound), or 12-bit ones when every tiled pass
    of that plan gets a specialised kernel (fewer passes, and twice the work per
    tile against each tile's barriers)."""
    if dtype == torch.complex64 and wide_tiles and n >= 12:
        from ..circuits import jit
        wide = PauliPlan(terms, n, n_qubits, tile_bits=12)
        if all(int(p['tile_bits']) == 0 or (int(p['term_end']) - int(p['term_begin']) <= jit.MAX_PAULI_TERMS and
                                            int(p['tile_bits']) - int(p['low_bits']) <= 8) for p in wide.passes):
            return wide
    return PauliPlan(terms, n, n_qubits, tile_bits=11 if dtype == torch.complex64 else 10)


def plan_for(terms, n: int, n_qubits=None, dtype=torch.complex128, wide_tiles=None) -> PauliPlan:
    """Cached Pauli plan; wide_tiles (default: the specialised kernels are in
    use at this size) allows 12-bit tiles for complex64."""
    if wide_tiles is None:
        from ..circuits import jit
        wide_tiles = jit.enabled(n)
    wide_tiles = bool(wide_tiles)
    terms = list(terms)
    key = _terms_key(terms, n, n_qubits)
    if key is not None:
        key = key + (dtype == torch.complex64, wide_tiles)
        p = _plan_cache.get(key)
        if p is None:
            p = _plan(terms, n, n_qubits, dtype, wide_tiles)
            if len(_plan_cache) > 64:
                _plan_cache.clear()
            _plan_cache[key] = p
        return p
    return _plan(terms, n, n_qubits, dtype, wide_tiles)


def _to_device_state(statevector) -> Tuple[torch.Tensor, bool]:
    """(CUDA tensor, came_from_numpy)."""
    if isinstance(statevector, torch.Tensor):
        t = statevector.reshape(-1)
        if not t.is_cuda:
            t = t.to(N.require_cuda())
        if t.dtype not in (torch.complex64, torch.complex128):
            t = t.to(torch.complex128)
        return t.contiguous(), False
    arr = np.asarray(statevector).reshape(-1).astype(np.complex128)
    return torch.from_numpy(arr).to(N.require_cuda()), True


# ---------------------------------------------------------------------------
# public functions
# ---------------------------------------------------------------------------

def pauli_expectation(statevector, pauli_terms, n_qubits=None) -> float:
    """<psi|P|psi> of one Pauli string (observables.py:97-149)."""
    if not isinstance(statevector, torch.Tensor):
        dim = np.asarray(statevector).shape[0]
    else:
        dim = statevector.reshape(-1).shape[0]
    n = _n_of(dim, 'statevector')
    plan = plan_for([(1.0, pauli_terms)], n, n_qubits)
    psi, _ = _to_device_state(statevector)
    return float(plan.expect(psi)[0].item())


def pauli_sum_expectation(statevector, terms, n_qubits=None):
    """sum_i coeff_i <psi|P_i|psi> in one fused GPU reduction (observables.py:152-186)."""
    terms = list(terms)
    if not terms:
        return 0.0
    dim = statevector.reshape(-1).shape[0] if isinstance(statevector, torch.Tensor) else np.asarray(statevector).shape[0]
    n = _n_of(dim, 'statevector')
    psi, _ = _to_device_state(statevector)
    plan = plan_for(terms, n, n_qubits, psi.dtype)
    r = plan.expect(psi).cpu().numpy()
    return float(r[0]) if plan.all_real else complex(r[0], r[1])


def pauli_sum_matvec(vector, terms, n_qubits=None):
    """H @ vector without building H (observables.py:250-308).  NumPy in ->
    NumPy complex128 out; CUDA tensor in -> CUDA tensor out."""
    was_tensor = isinstance(vector, torch.Tensor)
    v, _ = _to_device_state(vector if was_tensor else np.asarray(vector, dtype=np.complex128))
    n = _n_of(v.shape[0], 'vector')
    plan = plan_for(list(terms), n, n_qubits, v.dtype)
    out = plan.matvec(v)
    return out if was_tensor else out.cpu().numpy()


def pauli_hamiltonian_to_matrix(terms, n_qubits):
    """Dense H = sum c_k P_k (observables.py:189-247); host-side, small n only."""
    if n_qubits < 1:
        raise ValueError(f"n_qubits must be >= 1, got {n_qubits}")
    dim = 1 << n_qubits
    H = np.zeros((dim, dim), dtype=np.complex128)
    for coeff, pt in terms:
        t = _normalize_terms(pt, n_qubits)
        if t and max(t) >= n_qubits:
            raise ValueError(f"term references qubit {max(t)}, but n_qubits={n_qubits}")
        m = np.array([[1.0]], dtype=np.complex128)
        for q in range(n_qubits):
            m = np.kron(m, _PAULI_MATRICES[t.get(q, 'I')])
        H += coeff * m
    return H


def pauli_sum_matvec_jax(vector, terms, n_qubits=None):
    """Tensor-in/tensor-out matvec (the name of the reference's JAX twin,
    observables.py:344-402): a CUDA tensor input stays on the device."""
    return pauli_sum_matvec(vector, terms, n_qubits)


def pauli_sum_expectation_jax(statevector, terms, n_qubits=None):
    return pauli_sum_expectation(statevector, terms, n_qubits)


class PauliSumOperator:
    """Matrix-free Hamiltonian usable as `h_matrix` of an energy function:
    `op @ psi` is the fused GPU matvec (observables.py:432-450)."""

    def __init__(self, terms, n_qubits):
        self.terms = list(terms)
        self.n_qubits = n_qubits

    def plan(self, dtype=torch.complex128) -> PauliPlan:
        return plan_for(self.terms, self.n_qubits, self.n_qubits, dtype)

    def __matmul__(self, vector):
        return pauli_sum_matvec(vector, self.terms, n_qubits=self.n_qubits)


_SAME_QUBIT_PAULI_PRODUCT = {
    ('X', 'X'): (1, None), ('Y', 'Y'): (1, None), ('Z', 'Z'): (1, None),
    ('X', 'Y'): (1j, 'Z'), ('Y', 'X'): (-1j, 'Z'),
    ('Y', 'Z'): (1j, 'X'), ('Z', 'Y'): (-1j, 'X'),
    ('Z', 'X'): (1j, 'Y'), ('X', 'Z'): (-1j, 'Y'),
}


def multiply_pauli_terms(factors):
    """Operator product of Pauli strings, left factor first, tracking the i^k
    phases of same-qubit products (observables.py:461-523)."""
    merged = {}
    total = 1.0 + 0j
    for coeff, pt in factors:
        total *= coeff
        for q, p in _normalize_terms(pt).items():
            if q not in merged:
                merged[q] = p
            else:
                ph, new = _SAME_QUBIT_PAULI_PRODUCT[(merged[q], p)]
                total *= ph
                if new is None:
                    del merged[q]
                else:
                    merged[q] = new
    return total, merged
