"""Plan-specialised fused-pass kernels.

A compacted pass (the op records that ``PackedPlan.compact`` uploads for the
fused interpreter ``k_fused_pass``) is written out as CUDA source in which
every structural field is a constant: the register bit positions of each
stage, the op bodies picked by their dispatch codes, the matrix offsets, the
thread predicates and the +-1 sign masks.  libdesv compiles the source with
NVRTC for sm_100a (``desv_jit_load``) against ``csrc/jit_pass.cuh``, which
reuses the interpreter's tile pipeline and op bodies, and launches it with
``desv_jit_pass``.  The matrix values stay in the same device pool, so new
angles need no recompile; a kernel is cached per source text.

The op bodies and their order are the interpreter's, so a specialised pass
computes what the interpreter computes (tests compare the two).
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import threading
from concurrent.futures import ThreadPoolExecutor
from typing import List, Optional, Sequence

import numpy as np

from .. import _native as N

_PKG = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
CSRC = os.path.join(_PKG, 'csrc')
INCLUDE = os.path.join(os.path.dirname(_PKG), 'include')
INCLUDE_PATH = CSRC + ':' + INCLUDE
V_ANTI, V_BREAL = 4, 5   # m1_variant codes of stage_ops.cuh
PRED = 0x8000


def _hex(v: int) -> str:
    return f'0x{int(v):x}ull'


def _signs_code(words: np.ndarray, w0: int, npairs: int) -> str:
    """Code of a +-1 group (dispatch code 152) with its normal-form record as
    immediates: neg = c ^ par(x) * 0xFFFF ^ sum_S par(tg & L_S) * slot mask S."""
    q = [int(words[w0 + 2 * i]) | int(words[w0 + 2 * i + 1]) << 32 for i in range(6 + 2 * npairs)]
    c, lall, ls = q[0] & 0xFFFF, q[1], q[2:6]
    xs = [f'(tg & {_hex(lall)})'] if lall else []
    for i in range(npairs):
        d, m = q[6 + 2 * i], q[7 + 2 * i]
        if m:
            xs.append(f'(tg & (tg >> {d}) & {_hex(m)})')
    terms = [f'0x{c:x}u'] if c else []
    if xs:
        terms.append(f'parity_mask({" ^ ".join(xs)}, 0xFFFFu)')
    for s, (l, sm) in enumerate(zip(ls, (0xAAAA, 0xCCCC, 0xF0F0, 0xFF00))):
        if l:
            terms.append(f'parity_mask(tg & {_hex(l)}, 0x{sm:X}u)')
    if not terms:
        return ''
    return f'sign_flips(a, {" ^ ".join(terms)});'


def mat_values(words: Optional[np.ndarray], off: int, wpe: int, count: int = 4) -> Optional[List[complex]]:
    """The complex values mats[off:off+count] from the pool's 32-bit words
    (wpe words per element: 2 for complex64, 4 for complex128)."""
    if words is None or (off + count) * wpe > len(words):
        return None
    w = np.ascontiguousarray(words[off * wpe:(off + count) * wpe])
    v = w.view(np.float32 if wpe == 2 else np.float64)
    return [complex(float(v[2 * i]), float(v[2 * i + 1])) for i in range(count)]


def _is_x(m: Optional[List[complex]]) -> bool:
    return m is not None and m[0] == 0 and m[1] == 1 and m[2] == 1 and m[3] == 0


def value_key(ops: np.ndarray, mats_host: np.ndarray) -> str:
    """Digest of the pool values the generated sources depend on (X matrices
    of anti-diagonal records become register swaps; generator values become
    immediates): with the op records, it keys a cache of generated kernels."""
    pool = np.ascontiguousarray(mats_host)
    if not len(ops) or not len(pool):
        return ''
    c = ops['code'].astype(np.int64) & 0x7FFF
    anti = ((c >= 1) & (c <= 20) & ((c - 1) % 5 == V_ANTI)) | ((c >= 21) & (c <= 52) & ((c - 21) % 2 == 0))
    sel = ((ops['kind'] == N.OP_GRAD) | (anti & (ops['kind'] != N.OP_STAGE))).nonzero()[0]
    if not len(sel):
        return ''
    idx = ops['mat'][sel].astype(np.int64)[:, None] + np.arange(4)
    return hashlib.sha1(pool[np.clip(idx, 0, len(pool) - 1)].tobytes()).hexdigest()


def _op_code(o, words: np.ndarray, wpe: int) -> str:
    c = int(o['code'])
    pred, c = c & PRED, c & 0x7FFF
    off = int(o['mat'])
    mp = f'mats + {off}'
    s0 = int(o['s0'])
    s1 = int(o['s1']) & 0xFF
    if 1 <= c <= 20:
        S, V = divmod(c - 1, 5)
        if V == V_ANTI and _is_x(mat_values(words, off, wpe)):
            call = f'swap_reg<{S}, -1>(a);'
        else:
            call = f'm1_reg<{S}, {V}, -1>(a, load_m22({mp}));'
    elif 21 <= c <= 52:
        x = c - 21
        S, CS = divmod(x // 2, 4)
        if not x & 1 and S != CS and _is_x(mat_values(words, off, wpe)):
            call = f'swap_reg<{S}, {CS}>(a);'
        else:
            call = f'm1_ctl_case<{S}, {CS}>(a, load_m22({mp}), {"false" if x & 1 else "true"});'
    elif 53 <= c <= 57:
        call = f'm1_lane_free<{c - 53}>(a, load_m22({mp}), {s0 - 16}, lane);'
    elif 58 <= c <= 107:
        sg = c < 83
        x = c - (58 if sg else 83)
        SA, SB = x // 5 - 1, x % 5 - 1
        w0y = (int(o['ga']) << 8) | (int(o['gb']) << 16)
        call = f'diag_case<{SA}, {SB}>(a, {mp}, 0x{w0y:x}u, tg, {"true" if sg else "false"});'
    elif 120 <= c <= 151:
        M, V = (c - 120, 0) if c < 136 else (c - 136, 1)
        call = f'multi_reg<{M}, {V}>(a, {mp});'
    elif c == 152:
        call = _signs_code(words, off * wpe, s0)
    elif c == 154:
        call = f'diag_group(a, {mp}, {s0}, tg);'
    elif 160 <= c <= 191:
        real = c >= 176
        M = c - (176 if real else 160)
        nreg = bin(M).count('1')
        parts = []
        if M:
            parts.append(f'multi_reg<{M}, {V_BREAL}>(a, {mp});' if real else f'multi_reg_packed<{M}>(a, {mp});')
        k = off + (4 if real else 8) * nreg
        for b in range(5):
            if (s1 >> b) & 1:
                parts.append(f'm1_lane_free<{V_BREAL if real else 0}>(a, load_m22(mats + {k}), {b}, lane);')
                k += 4
        call = ' '.join(parts)
    elif c == 192:
        cs = int(o['cslot'])
        call = (f'm1_lane(a, load_m22({mp}), m1_variant({int(o["flags"])}), {cs}, {s0 - 16}, '
                f'(tg & {_hex(o["cmask"])}) == {_hex(o["cval"])}, lane);')
    else:
        raise ValueError(f'dispatch code {c} has no specialised form')
    if pred and call:
        call = f'if ((tg & {_hex(o["cmask"])}) == {_hex(o["cval"])}) {{ {call} }}'
    return call


def grad_reads_pool(o, words: Optional[np.ndarray] = None, wpe: int = 2) -> bool:
    """True when the probe's code reads its generator from the pool at run time
    (False: the generator is compiled in as immediates, _grad_code's y, x and
    imaginary-diagonal forms)."""
    g = mat_values(words, int(o['mat']), wpe)
    if int(o['s1']) == 1:
        return not (g is not None and all(v.real == 0 for v in g))
    if int(o['s0']) >= 16:
        return True
    if g is not None and g[0] == 0 and g[3] == 0 and g[1].imag == 0 and g[2].imag == 0 and g[1] == -g[2]:
        return False
    if g is not None and g[0] == 0 and g[3] == 0 and g[1].real == 0 and g[2].real == 0 and g[1] == g[2]:
        return False
    return True


def _grad_code(o, words: Optional[np.ndarray] = None, wpe: int = 2, corr: bool = False) -> str:
    """A GRAD probe with its generator's placement compiled in (grad_term's
    forms); generators of the known shapes (ry: real antisymmetric, rx: -i h X,
    rz / p / cp / crz: imaginary diagonal) get probes with their values as
    immediates and no complex products."""
    mp = f'mats + {int(o["mat"])}'
    cs = int(o['cslot'])
    g = mat_values(words, int(o['mat']), wpe)
    if int(o['s1']) == 1:                          # diagonal generator over ga / gb
        sa, sb = int(o['sa']), int(o['sb'])
        ga, gb = int(o['ga']), int(o['gb'])
        fa = '0' if ga == 0xFF else f'(int)((tg >> {ga}) & 1ull)'
        fb = '0' if gb == 0xFF else f'(int)((tg >> {gb}) & 1ull)'
        if g is not None and all(v.real == 0 for v in g):
            hs = ', '.join(repr(float(v.imag)) for v in g)
            call = f'jit_grad_dim<{sa}, {sb}>(a, b, {hs}, {fa}, {fb})'
        else:
            call = f'jit_grad_diag<{sa}, {sb}>(a, b, {mp}, {fa}, {fb})'
    elif int(o['s0']) >= 16:                       # lane-bit generator
        call = f'jit_grad_lane<{cs}>(a, b, {mp}, {int(o["s0"]) - 16}, lane)'
    elif g is not None and g[0] == 0 and g[3] == 0 and g[1].imag == 0 and g[2].imag == 0 and g[1] == -g[2]:
        call = f'jit_grad_y<{int(o["s0"])}, {cs}>(a, b, {float(g[2].real)!r})'
    elif g is not None and g[0] == 0 and g[3] == 0 and g[1].real == 0 and g[2].real == 0 and g[1] == g[2]:
        call = f'jit_grad_x<{int(o["s0"])}, {cs}>(a, b, {-float(g[1].imag)!r})'
    else:
        call = f'jit_grad_reg<{int(o["s0"])}, {cs}>(a, b, {mp})'
    pred = f'(tg & {_hex(o["cmask"])}) == {_hex(o["cval"])}'
    # tangent passes: an immediate-form probe is scaled by the correction the
    # host writes into its (otherwise unread) pool slot
    cv = f' v *= (double)mats[{int(o["mat"])}].x;' if corr and not grad_reads_pool(o, words, wpe) else ''
    return (f'{{ double v = {call}; v = warp_sum_d({pred} ? v : 0.0);{cv} '
            f'if (lane == 0) acc[warp * nparams + {int(o["param"])}] += v; }}')


def adjoint_source(ops: np.ndarray, begin: int, end: int, tile_bits: int, nbuf: int, complex64: bool,
                   words: np.ndarray, wpe: int, tangent=None) -> str:
    """CUDA source of one specialised adjoint backward pass over ops[begin:end]
    (absolute indices into the op array the kernel receives): every inverse
    gate is applied to phi (a) and lambda (b); a GRAD op adds its probe
    2 Re<lambda|G|phi> (the factor 2 comes in the reduction) to its slot."""
    T = 'float2' if complex64 else 'double2'
    minb = _adjoint_min_blocks(tile_bits, nbuf, complex64)
    lines = ['#include "jit_pass.cuh"', 'using namespace desv;',
             f'extern "C" __global__ void __launch_bounds__({1 << (tile_bits - 4)}, {minb})',
             f'desv_jit_kernel({T} *phi, {T} *lam, TileGeom g, const desv_op *__restrict__ ops, '
             f'const {T} *__restrict__ mats, int nparams, double *part, RowStrides rs, '
             'const unsigned char *__restrict__ rflag, int want) {',
             '    extern __shared__ __align__(128) unsigned char smem[];',
             '    // rows launched twice per pass (tangent and general form): a row runs in the',
             '    // launch its flag selects, the other launch\'s CTAs of that row return at once',
             '    if (rflag != nullptr && (int)rflag[blockIdx.y] != want) return;',
             '    // rows: this grid row\'s (phi, lambda), pool and partial sums (zero strides: one state)',
             '    phi += blockIdx.y * rs.amps;',
             '    lam += blockIdx.y * rs.amps;',
             '    mats += blockIdx.y * rs.mats;',
             '    part += blockIdx.y * rs.part;',
             '    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;',
             f'    auto stages = [=]({T} *sphi, {T} *slam, uint64_t base, const uint64_t *ctab, int L, double *acc) {{',
             f'        {T} a[16], b[16];']
    k = begin
    while k < end:
        st = ops[k]
        if int(st['kind']) != N.OP_STAGE:
            raise ValueError('pass does not start with a stage record')
        cnt = int(st['mat'])
        g = [int(x) for x in st['g']]
        last = k + 1 + cnt >= end
        lines.append('        {')
        lines.append(f'            using S = JitStage<{T}, {g[0]}u, {g[1]}u, {g[2]}u, {g[3]}u>;')
        lines.append('            const uint32_t idx = S::index();')
        lines.append('            S::load(a, sphi, idx);')
        lines.append('            S::load(b, slam, idx);')
        lines.append('            const uint64_t tg = base | tl2g(ctab, L, idx);')
        for q in range(k + 1, k + 1 + cnt):
            o = ops[q]
            if int(o['kind']) == N.OP_GRAD:
                lines.append('            ' + _grad_code(o, words, wpe, corr=tangent is not None))
                continue
            if tangent is not None and q in tangent[0]:
                tv = f'mats[{int(o["mat"])}].x'
                if tangent[0][q] == 'rot':
                    S = (int(o['code']) - 1) // 5
                    lines.append(f'            {{ const auto t = {tv}; tan_rot<{S}>(a, t); tan_rot<{S}>(b, t); }}')
                else:
                    x = (int(o['code']) & 0x7FFF) - 83
                    SA = x // 5 - 1
                    fb = '0' if SA >= 0 else f'(int)((tg >> {int(o["ga"])}) & 1ull)'
                    lines.append(f'            {{ const auto t = {tv}; const int fb = {fb}; '
                                 f'tan_phase<{SA}>(a, t, fb); tan_phase<{SA}>(b, t, fb); }}')
                continue
            code = _op_code(o, words, wpe)
            if code:
                lines.append('            ' + code)
                lines.append('            ' + code.replace('(a, ', '(b, ').replace('(a);', '(b);'))
        if last and tangent is not None:
            lines.append(f'            scale_both(a, b, mats[{tangent[1]}].x);')
        if last:
            lines.append('            S::store_global(a, phi, tg, ctab, L);')
            lines.append('            S::store_global(b, lam, tg, ctab, L);')
        else:
            lines.append(f'            JitStage2<{T}, S>::store_smem(a, b, sphi, slam, idx);')
        lines.append('        }')
        k += 1 + cnt
    lines += ['    };', f'    jit_adjoint_kernel<{T}, {tile_bits}, {nbuf}>(phi, lam, g, smem, nparams, part, stages);',
              '}', '']
    return '\n'.join(lines)


def adjoint_nbuf_for(tile_bits: int, complex64: bool) -> int:
    """Ring depth of the adjoint interpreter for this tile width (k_adjoint.cu);
    DESV_ADJ_NBUF overrides it for the specialised complex64 kernels (tuning)."""
    if complex64:
        v = os.environ.get('DESV_ADJ_NBUF', '')
        if v in ('2', '3', '4'):
            return int(v)
        return 3 if tile_bits >= 11 else 4
    return 3 if tile_bits >= 10 else 4


def _adjoint_min_blocks(tile_bits: int, nbuf: int, complex64: bool) -> int:
    """CTAs per SM the specialised adjoint kernel's registers are bounded for:
    shared memory holds two CTAs of 11-bit tiles with three ring slots (no
    register bound needed), three with two slots (at most 170 registers)."""
    if complex64 and tile_bits == 11 and nbuf == 2:
        return 3
    return 1


def pass_source(ops: np.ndarray, begin: int, end: int, tile_bits: int, nbuf: int, complex64: bool,
                words: np.ndarray, wpe: int) -> str:
    """CUDA source of one specialised pass over ops[begin:end]."""
    T = 'float2' if complex64 else 'double2'
    lines = ['#include "jit_pass.cuh"', 'using namespace desv;',
             f'extern "C" __global__ void __launch_bounds__({1 << (tile_bits - 4)}, {2 if complex64 else 1})',
             f'desv_jit_kernel({T} *sv, TileGeom g, const {T} *__restrict__ mats, RowStrides rs) {{',
             '    extern __shared__ __align__(128) unsigned char smem[];',
             '    // rows: this grid row\'s state and pool (zero strides: one state)',
             '    sv += blockIdx.y * rs.amps;',
             '    mats += blockIdx.y * rs.mats;',
             '    const int lane = threadIdx.x & 31;',
             f'    auto stages = [=]({T} *s, uint64_t base, const uint64_t *ctab, int L) {{',
             f'        {T} a[16];']
    k = begin
    while k < end:
        st = ops[k]
        if int(st['kind']) != N.OP_STAGE:
            raise ValueError('pass does not start with a stage record')
        cnt = int(st['mat'])
        g = [int(x) for x in st['g']]
        last = k + 1 + cnt >= end
        lines.append('        {')
        lines.append(f'            using S = JitStage<{T}, {g[0]}u, {g[1]}u, {g[2]}u, {g[3]}u>;')
        lines.append('            const uint32_t idx = S::index();')
        lines.append('            S::load(a, s, idx);')
        lines.append('            const uint64_t tg = base | tl2g(ctab, L, idx);')
        for o in ops[k + 1:k + 1 + cnt]:
            code = _op_code(o, words, wpe)
            if code:
                lines.append('            ' + code)
        lines.append('            S::store_global(a, sv, tg, ctab, L);' if last else '            S::store_smem(a, s, idx);')
        lines.append('        }')
        k += 1 + cnt
    lines += ['    };', f'    jit_pass_kernel<{T}, {tile_bits}, {nbuf}>(sv, g, smem, stages);', '}', '']
    return '\n'.join(lines)


# Pauli passes: more terms than this stay on the interpreter
MAX_PAULI_TERMS = 64


def _tile_local(m: int, L: int, high) -> int:
    """Tile-local form of the global bit mask m (bits 0..L-1, then high[i] -> L + i)."""
    x = m & ((1 << L) - 1)
    for i, h in enumerate(high):
        if (m >> h) & 1:
            x |= 1 << (L + i)
    return x


def _expect_source(terms: np.ndarray, K: int, L: int, high, complex64: bool) -> str:
    """CUDA source of one specialised <H> pass (mode 0).

    Per amplitude only single-precision work: the product w = Re(conj(a) p)
    with the partner p = psi[j ^ x] (and Im(conj(a) p) where a term needs it)
    in the state's precision, added with its integer sign weight into
    per-thread sums, one per coefficient class of the pass.  Once per tile each
    sum is widened and multiplied by its FP64 coefficient into the FP64
    energy.  The interpreter widens every partner to FP64 for every flip mask
    (two conversions per mask and amplitude); those conversions bound it.

    Terms: (P psi)[i] = psi[i ^ x] c (-1)^popcount((i ^ x) & z) with c the
    coefficient times i^(number of Y).  S = sum_i sign conj(a_i) p_i is real
    when the number of Y is even and imaginary when it is odd, so a term with a
    real c and an even Y count adds c S_re to Re<H> and nothing to Im<H>; every
    other term keeps both parts."""
    T = 'float2' if complex64 else 'double2'
    R = 'float' if complex64 else 'double'
    high = [int(h) for h in high[:K - L]]
    tile_mask = ((1 << L) - 1) | sum(1 << h for h in high)
    # as many CTAs per SM as the ring allows (three for 64 KB): without the
    # bound the compiler took 128 registers for 8-mask passes of 12-bit tiles,
    # which left two CTAs (16 warps) per SM; with it they take 80, no spills
    lines = ['#include "jit_pass.cuh"', 'using namespace desv;',
             f'extern "C" __global__ void __launch_bounds__(256, {_pauli_min_blocks(K, complex64)})',
             f'desv_jit_kernel(const {T} *psi, {T} *out, TileGeom g, int want_e, double *part) {{',
             '    extern __shared__ __align__(128) unsigned char smem[];',
             f'    auto body = [=]({T} *s, uint64_t base, const uint64_t *ctab, int L, double &ere, double &eim) {{']
    groups = {}
    for k, t in enumerate(terms):
        groups.setdefault(int(t['xmask']), []).append(k)
    for k, t in enumerate(terms):
        zo = int(t['zmask']) & ~tile_mask
        if zo:
            lines.append(f'        const uint32_t pb{k} = (uint32_t)__popcll(base & {_hex(zo)}) & 1u;')
    plan = []
    acc = []            # accumulator names
    for gi, (x, ks) in enumerate(groups.items()):
        xl = _tile_local(x, L, high)
        classes, outside, single, cplx = [], [], [], []
        for k in ks:
            t = terms[k]
            zl = _tile_local(int(t['zmask']) & tile_mask, L, high)
            zo = int(t['zmask']) & ~tile_mask
            cre, cim = float(t['cre']), float(t['cim'])
            ny_odd = bin(int(t['xmask']) & int(t['zmask'])).count('1') & 1
            if cim != 0.0 or ny_odd:
                cplx.append((k, zl, zo, cre, cim))
            elif zl == 0:
                outside.append((k, zo, cre))
            elif zo == 0 and bin(zl).count('1') <= 2:
                lo = (zl & -zl).bit_length() - 1
                d = zl.bit_length() - 1 - lo
                for cl in classes:
                    if cl[0] == cre and cl[1] == d and not (cl[2] >> lo) & 1:
                        cl[2] |= 1 << lo
                        cl[3] += 1
                        break
                else:
                    classes.append([cre, d, 1 << lo, 1])
            else:
                single.append((k, zl, zo, cre))
        plan.append((xl, classes, outside, single, cplx))
    # per-thread sums of this tile's amplitudes
    decl = []
    for gi, (xl, classes, outside, single, cplx) in enumerate(plan):
        if outside:
            decl.append(f'so{gi}')
        decl += [f'sc{gi}_{ci}' for ci in range(len(classes))]
        decl += [f'ss{gi}_{si}' for si in range(len(single))]
        for k, *_ in cplx:
            decl += [f'sr{k}', f'si{k}']
    lines += [f'        {R} {", ".join(n + " = 0" for n in decl)};'] if decl else []
    # Amplitude j = t | (k << 8) of the tile (t the thread, k the unrolled row):
    # its partner j ^ x is (t ^ x_lo) ^ ((k ^ x_hi) << 8), a per-thread part
    # formed once per flip mask and a compile-time offset, so no index
    # arithmetic is left per amplitude (the form j0 + r * 256 hid that from the
    # compiler, which cannot know threadIdx.x < 256 from it)
    if K < 8:
        raise ValueError('specialised <H> passes need tiles of at least 8 bits')
    lines.append('        const uint32_t t = threadIdx.x & 255u;')
    for gi, (xl, *_rest) in enumerate(plan):
        lines.append(f'        const uint32_t tx{gi} = t ^ {xl & 255}u;')
        lines.append(f'        const {T} *q{gi} = s + tx{gi};')
    lines += ['#pragma unroll',
              f'        for (uint32_t k = 0; k < {1 << (K - 8)}u; ++k) {{',
              '            {',
              f'                const {T} a = s[t + (k << 8)];']
    for gi, (xl, classes, outside, single, cplx) in enumerate(plan):
        lines.append('                {')
        lines.append(f'                    const uint32_t kx = (k ^ {xl >> 8}u) << 8;')
        lines.append(f'                    const uint32_t jx = tx{gi} ^ kx;')
        lines.append(f'                    const {T} q = q{gi}[kx];')
        lines.append(f'                    const {R} w = a.x * q.x + a.y * q.y;')
        if cplx:
            lines.append(f'                    const {R} wi = a.x * q.y - a.y * q.x;')
        if outside:
            lines.append(f'                    so{gi} += w;')
        for ci, (c, d, m, cnt) in enumerate(classes):
            pc = f'__popc(jx & {m}u)' if d == 0 else f'__popc((jx ^ (jx >> {d})) & {m}u)'
            lines.append(f'                    sc{gi}_{ci} += small_int_to_{R}({cnt} - 2 * (int){pc}) * w;')
        for si, (k, zl, zo, c) in enumerate(single):
            lines.append(f'                    ss{gi}_{si} += (__popc(jx & {zl}u) & 1u) ? -w : w;')
        for k, zl, zo, cre, cim in cplx:
            if zl:
                lines.append(f'                    {{ const bool ng = (__popc(jx & {zl}u) & 1u) != 0; '
                             f'sr{k} += ng ? -w : w; si{k} += ng ? -wi : wi; }}')
            else:
                lines.append(f'                    sr{k} += w; si{k} += wi;')
        lines.append('                }')
    lines += ['            }', '        }']
    # widen once per tile: FP64 coefficients times the sums
    er, ei = [], []
    for gi, (xl, classes, outside, single, cplx) in enumerate(plan):
        if outside:
            const = sum(c for (_, zo, c) in outside if not zo)
            ts = [f'(pb{k} ? {-c!r} : {c!r})' for (k, zo, c) in outside if zo]
            er.append(f'({" + ".join(([repr(const)] if const else []) + ts) or "0.0"}) * (double)so{gi}')
        for ci, (c, d, m, cnt) in enumerate(classes):
            er.append(f'{c!r} * (double)sc{gi}_{ci}')
        for si, (k, zl, zo, c) in enumerate(single):
            cc = f'(pb{k} ? {-c!r} : {c!r})' if zo else repr(c)
            er.append(f'{cc} * (double)ss{gi}_{si}')
        for k, zl, zo, cre, cim in cplx:
            sg = f'(pb{k} ? -1.0 : 1.0) * ' if zo else ''
            er.append(f'{sg}({cre!r} * (double)sr{k} - {cim!r} * (double)si{k})')
            ei.append(f'{sg}({cre!r} * (double)si{k} + {cim!r} * (double)sr{k})')
    if er:
        lines.append('        ere += ' + ' + '.join(er) + ';')
    if ei:
        lines.append('        eim += ' + ' + '.join(ei) + ';')
    lines += ['    };', f'    jit_pauli_kernel<{T}, {K}, {pauli_nbuf(K)}>(psi, g, want_e, part, smem, body);', '}', '']
    return '\n'.join(lines)


def pauli_source(terms: np.ndarray, tile_bits: int, low_bits: int, high, mode: int, complex64: bool,
                 syms: Optional[Sequence[Optional[int]]] = None) -> str:
    """CUDA source of one specialised Pauli pass (the interpreter k_pauli with
    the pass's terms compiled in): mode 0 <H> only, 1 write H psi, 2 add into
    H psi.  Terms with one flip mask share the partner amplitude; real
    coefficients take the two-FMA form.  (P psi)[i] = psi[i ^ x] c
    (-1)^popcount((i ^ x) & z); the z bits outside the tile give a per-tile
    parity.

    syms (H psi modes, rows launches): per term None (its coefficient is
    compiled in) or the index of a per-row coefficient that multiplies it:
    the kernel then runs one grid row per state and reads its row's values
    from csym[blockIdx.y * nsym + ...] (terms with equal per-row values share
    an index and still fold into one class)."""
    if mode == 0:
        return _expect_source(terms, tile_bits, low_bits, high, complex64)
    T = 'float2' if complex64 else 'double2'
    R = 'float' if complex64 else 'double'
    K, L = tile_bits, low_bits
    high = [int(h) for h in high[:K - L]]
    tile_mask = ((1 << L) - 1) | sum(1 << h for h in high)
    rows = syms is not None
    if not rows:
        syms = [None] * len(terms)
    nsym = 1 + max([x for x in syms if x is not None], default=-1)

    def cx(v: float, sym) -> str:
        """the coefficient v (times the row's value of symbol sym) as an expression"""
        return repr(v) if sym is None else f'({v!r} * C{sym})'

    if rows:
        lines = ['#include "jit_pass.cuh"', 'using namespace desv;',
                 'extern "C" __global__ void __launch_bounds__(256)',
                 f'desv_jit_kernel(const {T} *psi, {T} *out, TileGeom g, int want_e, double *part, '
                 'const double *__restrict__ csym, int nsym, RowStrides rs) {',
                 '    extern __shared__ __align__(128) unsigned char smem[];',
                 '    // rows: this grid row\'s state, output, partial sums and coefficients',
                 '    psi += blockIdx.y * rs.amps;',
                 '    out += blockIdx.y * rs.amps;',
                 '    part += blockIdx.y * rs.part;',
                 '    csym += (size_t)blockIdx.y * nsym;']
        lines += [f'    const double C{k} = csym[{k}];' for k in range(nsym)]
        lines.append(f'    auto body = [=]({T} *s, uint64_t base, const uint64_t *ctab, int L, double &ere, double &eim) {{')
    else:
        lines = ['#include "jit_pass.cuh"', 'using namespace desv;',
                 'extern "C" __global__ void __launch_bounds__(256)',
                 f'desv_jit_kernel(const {T} *psi, {T} *out, TileGeom g, int want_e, double *part) {{',
                 '    extern __shared__ __align__(128) unsigned char smem[];',
                 f'    auto body = [=]({T} *s, uint64_t base, const uint64_t *ctab, int L, double &ere, double &eim) {{']
    groups = {}
    for k, t in enumerate(terms):
        groups.setdefault(int(t['xmask']), []).append(k)
    for k, t in enumerate(terms):
        zo = int(t['zmask']) & ~tile_mask
        if zo:
            lines.append(f'        const uint32_t pb{k} = (uint32_t)__popcll(base & {_hex(zo)}) & 1u;')
    # Per flip mask: real-coefficient terms fold into one real factor per
    # amplitude -- sign masks of one bit, or of two bits at a fixed tile-local
    # distance, become one popcount per class (sum of c (-1)^bit... over the
    # class = c (count - 2 popcount)); sign masks wholly outside the tile give a
    # per-tile constant; the rest add their signed coefficient.  Complex
    # coefficients keep the per-term complex FMA.
    plan = []
    for gi, (x, ks) in enumerate(groups.items()):
        xl = _tile_local(x, L, high)
        classes, outside, single, cplx = [], [], [], []
        for k in ks:
            t = terms[k]
            zl = _tile_local(int(t['zmask']) & tile_mask, L, high)
            zo = int(t['zmask']) & ~tile_mask
            cre, cim = float(t['cre']), float(t['cim'])
            sy = syms[k]
            if cim != 0.0:
                cplx.append((k, zl, zo, cre, cim, sy))
            elif zl == 0:
                outside.append((k, zo, cre, sy))
            elif zo == 0 and bin(zl).count('1') <= 2:
                lo = (zl & -zl).bit_length() - 1
                d = zl.bit_length() - 1 - lo
                for cl in classes:
                    if cl[0] == (cre, sy) and cl[1] == d and not (cl[2] >> lo) & 1:
                        cl[2] |= 1 << lo
                        cl[3] += 1
                        break
                else:
                    classes.append([(cre, sy), d, 1 << lo, 1])
            else:
                single.append((k, zl, zo, cre, sy))
        plan.append((xl, classes, outside, single, cplx))
        const = [cx(c, sy) for (_, zo, c, sy) in outside if not zo]
        ts = [f'(pb{k} ? {cx(-c, sy)} : {cx(c, sy)})' for (k, zo, c, sy) in outside if zo]
        if const or ts:
            lines.append(f'        const double dg{gi} = {" + ".join(const + ts)};')
    lines += ['#pragma unroll 1',
              f'        for (uint32_t j0 = threadIdx.x; j0 < {1 << K}u; j0 += 1024u) {{',
              '            double2 v[4];',
              '#pragma unroll',
              '            for (int r = 0; r < 4; ++r) v[r] = make_double2(0.0, 0.0);']
    for gi, (xl, classes, outside, single, cplx) in enumerate(plan):
        lines.append('            {')
        lines.append('                double2 p[4];')
        lines.append('#pragma unroll')
        lines.append(f'                for (int r = 0; r < 4; ++r) {{ const {T} q = s[(j0 + r * 256u) ^ {xl}u]; '
                     'p[r] = make_double2((double)q.x, (double)q.y); }')
        lines.append('#pragma unroll')
        lines.append('                for (int r = 0; r < 4; ++r) {')
        lines.append(f'                    const uint32_t jx = (j0 + r * 256u) ^ {xl}u;')
        real = bool(classes or outside or single)
        if real:
            lines.append(f'                    double cr = {"dg%d" % gi if outside else "0.0"};')
            for (c, sy), d, m, cnt in classes:
                pc = f'__popc(jx & {m}u)' if d == 0 else f'__popc((jx ^ (jx >> {d})) & {m}u)'
                lines.append(f'                    cr = fma({cx(c, sy)}, (double)({cnt} - 2 * (int){pc}), cr);')
            for k, zl, zo, c, sy in single:
                parts = [f'__popc(jx & {zl}u)'] + ([f'pb{k}'] if zo else [])
                lines.append(f'                    cr += (({" ^ ".join(parts)}) & 1u) ? {cx(-c, sy)} : {cx(c, sy)};')
            lines.append('                    v[r].x = fma(cr, p[r].x, v[r].x); v[r].y = fma(cr, p[r].y, v[r].y);')
        for k, zl, zo, cre, cim, sy in cplx:
            parts = ([f'__popc(jx & {zl}u)'] if zl else []) + ([f'pb{k}'] if zo else [])
            sg = f'(({" ^ ".join(parts)}) & 1u)' if parts else None
            pos = f'make_double2({cx(cre, sy)}, {cx(cim, sy)})'
            ng = f'make_double2({cx(-cre, sy)}, {cx(-cim, sy)})'
            c = pos if sg is None else f'({sg} ? {ng} : {pos})'
            lines.append(f'                    v[r] = cfma({c}, p[r], v[r]);')
        lines.append('                }')
        lines.append('            }')
    lines += ['#pragma unroll',
              '            for (int r = 0; r < 4; ++r) {',
              '                const uint32_t j = j0 + r * 256u;',
              '                { const ' + T + ' a = s[j]; ere += (double)a.x * v[r].x + (double)a.y * v[r].y; '
              'eim += (double)a.x * v[r].y - (double)a.y * v[r].x; }',
              '                const uint64_t gi = base + tl2g(ctab, L, j);']
    if mode == 1:
        lines.append(f'                out[gi] = mk(({R})v[r].x, ({R})v[r].y);')
    else:
        lines.append(f'                {{ {T} o = out[gi]; o.x = ({R})((double)o.x + v[r].x); '
                     f'o.y = ({R})((double)o.y + v[r].y); out[gi] = o; }}')
    lines += ['            }', '        }', '    };',
              f'    jit_pauli_kernel<{T}, {K}, {pauli_nbuf(K)}>(psi, g, want_e, part, smem, body);', '}', '']
    return '\n'.join(lines)


def pauli_nbuf(tile_bits: int) -> int:
    """Ring slots of a specialised Pauli pass: four for tiles of up to 11 bits,
    two for 12-bit tiles (three CTAs of 64 KB per SM; DESV_PAULI_NBUF12
    overrides the latter, for tuning)."""
    if tile_bits >= 12:
        return int(os.environ.get('DESV_PAULI_NBUF12', '2'))
    return 4


def _pauli_min_blocks(tile_bits: int, complex64: bool) -> int:
    """CTAs per SM the ring of a Pauli pass leaves room for (at most three)."""
    ring = pauli_nbuf(tile_bits) * ((8 if complex64 else 16) << tile_bits) + 4096
    return max(1, min(3, (220 << 10) // ring))


def pauli_modes(passes: np.ndarray, matvec: bool) -> list:
    """The kernel mode each pass runs in, as desv_jit_pauli walks them (None:
    skipped): <H> passes 0; H psi: 1 for the first pass run, 2 after it."""
    out, wrote = [], False
    for p in passes:
        nt = int(p['term_end']) - int(p['term_begin'])
        if nt == 0 and (not matvec or wrote):
            out.append(None)
            continue
        out.append((2 if wrote else 1) if matvec else 0)
        wrote = True
    return out


def compile_pauli(terms: np.ndarray, passes: np.ndarray, matvec: bool, complex64: bool, device: int,
                  workers: int = 0) -> list:
    """One specialised kernel per tiled Pauli pass in the mode that call runs it
    (None: the interpreter runs that pass)."""
    code = N.DESV_C64 if complex64 else N.DESV_C128
    jobs, kinds = [], []
    for p, mode in zip(passes, pauli_modes(passes, matvec)):
        K, L = int(p['tile_bits']), int(p['low_bits'])
        b, e = int(p['term_begin']), int(p['term_end'])
        if mode is None or K < 10 or K - L > 8 or not 0 < e - b <= MAX_PAULI_TERMS:
            jobs.append(None)
            kinds.append(None)
            continue
        jobs.append((pauli_source(terms[b:e], K, L, p['high'], mode, complex64), K, pauli_nbuf(K)))
        kinds.append(KIND_PAULI + mode)
    workers = workers or min(32, os.cpu_count() or 1, max(1, len(jobs)))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(lambda a: None if a[0] is None else _load(a[0][0], a[0][1], a[0][2], code, device, a[1]),
                           zip(jobs, kinds)))


def compile_pauli_rows(terms: np.ndarray, passes: np.ndarray, syms: Sequence[Optional[int]], complex64: bool,
                       device: int, workers: int = 0) -> list:
    """H psi kernels for rows launches (desv_jit_pauli_matvec_rows): one per
    tiled pass in the mode the rows driver runs it, with the terms' per-row
    coefficient symbols (None: the term's coefficient is compiled in)."""
    code = N.DESV_C64 if complex64 else N.DESV_C128
    jobs, kinds = [], []
    for p, mode in zip(passes, pauli_modes(passes, True)):
        K, L = int(p['tile_bits']), int(p['low_bits'])
        b, e = int(p['term_begin']), int(p['term_end'])
        if mode is None or K < 10 or K - L > 8 or not 0 < e - b <= MAX_PAULI_TERMS:
            jobs.append(None)
            kinds.append(None)
            continue
        jobs.append((pauli_source(terms[b:e], K, L, p['high'], mode, complex64, syms=list(syms[b:e])), K,
                     pauli_nbuf(K)))
        kinds.append(KIND_PAULI + mode)
    workers = workers or min(32, os.cpu_count() or 1, max(1, len(jobs)))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(lambda a: None if a[0] is None else _load(a[0][0], a[0][1], a[0][2], code, device, a[1]),
                           zip(jobs, kinds)))


def nbuf_for(tile_bits: int) -> int:
    """Ring depth of the interpreter for this tile width (k_fused.cu)."""
    return 3 if tile_bits >= 12 else 4


# below this size a pass is too short for its compile to pay off
MIN_QUBITS = 20
# passes with more op records than this stay on the interpreter: every op is
# unrolled over 16 amplitudes, and compile time grows with the pass
MAX_OPS = 96
_available = None


def available() -> bool:
    """NVRTC and the CUDA driver can be opened (libdesv loads them with dlopen)."""
    global _available
    if _available is None:
        buf = ctypes.create_string_buffer(256)
        _available = bool(N.lib().desv_jit_available(buf, 256))
    return _available


def enabled(n: int) -> bool:
    """Use specialised kernels for an n-qubit plan: DESV_JIT=1 / 0 forces the
    choice; by default from MIN_QUBITS qubits on."""
    v = os.environ.get('DESV_JIT', '')
    if v in ('0', '1'):
        return v == '1'
    return n >= MIN_QUBITS and available()


class _Kernel:
    __slots__ = ('handle',)

    def __init__(self, handle):
        self.handle = handle

    def __del__(self):
        try:
            N.lib().desv_jit_free(self.handle)
        except Exception:
            pass


_cache: dict = {}
_cache_lock = threading.Lock()


KIND_PASS, KIND_ADJOINT, KIND_PAULI = 0, 1, 2   # Pauli: + mode (0, 1, 2)


def _load(src: str, tile_bits: int, nbuf: int, dtype_code: int, device: int, kind: int = KIND_PASS) -> _Kernel:
    key = (hashlib.sha1(src.encode()).hexdigest(), device, kind)
    with _cache_lock:
        k = _cache.get(key)
    if k is not None:
        return k
    h = ctypes.c_void_p()
    log = ctypes.create_string_buffer(8192)
    rc = N.lib().desv_jit_load(src.encode(), INCLUDE_PATH.encode(), kind, tile_bits, nbuf, dtype_code, device,
                               ctypes.byref(h), log, 8192)
    N.check(rc, 'desv_jit_load')
    k = _Kernel(h)
    with _cache_lock:
        _cache.setdefault(key, k)
        return _cache[key]


def _compile(jobs, code, device, kind, workers):
    """Kernels for the jobs (None stays None: that pass runs on the interpreter)."""
    workers = workers or min(32, os.cpu_count() or 1, max(1, len(jobs)))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(lambda j: None if j is None else _load(j[0], j[1], j[2], code, device, kind), jobs))


def compile_passes(ops: np.ndarray, passes: np.ndarray, mats_host: np.ndarray, complex64: bool, device: int,
                   workers: int = 0) -> list:
    """One specialised kernel per pass (NVRTC compiles run in parallel threads;
    the ctypes call releases the GIL)."""
    words = np.ascontiguousarray(mats_host).view(np.uint32)
    wpe = mats_host.dtype.itemsize // 4
    code = N.DESV_C64 if complex64 else N.DESV_C128
    jobs = []
    for p in passes:
        K = int(p['tile_bits'])
        nb = nbuf_for(K)
        b, e = int(p['op_begin']), int(p['op_end'])
        jobs.append((pass_source(ops, b, e, K, nb, complex64, words, wpe), K, nb) if 0 < e - b <= MAX_OPS else None)
    return _compile(jobs, code, device, KIND_PASS, workers)


def compile_adjoint(ops: np.ndarray, passes: np.ndarray, mats_host: np.ndarray, complex64: bool, device: int,
                    workers: int = 0, tangents=None) -> list:
    """One specialised adjoint backward kernel per pass (None for an empty pass).
    tangents: per pass None (the general form) or (records in tangent form,
    pool offset of the pass-end factor) for the tangent variant."""
    words = np.ascontiguousarray(mats_host).view(np.uint32)
    wpe = mats_host.dtype.itemsize // 4
    code = N.DESV_C64 if complex64 else N.DESV_C128
    jobs = []
    for i, p in enumerate(passes):
        K = int(p['tile_bits'])
        nb = adjoint_nbuf_for(K, complex64)
        b, e = int(p['op_begin']), int(p['op_end'])
        tg = tangents[i] if tangents is not None else None
        jobs.append((adjoint_source(ops, b, e, K, nb, complex64, words, wpe, tangent=tg), K, nb)
                    if 0 < e - b <= MAX_OPS else None)
    return _compile(jobs, code, device, KIND_ADJOINT, workers)


def run_adjoint(kernels: list, phi_ptr: int, lam_ptr: int, n: int, dtype_code: int, passes: np.ndarray,
                ops_ptr: int, mats_ptr: int, map_ptr: int, grad_ptr: int, scratch_ptr: int, scratch_bytes: int,
                stream):
    """The backward sweep, pass by pass: each launch is followed by the
    gradient reduction of its partial sums (desv_jit_adjoint)."""
    lib = N.lib()
    st = ctypes.c_void_p(stream)
    base = passes.ctypes.data
    for i, k in enumerate(kernels):
        pp = ctypes.c_void_p(base + i * passes.itemsize)
        if k is None:
            N.check(lib.desv_adjoint_passes(ctypes.c_void_p(phi_ptr), ctypes.c_void_p(lam_ptr), n, dtype_code, pp, 1,
                                            ctypes.c_void_p(ops_ptr), ctypes.c_void_p(mats_ptr),
                                            ctypes.c_void_p(map_ptr), ctypes.c_void_p(grad_ptr),
                                            ctypes.c_void_p(scratch_ptr), scratch_bytes, st), 'adjoint pass')
        else:
            N.check(lib.desv_jit_adjoint(k.handle, ctypes.c_void_p(phi_ptr), ctypes.c_void_p(lam_ptr), n, dtype_code,
                                         pp, ctypes.c_void_p(ops_ptr), ctypes.c_void_p(mats_ptr),
                                         ctypes.c_void_p(map_ptr), ctypes.c_void_p(grad_ptr),
                                         ctypes.c_void_p(scratch_ptr), scratch_bytes, st), 'desv_jit_adjoint')


def run_passes(kernels: list, sv_ptr: int, n: int, dtype_code: int, passes: np.ndarray, ops_ptr: int,
               mats_ptr: int, stream):
    """passes[i] through kernels[i], or through the interpreter where that is None."""
    lib = N.lib()
    st = ctypes.c_void_p(stream)
    base = passes.ctypes.data
    for i, k in enumerate(kernels):
        pp = ctypes.c_void_p(base + i * passes.itemsize)
        if k is None:
            N.check(lib.desv_apply_passes(ctypes.c_void_p(sv_ptr), n, dtype_code, pp, 1, ctypes.c_void_p(ops_ptr),
                                          ctypes.c_void_p(mats_ptr), st), 'apply fused pass')
        else:
            N.check(lib.desv_jit_pass(k.handle, ctypes.c_void_p(sv_ptr), n, dtype_code, pp,
                                      ctypes.c_void_p(mats_ptr), st), 'desv_jit_pass')
