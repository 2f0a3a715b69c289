"""NumPy interpreter of the packed fused-pass format (include/desv.h) -- test
infrastructure.  It executes desv_pass / desv_op records exactly as the CUDA
kernels define them (tile = low bits + high bits, stages of 4 register bits,
lanes = bits 0..4, controls / diagonal bits read from the global index), so
the host fusion pass and packer can be checked against the oracle on a CPU.
"""
from __future__ import annotations

import numpy as np

OP_STAGE, OP_M1, OP_M2, OP_DIAG, OP_GRAD = 0, 1, 2, 3, 4


def _tile_index_map(n, K, L, high):
    """global indices of every tile: array [ntiles, 2^K]"""
    rest = [b for b in range(n) if b >= L and b not in high]
    j = np.arange(1 << K, dtype=np.int64)
    loc = j & ((1 << L) - 1)
    for i, h in enumerate(high):
        loc |= ((j >> (L + i)) & 1) << h
    t = np.arange(1 << (n - K), dtype=np.int64)
    base = np.zeros_like(t)
    for i, b in enumerate(rest):
        base |= ((t >> i) & 1) << b
    return base[:, None] | loc[None, :]


def _bit(idx, b):
    return (idx >> b) & 1


def run_passes(sv, n, passes, ops, mats, lam=None, grad=None, param_map=None):
    """Apply passes in place to sv (and lam for adjoint passes); returns sv (, lam, grad)."""
    sv = sv.copy()
    lam = None if lam is None else lam.copy()
    for ps in passes:
        K, L = int(ps['tile_bits']), int(ps['low_bits'])
        high = [int(h) for h in ps['high'][:K - L]]
        gi = _tile_index_map(n, K, L, high)                 # [T, 2^K]
        a = sv[gi]
        b = None if lam is None else lam[gi]
        k = int(ps['op_begin'])
        end = int(ps['op_end'])
        nparams = int(ps['nparams']) if 'nparams' in (ps.dtype.names or ()) else 0
        while k < end:
            st = ops[k]
            assert st['kind'] == OP_STAGE
            cnt = int(st['mat'])
            g = [int(x) for x in st['g']]
            assert len(set(g)) == 4 and min(g) >= 5 and max(g) < K
            gmask = 0
            for x in g:
                gmask |= 1 << (x if x < L else high[x - L])
            tg = gi & ~gmask      # the kernel's per-thread index: register bits cleared
            for q in range(1, cnt + 1):
                op = ops[k + q]
                if op['kind'] in (OP_M1, OP_M2, OP_GRAD):
                    assert int(op['cmask']) & gmask == 0, 'control on a register bit must use cslot'
                if op['kind'] == OP_GRAD:
                    v = _grad(a, b, tg, op, g, mats, L, high)
                    grad[param_map[int(ps['map_begin']) + int(op['param'])]] += 2.0 * v
                    continue
                code = int(op['code'])
                a = _apply_coded(a, tg, op, g, mats, code) if code else _apply(a, tg, op, g, mats)
                if b is not None:
                    b = _apply_coded(b, tg, op, g, mats, code) if code else _apply(b, tg, op, g, mats)
            k += 1 + cnt
        sv[gi] = a
        if lam is not None:
            lam[gi] = b
    if lam is None:
        return sv
    return sv, lam, grad


def _target_local(op):
    s0 = int(op['s0'])
    return s0


def _pred(gi, op, g):
    # thread-level control on the amplitude's global index with register bits cleared
    cm, cv = int(op['cmask']), int(op['cval'])
    return (gi & cm) == cv


def _apply(a, gi, op, g, mats):
    kind = int(op['kind'])
    m0 = int(op['mat'])
    pred = _pred(gi, op, g)
    if kind == OP_M1:
        m = mats[m0:m0 + 4].reshape(2, 2)
        s0 = int(op['s0'])
        tl = (s0 - 16) if s0 >= 16 else g[s0]
        cs = int(op['cslot'])
        bit = (np.arange(a.shape[1]) >> tl) & 1
        partner = np.arange(a.shape[1]) ^ (1 << tl)
        p = a[:, partner]
        new = np.where(bit[None, :] == 0, m[0, 0] * a + m[0, 1] * p, m[1, 0] * p + m[1, 1] * a)
        ok = pred
        if cs >= 0:
            ok = ok & (((np.arange(a.shape[1]) >> g[cs]) & 1)[None, :] == 1)
        return np.where(ok, new, a)
    if kind == OP_M2:
        m = mats[m0:m0 + 16].reshape(4, 4)
        t0, t1 = g[int(op['s0'])], g[int(op['s1'])]
        j = np.arange(a.shape[1])
        r = ((j >> t1) & 1) * 2 + ((j >> t0) & 1)
        base = j & ~((1 << t0) | (1 << t1))
        cols = [base, base | (1 << t0), base | (1 << t1), base | (1 << t0) | (1 << t1)]
        new = sum(m[r, c][None, :] * a[:, cols[c]] for c in range(4))
        return np.where(pred, new, a)
    if kind == OP_DIAG:
        d = mats[m0:m0 + 4]
        ba, bb = _diag_bits(gi, op, g, a.shape[1])
        f = d[ba + 2 * bb]
        return np.where(pred, a * f, a)
    raise AssertionError(kind)


def _diag_bits(tg, op, g, width):
    j = np.arange(width)
    out = []
    for key, skey in (('ga', 'sa'), ('gb', 'sb')):
        gbit, slot = int(op[key]), int(op[skey])
        if slot >= 0:
            out.append(((j >> g[slot]) & 1)[None, :])
        elif gbit != 0xFF:
            out.append(_bit(tg, gbit))
        else:
            out.append(0)
    return out[0], out[1]


def _grad(a, b, gi, op, g, mats, L, high):
    m0 = int(op['mat'])
    pred = _pred(gi, op, g)
    if int(op['s1']) == 1:
        d = mats[m0:m0 + 4]
        ba, bb = _diag_bits(gi, op, g, a.shape[1])
        ga_ = d[ba + 2 * bb] * a
    else:
        m = mats[m0:m0 + 4].reshape(2, 2)
        s0 = int(op['s0'])
        tl = (s0 - 16) if s0 >= 16 else g[s0]
        j = np.arange(a.shape[1])
        bit = (j >> tl) & 1
        p = a[:, j ^ (1 << tl)]
        ga_ = np.where(bit[None, :] == 0, m[0, 0] * a + m[0, 1] * p, m[1, 0] * p + m[1, 1] * a)
        cs = int(op['cslot'])
        if cs >= 0:
            pred = pred & (((j >> g[cs]) & 1)[None, :] == 1)
    return float(np.real(np.sum(np.where(pred, np.conj(b) * ga_, 0))))


def _variant_pair(m, var, x0, x1):
    """The kernel's per-variant 2x2 formulas (a wrong variant gives a wrong result here too)."""
    if var == 2:                      # diagonal
        return m[0, 0] * x0, m[1, 1] * x1
    if var == 3:                      # phase on |1>
        return x0, m[1, 1] * x1
    if var == 4:                      # anti-diagonal
        return m[0, 1] * x1, m[1, 0] * x0
    if var == 1:                      # real
        return m[0, 0].real * x0 + m[0, 1].real * x1, m[1, 0].real * x0 + m[1, 1].real * x1
    return m[0, 0] * x0 + m[0, 1] * x1, m[1, 0] * x0 + m[1, 1] * x1


def _apply_coded(a, tg, op, g, mats, code):
    """Follow the dispatch code exactly as the kernel's switch does."""
    m0 = int(op['mat'])
    pred = _pred(tg, op, g) if code & 0x8000 else np.ones_like(tg, dtype=bool)
    c = code & 0x7FFF
    j = np.arange(a.shape[1])
    if 1 <= c <= 57:
        m = mats[m0:m0 + 4].reshape(2, 2)
        if c <= 20:
            S, var, cs = (c - 1) // 5, (c - 1) % 5, -1
            tl = g[S]
        elif c <= 52:
            k = c - 21
            var = 4 if k % 2 == 0 else 0
            S, cs = (k // 2) // 4, (k // 2) % 4
            tl = g[S]
        else:
            var, cs = c - 53, -1
            tl = int(op['s0']) - 16
        bit = (j >> tl) & 1
        lo = j[bit == 0]
        hi = lo | (1 << tl)
        n0, n1 = _variant_pair(m, var, a[:, lo], a[:, hi])
        out = a.copy()
        out[:, lo], out[:, hi] = n0, n1
        ok = pred
        if cs >= 0:
            ok = ok & (((j >> g[cs]) & 1)[None, :] == 1)
        return np.where(ok, out, a)
    if 58 <= c <= 107:
        sign = c < 83
        k = c - (58 if sign else 83)
        SA, SB = k // 5 - 1, k % 5 - 1
        d = mats[m0:m0 + 4]
        ba = ((j >> g[SA]) & 1)[None, :] if SA >= 0 else (_bit(tg, int(op['ga'])) if int(op['ga']) != 0xFF else 0)
        bb = ((j >> g[SB]) & 1)[None, :] if SB >= 0 else (_bit(tg, int(op['gb'])) if int(op['gb']) != 0xFF else 0)
        f = d[ba + 2 * bb]
        if sign:
            f = np.where(np.real(f) < 0, -1.0, 1.0)
        return np.where(pred, a * f, a)
    if 120 <= c <= 151:
        real, mask = c >= 136, c - (136 if c >= 136 else 120)
        out = a
        k = 0
        for S in range(4):
            if not (mask >> S) & 1:
                continue
            m = mats[m0 + 4 * k:m0 + 4 * k + 4].reshape(2, 2)
            k += 1
            tl = g[S]
            lo = j[((j >> tl) & 1) == 0]
            hi = lo | (1 << tl)
            n0, n1 = _variant_pair(m, 1 if real else 0, out[:, lo], out[:, hi])
            out = out.copy()
            out[:, lo], out[:, hi] = n0, n1
        return np.where(pred, out, a)
    if 160 <= c <= 191:
        real, mask = c >= 176, c - (176 if c >= 176 else 160)
        lmask = int(op['s1']) & 0x1F
        out = a.copy()
        k = m0
        tls = [(g[S], True) for S in range(4) if (mask >> S) & 1] + [(b, False) for b in range(5) if (lmask >> b) & 1]
        for tl, slot in tls:
            if slot and not real:
                pk = mats[k:k + 8]          # packed form: (re, re), (-im, im) per entry
                m = (pk[0::2].real + 1j * pk[1::2].imag).reshape(2, 2)
                k += 8
            else:
                m = mats[k:k + 4].reshape(2, 2)
                k += 4
            lo = j[((j >> tl) & 1) == 0]
            hi = lo | (1 << tl)
            n0, n1 = _variant_pair(m, 1 if real else 0, out[:, lo], out[:, hi])
            out[:, lo], out[:, hi] = n0, n1
        return np.where(pred, out, a)
    if c == 154:
        cnt = int(op['s0'])
        wpe = mats.dtype.itemsize // 4
        raw = np.ascontiguousarray(mats).view(np.uint32)
        f = np.ones(a.shape, dtype=np.complex128)

        def bit(x):
            if x < 4:
                return ((j >> g[x]) & 1)[None, :]
            if x == 0xFF:
                return np.zeros((1, a.shape[1]), np.int64)
            return _bit(tg, x & 63)
        for e in range(cnt):
            hdr = int(raw[(m0 + 5 * e) * wpe])
            ba, bb = bit(hdr & 0xFF), bit((hdr >> 8) & 0xFF)
            kind = (hdr >> 16) & 0xF
            k = ba + 2 * bb
            if kind == 0:
                f = f * np.where(((hdr >> 20) >> k) & 1, -1.0, 1.0)
            else:
                d = mats[m0 + 5 * e + 1:m0 + 5 * e + 5]
                f = f * d[k]
        return np.where(pred, a * f, a)
    if c == 192:
        return _apply(a, tg, op, g, mats)
    if c == 152:
        npairs = int(op['s0'])
        wpe = mats.dtype.itemsize // 4
        w = np.ascontiguousarray(mats).view(np.uint32)[m0 * wpe:m0 * wpe + 2 * (6 + 2 * npairs)].astype(np.uint64)
        q = [int(w[2 * i]) | int(w[2 * i + 1]) << 32 for i in range(6 + 2 * npairs)]
        t = tg.astype(np.uint64)

        def par(x):
            x = x.astype(np.uint64)
            for sh in (32, 16, 8, 4, 2, 1):
                x = x ^ (x >> np.uint64(sh))
            return (x & np.uint64(1)).astype(np.int64)
        x = t & np.uint64(q[1])
        for i in range(npairs):
            x = x ^ (t & (t >> np.uint64(q[6 + 2 * i])) & np.uint64(q[7 + 2 * i]))
        reg = np.zeros(a.shape[1], np.int64)  # register index of every tile position
        for s_, gp in enumerate(g):
            reg |= ((j >> gp) & 1) << s_
        neg = ((q[0] & 0xFFFF) >> reg[None, :]) & 1
        neg = neg ^ par(x)
        for s_ in range(4):
            neg = neg ^ (par(t & np.uint64(q[2 + s_])) * ((reg[None, :] >> s_) & 1))
        return np.where(pred & (neg == 1), -a, a)
    raise AssertionError(f'unknown dispatch code {code}')
