"""Tile-level NumPy emulation of the rotation-pass kernels (test
infrastructure): it walks every tile of a pass the way the generated CUDA
does -- the same thread-to-index deposits (rotation.runs), register offsets,
padded shared-memory layout, item order, tangent / general rotation forms,
tables, sign words and end factors -- so the planner, the value program and
the kernels' index arithmetic can be checked against the oracle on the CPU."""
from __future__ import annotations

import numpy as np

from dense_evolution.circuits import rotation as R


def _deposit(t: np.ndarray, rs) -> np.ndarray:
    out = np.zeros_like(t, dtype=np.int64)
    for s, d, ln in rs:
        out |= ((t >> s) & ((1 << ln) - 1)) << d
    return out


def run(plan: R.RotationPlan, sv: np.ndarray, blocks) -> np.ndarray:
    """Apply every pass of the plan to sv (complex128, in place) and return it."""
    for ps, v in zip(plan.passes, blocks):
        _pass(plan, ps, sv, np.asarray(v, dtype=np.float64))
    return sv


def _pass(plan, ps, sv, v):
    n, K, L, high = plan.n, ps.K, ps.L, ps.high
    NA = 1 << R.RB
    NT = 1 << (K - R.RB)
    tile_bits = list(range(L)) + list(high)
    gmap = [b if b < L else high[b - L] for b in range(K)]
    rest = [b for b in range(n) if b not in tile_bits]
    ntiles = 1 << (n - K)
    tid = np.arange(ntiles, dtype=np.int64)
    base = np.zeros(ntiles, dtype=np.int64)
    for k, b in enumerate(rest):
        base |= ((tid >> k) & 1) << b
    # tile-local index -> global offset inside the tile
    loc = np.arange(1 << K, dtype=np.int64)
    tl2g = np.zeros(1 << K, dtype=np.int64)
    for p in range(K):
        tl2g |= ((loc >> p) & 1) << gmap[p]
    smem = np.zeros((ntiles, R.slot_elems(K)), dtype=np.complex128)
    smem[:, :1 << K] = sv[base[:, None] + tl2g[None, :]]
    t = np.arange(NT, dtype=np.int64)
    nst = len(ps.stages)
    for si, st in enumerate(ps.stages):
        first, last = si == 0, si == nst - 1
        regs = list(st.regs)
        nr = R.nonreg_bits(K, regs)
        lb = _deposit(t, R.runs(nr))
        gthr = _deposit(t, R.runs([gmap[b] for b in nr]))
        offs = np.array([R.reg_offset(j, regs) for j in range(NA)], dtype=np.int64)
        goffs = np.array([R.reg_offset(j, [gmap[p] for p in regs]) for j in range(NA)], dtype=np.int64)
        if first:
            a = smem[:, lb[:, None] + offs[None, :]]                        # [tile, thread, j]
        else:
            a = smem[:, R.padded(lb)[:, None] + R.padded(offs)[None, :]]
        gi = base[:, None] | gthr[None, :]                                  # [tile, thread]
        for kind, x in st.items:
            if kind == 'rot':
                pi, s, off = x
                tt, c, sn, form = v[off:off + 4]
                for j in range(NA):
                    if (j >> s) & 1:
                        continue
                    j1 = j | (1 << s)
                    x0, x1 = a[:, :, j].copy(), a[:, :, j1].copy()
                    if form == 0.0:
                        a[:, :, j], a[:, :, j1] = x0 - tt * x1, x1 + tt * x0
                    else:
                        a[:, :, j], a[:, :, j1] = c * x0 - sn * x1, sn * x0 + c * x1
            else:
                _group(x, a, gi, v)
        if last:
            if ps.end_scale_off >= 0:
                o = ps.end_scale_off
                f = complex(v[o], v[o + 1]) if ps.end_complex else v[o]
                a = a * f
            sv[gi[:, :, None] + goffs[None, None, :]] = a
        else:
            if first:
                smem = np.zeros_like(smem)    # the barrier before the padded re-layout
            smem[:, R.padded(lb)[:, None] + R.padded(offs)[None, :]] = a


def _bit(gi, x):
    return (gi >> x) & 1


def _group(g, a, gi, v):
    NA = a.shape[2]
    slots = [q for q in range(R.RB) if (g.reg_mask >> q) & 1]
    F = np.ones(gi.shape, dtype=np.complex128)
    for it in g.f_items:
        if it[0] == 'ph':
            _, pi, x, off = it
            F = F * np.where(_bit(gi, x) == 1, complex(v[off], v[off + 1]), 1.0)
        else:
            _, pi, xa, xb, off = it
            k = _bit(gi, xa) | (_bit(gi, xb) << 1)
            vals = v[off:off + 8:2] + 1j * v[off + 1:off + 8:2]
            F = F * vals[k]
    for j in range(NA):
        k = 0
        for i, q in enumerate(slots):
            if (j >> q) & 1:
                k |= 1 << i
        if g.has_table and k:
            o = g.t_off + 2 * k
            a[:, :, j] *= complex(v[o], v[o + 1])
        if g.f_items:
            a[:, :, j] *= F
    for pi, s, x, off in g.mixed_items:
        X = _bit(gi, x)
        vals = v[off:off + 8:2] + 1j * v[off + 1:off + 8:2]     # (x, y) -> vals[2 x + y]
        for j in range(NA):
            y = (j >> s) & 1
            a[:, :, j] *= vals[2 * X + y]
    for j in range(NA):
        sgn = np.zeros(gi.shape, dtype=np.int64)
        for s, x in g.signs_mixed:
            if (j >> s) & 1:
                sgn ^= _bit(gi, x)
        for x, y in g.signs_thread:
            sgn ^= _bit(gi, x) & _bit(gi, y)
        neg = sum(1 for sa, sb in g.signs_reg if (j >> sa) & 1 and (j >> sb) & 1) & 1
        sgn ^= neg
        a[:, :, j] *= np.where(sgn == 1, -1.0, 1.0)
