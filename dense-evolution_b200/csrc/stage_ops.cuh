// Register-stage interpreter of a fused pass.
//
// A stage owns 4 tile-local index bits g[0..3] (all >= 5): each of the
// 2^(K-4) threads holds the 16 amplitudes that differ only in those bits, in
// registers.  Index bits 0..4 are the lane id, so a gate on them is a warp
// shuffle with lane ^ (1 << bit).  Every other bit is fixed per thread, so
// controls and diagonal factors on them are per-thread predicates / scalars.
// Gates on the 4 register slots are unrolled with compile-time register
// indices (slot chosen by a uniform switch), so nothing spills to local memory.
#pragma once

#include "desv_common.cuh"

namespace desv {

enum : int { V_GEN = 0, V_REAL, V_DIAG, V_PHASE1, V_ANTI };

__device__ __forceinline__ int m1_variant(int flags) {
    if (flags & DESV_F_PHASE1) return V_PHASE1;
    if (flags & DESV_F_DIAG) return V_DIAG;
    if (flags & DESV_F_ANTI) return V_ANTI;
    if (flags & DESV_F_REAL) return V_REAL;
    return V_GEN;
}

template <typename T> struct M22 { T m00, m01, m10, m11; };

template <typename T> __device__ __forceinline__ M22<T> load_m22(const T *p) {
    M22<T> m;
    m.m00 = p[0]; m.m01 = p[1]; m.m10 = p[2]; m.m11 = p[3];
    return m;
}

// 16-bit mask of the register indices j whose bit `slot` is set
__device__ __forceinline__ uint32_t slot_mask(int slot) {
    return slot == 0 ? 0xAAAAu : slot == 1 ? 0xCCCCu : slot == 2 ? 0xF0F0u : 0xFF00u;
}

// 2x2 on register slot S (pairs j, j | 1<<S).  CTRL: only pairs whose bit in
// the 16-bit mask `act` is set are updated (control on a register slot).
template <int S, int VAR, bool CTRL, typename T>
__device__ __forceinline__ void m1_reg(T (&a)[16], const M22<T> &m, uint32_t act) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j & (1 << S)) continue;
        const int j1 = j | (1 << S);
        if (CTRL && !((act >> j) & 1u)) continue;
        const T x0 = a[j], x1 = a[j1];
        if (VAR == V_DIAG) {
            a[j] = cmul(m.m00, x0);
            a[j1] = cmul(m.m11, x1);
        } else if (VAR == V_PHASE1) {
            a[j1] = cmul(m.m11, x1);
        } else if (VAR == V_ANTI) {
            a[j] = cmul(m.m01, x1);
            a[j1] = cmul(m.m10, x0);
        } else if (VAR == V_REAL) {
            a[j] = rfma(m.m01.x, x1, rfma(m.m00.x, x0, mk(decltype(x0.x)(0), decltype(x0.x)(0))));
            a[j1] = rfma(m.m11.x, x1, rfma(m.m10.x, x0, mk(decltype(x0.x)(0), decltype(x0.x)(0))));
        } else {
            a[j] = cfma(m.m01, x1, cmul(m.m00, x0));
            a[j1] = cfma(m.m11, x1, cmul(m.m10, x0));
        }
    }
}

template <int S, bool CTRL, typename T>
__device__ __forceinline__ void m1_reg_var(T (&a)[16], const M22<T> &m, int var, uint32_t act) {
    switch (var) {
        case V_DIAG: m1_reg<S, V_DIAG, CTRL>(a, m, act); break;
        case V_PHASE1: m1_reg<S, V_PHASE1, CTRL>(a, m, act); break;
        case V_ANTI: m1_reg<S, V_ANTI, CTRL>(a, m, act); break;
        case V_REAL: m1_reg<S, V_REAL, CTRL>(a, m, act); break;
        default: m1_reg<S, V_GEN, CTRL>(a, m, act); break;
    }
}

template <int S, typename T>
__device__ __forceinline__ void m1_reg_dispatch(T (&a)[16], const M22<T> &m, int var, int cs) {
    if (cs < 0) m1_reg_var<S, false>(a, m, var, 0xFFFFu);
    else m1_reg_var<S, true>(a, m, var, slot_mask(cs));
}

// 2x2 on lane bit lb: the partner amplitude lives in lane ^ (1 << lb).
template <typename T>
__device__ __forceinline__ void m1_lane(T (&a)[16], const M22<T> &m, int var, int cs, int lb, bool pred, int lane) {
    const int mine = (lane >> lb) & 1;
    const T cself = mine ? m.m11 : m.m00;
    const T coth = mine ? m.m10 : m.m01;
    const uint32_t act = cs < 0 ? 0xFFFFu : slot_mask(cs);
    if (var == V_DIAG || var == V_PHASE1) {
        if (!pred || (var == V_PHASE1 && !mine)) return;
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if ((act >> j) & 1u) a[j] = cmul(cself, a[j]);
        return;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (!((act >> j) & 1u)) continue;  // uniform across the warp
        const T p = shfl_xor(a[j], 1 << lb);
        T r;
        if (var == V_ANTI) r = cmul(coth, p);
        else if (var == V_REAL) r = rfma(coth.x, p, rfma(cself.x, a[j], mk(decltype(p.x)(0), decltype(p.x)(0))));
        else r = cfma(coth, p, cmul(cself, a[j]));
        if (pred) a[j] = r;
    }
}

// 4x4 on register slots S0 < S1; row index = 2*bit(S1) + bit(S0).
template <int S0, int S1, typename T>
__device__ __forceinline__ void m2_reg(T (&a)[16], const T *mp) {
    T m[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) m[k] = mp[k];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j & ((1 << S0) | (1 << S1))) continue;
        const int i1 = j | (1 << S0), i2 = j | (1 << S1), i3 = j | (1 << S0) | (1 << S1);
        const T v0 = a[j], v1 = a[i1], v2 = a[i2], v3 = a[i3];
        T o[4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
            o[r] = cfma(m[4 * r + 3], v3, cfma(m[4 * r + 2], v2, cfma(m[4 * r + 1], v1, cmul(m[4 * r], v0))));
        a[j] = o[0]; a[i1] = o[1]; a[i2] = o[2]; a[i3] = o[3];
    }
}

template <typename T>
__device__ __forceinline__ void m2_dispatch(T (&a)[16], const T *mp, int s0, int s1) {
    switch (s0 * 4 + s1) {
        case 1: m2_reg<0, 1>(a, mp); break;
        case 2: m2_reg<0, 2>(a, mp); break;
        case 3: m2_reg<0, 3>(a, mp); break;
        case 6: m2_reg<1, 2>(a, mp); break;
        case 7: m2_reg<1, 3>(a, mp); break;
        case 11: m2_reg<2, 3>(a, mp); break;
        default: break;
    }
}

// diagonal factor d[bit(ga) + 2 bit(gb)]; bits come from register slots sa/sb
// or the thread index.  The per-amplitude selection uses 16-bit masks
// computed once per op.
template <typename T>
__device__ __forceinline__ void diag_apply(T (&a)[16], const T *dp, int sa, int sb, int fa, int fb, bool sign_only) {
    const T d0 = dp[0], d1 = dp[1], d2 = dp[2], d3 = dp[3];
    if (sa < 0 && sb < 0) {
        const int k = fa | (fb << 1);
        const T f = k == 0 ? d0 : k == 1 ? d1 : k == 2 ? d2 : d3;
        if (sign_only) {
            if (f.x < 0)
#pragma unroll
                for (int j = 0; j < 16; ++j) a[j] = cneg(a[j]);
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) a[j] = cmul(f, a[j]);
        }
        return;
    }
    const uint32_t A = sa >= 0 ? slot_mask(sa) : (fa ? 0xFFFFu : 0u);
    const uint32_t B = sb >= 0 ? slot_mask(sb) : (fb ? 0xFFFFu : 0u);
    const uint32_t m0 = ~A & ~B & 0xFFFFu, m1 = A & ~B & 0xFFFFu, m2 = ~A & B & 0xFFFFu, m3 = A & B;
    if (sign_only) {
        const uint32_t neg = (d0.x < 0 ? m0 : 0u) | (d1.x < 0 ? m1 : 0u) | (d2.x < 0 ? m2 : 0u) | (d3.x < 0 ? m3 : 0u);
        if (neg)
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if ((neg >> j) & 1u) a[j] = cneg(a[j]);
        return;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const T f = ((m3 >> j) & 1u) ? d3 : ((m2 >> j) & 1u) ? d2 : ((m1 >> j) & 1u) ? d1 : d0;
        a[j] = cmul(f, a[j]);
    }
}

// Apply one op to the thread's registers.  `tg` is the global index of the
// thread's register-amplitude 0 (register bits zero).
template <typename T>
__device__ __forceinline__ void apply_one_op(T (&a)[16], const desv_op &op, const T *mats, uint64_t tg, int lane) {
    {
        const bool pred = (tg & op.cmask) == op.cval;
        const T *mp = mats + op.mat;
        if (op.kind == DESV_OP_M1) {
            const int var = m1_variant(op.flags);
            const M22<T> m = load_m22(mp);
            if (op.s0 >= 16) {
                m1_lane(a, m, var, op.cslot, op.s0 - 16, pred, lane);
            } else if (pred) {
                switch (op.s0) {
                    case 0: m1_reg_dispatch<0>(a, m, var, op.cslot); break;
                    case 1: m1_reg_dispatch<1>(a, m, var, op.cslot); break;
                    case 2: m1_reg_dispatch<2>(a, m, var, op.cslot); break;
                    default: m1_reg_dispatch<3>(a, m, var, op.cslot); break;
                }
            }
        } else if (op.kind == DESV_OP_M2) {
            if (pred) m2_dispatch(a, mp, op.s0, op.s1);
        } else if (op.kind == DESV_OP_DIAG) {
            if (pred) {
                const int fa = op.ga == 0xFF ? 0 : (int)((tg >> op.ga) & 1ull);
                const int fb = op.gb == 0xFF ? 0 : (int)((tg >> op.gb) & 1ull);
                diag_apply(a, mp, op.sa, op.sb, fa, fb, (op.flags & DESV_F_SIGN) != 0);
            }
        }
    }
}

// Apply ops[0..nops) of one stage to the thread's registers.
template <typename T>
__device__ __forceinline__ void run_stage_ops(T (&a)[16], const desv_op *ops, int nops, const T *mats, uint64_t tg,
                                              int lane) {
#pragma unroll 1
    for (int k = 0; k < nops; ++k) {
        const desv_op op = ops[k];
        apply_one_op(a, op, mats, tg, lane);
    }
}

// Thread's tile-local index with zeros at the 4 register bits g[0..3] (ascending).
__device__ __forceinline__ uint32_t stage_base(uint32_t t, const uint8_t *g) {
    uint32_t x = t;
#pragma unroll
    for (int s = 0; s < 4; ++s) x = (uint32_t)insert0(x, g[s]);
    return x;
}

}  // namespace desv
