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

enum : int { V_GEN = 0, V_REAL, V_DIAG, V_PHASE1, V_ANTI, V_BREAL };

// Element-wise products for real matrices stored duplicated as (v, v): one
// packed FP32 instruction per complex amplitude on sm_100 (fma.rn.f32x2).
__device__ __forceinline__ float2 bmul(const float2 &m, const float2 &x) { return __fmul2_rn(m, x); }
__device__ __forceinline__ float2 bfma(const float2 &m, const float2 &x, const float2 &c) {
    return __ffma2_rn(m, x, c);
}
__device__ __forceinline__ double2 bmul(const double2 &m, const double2 &x) { return make_double2(m.x * x.x, m.y * x.y); }
__device__ __forceinline__ double2 bfma(const double2 &m, const double2 &x, const double2 &c) {
    return make_double2(fma(m.x, x.x, c.x), fma(m.y, x.y, c.y));
}

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

// 2x2 on register slot S (pairs j, j | 1<<S).  CS >= 0: only pairs whose
// register bit CS is set are updated (control on a register slot); every
// register index is a compile-time constant.
template <int S, int VAR, int CS, typename T>
__device__ __forceinline__ void m1_reg(T (&a)[16], const M22<T> &m) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j & (1 << S)) continue;
        if (CS >= 0 && !((j >> CS) & 1)) continue;
        const int j1 = j | (1 << S);
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
            // (v, v) pairs of the real entries: one packed multiply and one packed
            // FMA per amplitude (the same roundings as the scalar form)
            const T p00 = mk(m.m00.x, m.m00.x), p01 = mk(m.m01.x, m.m01.x);
            const T p10 = mk(m.m10.x, m.m10.x), p11 = mk(m.m11.x, m.m11.x);
            a[j] = bfma(p01, x1, bmul(p00, x0));
            a[j1] = bfma(p11, x1, bmul(p10, x0));
        } else if (VAR == V_BREAL) {
            a[j] = bfma(m.m01, x1, bmul(m.m00, x0));
            a[j1] = bfma(m.m11, x1, bmul(m.m10, x0));
        } else {
            a[j] = cfma(m.m01, x1, cmul(m.m00, x0));
            a[j1] = cfma(m.m11, x1, cmul(m.m10, x0));
        }
    }
}

template <int S, typename T>
__device__ __forceinline__ void m1_reg_uncontrolled(T (&a)[16], const M22<T> &m, int var) {
    switch (var) {
        case V_DIAG: m1_reg<S, V_DIAG, -1>(a, m); break;
        case V_PHASE1: m1_reg<S, V_PHASE1, -1>(a, m); break;
        case V_ANTI: m1_reg<S, V_ANTI, -1>(a, m); break;
        case V_REAL: m1_reg<S, V_REAL, -1>(a, m); break;
        default: m1_reg<S, V_GEN, -1>(a, m); break;
    }
}

// controlled by register slot CS: anti-diagonal (CX-like) or general
template <int S, int CS, typename T>
__device__ __forceinline__ void m1_reg_ctl(T (&a)[16], const M22<T> &m, int var) {
    if (var == V_ANTI) m1_reg<S, V_ANTI, CS>(a, m);
    else m1_reg<S, V_GEN, CS>(a, m);
}

template <int S, typename T>
__device__ __forceinline__ void m1_reg_dispatch(T (&a)[16], const M22<T> &m, int var, int cs) {
    switch (cs) {
        case -1: m1_reg_uncontrolled<S>(a, m, var); break;
        case 0: if (S != 0) m1_reg_ctl<S, (S != 0 ? 0 : 1)>(a, m, var); break;
        case 1: if (S != 1) m1_reg_ctl<S, (S != 1 ? 1 : 0)>(a, m, var); break;
        case 2: if (S != 2) m1_reg_ctl<S, (S != 2 ? 2 : 0)>(a, m, var); break;
        default: if (S != 3) m1_reg_ctl<S, (S != 3 ? 3 : 0)>(a, m, var); break;
    }
}

// 2x2 on lane bit lb: the partner amplitude lives in lane ^ (1 << lb).
// Uncontrolled (no thread predicate, no register control): no selects.
template <int VAR, typename T>
__device__ __forceinline__ void m1_lane_free(T (&a)[16], const M22<T> &m, int lb, int lane) {
    const int mine = (lane >> lb) & 1;
    const T cself = mine ? m.m11 : m.m00;
    const T coth = mine ? m.m10 : m.m01;
    if (VAR == V_DIAG || VAR == V_PHASE1) {
        if (VAR == V_PHASE1 && !mine) return;
#pragma unroll
        for (int j = 0; j < 16; ++j) a[j] = cmul(cself, a[j]);
        return;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const T p = shfl_xor(a[j], 1 << lb);
        if (VAR == V_BREAL) { a[j] = bfma(coth, p, bmul(cself, a[j])); continue; }
        if (VAR == V_ANTI) a[j] = cmul(coth, p);
        else if (VAR == V_REAL) a[j] = rfma(coth.x, p, rfma(cself.x, a[j], mk(decltype(p.x)(0), decltype(p.x)(0))));
        else a[j] = cfma(coth, p, cmul(cself, a[j]));
    }
}

// controlled variant: thread predicate `pred` and/or register control slot `cs`
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

// diagonal factor d[bit(ga) + 2 bit(gb)] per amplitude.  SA / SB: register
// slot holding that bit (compile-time) or -1 when the bit is fixed for the
// thread (values fa / fb); the factor of every amplitude is then picked at
// compile time from four per-op registers.
template <int SA, int SB, typename T>
__device__ __forceinline__ void diag_slots(T (&a)[16], const T *dp, int fa, int fb, bool sign_only) {
    const T d[4] = {dp[0], dp[1], dp[2], dp[3]};
    if (sign_only) {
        const bool n0 = d[0].x < 0, n1 = d[1].x < 0, n2 = d[2].x < 0, n3 = d[3].x < 0;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int ba = SA >= 0 ? ((j >> SA) & 1) : fa;
            const int bb = SB >= 0 ? ((j >> SB) & 1) : fb;
            const int k = ba | (bb << 1);
            const bool neg = k == 0 ? n0 : k == 1 ? n1 : k == 2 ? n2 : n3;
            if (neg) a[j] = cneg(a[j]);
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int ba = SA >= 0 ? ((j >> SA) & 1) : fa;
        const int bb = SB >= 0 ? ((j >> SB) & 1) : fb;
        a[j] = cmul(d[ba | (bb << 1)], a[j]);
    }
}

template <int SA, typename T>
__device__ __forceinline__ void diag_sb(T (&a)[16], const T *dp, int sb, int fa, int fb, bool sg) {
    switch (sb) {
        case -1: diag_slots<SA, -1>(a, dp, fa, fb, sg); break;
        case 0: diag_slots<SA, 0>(a, dp, fa, fb, sg); break;
        case 1: diag_slots<SA, 1>(a, dp, fa, fb, sg); break;
        case 2: diag_slots<SA, 2>(a, dp, fa, fb, sg); break;
        default: diag_slots<SA, 3>(a, dp, fa, fb, sg); break;
    }
}

template <typename T>
__device__ __forceinline__ void diag_apply(T (&a)[16], const T *dp, int sa, int sb, int fa, int fb, bool sign_only) {
    if (sa < 0 && sb < 0) {
        const int k = fa | (fb << 1);
        const T f = dp[k];
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
    switch (sa) {
        case -1: diag_sb<-1>(a, dp, sb, fa, fb, sign_only); break;
        case 0: diag_sb<0>(a, dp, sb, fa, fb, sign_only); break;
        case 1: diag_sb<1>(a, dp, sb, fa, fb, sign_only); break;
        case 2: diag_sb<2>(a, dp, sb, fa, fb, sign_only); break;
        default: diag_sb<3>(a, dp, sb, fa, fb, sign_only); break;
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
                if (op.cmask == 0 && op.cslot < 0) {
                    const int lb = op.s0 - 16;
                    switch (var) {
                        case V_DIAG: m1_lane_free<V_DIAG>(a, m, lb, lane); break;
                        case V_PHASE1: m1_lane_free<V_PHASE1>(a, m, lb, lane); break;
                        case V_ANTI: m1_lane_free<V_ANTI>(a, m, lb, lane); break;
                        case V_REAL: m1_lane_free<V_REAL>(a, m, lb, lane); break;
                        default: m1_lane_free<V_GEN>(a, m, lb, lane); break;
                    }
                } else {
                    m1_lane(a, m, var, op.cslot, op.s0 - 16, pred, lane);
                }
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

// Host-computed dispatch codes (desv_op bytes 13-14, see include/desv.h):
//   1 + S*5 + VAR                        2x2 on register slot S, uncontrolled
//   21 + (S*4 + CS)*2 + (VAR != ANTI)    2x2 on slot S controlled by slot CS
//   53 + VAR                             2x2 on a lane bit, uncontrolled
//   58 + (SA+1)*5 + (SB+1)               sign-only diagonal (slots SA/SB, -1 = thread bit)
//   83 + (SA+1)*5 + (SB+1)               diagonal
//   | 0x8000                             the thread predicate (cmask/cval) applies
//   0                                    invalid in a plan (sets DESV_DEV_BADPLAN)
#define DESV_CODE_PRED 0x8000u
#define DESV_CODE_MULTI 120u      // + slot mask 1..15: general 2x2 on each slot in the mask
#define DESV_CODE_MULTI_REAL 136u // + slot mask: real 2x2 on each slot in the mask
#define DESV_CODE_SIGNS 152u      // group of +-1 diagonals: normal-form record, s0 product pairs
#define DESV_CODE_DIAG_GROUP 154u // group of diagonals, s0 entries of 5 elements at the op's matrix offset
#define DESV_CODE_LAYER 160u      // + slot mask 0..15: general 2x2 on those slots (packed form, 8 elements
                                  // per matrix) and on the lane bits in s1 (plain form)
#define DESV_CODE_LAYER_REAL 176u // + slot mask: the same with real matrices stored as (v, v) pairs
#define DESV_CODE_LANE_CTL 192u   // 2x2 on lane bit s0-16 with a register control (cslot) and/or predicate

template <int S, int CS, typename T>
__device__ __forceinline__ void m1_ctl_case(T (&a)[16], const M22<T> &m, bool anti) {
    if (CS == S) return;
    if (anti) m1_reg<S, V_ANTI, (CS == S ? -1 : CS)>(a, m);
    else m1_reg<S, V_GEN, (CS == S ? -1 : CS)>(a, m);
}

template <int SA, int SB, typename T>
__device__ __forceinline__ void diag_case(T (&a)[16], const T *mp, uint32_t w0y, uint64_t tg, bool sg) {
    // thread-fixed bit values, read only when the bit is not in a register slot
    const int fa = SA >= 0 ? 0 : (((w0y >> 8) & 0xFFu) == 0xFFu ? 0 : (int)((tg >> ((w0y >> 8) & 0xFFu)) & 1ull));
    const int fb = SB >= 0 ? 0 : (((w0y >> 16) & 0xFFu) == 0xFFu ? 0 : (int)((tg >> ((w0y >> 16) & 0xFFu)) & 1ull));
    diag_slots<SA, SB>(a, mp, fa, fb, sg);
}

#define DESV_M1U(S)                                                              \
    case 1 + S * 5 + V_GEN: m1_reg<S, V_GEN, -1>(a, load_m22(mp)); break;        \
    case 1 + S * 5 + V_REAL: m1_reg<S, V_REAL, -1>(a, load_m22(mp)); break;      \
    case 1 + S * 5 + V_DIAG: m1_reg<S, V_DIAG, -1>(a, load_m22(mp)); break;      \
    case 1 + S * 5 + V_PHASE1: m1_reg<S, V_PHASE1, -1>(a, load_m22(mp)); break;  \
    case 1 + S * 5 + V_ANTI: m1_reg<S, V_ANTI, -1>(a, load_m22(mp)); break;
#define DESV_M1C(S, CS)                                                                   \
    case 21 + (S * 4 + CS) * 2: m1_ctl_case<S, CS>(a, load_m22(mp), true); break;         \
    case 21 + (S * 4 + CS) * 2 + 1: m1_ctl_case<S, CS>(a, load_m22(mp), false); break;
#define DESV_DG(SA, SB)                                                                     \
    case 58 + (SA + 1) * 5 + (SB + 1): diag_case<SA, SB>(a, mp, w0y, tg, true); break;    \
    case 83 + (SA + 1) * 5 + (SB + 1): diag_case<SA, SB>(a, mp, w0y, tg, false); break;
#define DESV_DGROW(SA) DESV_DG(SA, -1) DESV_DG(SA, 0) DESV_DG(SA, 1) DESV_DG(SA, 2) DESV_DG(SA, 3)

// 2x2 gates on every register slot in the compile-time set M (ascending slot
// order, commuting: the slots are distinct); matrices are consecutive in the pool.
template <int M, int VAR, typename T>
__device__ __forceinline__ void multi_reg(T (&a)[16], const T *mp) {
    constexpr int k1 = (M & 1) ? 1 : 0;
    constexpr int k2 = k1 + ((M & 2) ? 1 : 0);
    constexpr int k3 = k2 + ((M & 4) ? 1 : 0);
    if (M & 1) m1_reg<0, VAR, -1>(a, load_m22(mp));
    if (M & 2) m1_reg<1, VAR, -1>(a, load_m22(mp + 4 * k1));
    if (M & 4) m1_reg<2, VAR, -1>(a, load_m22(mp + 4 * k2));
    if (M & 8) m1_reg<3, VAR, -1>(a, load_m22(mp + 4 * k3));
}

// 16-bit mask of the register indices j whose selected bit is 1: x < 4 is a
// register slot, 0x40 | b is global index bit b (fixed for the thread), 0xFF
// is an absent bit (always 0).
__device__ __forceinline__ uint32_t sign_bit_mask(uint32_t x, uint64_t tg) {
    if (x < 4u) return (uint32_t)(0xFF00F0F0CCCCAAAAull >> (16u * x)) & 0xFFFFu;
    if (x == 0xFFu) return 0u;
    return ((tg >> (x & 63u)) & 1ull) ? 0xFFFFu : 0u;
}

__device__ __forceinline__ void flip_sign(float2 &v, uint32_t s) {
    v.x = __uint_as_float(__float_as_uint(v.x) ^ s);
    v.y = __uint_as_float(__float_as_uint(v.y) ^ s);
}
__device__ __forceinline__ void flip_sign(double2 &v, uint32_t s) {
    const unsigned long long t = (unsigned long long)s << 32;
    v.x = __longlong_as_double(__double_as_longlong(v.x) ^ (long long)t);
    v.y = __longlong_as_double(__double_as_longlong(v.y) ^ (long long)t);
}

// A group of +-1 diagonals (cz, and cp / crz at angles that give signs) in
// algebraic normal form over the thread-fixed index bits, precomputed on the
// host.  Record (64-bit words at the op's matrix offset): q[0] the 16-bit
// negation mask shared by every thread; q[1] the global bits whose parity
// negates all 16 register amplitudes; q[2 + S] the global bits whose parity
// negates the amplitudes with register bit S set; then npairs pairs (d, M):
// the parity of bit(i) & bit(i + d) over i in M negates all 16.  tg has zeros
// at the register bits, so only thread-fixed bits enter.  The negations fold
// into one 16-bit mask per thread, applied once as sign-bit flips; every load
// of the record is independent of the others.
__device__ __forceinline__ uint32_t parity_mask(uint64_t x, uint32_t m) {
    return (0u - ((uint32_t)__popcll(x) & 1u)) & m;
}

// negate the register amplitudes j whose bit j of `neg` is set
template <typename T> __device__ __forceinline__ void sign_flips(T (&a)[16], uint32_t neg) {
#pragma unroll
    for (int j = 0; j < 16; ++j) flip_sign(a[j], (neg << (31 - j)) & 0x80000000u);
}

template <typename T>
__device__ __forceinline__ void signs_group(T (&a)[16], const uint64_t *q, int npairs, uint64_t tg) {
    const uint64_t c = q[0], lall = q[1], l0 = q[2], l1 = q[3], l2 = q[4], l3 = q[5];
    uint64_t x = tg & lall;
    if (npairs > 0) {
        const uint64_t d0 = q[6], m0 = q[7];
        x ^= tg & (tg >> (uint32_t)d0) & m0;
#pragma unroll 1
        for (int i = 1; i < npairs; ++i) x ^= tg & (tg >> (uint32_t)q[6 + 2 * i]) & q[7 + 2 * i];
    }
    const uint32_t neg = ((uint32_t)c & 0xFFFFu) ^ parity_mask(x, 0xFFFFu) ^ parity_mask(tg & l0, 0xAAAAu) ^
                         parity_mask(tg & l1, 0xCCCCu) ^ parity_mask(tg & l2, 0xF0F0u) ^
                         parity_mask(tg & l3, 0xFF00u);
    sign_flips(a, neg);
}

// 2x2 on register slot S with the matrix in packed form: for every entry m the
// pool holds A = (re m, re m) and B = (-im m, im m), so that
// m x = A * x + B * swap(x) element-wise -- four packed FP32 instructions per
// output amplitude (fma.rn.f32x2), the swapped inputs shared by both outputs.
template <typename T> __device__ __forceinline__ void load_packed8(const T *mp, T (&m)[8]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) m[k] = mp[k];
}
template <int S, typename T> __device__ __forceinline__ void m1_reg_packed(T (&a)[16], const T *mp) {
    T m[8];
    load_packed8(mp, m);
    const T A00 = m[0], B00 = m[1], A01 = m[2], B01 = m[3], A10 = m[4], B10 = m[5], A11 = m[6], B11 = m[7];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j & (1 << S)) continue;
        const int j1 = j | (1 << S);
        const T x0 = a[j], x1 = a[j1];
        const T s0 = mk(x0.y, x0.x), s1 = mk(x1.y, x1.x);
        a[j] = bfma(B01, s1, bfma(A01, x1, bfma(B00, s0, bmul(A00, x0))));
        a[j1] = bfma(B11, s1, bfma(A11, x1, bfma(B10, s0, bmul(A10, x0))));
    }
}

// packed-form gates on every register slot in M (8 elements per matrix)
template <int M, typename T> __device__ __forceinline__ void multi_reg_packed(T (&a)[16], const T *mp) {
    constexpr int k1 = (M & 1) ? 1 : 0;
    constexpr int k2 = k1 + ((M & 2) ? 1 : 0);
    constexpr int k3 = k2 + ((M & 4) ? 1 : 0);
    if (M & 1) m1_reg_packed<0>(a, mp);
    if (M & 2) m1_reg_packed<1>(a, mp + 8 * k1);
    if (M & 4) m1_reg_packed<2>(a, mp + 8 * k2);
    if (M & 8) m1_reg_packed<3>(a, mp + 8 * k3);
}

// 2x2 gates on the lane bits in `lmask` (bit b: lane bit b), commuting,
// matrices consecutive (ascending lane bit).
template <int VAR, typename T>
__device__ __forceinline__ void multi_lane(T (&a)[16], const T *mp, uint32_t lmask, int lane) {
#pragma unroll 1
    while (lmask) {
        const int lb = __ffs(lmask) - 1;
        lmask &= lmask - 1u;
        m1_lane_free<VAR>(a, load_m22(mp), lb, lane);
        mp += 4;
    }
}

// One layer of commuting uncontrolled 2x2 gates of a stage: register slots in
// M (compile time), then the lane bits in lmask.
template <int M, int VAR, typename T>
__device__ __forceinline__ void layer_op(T (&a)[16], const T *mp, uint32_t lmask, int lane) {
    constexpr int nreg = ((M & 1) ? 1 : 0) + ((M & 2) ? 1 : 0) + ((M & 4) ? 1 : 0) + ((M & 8) ? 1 : 0);
    if (M) multi_reg<M, VAR>(a, mp);
    multi_lane<VAR>(a, mp + 4 * nreg, lmask, lane);
}

// ---- diagonal groups (code DESV_CODE_DIAG_GROUP) ----------------------------
// Entry i: element 5i holds the header word a | b << 8 | kind << 16 | sign
// pattern << 20; elements 5i+1..5i+4 hold d[bit(a) + 2 bit(b)].  Entries with a
// register slot are normalised on the host so that d[0] == 1.
enum : uint32_t { DG_SIGN = 0, DG_THREAD = 1, DG_SLOT_A = 2, DG_SLOT_B = 3, DG_TWO = 4 };

__device__ __forceinline__ uint32_t dg_bit(uint32_t x, uint64_t tg) {
    return x == 0xFFu ? 0u : (uint32_t)((tg >> (x & 63u)) & 1ull);
}

template <typename T> __device__ __forceinline__ T cdiv(const T &x, const T &y) {
    const auto inv = decltype(y.x)(1) / (y.x * y.x + y.y * y.y);
    return mk((x.x * y.x + x.y * y.y) * inv, (x.y * y.x - x.x * y.y) * inv);
}

// amplitudes with register bit S == 0 times g0, == 1 times g1
template <int S, typename T> __device__ __forceinline__ void dg_slot16(T (&a)[16], const T &g0, const T &g1) {
#pragma unroll
    for (int j = 0; j < 16; ++j) a[j] = cmul((j >> S) & 1 ? g1 : g0, a[j]);
}
// amplitudes with register bit S == 1 times r
template <int S, typename T> __device__ __forceinline__ void dg_slot8(T (&a)[16], const T &r) {
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if ((j >> S) & 1) a[j] = cmul(r, a[j]);
}
template <typename T>
__device__ __forceinline__ void dg_slot(T (&a)[16], uint32_t s, bool full, const T &g0, const T &g1) {
    switch (s) {
        case 0: if (full) dg_slot16<0>(a, g0, g1); else dg_slot8<0>(a, g1); break;
        case 1: if (full) dg_slot16<1>(a, g0, g1); else dg_slot8<1>(a, g1); break;
        case 2: if (full) dg_slot16<2>(a, g0, g1); else dg_slot8<2>(a, g1); break;
        default: if (full) dg_slot16<3>(a, g0, g1); else dg_slot8<3>(a, g1); break;
    }
}

template <typename T>
__device__ __forceinline__ void diag_group(T (&a)[16], const T *e, int cnt, uint64_t tg) {
    using R = decltype(a[0].x);
    const T one = mk(R(1), R(0));
    T ps = one;
    uint32_t neg = 0;
    // thread-fixed factors (and the thread-dependent normalisation of slot entries)
#pragma unroll 1
    for (int i = 0; i < cnt; ++i) {
        const uint32_t h = *reinterpret_cast<const uint32_t *>(e + 5 * i);
        const uint32_t sa = h & 0xFFu, sb = (h >> 8) & 0xFFu, kind = (h >> 16) & 0xFu;
        if (kind == DG_SIGN) {
            const uint32_t ma1 = sign_bit_mask(sa, tg), mb1 = sign_bit_mask(sb, tg);
            const uint32_t ma0 = ~ma1 & 0xFFFFu, mb0 = ~mb1 & 0xFFFFu;
            const uint32_t p = h >> 20;
            neg ^= (ma0 & mb0 & (0u - (p & 1u))) ^ (ma1 & mb0 & (0u - ((p >> 1) & 1u))) ^
                   (ma0 & mb1 & (0u - ((p >> 2) & 1u))) ^ (ma1 & mb1 & (0u - ((p >> 3) & 1u)));
        } else if (kind == DG_THREAD) {
            ps = cmul(ps, e[5 * i + 1 + dg_bit(sa, tg) + 2 * dg_bit(sb, tg)]);
        } else if (kind == DG_SLOT_A) {
            if (dg_bit(sb, tg)) ps = cmul(ps, e[5 * i + 3]);
        } else if (kind == DG_SLOT_B) {
            if (dg_bit(sa, tg)) ps = cmul(ps, e[5 * i + 2]);
        }
    }
    // register-slot factors; the first one also carries ps
    bool first = true;
#pragma unroll 1
    for (int i = 0; i < cnt; ++i) {
        const uint32_t h = *reinterpret_cast<const uint32_t *>(e + 5 * i);
        const uint32_t sa = h & 0xFFu, sb = (h >> 8) & 0xFFu, kind = (h >> 16) & 0xFu;
        if (kind == DG_SLOT_A || kind == DG_SLOT_B) {
            const bool isa = kind == DG_SLOT_A;
            const uint32_t v = dg_bit(isa ? sb : sa, tg);
            const T *d = e + 5 * i + 1;
            // factor for slot bit 0 / 1 at this thread's other bit v (f0 == 1 when v == 0)
            const T f0 = v ? d[isa ? 2 : 1] : one;
            const T f1 = v ? d[3] : d[isa ? 1 : 2];
            const T r = v ? cdiv(f1, f0) : f1;
            if (first) dg_slot(a, isa ? sa : sb, true, ps, cmul(ps, r));
            else dg_slot(a, isa ? sa : sb, false, one, r);
            first = false;
        } else if (kind == DG_TWO) {
            // two register slots (rare: a non-sign diagonal inside the register set);
            // d[0] == 1, so only amplitudes with a slot bit set change
            const T *d = e + 5 * i + 1;
            const T d1 = d[1], d2 = d[2], d3 = d[3];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const uint32_t ba = (j >> sa) & 1u, bb = (j >> sb) & 1u;
                if (ba | bb) a[j] = cmul(bb ? (ba ? d3 : d2) : d1, a[j]);
            }
        }
    }
    if (first) {
#pragma unroll
        for (int j = 0; j < 16; ++j) a[j] = cmul(ps, a[j]);
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) flip_sign(a[j], (neg << (31 - j)) & 0x80000000u);
}

// general layer with the register-slot matrices in packed form, then the lane
// gates in plain form
template <int M, typename T>
__device__ __forceinline__ void layer_packed(T (&a)[16], const T *mp, uint32_t lmask, int lane) {
    constexpr int nreg = ((M & 1) ? 1 : 0) + ((M & 2) ? 1 : 0) + ((M & 4) ? 1 : 0) + ((M & 8) ? 1 : 0);
    if (M) multi_reg_packed<M>(a, mp);
    multi_lane<V_GEN>(a, mp + 8 * nreg, lmask, lane);
}

#define DESV_LAYER(M)                                                                        \
    case DESV_CODE_LAYER + M: layer_packed<M>(a, mp, (w0.x >> 24) & 0x1Fu, lane); break;     \
    case DESV_CODE_LAYER_REAL + M: layer_op<M, V_BREAL>(a, mp, (w0.x >> 24) & 0x1Fu, lane); break;

#define DESV_MULTI(M)                                              \
    case DESV_CODE_MULTI + M: multi_reg<M, V_GEN>(a, mp); break;   \
    case DESV_CODE_MULTI_REAL + M: multi_reg<M, V_REAL>(a, mp); break;

// First 24 bytes of an op record: bytes 0..15 (kinds, slots, code) and the
// matrix offset (bytes 16..19).  Records are 40 bytes, so only 8-byte loads
// are aligned for every record.
struct OpHead {
    uint4 w;
    uint32_t mat;
};

__device__ __forceinline__ OpHead load_head(const desv_op *opp) {
    const uint2 *p = reinterpret_cast<const uint2 *>(opp);
    const uint2 lo = p[0], hi = p[1], m = p[2];
    OpHead h;
    h.w = make_uint4(lo.x, lo.y, hi.x, hi.y);
    h.mat = m.x;
    return h;
}

// Apply the op whose header is `h` (record at `opp`) to the thread's registers.
template <typename T>
__device__ __forceinline__ void apply_op_head(T (&a)[16], const OpHead &h, const desv_op *opp, const T *mats,
                                              uint64_t tg, int lane) {
    const uint4 w0 = h.w;
    const uint32_t code = (w0.w >> 8) & 0xFFFFu;
    const T *mp = mats + h.mat;
    if (code & DESV_CODE_PRED) {
        if ((tg & opp->cmask) != opp->cval) return;
    }
    const uint32_t w0y = w0.y;  // bytes 4..7: cslot, ga, gb, sa
    switch (code & 0x7FFFu) {
        DESV_M1U(0) DESV_M1U(1) DESV_M1U(2) DESV_M1U(3)
        DESV_M1C(0, 1) DESV_M1C(0, 2) DESV_M1C(0, 3)
        DESV_M1C(1, 0) DESV_M1C(1, 2) DESV_M1C(1, 3)
        DESV_M1C(2, 0) DESV_M1C(2, 1) DESV_M1C(2, 3)
        DESV_M1C(3, 0) DESV_M1C(3, 1) DESV_M1C(3, 2)
        case 53 + V_GEN: m1_lane_free<V_GEN>(a, load_m22(mp), (int)((w0.x >> 16) & 0xFFu) - 16, lane); break;
        case 53 + V_REAL: m1_lane_free<V_REAL>(a, load_m22(mp), (int)((w0.x >> 16) & 0xFFu) - 16, lane); break;
        case 53 + V_DIAG: m1_lane_free<V_DIAG>(a, load_m22(mp), (int)((w0.x >> 16) & 0xFFu) - 16, lane); break;
        case 53 + V_PHASE1: m1_lane_free<V_PHASE1>(a, load_m22(mp), (int)((w0.x >> 16) & 0xFFu) - 16, lane); break;
        case 53 + V_ANTI: m1_lane_free<V_ANTI>(a, load_m22(mp), (int)((w0.x >> 16) & 0xFFu) - 16, lane); break;
        DESV_DGROW(-1) DESV_DGROW(0) DESV_DGROW(1) DESV_DGROW(2) DESV_DGROW(3)
        DESV_MULTI(1) DESV_MULTI(2) DESV_MULTI(3) DESV_MULTI(4) DESV_MULTI(5) DESV_MULTI(6) DESV_MULTI(7)
        DESV_MULTI(8) DESV_MULTI(9) DESV_MULTI(10) DESV_MULTI(11) DESV_MULTI(12) DESV_MULTI(13) DESV_MULTI(14)
        DESV_MULTI(15)
        DESV_LAYER(0) DESV_LAYER(1) DESV_LAYER(2) DESV_LAYER(3) DESV_LAYER(4) DESV_LAYER(5) DESV_LAYER(6)
        DESV_LAYER(7) DESV_LAYER(8) DESV_LAYER(9) DESV_LAYER(10) DESV_LAYER(11) DESV_LAYER(12) DESV_LAYER(13)
        DESV_LAYER(14) DESV_LAYER(15)
        case DESV_CODE_SIGNS:
            signs_group(a, reinterpret_cast<const uint64_t *>(mp), (int)((w0.x >> 16) & 0xFFu), tg);
            break;
        case DESV_CODE_DIAG_GROUP: diag_group(a, mp, (int)((w0.x >> 16) & 0xFFu), tg); break;
        case DESV_CODE_LANE_CTL:
            m1_lane(a, load_m22(mp), m1_variant((int)((w0.x >> 8) & 0xFFu)), (int)(int8_t)(w0.y & 0xFFu),
                    (int)((w0.x >> 16) & 0xFFu) - 16, (tg & opp->cmask) == opp->cval, lane);
            break;
        default: atomicOr(&g_dev_status, DESV_DEV_BADPLAN); break;
    }
}

template <typename T>
__device__ __forceinline__ void apply_op_at(T (&a)[16], const desv_op *opp, const T *mats, uint64_t tg, int lane) {
    apply_op_head(a, load_head(opp), opp, mats, tg, lane);
}

// Apply ops[0..nops) of one stage to the thread's registers; the next op's
// header is loaded while the current op runs.
template <typename T>
__device__ __forceinline__ void run_stage_ops(T (&a)[16], const desv_op *ops, int nops, const T *mats, uint64_t tg,
                                              int lane) {
    if (nops <= 0) return;
    OpHead h = load_head(ops);
#pragma unroll 1
    for (int k = 0; k < nops; ++k) {
        const OpHead hn = load_head(ops + (k + 1 < nops ? k + 1 : k));
        apply_op_head(a, h, ops + k, mats, tg, lane);
        h = hn;
    }
}
#undef DESV_MULTI
#undef DESV_LAYER
#undef DESV_M1U
#undef DESV_M1C
#undef DESV_DG
#undef DESV_DGROW

// Thread's tile-local index with zeros at the 4 register bits g[0..3] (ascending).
// thread t's register-amplitude-0 index: zero bits inserted at the four register
// positions g0 < g1 < g2 < g3 (scalar arguments keep everything in registers)
__device__ __forceinline__ uint32_t stage_base4(uint32_t t, uint32_t g0, uint32_t g1, uint32_t g2, uint32_t g3) {
    uint32_t x = (uint32_t)insert0(t, (int)g0);
    x = (uint32_t)insert0(x, (int)g1);
    x = (uint32_t)insert0(x, (int)g2);
    return (uint32_t)insert0(x, (int)g3);
}

__device__ __forceinline__ uint32_t stage_base(uint32_t t, const uint8_t *g) {
    uint32_t x = t;
#pragma unroll
    for (int s = 0; s < 4; ++s) x = (uint32_t)insert0(x, g[s]);
    return x;
}

}  // namespace desv
