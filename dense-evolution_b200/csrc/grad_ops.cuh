// Gradient probes of the adjoint passes: Re sum conj(lambda) (G phi) over a
// thread's register amplitudes for a GRAD op (see DESV_OP_GRAD).
#pragma once

#include "desv_common.cuh"

namespace desv {

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Re sum conj(b) (G a) for a 2x2 generator on register slot S (compile-time
// register indices keep a[] and b[] in registers).
template <int S, typename T>
__device__ __forceinline__ decltype(T().x) grad_reg(const T (&a)[16], const T (&b)[16], T g00, T g01, T g10, T g11,
                                                    int cs) {
    decltype(T().x) acc = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if ((j >> S) & 1) continue;
        if (cs >= 0 && !((j >> cs) & 1)) continue;
        const int j1 = j | (1 << S);
        const T v0 = cfma(g01, a[j1], cmul(g00, a[j]));
        const T v1 = cfma(g11, a[j1], cmul(g10, a[j]));
        acc += b[j].x * v0.x + b[j].y * v0.y + b[j1].x * v1.x + b[j1].y * v1.y;
    }
    return acc;
}

// Re sum conj(b) (G a) over the thread's amplitudes for a GRAD op.
//   s1 == 0: G = 2x2 generator on register slot / lane bit s0 (controls as M1)
//   s1 == 1: G = diagonal over global bits ga, gb (factor d[bit(ga) + 2 bit(gb)])
template <typename T>
__device__ __forceinline__ double grad_term(const T (&a)[16], const T (&b)[16], const desv_op &op, const T *mp,
                                            uint64_t tg, int lane) {
    // predicate is applied at the end: lane-bit generators shuffle with every lane
    const bool pred = (tg & op.cmask) == op.cval;
    typedef decltype(a[0].x) R;
    R acc = 0;
    if (op.s1 == 1) {
        const T d0 = mp[0], d1 = mp[1], d2 = mp[2], d3 = mp[3];
        const int fa = op.ga == 0xFF ? 0 : (int)((tg >> op.ga) & 1ull);
        const int fb = op.gb == 0xFF ? 0 : (int)((tg >> op.gb) & 1ull);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int ba = op.sa >= 0 ? ((j >> op.sa) & 1) : fa;
            const int bb = op.sb >= 0 ? ((j >> op.sb) & 1) : fb;
            const int k = ba | (bb << 1);
            const T f = k == 0 ? d0 : k == 1 ? d1 : k == 2 ? d2 : d3;
            const T ga = cmul(f, a[j]);
            acc += b[j].x * ga.x + b[j].y * ga.y;
        }
        return pred ? (double)acc : 0.0;
    }
    const T g00 = mp[0], g01 = mp[1], g10 = mp[2], g11 = mp[3];
    const int cs = op.cslot;
    if (op.s0 >= 16) {
        const int lb = op.s0 - 16;
        const int mine = (lane >> lb) & 1;
        const T cself = mine ? g11 : g00, coth = mine ? g10 : g01;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            if (cs >= 0 && !((j >> cs) & 1)) continue;
            const T p = shfl_xor(a[j], 1 << lb);
            const T v = cfma(coth, p, cmul(cself, a[j]));
            acc += b[j].x * v.x + b[j].y * v.y;
        }
        return pred ? (double)acc : 0.0;
    }
    switch (op.s0) {
        case 0: acc = grad_reg<0>(a, b, g00, g01, g10, g11, cs); break;
        case 1: acc = grad_reg<1>(a, b, g00, g01, g10, g11, cs); break;
        case 2: acc = grad_reg<2>(a, b, g00, g01, g10, g11, cs); break;
        default: acc = grad_reg<3>(a, b, g00, g01, g10, g11, cs); break;
    }
    return pred ? (double)acc : 0.0;
}

}  // namespace desv
