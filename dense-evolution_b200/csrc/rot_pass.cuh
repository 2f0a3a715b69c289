// Device helpers of the rotation passes (plan-specialised complex64 passes
// compiled at run time by NVRTC; the host planner and code generator are
// dense_evolution/circuits/rotation.py).
//
// A thread holds the 32 amplitudes a[0..31] of one register stage: amplitude
// j has register slot k of its tile-local index set when bit k of j is.
// Everything here works on those registers with compile-time slot numbers,
// so the arrays stay in registers.
#pragma once

#include "desv_common.cuh"
#include "tile_pipeline.cuh"

namespace desv {

constexpr int ROT_NA = 32;   // amplitudes per thread (5 register slots)

// (re, im) * (cr + i ci)
__device__ __forceinline__ float2 cmulc(float2 a, float cr, float ci) {
    return make_float2(fmaf(a.x, cr, -a.y * ci), fmaf(a.x, ci, a.y * cr));
}

// Real rotation [[c, -s], [s, c]] on register slot S.  p[0..3] = (t, c, s,
// form): form 0 is the tangent form x0 -= t x1, x1 += t x0 (one packed FP32
// FMA per amplitude; the state is then 1/c too large, which a later table or
// end factor corrects), form 1 the general form.  The form is uniform across
// the grid (a parameter), so the branch never diverges.
template <int S> __device__ __forceinline__ void rot(float2 (&a)[ROT_NA], const float *p) {
    if (p[3] == 0.f) {
        const float t = p[0];
        const float2 pt = make_float2(t, t), nt = make_float2(-t, -t);
#pragma unroll
        for (int j = 0; j < ROT_NA; ++j) {
            if (j & (1 << S)) continue;
            const float2 x0 = a[j], x1 = a[j | (1 << S)];
            a[j] = __ffma2_rn(nt, x1, x0);
            a[j | (1 << S)] = __ffma2_rn(pt, x0, x1);
        }
    } else {
        const float c = p[1], s = p[2];
        const float2 pc = make_float2(c, c), ps = make_float2(s, s), ns = make_float2(-s, -s);
#pragma unroll
        for (int j = 0; j < ROT_NA; ++j) {
            if (j & (1 << S)) continue;
            const float2 x0 = a[j], x1 = a[j | (1 << S)];
            a[j] = __ffma2_rn(ns, x1, __fmul2_rn(pc, x0));
            a[j | (1 << S)] = __ffma2_rn(ps, x0, __fmul2_rn(pc, x1));
        }
    }
}

// every amplitude times the real f
__device__ __forceinline__ void scale_all(float2 (&a)[ROT_NA], float f) {
    const float2 ff = make_float2(f, f);
#pragma unroll
    for (int j = 0; j < ROT_NA; ++j) a[j] = __fmul2_rn(ff, a[j]);
}

// every amplitude times the complex (fr + i fi)
__device__ __forceinline__ void scale_all_c(float2 (&a)[ROT_NA], float fr, float fi) {
#pragma unroll
    for (int j = 0; j < ROT_NA; ++j) a[j] = cmulc(a[j], fr, fi);
}

// negate the amplitude when bit 31 of w is set (sign-bit flips of re and im)
__device__ __forceinline__ void flip(float2 &v, uint32_t w) {
    v.x = __uint_as_float(__float_as_uint(v.x) ^ w);
    v.y = __uint_as_float(__float_as_uint(v.y) ^ w);
}

}  // namespace desv
