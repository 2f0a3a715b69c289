// Plan-specialised fused pass.  The tile pipeline and register stages are
// those of k_fused_pass; the difference is that the pass's op list is compiled
// in.  The host writes one source per pass that calls the stage helpers below
// and the op bodies of stage_ops.cuh with every structural field -- register
// bit positions, dispatch code, matrix offsets, the +-1 sign masks -- as a
// compile-time constant, and compiles it with NVRTC for sm_100a
// (desv_jit.cu).  Only the matrix values are read at run time, at constant
// offsets, so the compiler can issue every coefficient load of a stage early
// and no per-op dispatch (header load, jump table) remains.
#pragma once

#include "desv_common.cuh"
#include "grad_ops.cuh"
#include "stage_ops.cuh"
#include "tile_pipeline.cuh"

namespace desv {

// Register stage on tile-local bits G0 < G1 < G2 < G3 (all >= 5).
template <typename T, uint32_t G0, uint32_t G1, uint32_t G2, uint32_t G3> struct JitStage {
    static __device__ __forceinline__ uint32_t off(int j) {
        return ((j & 1) ? (1u << G0) : 0u) + ((j & 2) ? (1u << G1) : 0u) + ((j & 4) ? (1u << G2) : 0u) +
               ((j & 8) ? (1u << G3) : 0u);
    }
    static __device__ __forceinline__ uint32_t index() { return stage_base4(threadIdx.x, G0, G1, G2, G3); }
    static __device__ __forceinline__ void load(T (&a)[16], const T *s, uint32_t idx) {
#pragma unroll
        for (int j = 0; j < 16; ++j) a[j] = s[idx + off(j)];
    }
    // back to the tile in shared memory for the next stage
    static __device__ __forceinline__ void store_smem(const T (&a)[16], T *s, uint32_t idx) {
#pragma unroll
        for (int j = 0; j < 16; ++j) s[idx + off(j)] = a[j];
        __syncthreads();
        // the next bulk load into this slot (async proxy) must follow these writes
        fence_proxy_async_smem();
    }
    // last stage: straight to HBM; lanes are index bits 0..4, so every warp
    // store covers 32 consecutive amplitudes
    static __device__ __forceinline__ void store_global(const T (&a)[16], T *sv, uint64_t tg, const uint64_t *ctab,
                                                        int L) {
        const uint64_t q0 = tl_bit(ctab, L, G0), q1 = tl_bit(ctab, L, G1), q2 = tl_bit(ctab, L, G2),
                       q3 = tl_bit(ctab, L, G3);
        T *out = sv + tg;
#pragma unroll
        for (int j = 0; j < 16; ++j)
            out[((j & 1) ? q0 : 0ull) + ((j & 2) ? q1 : 0ull) + ((j & 4) ? q2 : 0ull) + ((j & 8) ? q3 : 0ull)] = a[j];
    }
};

// Two arrays in lockstep (the adjoint pass's phi and lambda).
template <typename T, class S> struct JitStage2 {
    static __device__ __forceinline__ void store_smem(const T (&a)[16], const T (&b)[16], T *sa, T *sb,
                                                      uint32_t idx) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            sa[idx + S::off(j)] = a[j];
            sb[idx + S::off(j)] = b[j];
        }
        __syncthreads();
        fence_proxy_async_smem();
    }
};

// The pass: `stages(slot, tile_base, ctab, L)` applies every stage of one tile.
template <typename T, int K, int NBUF, class Stages>
__device__ __forceinline__ void jit_pass_kernel(T *sv, const TileGeom &g, unsigned char *smem, Stages &stages) {
    PipeArrays<T, 1> A;
    A.ptr[0] = sv;
    A.load[0] = true;
    A.store[0] = false;
    const int L = g.L;
    auto body = [=, &stages](T *const *sp, uint64_t base, uint64_t) { stages(sp[0], base, pipe_ctab(smem), L); };
    run_tiles<T, K, NBUF, 1>(g, A, body, smem);
}

// Gradient probes Re sum conj(b) (G a) with the generator's placement as
// compile-time constants (the forms of grad_term in grad_ops.cuh).  The thread
// predicate is applied by the caller after the call, since lane-bit
// generators shuffle with every lane.
template <int S, int CS, typename T>
__device__ __forceinline__ double jit_grad_reg(const T (&a)[16], const T (&b)[16], const T *mp) {
    return (double)grad_reg<S>(a, b, mp[0], mp[1], mp[2], mp[3], CS);
}
template <int CS, typename T>
__device__ __forceinline__ double jit_grad_lane(const T (&a)[16], const T (&b)[16], const T *mp, int lb, int lane) {
    const T g00 = mp[0], g01 = mp[1], g10 = mp[2], g11 = mp[3];
    const int mine = (lane >> lb) & 1;
    const T cself = mine ? g11 : g00, coth = mine ? g10 : g01;
    decltype(a[0].x) acc = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (CS >= 0 && !((j >> CS) & 1)) continue;
        const T p = shfl_xor(a[j], 1 << lb);
        const T v = cfma(coth, p, cmul(cself, a[j]));
        acc += b[j].x * v.x + b[j].y * v.y;
    }
    return (double)acc;
}
// Probes whose generator is known when the pass is generated (the generators
// of rx, ry, rz, p, cp and crz do not depend on the angle).  Four partial sums
// keep the multiply-adds independent.
//
// Y type, G = [[0, -h], [h, 0]] with h real (ry): Re sum conj(b) G a over the
// pairs on register slot S is h (Re conj(b1) a0 - Re conj(b0) a1).
template <int S, int CS, typename T>
__device__ __forceinline__ double jit_grad_y(const T (&a)[16], const T (&b)[16], decltype(T().x) h) {
    typedef decltype(T().x) R;
    // (s0, s1) and (s2, s3) as packed pairs: one packed FMA per pair and product
    T s01 = mk(R(0), R(0)), s23 = mk(R(0), R(0));
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if ((j >> S) & 1) continue;
        if (CS >= 0 && !((j >> CS) & 1)) continue;
        const int j1 = j | (1 << S);
        s01 = bfma(b[j1], a[j], s01);
        s23 = bfma(b[j], a[j1], s23);
    }
    return (double)(((s01.x + s01.y) - (s23.x + s23.y)) * h);
}
// X type, G = [[0, -i h], [-i h, 0]] with h real (rx): h (Im conj(b0) a1 + Im conj(b1) a0),
// Im conj(b) a = b.x a.y - b.y a.x.
template <int S, int CS, typename T>
__device__ __forceinline__ double jit_grad_x(const T (&a)[16], const T (&b)[16], decltype(T().x) h) {
    typedef decltype(T().x) R;
    R s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if ((j >> S) & 1) continue;
        if (CS >= 0 && !((j >> CS) & 1)) continue;
        const int j1 = j | (1 << S);
        s0 = fma(b[j].x, a[j1].y, s0);
        s1 = fma(b[j].y, a[j1].x, s1);
        s2 = fma(b[j1].x, a[j].y, s2);
        s3 = fma(b[j1].y, a[j].x, s3);
    }
    return (double)(((s0 - s1) + (s2 - s3)) * h);
}
// Imaginary diagonal, G = diag(i h_k) with k = bit(ga) + 2 bit(gb) (rz, p, cp,
// crz): Re conj(b) (i h) a = h (b.y a.x - b.x a.y), summed per class k.  The
// register part of k is a compile-time constant per amplitude; the bits on
// thread-fixed positions (fa, fb) complete it per thread.
template <int SA, int SB, typename T>
__device__ __forceinline__ double jit_grad_dim(const T (&a)[16], const T (&b)[16], decltype(T().x) h0,
                                               decltype(T().x) h1, decltype(T().x) h2, decltype(T().x) h3, int fa,
                                               int fb) {
    typedef decltype(T().x) R;
    R s[4] = {0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int kr = (SA >= 0 ? ((j >> SA) & 1) : 0) | (SB >= 0 ? (((j >> SB) & 1) << 1) : 0);
        s[kr] = fma(b[j].y, a[j].x, s[kr]);
        s[kr] = fma(-b[j].x, a[j].y, s[kr]);
    }
    const int kf = (SA >= 0 ? 0 : fa) | (SB >= 0 ? 0 : (fb << 1));
    R acc = 0;
#pragma unroll
    for (int kr = 0; kr < 4; ++kr) {
        if ((SA < 0 && (kr & 1)) || (SB < 0 && (kr & 2))) continue;
        const int k = kr | kf;   // selects, not an indexed array: no local memory
        const R hk = k == 0 ? h0 : k == 1 ? h1 : k == 2 ? h2 : h3;
        acc = fma(hk, s[kr], acc);
    }
    return (double)acc;
}

// Tangent forms of the adjoint passes (the tangent variant of a backward pass).
// A real rotation [[c, -s], [s, c]] on register slot S becomes
// x0 -= t x1, x1 += t x0 with t = s / c: one packed FMA per amplitude, and the
// result is 1/c times the exact one.  A conjugate pair of phases
// diag(c + i s, c - i s) on index bit b becomes x += i t x (bit 0) or
// x -= i t x (bit 1): two FMAs per amplitude, again 1/c times the exact one.
// The host keeps the running product of the 1/c of a pass: every gradient
// probe is multiplied by the inverse square of it (both arrays carry it) and
// the pass ends by multiplying both arrays by its inverse.
template <int S, typename T>
__device__ __forceinline__ void tan_rot(T (&a)[16], decltype(T().x) t) {
    const T pt = mk(t, t), nt = mk(-t, -t);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if ((j >> S) & 1) continue;
        const int j1 = j | (1 << S);
        const T x0 = a[j], x1 = a[j1];
        a[j] = bfma(nt, x1, x0);
        a[j1] = bfma(pt, x0, x1);
    }
}
// SA >= 0: the phase's bit is register slot SA; SA < 0: the thread-fixed bit fbit
template <int SA, typename T>
__device__ __forceinline__ void tan_phase(T (&a)[16], decltype(T().x) t, int fbit) {
    typedef decltype(T().x) R;
    const R tf = fbit ? -t : t;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const R tt = SA >= 0 ? (((j >> SA) & 1) ? -t : t) : tf;
        const R re = a[j].x, im = a[j].y;
        a[j].x = fma(-tt, im, re);
        a[j].y = fma(tt, re, im);
    }
}
template <typename T>
__device__ __forceinline__ void scale_both(T (&a)[16], T (&b)[16], decltype(T().x) f) {
    const T ff = mk(f, f);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        a[j] = bmul(ff, a[j]);
        b[j] = bmul(ff, b[j]);
    }
}

// Controlled X on register slot S (control register slot CS, or none): a
// swap of register pairs, no arithmetic.
template <int S, int CS, typename T>
__device__ __forceinline__ void swap_reg(T (&a)[16]) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if ((j >> S) & 1) continue;
        if (CS >= 0 && !((j >> CS) & 1)) continue;
        const T t = a[j];
        a[j] = a[j | (1 << S)];
        a[j | (1 << S)] = t;
    }
}

template <int SA, int SB, typename T>
__device__ __forceinline__ double jit_grad_diag(const T (&a)[16], const T (&b)[16], const T *mp, int fa, int fb) {
    const T d0 = mp[0], d1 = mp[1], d2 = mp[2], d3 = mp[3];
    decltype(a[0].x) acc = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int ba = SA >= 0 ? ((j >> SA) & 1) : fa;
        const int bb = SB >= 0 ? ((j >> SB) & 1) : fb;
        const int k = ba | (bb << 1);
        const T f = k == 0 ? d0 : k == 1 ? d1 : k == 2 ? d2 : d3;
        const T ga = cmul(f, a[j]);
        acc += b[j].x * ga.x + b[j].y * ga.y;
    }
    return (double)acc;
}

// Adjoint backward pass over (phi, lambda): `stages(sphi, slam, base, ctab, L,
// acc)` walks one tile; GRAD probes add into the per-warp FP64 accumulators
// acc[warp * nparams + p] in shared memory, reduced per CTA into part[] at the
// end (the layout k_grad_reduce reads).
template <typename T, int K, int NBUF, class Stages>
__device__ __forceinline__ void jit_adjoint_kernel(T *phi, T *lam, const TileGeom &g, unsigned char *smem, int nparams,
                                                   double *part, Stages &stages) {
    constexpr int NW = (1 << (K - 4)) / 32 > 0 ? (1 << (K - 4)) / 32 : 1;
    double *acc = reinterpret_cast<double *>(smem + PIPE_HDR_BYTES + (size_t)NBUF * 2 * (1u << K) * sizeof(T));
    for (int i = threadIdx.x; i < NW * nparams; i += blockDim.x) acc[i] = 0.0;
    PipeArrays<T, 2> A;
    A.ptr[0] = phi;
    A.ptr[1] = lam;
    A.load[0] = A.load[1] = true;
    A.store[0] = A.store[1] = false;
    const int L = g.L;
    auto body = [=, &stages](T *const *sp, uint64_t base, uint64_t) {
        stages(sp[0], sp[1], base, pipe_ctab(smem), L, acc);
    };
    __syncthreads();
    run_tiles<T, K, NBUF, 2>(g, A, body, smem);
    __syncthreads();
    for (int p = threadIdx.x; p < nparams; p += blockDim.x) {
        double s = 0;
        for (int w = 0; w < NW; ++w) s += acc[w * nparams + p];
        part[(size_t)blockIdx.x * nparams + p] = s;
    }
}

// n (|n| < 2^22) as a float without the conversion unit: 1.5 * 2^23 + n has
// the bits 0x4B400000 + n, from which 1.5 * 2^23 is subtracted exactly
__device__ __forceinline__ float small_int_to_float(int n) {
    return __int_as_float(0x4B400000 + n) - 12582912.0f;
}
__device__ __forceinline__ double small_int_to_double(int n) { return (double)n; }

// Pauli-sum pass over psi tiles (MODE 0: <H> only, 1: write H psi, 2: add
// into H psi): `body(tile, base, ctab, L, ere, eim)` evaluates the pass's terms
// (compiled in) for the tile's amplitudes.  The FP64 energy partials are
// reduced per CTA into part[2 * blockIdx.x + {0, 1}], the layout the
// interpreter k_pauli writes.
template <typename T, int K, int NBUF, class Body>
__device__ __forceinline__ void jit_pauli_kernel(const T *psi, const TileGeom &g, int want_e, double *part,
                                                 unsigned char *smem, Body &body) {
    PipeArrays<T, 1> A;
    A.ptr[0] = const_cast<T *>(psi);
    A.load[0] = true;
    A.store[0] = false;
    const int L = g.L;
    double ere = 0, eim = 0;
    auto tb = [=, &ere, &eim, &body](T *const *sp, uint64_t base, uint64_t) {
        body(sp[0], base, pipe_ctab(smem), L, ere, eim);
    };
    __syncthreads();
    run_tiles<T, K, NBUF, 1>(g, A, tb, smem);
    if (want_e) {
        __shared__ double sh[32];
        const double r = warp_sum_d(ere), i2 = warp_sum_d(eim);
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        __syncthreads();
        if (l == 0) sh[w] = r;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
            part[2 * blockIdx.x] = t;
        }
        __syncthreads();
        if (l == 0) sh[w] = i2;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
            part[2 * blockIdx.x + 1] = t;
        }
    }
}

}  // namespace desv
