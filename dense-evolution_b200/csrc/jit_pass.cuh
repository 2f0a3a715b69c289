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

}  // namespace desv
