// Fused gate pass: one HBM read + one HBM write of the state per pass, all of
// the pass's gates applied to shared-memory tiles in register stages.
// Replaces the per-gate lax.scan step of the reference
// (dense_evolution/circuits/compiler.py:136-355), which reads, gathers and
// writes the full state once per gate.
#include "desv_common.cuh"
#include "stage_ops.cuh"
#include "tile_pipeline.cuh"

namespace desv {

template <typename T, int K>
__device__ __forceinline__ void fused_tile_body(T *s, T *sv, uint64_t base, const uint64_t *ctab, int L,
                                                const desv_op *ops, int nops, const T *mats) {
    const int lane = threadIdx.x & 31;
    int k = 0;
#pragma unroll 1
    while (k < nops) {
        // stage record: register bit positions g[0..3] (bytes 9..12), op count (mat)
        const OpHead sh = load_head(ops + k);
        const int cnt = (int)sh.mat;
        const uint32_t g0 = (sh.w.z >> 8) & 0xFFu, g1 = (sh.w.z >> 16) & 0xFFu, g2 = sh.w.z >> 24,
                       g3 = sh.w.w & 0xFFu;
        const uint32_t idx = stage_base4(threadIdx.x, g0, g1, g2, g3);
        const uint32_t o0 = 1u << g0, o1 = 1u << g1, o2 = 1u << g2, o3 = 1u << g3;
        T a[16];
#pragma unroll
        for (int j = 0; j < 16; ++j)
            a[j] = s[idx + ((j & 1) ? o0 : 0u) + ((j & 2) ? o1 : 0u) + ((j & 4) ? o2 : 0u) + ((j & 8) ? o3 : 0u)];
        const uint64_t tg = base | tl2g(ctab, L, idx);
        run_stage_ops(a, ops + k + 1, cnt, mats, tg, lane);
        k += 1 + cnt;
        if (k >= nops) {
            // last stage: straight from registers to HBM.  Lanes are index bits
            // 0..4, so every store instruction of a warp writes 32 consecutive
            // amplitudes.
            const uint64_t q0 = tl_bit(ctab, L, g0), q1 = tl_bit(ctab, L, g1), q2 = tl_bit(ctab, L, g2),
                           q3 = tl_bit(ctab, L, g3);
            T *out = sv + tg;
#pragma unroll
            for (int j = 0; j < 16; ++j)
                out[((j & 1) ? q0 : 0ull) + ((j & 2) ? q1 : 0ull) + ((j & 4) ? q2 : 0ull) + ((j & 8) ? q3 : 0ull)] =
                    a[j];
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j)
                s[idx + ((j & 1) ? o0 : 0u) + ((j & 2) ? o1 : 0u) + ((j & 4) ? o2 : 0u) + ((j & 8) ? o3 : 0u)] = a[j];
            __syncthreads();
            // the next bulk load into this slot (async proxy) must follow these writes
            fence_proxy_async_smem();
        }
    }
}

// Loads run NBUF-1 tiles ahead (bulk copies into the shared-memory ring); the
// last register stage of every tile writes its amplitudes straight to HBM, so
// no ring slot waits for a store to drain.
template <typename T, int K, int NBUF>
__global__ void __launch_bounds__(1 << (K - 4)) k_fused_pass(T *sv, TileGeom g, const desv_op *ops, int nops,
                                                              const T *mats, RowStrides rs) {
    extern __shared__ __align__(128) unsigned char smem[];
    sv += blockIdx.y * rs.amps;
    mats += blockIdx.y * rs.mats;
    PipeArrays<T, 1> A;
    A.ptr[0] = sv;
    A.load[0] = true;
    A.store[0] = false;
    const int L = g.L;
    auto body = [=](T *const *sp, uint64_t base, uint64_t) {
        fused_tile_body<T, K>(sp[0], sv, base, pipe_ctab(smem), L, ops, nops, mats);
    };
    run_tiles<T, K, NBUF, 1>(g, A, body, smem);
}

template <typename T, int K, int NBUF>
static int launch_fused(T *sv, const TileGeom &g, const desv_op *ops, int nops, const T *mats, int rows,
                        const RowStrides &rs, cudaStream_t st) {
    static int bps[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = PIPE_HDR_BYTES + (size_t)NBUF * (1u << K) * sizeof(T);
    if (bps[dev & 63] == 0) {
        cudaFuncSetAttribute(k_fused_pass<T, K, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_fused_pass<T, K, NBUF>, 1 << (K - 4), smem);
        bps[dev & 63] = b > 0 ? b : 1;
    }
    const uint64_t ntiles = 1ull << (g.n - K);
    const uint64_t cap = (uint64_t)sm_count() * bps[dev & 63];
    const int grid = rs.amps != 0 ? rows_grid_x(ntiles, cap, rows) : (int)(ntiles < cap ? ntiles : cap);
    k_fused_pass<T, K, NBUF><<<dim3(grid, rows), 1 << (K - 4), smem, st>>>(sv, g, ops, nops, mats, rs);
    return check_launch("fused pass");
}

// one fused pass over `rows` states (rs: their strides; rows = 1, rs = {} for one state)
int fused_pass_rows(void *sv, int dtype, const TileGeom &g, const desv_op *ops, int nops, const void *mats, int rows,
                    const RowStrides &rs, cudaStream_t st) {
    if (dtype == DESV_C64) {
        float2 *p = static_cast<float2 *>(sv);
        const float2 *m = static_cast<const float2 *>(mats);
        switch (g.K) {
            case 9: return launch_fused<float2, 9, 4>(p, g, ops, nops, m, rows, rs, st);
            case 10: return launch_fused<float2, 10, 4>(p, g, ops, nops, m, rows, rs, st);
            case 11: return launch_fused<float2, 11, 4>(p, g, ops, nops, m, rows, rs, st);
            case 12: return launch_fused<float2, 12, 3>(p, g, ops, nops, m, rows, rs, st);
            case 13: return launch_fused<float2, 13, 3>(p, g, ops, nops, m, rows, rs, st);
            default: return fail(DESV_EINVAL, "fused pass: complex64 tile_bits must be 9..13");
        }
    }
    double2 *p = static_cast<double2 *>(sv);
    const double2 *m = static_cast<const double2 *>(mats);
    switch (g.K) {
        case 9: return launch_fused<double2, 9, 4>(p, g, ops, nops, m, rows, rs, st);
        case 10: return launch_fused<double2, 10, 4>(p, g, ops, nops, m, rows, rs, st);
        case 11: return launch_fused<double2, 11, 4>(p, g, ops, nops, m, rows, rs, st);
        case 12: return launch_fused<double2, 12, 3>(p, g, ops, nops, m, rows, rs, st);
        default: return fail(DESV_EINVAL, "fused pass: complex128 tile_bits must be 9..12");
    }
}

int fused_pass(void *sv, int dtype, const TileGeom &g, const desv_op *ops, int nops, const void *mats,
               cudaStream_t st) {
    return fused_pass_rows(sv, dtype, g, ops, nops, mats, 1, RowStrides{0, 0, 0, 0}, st);
}

}  // namespace desv
