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

constexpr int ROT_NA = 32;   // amplitudes per thread with 5 register slots (the default; 6 slots: 64)

// (re, im) * (cr + i ci)
__device__ __forceinline__ float2 cmulc(float2 a, float cr, float ci) {
    return make_float2(fmaf(a.x, cr, -a.y * ci), fmaf(a.x, ci, a.y * cr));
}

// Real rotation [[c, -s], [s, c]] on register slot S.  form 0 is the tangent
// form x0 -= t x1, x1 += t x0 (one packed FP32 FMA per amplitude; the state is
// then 1/c too large, which the pass-end factor corrects), form 1 the general
// form.  The values are kernel parameters (uniform across the grid), so the
// branch never diverges.
template <int S, int NA>
__device__ __forceinline__ void rot(float2 (&a)[NA], float t, float c, float s, float form) {
    if (form == 0.f) {
        const float2 pt = make_float2(t, t), nt = make_float2(-t, -t);
#pragma unroll
        for (int j = 0; j < NA; ++j) {
            if (j & (1 << S)) continue;
            const float2 x0 = a[j], x1 = a[j | (1 << S)];
            a[j] = __ffma2_rn(nt, x1, x0);
            a[j | (1 << S)] = __ffma2_rn(pt, x0, x1);
        }
    } else {
        const float2 pc = make_float2(c, c), ps = make_float2(s, s), ns = make_float2(-s, -s);
#pragma unroll
        for (int j = 0; j < NA; ++j) {
            if (j & (1 << S)) continue;
            const float2 x0 = a[j], x1 = a[j | (1 << S)];
            a[j] = __ffma2_rn(ns, x1, __fmul2_rn(pc, x0));
            a[j | (1 << S)] = __ffma2_rn(ps, x0, __fmul2_rn(pc, x1));
        }
    }
}

// The tangent form alone: the pass variant run when every rotation of the
// call takes the tangent form (the usual case), without the general form's
// code, which doubles the size of a pass.
template <int S, int NA>
__device__ __forceinline__ void rot_t(float2 (&a)[NA], float t) {
    const float2 pt = make_float2(t, t), nt = make_float2(-t, -t);
#pragma unroll
    for (int j = 0; j < NA; ++j) {
        if (j & (1 << S)) continue;
        const float2 x0 = a[j], x1 = a[j | (1 << S)];
        a[j] = __ffma2_rn(nt, x1, x0);
        a[j | (1 << S)] = __ffma2_rn(pt, x0, x1);
    }
}

// Shared-memory and global accesses of the generated stages.  With
// DESV_ROT_CHECK defined (a diagnostic build of a pass) every index is checked
// against its array first; an access out of range is skipped and recorded in
// the module's status word (DESV_DEV_BADPLAN) instead of being made.
#ifdef DESV_ROT_CHECK
#define ROT_SLD(dst, s, idx)                                          \
    do {                                                              \
        const uint32_t i_ = (idx);                                    \
        if (i_ < ROT_SLOT_ELEMS) (dst) = (s)[i_];                     \
        else atomicOr(&g_dev_status, DESV_DEV_BADPLAN);               \
    } while (0)
#define ROT_SST(s, idx, v)                                            \
    do {                                                              \
        const uint32_t i_ = (idx);                                    \
        if (i_ < ROT_SLOT_ELEMS) (s)[i_] = (v);                       \
        else atomicOr(&g_dev_status, DESV_DEV_BADPLAN);               \
    } while (0)
#define ROT_GST(sv, idx, v)                                           \
    do {                                                              \
        const uint64_t i_ = (idx);                                    \
        if (i_ < (1ull << g.n)) (sv)[i_] = (v);                       \
        else atomicOr(&g_dev_status, DESV_DEV_BADPLAN);               \
    } while (0)
#else
#define ROT_SLD(dst, s, idx) ((dst) = (s)[(idx)])
#define ROT_SST(s, idx, v) ((s)[(idx)] = (v))
#define ROT_GST(sv, idx, v) ((sv)[(idx)] = (v))
#endif

// every amplitude times the real f
template <int NA> __device__ __forceinline__ void scale_all(float2 (&a)[NA], float f) {
    const float2 ff = make_float2(f, f);
#pragma unroll
    for (int j = 0; j < NA; ++j) a[j] = __fmul2_rn(ff, a[j]);
}

// every amplitude times the complex (fr + i fi)
template <int NA> __device__ __forceinline__ void scale_all_c(float2 (&a)[NA], float fr, float fi) {
#pragma unroll
    for (int j = 0; j < NA; ++j) a[j] = cmulc(a[j], fr, fi);
}

// negate the amplitude when bit 31 of w is set (sign-bit flips of re and im)
__device__ __forceinline__ void flip(float2 &v, uint32_t w) {
    v.x = __uint_as_float(__float_as_uint(v.x) ^ w);
    v.y = __uint_as_float(__float_as_uint(v.y) ^ w);
}

// Load-only tile ring of a rotation pass (the schedule of run_tiles in
// tile_pipeline.cuh, with the tile loop left to the generated kernel so that
// its stage code reads the per-call values straight from the kernel's
// parameter block): ring slots of SLOT amplitudes hold the natural layout of
// a 2^K tile as the bulk copies leave it, with room for the padded layout the
// stages re-lay it into.  Loads run NBUF-1 tiles ahead; with one slot the
// next tile's load starts once the last stage has read the slot (release).
template <int K, int NBUF, uint32_t SLOT> struct RotRing {
    // every slot must start on a 16-byte boundary (bulk-copy destinations) and
    // hold the padded layout of a tile
    static_assert(SLOT % 2 == 0, "ring slots of whole 16-byte units");
    static_assert(SLOT >= (1u << K) + ((1u << K) - 1) / 16, "a slot holds the padded tile");
    uint64_t *full;
    float2 *bufs;
    uint32_t tid, nthr, lane, ntile, nchunks, chunk_bytes, warp_bytes, cnt;
    uint64_t my_off, my_off2, rmask, tstride, lbase, cbase;
    const float2 *src;

    __device__ __forceinline__ void init(const TileGeom &geom, const float2 *sv, unsigned char *smem) {
        src = sv;
        full = reinterpret_cast<uint64_t *>(smem);
        bufs = reinterpret_cast<float2 *>(smem + PIPE_HDR_BYTES);
        tid = threadIdx.x;
        nthr = blockDim.x;
        lane = tid & 31;
        const uint32_t ntiles = 1u << (geom.n - K);
        cnt = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
        nchunks = 1u << (K - geom.L);
        chunk_bytes = (1u << geom.L) * (uint32_t)sizeof(float2);
        const uint32_t mine = tid < nchunks ? (nchunks - tid + nthr - 1) / nthr : 0u;
        warp_bytes = __reduce_add_sync(0xffffffffu, mine) * chunk_bytes;
        if (tid == 0) {
            for (int b = 0; b < NBUF; ++b) mbar_init(&full[b], nthr / 32);
            fence_mbar_init();
        }
        my_off = tid < nchunks ? chunk_offset(geom, tid) : 0ull;
        // with 6 register slots a tile has up to twice as many runs as threads
        my_off2 = tid + nthr < nchunks ? chunk_offset(geom, tid + nthr) : 0ull;
        rmask = 0;
        for (int r = 0; r < geom.nrest; ++r) rmask |= 1ull << geom.rest[r];
        tstride = tile_base(geom, gridDim.x);
        lbase = cbase = tile_base(geom, blockIdx.x);
        __syncthreads();
        for (uint32_t i = 0; i < (NBUF > 1 ? NBUF - 1 : 1) && i < cnt; ++i) issue(i);
    }
    __device__ __forceinline__ uint64_t next(uint64_t b) const { return ((b | ~rmask) + tstride) & rmask; }
    __device__ __forceinline__ float2 *slot(uint32_t i) const { return bufs + (size_t)(i % NBUF) * SLOT; }
    __device__ __forceinline__ void issue(uint32_t i) {
        const uint32_t sl = i % NBUF;
        const uint64_t base = lbase;
        lbase = next(lbase);
        if (lane == 0) mbar_arrive_expect_tx(&full[sl], warp_bytes);
        __syncwarp();
        // runs c = tid and tid + threads: nchunks = 2^(K-L) <= 2^(K-5) and threads =
        // 2^(K - register slots), so at most two runs per thread for up to 6 slots
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const uint32_t c = tid + (uint32_t)r * nthr;
            if (c >= nchunks) break;
            float2 *dst = slot(i) + (size_t)c * (chunk_bytes / sizeof(float2));
            const float2 *from = src + base + (r ? my_off2 : my_off);
#ifdef DESV_ROT_CHECK
            if ((reinterpret_cast<uint64_t>(from) & 15u) || (smem_addr(dst) & 15u) || (chunk_bytes & 15u)) {
                atomicOr(&g_dev_status, DESV_DEV_BADPLAN);  // the tile's bounded wait then gives up
                return;
            }
#endif
            bulk_g2s(dst, from, chunk_bytes, &full[sl]);
        }
    }
    // Wait for tile i and, with NBUF >= 2, start the load NBUF-1 tiles ahead
    // (into the slot of tile i-1, whose stages are done: the caller ends every
    // tile with a barrier).  Returns false (for every thread) if a bounded wait
    // gave up.
    __device__ __forceinline__ bool begin(uint32_t i, uint64_t &tb) {
        const bool waited = mbar_wait_bounded(&full[i % NBUF], (i / NBUF) & 1u);
        if (!__syncthreads_and(waited)) return false;
        if (NBUF > 1 && i + NBUF - 1 < cnt) issue(i + NBUF - 1);
        tb = cbase;
        cbase = next(cbase);
        return true;
    }
    // With one slot: the last stage of tile i has read the slot into registers
    // (the caller has passed a barrier), so the load of tile i+1 can overwrite
    // it while the last stage computes and stores to HBM.
    __device__ __forceinline__ void release(uint32_t i) {
        if (NBUF == 1 && i + 1 < cnt) issue(i + 1);
    }
    // after a failed wait: let the loads still in flight land (bounded)
    __device__ __forceinline__ void drain(uint32_t i) {
        for (uint32_t j = i; j < cnt && j < i + NBUF; ++j) mbar_wait_bounded(&full[j % NBUF], (j / NBUF) & 1u, 1u << 16);
    }
};

}  // namespace desv
