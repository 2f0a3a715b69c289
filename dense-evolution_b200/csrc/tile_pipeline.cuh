// Tile geometry and the persistent bulk-copy pipeline shared by the fused
// gate kernel, the Pauli kernels and the adjoint kernel.
//
// A tile is 2^K amplitudes: the L lowest index bits (contiguous runs of 2^L
// amplitudes in HBM) plus K-L arbitrary higher bits `high[]`.  In shared
// memory a tile is stored densely by its tile-local index j: bits 0..L-1 of j
// are index bits 0..L-1, bit L+i of j is index bit high[i].  Tiles are
// enumerated by the remaining n-K index bits `rest[]` (ascending), so
// consecutive tile ids are neighbours in memory.
//
// Each CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ... through a ring
// of NBUF shared-memory slots.  Every thread issues cp.async.bulk copies for
// its share of the 2^L-runs (loads complete on the slot's mbarrier, stores go
// into per-thread bulk groups); every thread runs the body on the slot.  Loads
// run D = NBUF-2 tiles ahead when the body's results are stored (one slot is
// still draining its store), NBUF-1 tiles ahead otherwise.
#pragma once

#include "desv_common.cuh"

namespace desv {

struct TileGeom {
    int n, K, L, nrest;
    uint8_t high[16];
    uint8_t rest[40];
};

__device__ __forceinline__ uint64_t tile_local_to_global(const TileGeom &g, uint32_t j) {
    uint64_t x = j & ((1u << g.L) - 1u);
    const int nh = g.K - g.L;
#pragma unroll 1
    for (int i = 0; i < nh; ++i)
        if ((j >> (g.L + i)) & 1u) x |= 1ull << g.high[i];
    return x;
}

__device__ __forceinline__ uint64_t tile_base(const TileGeom &g, uint64_t t) {
    uint64_t b = 0;
#pragma unroll 1
    for (int i = 0; i < g.nrest; ++i)
        if ((t >> i) & 1ull) b |= 1ull << g.rest[i];
    return b;
}

__device__ __forceinline__ uint64_t chunk_offset(const TileGeom &g, uint32_t c) {
    uint64_t o = 0;
    const int nh = g.K - g.L;
#pragma unroll 1
    for (int i = 0; i < nh; ++i)
        if ((c >> i) & 1u) o |= 1ull << g.high[i];
    return o;
}

// Shared-memory header of a pipelined kernel: 128 bytes of mbarriers, then
// the chunk table ctab[c] = global offset of the tile's 2^L-run c (built when
// the tile has at most PIPE_CTAB_MAX runs), then the NBUF x NARR tile slots.
constexpr uint32_t PIPE_CTAB_MAX = 256;
constexpr size_t PIPE_HDR_BYTES = 128 + 8 * PIPE_CTAB_MAX;

__device__ __forceinline__ const uint64_t *pipe_ctab(const unsigned char *smem) {
    return reinterpret_cast<const uint64_t *>(smem + 128);
}

// tile-local index j -> global offset inside the tile (table lookup; valid when
// the tile has at most PIPE_CTAB_MAX runs)
__device__ __forceinline__ uint64_t tl2g(const uint64_t *ctab, int L, uint32_t j) {
    return ctab[j >> L] | (uint64_t)(j & ((1u << L) - 1u));
}

// global offset of tile-local bit position p (a single set bit)
__device__ __forceinline__ uint64_t tl_bit(const uint64_t *ctab, int L, uint32_t p) {
    return p < (uint32_t)L ? (1ull << p) : ctab[1u << (p - L)];
}

// Arrays taking part in a pipelined sweep.  Array 0 is always loaded.
template <typename T, int NARR> struct PipeArrays {
    T *ptr[NARR];
    bool load[NARR];
    bool store[NARR];
};

// Run `body(smem_slot_arrays, tile_base, tile_id)` over every tile.  Returns
// false (after draining in-flight copies) if a bounded wait gave up.  SLOT is
// the ring slot size in elements per array: the tile's 2^K by default, more
// when the body re-lays the tile out in a padded layout inside its slot.
//
// Every thread issues the bulk copies of the 2^L-runs c = threadIdx.x,
// threadIdx.x + blockDim.x, ...; each warp announces its own byte count on the
// slot's mbarrier (initialised with one arrival per warp), so no warp
// serialises the copy issue of the whole tile.
template <typename T, int K, int NBUF, int NARR, uint32_t SLOT = (1u << K), class Body>
__device__ bool run_tiles(const TileGeom &g, const PipeArrays<T, NARR> &A, Body &body, unsigned char *smem) {
    static_assert(SLOT >= (1u << K), "a ring slot holds at least one tile");
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *ctab = reinterpret_cast<uint64_t *>(smem + 128);
    T *bufs = reinterpret_cast<T *>(smem + PIPE_HDR_BYTES);
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31;
    const uint32_t ntiles = 1u << (g.n - K);
    const uint32_t cnt = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const uint32_t chunk = 1u << g.L, nchunks = 1u << (K - g.L);
    const uint32_t chunk_bytes = chunk * sizeof(T);

    bool any_store = false;
    uint32_t nload = 0;
#pragma unroll
    for (int a = 0; a < NARR; ++a) {
        any_store |= A.store[a];
        nload += A.load[a] ? 1u : 0u;
    }
    const uint32_t D = any_store ? (NBUF - 2) : (NBUF - 1);
    // bytes this warp's copies deliver per tile
    const uint32_t mine = tid < nchunks ? (nchunks - tid + nthr - 1) / nthr : 0u;
    const uint32_t warp_bytes = __reduce_add_sync(0xffffffffu, mine) * chunk_bytes * nload;

    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&full[b], nthr / 32);
        fence_mbar_init();
    }
    // geometry, once per CTA: the chunk table, this thread's run offsets and the
    // tile bases.  Tile t's base deposits the bits of t into the rest bits;
    // consecutive tiles of this CTA differ by a constant deposited stride, added
    // with carries running through the non-rest bits ((b | ~M) + s) & M.
    if (nchunks <= PIPE_CTAB_MAX)
        for (uint32_t c = tid; c < nchunks; c += nthr) ctab[c] = chunk_offset(g, c);
    const uint64_t my_off = tid < nchunks ? chunk_offset(g, tid) : 0ull;
    uint64_t rmask = 0;
#pragma unroll 1
    for (int r = 0; r < g.nrest; ++r) rmask |= 1ull << g.rest[r];
    const uint64_t tstride = tile_base(g, gridDim.x);
    const uint64_t base0 = tile_base(g, blockIdx.x);
    __syncthreads();
    uint64_t lbase = base0;  // base of the next tile to load
    uint64_t cbase = base0;  // base of the next tile to process
    auto next_base = [&](uint64_t b) { return ((b | ~rmask) + tstride) & rmask; };

    auto slot_ptr = [&](uint32_t slot, int a) { return bufs + (size_t)(slot * NARR + a) * SLOT; };
    auto issue_load = [&](uint32_t i) {
        const uint32_t slot = i % NBUF;
        const uint64_t base = lbase;
        lbase = next_base(lbase);
        if (lane == 0) mbar_arrive_expect_tx(&full[slot], warp_bytes);
        __syncwarp();
        for (uint32_t c = tid; c < nchunks; c += nthr) {
            const uint64_t off = base + (c == tid ? my_off : chunk_offset(g, c));
#pragma unroll
            for (int a = 0; a < NARR; ++a)
                if (A.load[a]) bulk_g2s(slot_ptr(slot, a) + (size_t)c * chunk, A.ptr[a] + off, chunk_bytes, &full[slot]);
        }
    };

    for (uint32_t i = 0; i < D && i < cnt; ++i) issue_load(i);

    bool ok = true;
    uint32_t i = 0;
    for (; i < cnt; ++i) {
        const uint32_t slot = i % NBUF;
        const bool waited = mbar_wait_bounded(&full[slot], (i / NBUF) & 1u);
        if (any_store) bulk_wait_read<1>();  // this thread's stores older than the last group have left smem
        if (!__syncthreads_and(waited)) { ok = false; break; }
        if (i + D < cnt) issue_load(i + D);  // into the slot of tile i+D-NBUF (drained above)
        T *sp[NARR];
#pragma unroll
        for (int a = 0; a < NARR; ++a) sp[a] = slot_ptr(slot, a);
        const uint64_t tix = blockIdx.x + (uint64_t)i * gridDim.x;
        const uint64_t base = cbase;
        cbase = next_base(cbase);
        body(sp, base, tix);
        if (any_store) {
            fence_proxy_async_smem();
            __syncthreads();
            for (uint32_t c = tid; c < nchunks; c += nthr) {
                const uint64_t off = base + (c == tid ? my_off : chunk_offset(g, c));
#pragma unroll
                for (int a = 0; a < NARR; ++a)
                    if (A.store[a]) bulk_s2g(A.ptr[a] + off, sp[a] + (size_t)c * chunk, chunk_bytes);
            }
            bulk_commit();
        } else {
            __syncthreads();
        }
    }
    if (!ok) {
        // drain loads still in flight (bounded) so no copy targets freed shared memory
        for (uint32_t j = i; j < cnt && j < i + D + 1; ++j) mbar_wait_bounded(&full[j % NBUF], (j / NBUF) & 1u, 1u << 16);
    }
    if (any_store) bulk_wait_all();
    return ok;
}

#ifndef __CUDACC_RTC__
// host-side geometry builder
inline bool make_geom(TileGeom &g, int n, int K, int L, const uint8_t *high) {
    if (K > n || L < 1 || L > K || n > 34) return false;
    g.n = n; g.K = K; g.L = L;
    uint64_t tmask = (1ull << L) - 1ull;
    for (int i = 0; i < K - L; ++i) {
        if (high[i] < L || high[i] >= n) return false;
        if (i && high[i] <= high[i - 1]) return false;
        g.high[i] = high[i];
        tmask |= 1ull << high[i];
    }
    int r = 0;
    for (int b = 0; b < n; ++b)
        if (!((tmask >> b) & 1ull)) g.rest[r++] = (uint8_t)b;
    g.nrest = r;
    return r == n - K;
}
#endif

}  // namespace desv
