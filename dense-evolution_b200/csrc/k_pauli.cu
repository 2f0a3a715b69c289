// Fused Pauli-sum kernels: <psi|H|psi> and H|psi> for H = sum_k c_k P_k.
//
// The reference applies one term at a time, each as >= 4 full passes
// (arange, XOR, a per-qubit coefficient array, a gather -- physics/
// observables.py:63-94,152-186,250-308).  Here the host groups terms into
// tile passes: every term whose flip mask lies inside a pass's tile bits is
// evaluated from the shared-memory tile, so all terms of a pass cost one read
// of psi.  (P_k psi)[i] = psi[i ^ x_k] * c_k * (-1)^popcount((i ^ x_k) & z_k),
// where c_k already carries the i^(#Y) factor.  The per-amplitude term sum and
// the expectation are accumulated in FP64 (only H psi is stored in the state's
// precision).
#include "desv_common.cuh"
#include "tile_pipeline.cuh"

namespace desv {

constexpr int PAULI_THREADS = 256;
constexpr int PAULI_MAX_ROWS_X = 64;  // CTAs per state of a rows pass (partial-sum rows per state and pass)
// an SM holds at most 2048 threads, so the occupancy of a tiled pass can never
// exceed the per-SM grid bound the partial-sum buffers are sized for
static_assert(2048 / PAULI_THREADS <= PAULI_MAX_BLOCKS_PER_SM, "Pauli grid bound");

template <typename T> struct TermTab {
    uint32_t xl[PAULI_MAX_TERMS];
    uint32_t zl[PAULI_MAX_TERMS];
    double2 c[PAULI_MAX_TERMS];
    uint8_t pb[PAULI_MAX_TERMS];
};

__device__ __forceinline__ uint32_t global_to_tile_local(const TileGeom &g, uint64_t m) {
    uint32_t x = (uint32_t)(m & ((1ull << g.L) - 1ull));
    for (int i = 0; i < g.K - g.L; ++i)
        if ((m >> g.high[i]) & 1ull) x |= 1u << (g.L + i);
    return x;
}

// MODE 0: expectation only; 1: matvec overwrite (+ optional expectation); 2: matvec accumulate
template <typename T, int K, int NBUF, int MODE>
__global__ void __launch_bounds__(PAULI_THREADS) k_pauli(const T *psi, T *out, TileGeom g, const desv_pauli_term *terms,
                                                         int nterms, int want_e, double *part, RowStrides rs) {
    extern __shared__ __align__(128) unsigned char smem[];
    // rows: this grid row's state, output, term table and partial sums
    psi += blockIdx.y * rs.amps;
    if (MODE != 0) out += blockIdx.y * rs.amps;
    terms += blockIdx.y * rs.terms;
    part += blockIdx.y * rs.part;
    // only psi travels through the shared-memory ring; H psi is written (MODE 1)
    // or accumulated (MODE 2) straight in HBM, amplitude j of a tile by thread
    // j mod 256, so consecutive threads touch consecutive addresses
    constexpr int NARR = 1;
    TermTab<T> *tab = reinterpret_cast<TermTab<T> *>(smem + PIPE_HDR_BYTES + (size_t)NBUF * NARR * (1u << K) * sizeof(T));
    for (int k = threadIdx.x; k < nterms; k += blockDim.x) {
        const desv_pauli_term tm = terms[k];
        tab->xl[k] = global_to_tile_local(g, tm.xmask);
        tab->zl[k] = global_to_tile_local(g, tm.zmask);
        tab->c[k] = make_double2(tm.cre, tm.cim);
    }
    PipeArrays<T, NARR> A;
    A.ptr[0] = const_cast<T *>(psi);
    A.load[0] = true;
    A.store[0] = false;
    const bool have_ctab = (1u << (K - g.L)) <= PIPE_CTAB_MAX;
    double ere = 0, eim = 0;
    auto body = [=, &ere, &eim](T *const *sp, uint64_t base, uint64_t) {
        const uint64_t *ctab = pipe_ctab(smem);
        // parity of the tile's fixed bits under each term's sign mask
        for (int k = threadIdx.x; k < nterms; k += blockDim.x)
            tab->pb[k] = (uint8_t)(__popcll(base & terms[k].zmask) & 1);
        __syncthreads();
        const T *s = sp[0];
        // R amplitudes per thread at a time, each with its own FP64 accumulator:
        // the term loop then carries R independent FMA chains instead of one
        constexpr int R = 4;
#pragma unroll 1
        for (uint32_t j0 = threadIdx.x; j0 < (1u << K); j0 += PAULI_THREADS * R) {
            double2 v[R], p[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                v[r] = make_double2(0.0, 0.0);
                p[r] = make_double2(0.0, 0.0);
            }
            uint32_t last_x = 0xFFFFFFFFu;
#pragma unroll 2
            for (int k = 0; k < nterms; ++k) {
                const uint32_t xl = tab->xl[k], zl = tab->zl[k];
                const uint32_t pb = tab->pb[k];
                if (xl != last_x) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const uint32_t j = j0 + (uint32_t)r * PAULI_THREADS;
                        if (j < (1u << K)) {
                            const T q = s[j ^ xl];
                            p[r] = make_double2((double)q.x, (double)q.y);
                        }
                    }
                    last_x = xl;
                }
                const double2 c = tab->c[k];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const uint32_t j = j0 + (uint32_t)r * PAULI_THREADS;
                    const bool sg = ((__popc((j ^ xl) & zl) ^ pb) & 1u) != 0;
                    const double2 cs = sg ? make_double2(-c.x, -c.y) : c;
                    v[r] = cfma(cs, p[r], v[r]);
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t j = j0 + (uint32_t)r * PAULI_THREADS;
                if (j >= (1u << K)) continue;
                if (MODE != 0 || want_e) {
                    const T a = s[j];
                    ere += (double)a.x * v[r].x + (double)a.y * v[r].y;
                    eim += (double)a.x * v[r].y - (double)a.y * v[r].x;
                }
                if (MODE != 0) {
                    const uint64_t gi = base + (have_ctab ? tl2g(ctab, g.L, j) : tile_local_to_global(g, j));
                    if (MODE == 1) {
                        out[gi] = mk((decltype(s[0].x))v[r].x, (decltype(s[0].x))v[r].y);
                    } else {
                        T o = out[gi];
                        o.x = (decltype(o.x))((double)o.x + v[r].x);
                        o.y = (decltype(o.y))((double)o.y + v[r].y);
                        out[gi] = o;
                    }
                }
            }
        }
    };
    __syncthreads();
    run_tiles<T, K, NBUF, NARR>(g, A, body, smem);
    if (want_e) {
        __shared__ double sh[32];
        double r = ere;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        double i2 = eim;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) i2 += __shfl_xor_sync(0xffffffffu, i2, o);
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        __syncthreads();
        if (l == 0) sh[w] = r;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int k = 0; k < PAULI_THREADS / 32; ++k) t += sh[k];
            part[2 * blockIdx.x] = t;
        }
        __syncthreads();
        if (l == 0) sh[w] = i2;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int k = 0; k < PAULI_THREADS / 32; ++k) t += sh[k];
            part[2 * blockIdx.x + 1] = t;
        }
    }
}

template <typename T, int K, int NBUF, int MODE>
static int launch_pauli(const T *psi, T *out, const TileGeom &g, const desv_pauli_term *terms, int nterms, int want_e,
                        double *part, int *grid_out, int nrows, const RowStrides &rs, cudaStream_t st) {
    static int bps[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    constexpr int NARR = 1;
    const size_t smem = PIPE_HDR_BYTES + (size_t)NBUF * NARR * (1u << K) * sizeof(T) + sizeof(TermTab<T>);
    if (bps[dev & 63] == 0) {
        cudaFuncSetAttribute(k_pauli<T, K, NBUF, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_pauli<T, K, NBUF, MODE>, PAULI_THREADS, smem);
        bps[dev & 63] = b < 1 ? 1 : b > PAULI_MAX_BLOCKS_PER_SM ? PAULI_MAX_BLOCKS_PER_SM : b;
    }
    const uint64_t ntiles = 1ull << (g.n - K);
    const uint64_t cap = (uint64_t)sm_count() * bps[dev & 63];
    int grid = (int)(ntiles < cap ? ntiles : cap);
    if (rs.amps != 0) {  // a rows launch (single-state launches pass zero strides)
        grid = rows_grid_x(ntiles, cap, nrows);
        if (grid > PAULI_MAX_ROWS_X) grid = PAULI_MAX_ROWS_X;
    }
    *grid_out = grid;
    k_pauli<T, K, NBUF, MODE><<<dim3(grid, nrows), PAULI_THREADS, smem, st>>>(psi, out, g, terms, nterms, want_e, part,
                                                                             rs);
    return check_launch("pauli pass");
}

// Terms whose flip mask spans more high bits than a tile holds: every thread
// reads psi[i] and psi[i ^ x] straight from global memory (i ^ x keeps
// consecutive i contiguous, so the loads stay coalesced).
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_pauli_direct(const T *psi, T *out, uint64_t dim,
                                                      const desv_pauli_term *terms, int nterms, int want_e,
                                                      double *part, RowStrides rs) {
    psi += blockIdx.y * rs.amps;
    if (MODE != 0) out += blockIdx.y * rs.amps;
    terms += blockIdx.y * rs.terms;
    part += blockIdx.y * rs.part;
    double ere = 0, eim = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        for (int k = 0; k < nterms; ++k) {
            const desv_pauli_term tm = terms[k];
            const uint64_t src = i ^ tm.xmask;
            const T q = psi[src];
            const double2 p = make_double2((double)q.x, (double)q.y);
            const double2 c = make_double2(tm.cre, tm.cim);
            v = (__popcll(src & tm.zmask) & 1) ? cfma(cneg(c), p, v) : cfma(c, p, v);
        }
        if (want_e) {
            const T a = psi[i];
            ere += (double)a.x * v.x + (double)a.y * v.y;
            eim += (double)a.x * v.y - (double)a.y * v.x;
        }
        if (MODE == 1) out[i] = mk((decltype(psi[0].x))v.x, (decltype(psi[0].x))v.y);
        if (MODE == 2) {
            T o = out[i];
            o.x = (decltype(o.x))((double)o.x + v.x);
            o.y = (decltype(o.y))((double)o.y + v.y);
            out[i] = o;
        }
    }
    if (want_e) {
        __shared__ double sh[32];
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ere += __shfl_xor_sync(0xffffffffu, ere, o);
            eim += __shfl_xor_sync(0xffffffffu, eim, o);
        }
        if (l == 0) sh[w] = ere;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
            part[2 * blockIdx.x] = t;
        }
        __syncthreads();
        if (l == 0) sh[w] = eim;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
            part[2 * blockIdx.x + 1] = t;
        }
    }
}

int pauli_direct_rows(const void *psi, void *out, int dtype, int mode, int n, const desv_pauli_term *terms,
                      int nterms, int want_e, double *part, int *grid_out, int nrows, const RowStrides &rs,
                      cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    uint64_t b = (dim + 255) / 256;
    const uint64_t cap = (uint64_t)sm_count() * PAULI_MAX_BLOCKS_PER_SM;
    int grid = (int)(b < cap ? b : cap);
    if (rs.amps != 0) {  // a rows launch (single-state launches pass zero strides)
        grid = rows_grid_x(b, cap, nrows);
        if (grid > PAULI_MAX_ROWS_X) grid = PAULI_MAX_ROWS_X;
    }
    *grid_out = grid;
#define DESV_PD(T, M)                                                                                             \
    k_pauli_direct<T, M><<<dim3(grid, nrows), 256, 0, st>>>(static_cast<const T *>(psi), static_cast<T *>(out), dim, \
                                                            terms, nterms, want_e, part, rs)
    if (dtype == DESV_C64) {
        if (mode == 0) DESV_PD(float2, 0);
        else if (mode == 1) DESV_PD(float2, 1);
        else DESV_PD(float2, 2);
    } else {
        if (mode == 0) DESV_PD(double2, 0);
        else if (mode == 1) DESV_PD(double2, 1);
        else DESV_PD(double2, 2);
    }
#undef DESV_PD
    return check_launch("pauli direct pass");
}

int pauli_direct(const void *psi, void *out, int dtype, int mode, int n, const desv_pauli_term *terms, int nterms,
                 int want_e, double *part, int *grid_out, cudaStream_t st) {
    return pauli_direct_rows(psi, out, dtype, mode, n, terms, nterms, want_e, part, grid_out, 1,
                             RowStrides{0, 0, 0, 0}, st);
}

template <typename T, int K, int MODE>
static int pauli_k(const T *p, T *o, const TileGeom &g, const desv_pauli_term *terms, int nterms, int want_e,
                   double *part, int *grid_out, int nrows, const RowStrides &rs, cudaStream_t st) {
    return launch_pauli<T, K, 4, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
}

template <typename T, int MODE>
static int pauli_dispatch(const T *p, T *o, const TileGeom &g, const desv_pauli_term *terms, int nterms, int want_e,
                          double *part, int *grid_out, int nrows, const RowStrides &rs, cudaStream_t st, int kmax) {
    if (g.K > kmax) return fail(DESV_EINVAL, "pauli pass: tile_bits too large for this precision");
    switch (g.K) {
        case 1: return pauli_k<T, 1, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 2: return pauli_k<T, 2, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 3: return pauli_k<T, 3, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 4: return pauli_k<T, 4, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 5: return pauli_k<T, 5, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 6: return pauli_k<T, 6, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 7: return pauli_k<T, 7, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 8: return pauli_k<T, 8, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 9: return pauli_k<T, 9, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        case 10: return pauli_k<T, 10, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
        default: return pauli_k<T, 11, MODE>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st);
    }
}

// Tile of up to 2^11 amplitudes for complex64 and 2^10 for complex128 (16 KB).
// nrows states (rs: strides) in one launch; nrows = 1, rs = {} for one state.
int pauli_pass_rows(const void *psi, void *out, int dtype, int mode, const TileGeom &g, const desv_pauli_term *terms,
                    int nterms, int want_e, double *part, int *grid_out, int nrows, const RowStrides &rs,
                    cudaStream_t st) {
    if (nterms > PAULI_MAX_TERMS) return fail(DESV_EINVAL, "pauli pass: more than 512 terms in one pass");
    if (g.K < 5 && g.K != g.n) return fail(DESV_EINVAL, "pauli pass: tile smaller than 2^5 must cover the state");
    if (dtype == DESV_C64) {
        const float2 *p = static_cast<const float2 *>(psi);
        float2 *o = static_cast<float2 *>(out);
        if (mode == 0) return pauli_dispatch<float2, 0>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st, 11);
        if (mode == 1) return pauli_dispatch<float2, 1>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st, 11);
        return pauli_dispatch<float2, 2>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st, 11);
    }
    const double2 *p = static_cast<const double2 *>(psi);
    double2 *o = static_cast<double2 *>(out);
    if (mode == 0) return pauli_dispatch<double2, 0>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st, 10);
    if (mode == 1) return pauli_dispatch<double2, 1>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st, 10);
    return pauli_dispatch<double2, 2>(p, o, g, terms, nterms, want_e, part, grid_out, nrows, rs, st, 10);
}

int pauli_pass(const void *psi, void *out, int dtype, int mode, const TileGeom &g, const desv_pauli_term *terms,
               int nterms, int want_e, double *part, int *grid_out, cudaStream_t st) {
    return pauli_pass_rows(psi, out, dtype, mode, g, terms, nterms, want_e, part, grid_out, 1, RowStrides{0, 0, 0, 0},
                           st);
}

}  // namespace desv
