// Fused adjoint backward pass (adjoint-method gradient of E = <psi|H|psi>).
//
// The reference differentiates with jax.grad through lax.scan
// (solvers/autodiff.py:136-166), which stores a residual state per gate.  The
// adjoint method needs two working states instead: phi (the circuit state,
// un-applied gate by gate) and lambda (= H psi, un-applied alongside).  For a
// gate U(theta) with dU/dtheta = G U, the derivative is 2 Re<lambda|G|phi>
// taken just before U is un-applied.  Here one tile pass loads the phi and
// lambda tiles, walks its stretch of the reversed circuit in registers -- GRAD
// ops accumulate the FP64 inner products, inverse-gate ops un-apply -- and
// writes both tiles back: 4 * 2^n amplitudes of HBM traffic per pass for any
// number of gates and gradient terms in it.
#include "desv_common.cuh"
#include "stage_ops.cuh"
#include "grad_ops.cuh"
#include "tile_pipeline.cuh"

namespace desv {

template <typename T, int K, int NBUF>
__global__ void __launch_bounds__(1 << (K - 4), 1) k_adjoint_pass(T *phi, T *lam, TileGeom g, const desv_op *ops,
                                                                int nops, const T *mats, int nparams, double *part,
                                                                RowStrides rs) {
    extern __shared__ __align__(128) unsigned char smem[];
    // rows: this grid row's (phi, lambda) pair, matrix pool and partial sums
    phi += blockIdx.y * rs.amps;
    lam += blockIdx.y * rs.amps;
    mats += blockIdx.y * rs.mats;
    part += blockIdx.y * rs.part;
    constexpr int NW = (1 << (K - 4)) / 32 > 0 ? (1 << (K - 4)) / 32 : 1;
    double *acc = reinterpret_cast<double *>(smem + PIPE_HDR_BYTES + (size_t)NBUF * 2 * (1u << K) * sizeof(T));
    for (int i = threadIdx.x; i < NW * nparams; i += blockDim.x) acc[i] = 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    PipeArrays<T, 2> A;
    A.ptr[0] = phi;
    A.ptr[1] = lam;
    A.load[0] = A.load[1] = true;
    // the last register stage stores both arrays straight to HBM: the ring only
    // serves loads, NBUF-1 tiles ahead
    A.store[0] = A.store[1] = false;
    const int L = g.L;
    auto body = [=](T *const *sp, uint64_t base, uint64_t) {
        T *sphi = sp[0], *slam = sp[1];
        const uint64_t *ctab = pipe_ctab(smem);
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
            T a[16], b[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const uint32_t off = idx + ((j & 1) ? o0 : 0u) + ((j & 2) ? o1 : 0u) + ((j & 4) ? o2 : 0u) +
                                     ((j & 8) ? o3 : 0u);
                a[j] = sphi[off];
                b[j] = slam[off];
            }
            const uint64_t tg = base | tl2g(ctab, L, idx);
#pragma unroll 1
            for (int q = 1; q <= cnt; ++q) {
                const desv_op &op = ops[k + q];
                if (op.kind == DESV_OP_GRAD) {
                    double v = grad_term(a, b, op, mats + op.mat, tg, lane);
                    v = warp_sum_d(v);
                    if (lane == 0) acc[warp * nparams + op.param] += v;
                } else {
                    apply_op_at(a, ops + k + q, mats, tg, lane);
                    apply_op_at(b, ops + k + q, mats, tg, lane);
                }
            }
            k += 1 + cnt;
            if (k >= nops) {
                const uint64_t q0 = tl_bit(ctab, L, g0), q1 = tl_bit(ctab, L, g1), q2 = tl_bit(ctab, L, g2),
                               q3 = tl_bit(ctab, L, g3);
                T *outa = phi + tg, *outb = lam + tg;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const uint64_t off = ((j & 1) ? q0 : 0ull) + ((j & 2) ? q1 : 0ull) + ((j & 4) ? q2 : 0ull) +
                                         ((j & 8) ? q3 : 0ull);
                    outa[off] = a[j];
                    outb[off] = b[j];
                }
            } else {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const uint32_t off = idx + ((j & 1) ? o0 : 0u) + ((j & 2) ? o1 : 0u) + ((j & 4) ? o2 : 0u) +
                                         ((j & 8) ? o3 : 0u);
                    sphi[off] = a[j];
                    slam[off] = b[j];
                }
                __syncthreads();
                // the next bulk load into this slot (async proxy) must follow these writes
                fence_proxy_async_smem();
            }
        }
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

// grad[map[p]] += 2 * sum_r part[r * np + p]   (fixed summation order); one
// block per state of a rows launch (part and grad offset by the row strides).
// One warp per parameter sums its column (lane-strided, then the warp tree);
// then the first record of each distinct map target adds, in record order, the
// sums of every record with that target, so a parameter that several records
// of the pass probe is updated by one thread, exactly as the records come.
constexpr int GRAD_REDUCE_THREADS = 512;
__global__ void __launch_bounds__(GRAD_REDUCE_THREADS)
k_grad_reduce(const double *part, int rows, int np, const int32_t *map, double *grad, int64_t part_stride,
              int64_t grad_stride) {
    extern __shared__ double sh[];  // np sums, then np map entries
    int32_t *mp = reinterpret_cast<int32_t *>(sh + np);
    part += blockIdx.x * part_stride;
    grad += blockIdx.x * grad_stride;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int p = threadIdx.x; p < np; p += blockDim.x) mp[p] = map[p];
    for (int p = w; p < np; p += nw) {
        double v = 0;
        for (int r = l; r < rows; r += 32) v += part[(size_t)r * np + p];
        v = warp_sum_d(v);
        if (l == 0) sh[p] = v;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const int32_t m = mp[p];
        bool first = true;
        for (int q = 0; q < p && first; ++q) first = mp[q] != m;
        if (!first) continue;
        double g = grad[m];
        for (int q = p; q < np; ++q)
            if (mp[q] == m) g += 2.0 * sh[q];
        grad[m] = g;
    }
}
static size_t grad_reduce_smem(int np) { return (size_t)(np > 0 ? np : 1) * (sizeof(double) + sizeof(int32_t)); }

constexpr int ADJ_MAX_PARAMS = 1024;
constexpr int ADJ_MAX_ROWS = 1184;  // partial-sum rows per pass (= grid bound)
constexpr int ADJ_MAX_ROWS_X = 64;  // CTAs per state of a rows pass (partial-sum rows per state)

template <typename T, int K, int NBUF> static size_t adj_smem(int nparams) {
    constexpr int NW = (1 << (K - 4)) / 32 > 0 ? (1 << (K - 4)) / 32 : 1;
    return PIPE_HDR_BYTES + (size_t)NBUF * 2 * (1u << K) * sizeof(T) + (size_t)NW * nparams * sizeof(double);
}

template <typename T, int K, int NBUF>
static int launch_adj(T *phi, T *lam, const TileGeom &g, const desv_op *ops, int nops, const T *mats, int nparams,
                      double *part, int *grid_out, int nrows, RowStrides rs, cudaStream_t st) {
    static bool attr[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smax = adj_smem<T, K, NBUF>(ADJ_MAX_PARAMS);
    if (!attr[dev & 63]) {
        cudaFuncSetAttribute(k_adjoint_pass<T, K, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
        attr[dev & 63] = true;
    }
    // resident CTAs for the shared memory this launch really uses
    int bps = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_adjoint_pass<T, K, NBUF>, 1 << (K - 4),
                                                  adj_smem<T, K, NBUF>(nparams));
    if (bps < 1) bps = 1;
    const uint64_t ntiles = 1ull << (g.n - K);
    uint64_t cap = (uint64_t)sm_count() * bps;
    int grid;
    if (rs.amps != 0) {  // a rows launch (single-state launches pass zero strides)
        grid = rows_grid_x(ntiles, cap, nrows);
        if (grid > ADJ_MAX_ROWS_X) grid = ADJ_MAX_ROWS_X;
        rs.part = (int64_t)grid * nparams;  // each state's partial-sum block: grid x nparams
    } else {
        if (cap > ADJ_MAX_ROWS) cap = ADJ_MAX_ROWS;
        grid = (int)(ntiles < cap ? ntiles : cap);
    }
    *grid_out = grid;
    k_adjoint_pass<T, K, NBUF><<<dim3(grid, nrows), 1 << (K - 4), adj_smem<T, K, NBUF>(nparams), st>>>(
        phi, lam, g, ops, nops, mats, nparams, part, rs);
    return check_launch("adjoint pass");
}

// One adjoint pass over `nrows` (phi, lambda) pairs; rs.amps / rs.mats are the
// state and pool strides (rs.part is set here: grid_out x nparams per state).
int adjoint_pass_rows(void *phi, void *lam, int dtype, const TileGeom &g, const desv_op *ops, int nops,
                      const void *mats, int nparams, double *part, int *grid_out, int nrows, const RowStrides &rs,
                      cudaStream_t st);

int adjoint_pass(void *phi, void *lam, int dtype, const TileGeom &g, const desv_op *ops, int nops, const void *mats,
                 int nparams, double *part, int *grid_out, cudaStream_t st) {
    return adjoint_pass_rows(phi, lam, dtype, g, ops, nops, mats, nparams, part, grid_out, 1, RowStrides{0, 0, 0, 0},
                             st);
}

int adjoint_pass_rows(void *phi, void *lam, int dtype, const TileGeom &g, const desv_op *ops, int nops,
                      const void *mats, int nparams, double *part, int *grid_out, int nrows, const RowStrides &rs,
                      cudaStream_t st) {
    if (nparams < 0 || nparams > ADJ_MAX_PARAMS) return fail(DESV_EINVAL, "adjoint pass: at most 1024 parameters");
    if (dtype == DESV_C64) {
        float2 *p = static_cast<float2 *>(phi), *l = static_cast<float2 *>(lam);
        const float2 *m = static_cast<const float2 *>(mats);
        switch (g.K) {
            case 9: return launch_adj<float2, 9, 4>(p, l, g, ops, nops, m, nparams, part, grid_out, nrows, rs, st);
            case 10: return launch_adj<float2, 10, 4>(p, l, g, ops, nops, m, nparams, part, grid_out, nrows, rs, st);
            case 11: return launch_adj<float2, 11, 3>(p, l, g, ops, nops, m, nparams, part, grid_out, nrows, rs, st);
            default: return fail(DESV_EINVAL, "adjoint pass: complex64 tile_bits must be 9..11");
        }
    }
    double2 *p = static_cast<double2 *>(phi), *l = static_cast<double2 *>(lam);
    const double2 *m = static_cast<const double2 *>(mats);
    switch (g.K) {
        case 9: return launch_adj<double2, 9, 4>(p, l, g, ops, nops, m, nparams, part, grid_out, nrows, rs, st);
        case 10: return launch_adj<double2, 10, 3>(p, l, g, ops, nops, m, nparams, part, grid_out, nrows, rs, st);
        default: return fail(DESV_EINVAL, "adjoint pass: complex128 tile_bits must be 9..10");
    }
}

int grad_reduce(const double *part, int rows, int np, const int32_t *map, double *grad, cudaStream_t st) {
    k_grad_reduce<<<1, GRAD_REDUCE_THREADS, grad_reduce_smem(np), st>>>(part, rows, np, map, grad, 0, 0);
    return check_launch("gradient reduce");
}

// the reduction of a rows adjoint pass: one block per state
int grad_reduce_rows(const double *part, int rows_x, int np, const int32_t *map, double *grad, int nrows,
                     int64_t grad_stride, cudaStream_t st) {
    k_grad_reduce<<<nrows, GRAD_REDUCE_THREADS, grad_reduce_smem(np), st>>>(part, rows_x, np, map, grad,
                                                                       (int64_t)rows_x * np, grad_stride);
    return check_launch("gradient reduce (rows)");
}

size_t adjoint_scratch_bytes(int max_params) {
    return (size_t)ADJ_MAX_ROWS * (size_t)(max_params > 0 ? max_params : 1) * sizeof(double) + 4096;
}

}  // namespace desv
