// Element-wise kernels, single-gate kernels and FP64 reductions.
//
// The single-gate kernels serve the one-gate API (apply_gate_1q/_2q, apply_cx,
// apply_rx ... of backends/statevector.py:167-268) and states too small for a
// fused tile; circuits go through the fused passes.
#include "desv_common.cuh"

namespace desv {

static int grid_for(uint64_t work, int threads, int per_sm = 8) {
    uint64_t b = (work + threads - 1) / threads;
    uint64_t cap = (uint64_t)sm_count() * per_sm;
    if (b > cap) b = cap;
    return (int)(b ? b : 1);
}

// ------------------------------------------------------------------ element-wise
template <typename T> __global__ void k_set_one(T *sv, uint64_t index) {
    T one;
    one.x = 1;
    one.y = 0;
    sv[index] = one;
}

template <typename T> __global__ void k_scale(T *sv, uint64_t dim, T f) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x)
        sv[i] = cmul(f, sv[i]);
}

template <typename T> __global__ void k_probs(const T *sv, uint64_t dim, double *out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
        const T a = sv[i];
        out[i] = (double)a.x * (double)a.x + (double)a.y * (double)a.y;
    }
}

template <typename T> __global__ void k_collapse(T *sv, uint64_t dim, int bit, int outcome, double scale) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
        T a = sv[i];
        if ((int)((i >> bit) & 1ull) != outcome) {
            a.x = 0;
            a.y = 0;
        } else {
            a.x = (decltype(a.x))((double)a.x * scale);
            a.y = (decltype(a.y))((double)a.y * scale);
        }
        sv[i] = a;
    }
}

// ------------------------------------------------------------------ single gates
template <typename T>
__global__ void k_gate1(T *sv, uint64_t npairs, int t, uint64_t cmask, uint64_t cval, T m00, T m01, T m10, T m11) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < npairs; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = insert0(p, t);
        if ((i0 & cmask) != cval) continue;
        const uint64_t i1 = i0 | (1ull << t);
        const T x0 = sv[i0], x1 = sv[i1];
        sv[i0] = cfma(m01, x1, cmul(m00, x0));
        sv[i1] = cfma(m11, x1, cmul(m10, x0));
    }
}

template <typename T> struct Mat4 { T m[16]; };

template <typename T>
__global__ void k_gate2(T *sv, uint64_t nquads, int t0, int t1, uint64_t cmask, uint64_t cval, Mat4<T> M) {
    const int lo = t0 < t1 ? t0 : t1, hi = t0 < t1 ? t1 : t0;
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < nquads; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i00 = insert0(insert0(p, lo), hi);
        if ((i00 & cmask) != cval) continue;
        const uint64_t idx[4] = {i00, i00 | (1ull << t0), i00 | (1ull << t1), i00 | (1ull << t0) | (1ull << t1)};
        T v[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = sv[idx[c]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            T o = cmul(M.m[4 * r], v[0]);
#pragma unroll
            for (int c = 1; c < 4; ++c) o = cfma(M.m[4 * r + c], v[c], o);
            sv[idx[r]] = o;
        }
    }
}

// ------------------------------------------------------------------ reductions
constexpr int RED_THREADS = 256;
constexpr int RED_MAX_BLOCKS = 2048;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum of `v`; result valid in thread 0
__device__ __forceinline__ double block_sum(double v, double *sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0;
    if (w == 0) {
        r = l < (int)(blockDim.x >> 5) ? sh[l] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// mode 0: sum |a|^2 ; mode 1: sum conj(a) b (2 outputs)
template <typename T> __global__ void k_dot_partial(const T *a, const T *b, uint64_t dim, int mode, double *part) {
    __shared__ double sh[32];
    double re = 0, im = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
        const T x = a[i];
        if (mode == 0) {
            re += (double)x.x * (double)x.x + (double)x.y * (double)x.y;
        } else {
            const T y = b[i];
            re += (double)x.x * (double)y.x + (double)x.y * (double)y.y;
            im += (double)x.x * (double)y.y - (double)x.y * (double)y.x;
        }
    }
    re = block_sum(re, sh);
    if (threadIdx.x == 0) part[2 * blockIdx.x] = re;
    im = block_sum(im, sh);
    if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = im;
}

// out[c] = sum over `rows` partial rows of part[row * stride + c], fixed order
__global__ void k_sum_rows(const double *part, int rows, int stride, int ncols, double *out) {
    __shared__ double sh[32];
    for (int c = 0; c < ncols; ++c) {
        double v = 0;
        for (int r = threadIdx.x; r < rows; r += blockDim.x) v += part[(size_t)r * stride + c];
        v = block_sum(v, sh);
        if (threadIdx.x == 0) out[c] = v;
    }
}

// Per-bit marginals sum_{i: bit b of i set} |a_i|^2 for every bit b < n, plus
// the total, as one row of n + 1 partial sums per CTA.  From 512 amplitudes on,
// each warp walks groups of 16 x 32 consecutive amplitudes: the lane is index
// bits 0..4 (fixed per thread, folded in at the end from the thread's total),
// u = bits 5..8 inside the group (sums over the eight u with the bit set), and
// the bits above are fixed per group (the group sum is added to each set bit).
// About seven FP64 operations per amplitude instead of one per bit.
template <typename T> __global__ void k_marg_partial(const T *a, uint64_t dim, int n, double *part) {
    __shared__ double sh[32];
    double acc[35];
#pragma unroll
    for (int b = 0; b < 35; ++b) acc[b] = 0;
    if (dim >= 512) {
        const int lane = threadIdx.x & 31;
        const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
        const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
        for (uint64_t grp = warp; grp < (dim >> 9); grp += nwarps) {
            const uint64_t base = grp << 9;
            double p[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const T x = a[base + ((uint64_t)u << 5) + lane];
                p[u] = (double)x.x * (double)x.x + (double)x.y * (double)x.y;
            }
            double h[4];  // h[k] = sum over u with bit k of u set
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                double t = 0;
#pragma unroll
                for (int u = 0; u < 16; ++u)
                    if ((u >> k) & 1) t += p[u];
                h[k] = t;
            }
            double sgrp = 0;
#pragma unroll
            for (int u = 0; u < 16; ++u) sgrp += p[u];
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[5 + k] += h[k];
            acc[34] += sgrp;
#pragma unroll
            for (int b = 9; b < 34; ++b)
                if ((base >> b) & 1ull) acc[b] += sgrp;
        }
#pragma unroll
        for (int b = 0; b < 5; ++b) acc[b] = ((lane >> b) & 1) ? acc[34] : 0.0;
    } else {
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim;
             i += (uint64_t)gridDim.x * blockDim.x) {
            const T x = a[i];
            const double p = (double)x.x * (double)x.x + (double)x.y * (double)x.y;
            acc[34] += p;
#pragma unroll
            for (int b = 0; b < 9; ++b)
                if ((i >> b) & 1ull) acc[b] += p;
        }
    }
    // unrolled with compile-time indices so acc[] stays in registers
#pragma unroll
    for (int b = 0; b < 34; ++b) {
        if (b >= n) break;
        const double v = block_sum(acc[b], sh);
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * (n + 1) + b] = v;
    }
    const double v = block_sum(acc[34], sh);
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * (n + 1) + n] = v;
}

// ------------------------------------------------------------------ host launchers
template <typename T> static T to_c(const double *m, int k) {
    T r;
    r.x = (decltype(r.x))m[2 * k];
    r.y = (decltype(r.y))m[2 * k + 1];
    return r;
}

int init_basis(void *sv, int n, int dtype, uint64_t index, cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    const size_t es = dtype == DESV_C64 ? 8 : 16;
    if (cudaMemsetAsync(sv, 0, dim * es, st) != cudaSuccess) return check_launch("init memset");
    if (dtype == DESV_C64) k_set_one<float2><<<1, 1, 0, st>>>(static_cast<float2 *>(sv), index);
    else k_set_one<double2><<<1, 1, 0, st>>>(static_cast<double2 *>(sv), index);
    return check_launch("init basis");
}

int scale(void *sv, int n, int dtype, double re, double im, cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    const int g = grid_for(dim, 256);
    if (dtype == DESV_C64) k_scale<float2><<<g, 256, 0, st>>>(static_cast<float2 *>(sv), dim, make_float2((float)re, (float)im));
    else k_scale<double2><<<g, 256, 0, st>>>(static_cast<double2 *>(sv), dim, make_double2(re, im));
    return check_launch("scale");
}

int probabilities(const void *sv, int n, int dtype, double *out, cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    const int g = grid_for(dim, 256);
    if (dtype == DESV_C64) k_probs<float2><<<g, 256, 0, st>>>(static_cast<const float2 *>(sv), dim, out);
    else k_probs<double2><<<g, 256, 0, st>>>(static_cast<const double2 *>(sv), dim, out);
    return check_launch("probabilities");
}

int collapse(void *sv, int n, int dtype, int bit, int outcome, double s, cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    const int g = grid_for(dim, 256);
    if (dtype == DESV_C64) k_collapse<float2><<<g, 256, 0, st>>>(static_cast<float2 *>(sv), dim, bit, outcome, s);
    else k_collapse<double2><<<g, 256, 0, st>>>(static_cast<double2 *>(sv), dim, bit, outcome, s);
    return check_launch("collapse");
}

int gate(void *sv, int n, int dtype, int nt, const int *tb, uint64_t cmask, uint64_t cval, const double *m,
         cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    if (nt == 1) {
        const uint64_t np = dim >> 1;
        const int g = grid_for(np, 256);
        if (dtype == DESV_C64)
            k_gate1<float2><<<g, 256, 0, st>>>(static_cast<float2 *>(sv), np, tb[0], cmask, cval, to_c<float2>(m, 0),
                                               to_c<float2>(m, 1), to_c<float2>(m, 2), to_c<float2>(m, 3));
        else
            k_gate1<double2><<<g, 256, 0, st>>>(static_cast<double2 *>(sv), np, tb[0], cmask, cval,
                                                to_c<double2>(m, 0), to_c<double2>(m, 1), to_c<double2>(m, 2),
                                                to_c<double2>(m, 3));
        return check_launch("gate 1q");
    }
    const uint64_t nq = dim >> 2;
    const int g = grid_for(nq, 256);
    if (dtype == DESV_C64) {
        Mat4<float2> M;
        for (int k = 0; k < 16; ++k) M.m[k] = to_c<float2>(m, k);
        k_gate2<float2><<<g, 256, 0, st>>>(static_cast<float2 *>(sv), nq, tb[0], tb[1], cmask, cval, M);
    } else {
        Mat4<double2> M;
        for (int k = 0; k < 16; ++k) M.m[k] = to_c<double2>(m, k);
        k_gate2<double2><<<g, 256, 0, st>>>(static_cast<double2 *>(sv), nq, tb[0], tb[1], cmask, cval, M);
    }
    return check_launch("gate 2q");
}

int dot(const void *a, const void *b, int n, int dtype, int mode, double *out, double *scratch, cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    int g = grid_for(dim, RED_THREADS, 4);
    if (g > RED_MAX_BLOCKS) g = RED_MAX_BLOCKS;
    if (dtype == DESV_C64)
        k_dot_partial<float2><<<g, RED_THREADS, 0, st>>>(static_cast<const float2 *>(a), static_cast<const float2 *>(b),
                                                         dim, mode, scratch);
    else
        k_dot_partial<double2><<<g, RED_THREADS, 0, st>>>(static_cast<const double2 *>(a),
                                                          static_cast<const double2 *>(b), dim, mode, scratch);
    k_sum_rows<<<1, RED_THREADS, 0, st>>>(scratch, g, 2, mode == 0 ? 1 : 2, out);
    return check_launch("dot");
}

int marginals(const void *a, int n, int dtype, double *out, double *scratch, cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    int g = grid_for(dim, RED_THREADS, 4);
    if (g > RED_MAX_BLOCKS) g = RED_MAX_BLOCKS;
    if (dtype == DESV_C64)
        k_marg_partial<float2><<<g, RED_THREADS, 0, st>>>(static_cast<const float2 *>(a), dim, n, scratch);
    else
        k_marg_partial<double2><<<g, RED_THREADS, 0, st>>>(static_cast<const double2 *>(a), dim, n, scratch);
    k_sum_rows<<<1, RED_THREADS, 0, st>>>(scratch, g, n + 1, n + 1, out);
    return check_launch("marginals");
}

// reductions: RED_MAX_BLOCKS rows of (n + 1) doubles; Pauli sums: up to 16
// passes x 4096 rows of 2 doubles
size_t scratch_bytes(int n) {
    const size_t red = (size_t)RED_MAX_BLOCKS * (size_t)(n + 2) * sizeof(double);
    const size_t pauli = (size_t)16 * 4096 * 2 * sizeof(double);
    return (red > pauli ? red : pauli) + 4096;
}

}  // namespace desv
