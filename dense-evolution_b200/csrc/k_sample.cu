// Finite-shot sampling of computational-basis outcomes on the GPU.
//
// Replaces the host path of the reference's sample_counts
// (utils/measurement.py:17-68: |a|^2 on the host, rng.choice with the
// probabilities, i.e. cumsum + searchsorted of rng.random(n_shots)).  Here the
// cumulative distribution never leaves the device:
//   prepare: FP64 sums of |a_i|^2 over blocks of 2^12 amplitudes (one CTA per
//            block, fixed reduction order), then one CTA turns them into an
//            inclusive prefix (fixed order) -- the CDF at block granularity;
//   pick:    one warp per shot finds the first block whose prefix exceeds
//            u * total (binary search), then scans that block 32 amplitudes at
//            a time with a warp prefix sum and takes the first amplitude whose
//            running sum exceeds the target -- searchsorted(cdf, u, 'right').
// The uniforms come from the caller (the host draws them exactly as
// rng.choice does), so a seeded generator reproduces the reference's draws;
// only a target within rounding (~1e-16 relative) of a CDF step could land on
// the neighbouring outcome.
#include "desv_common.cuh"

namespace desv {

constexpr int SAMPLE_BLOCK_BITS = 12;
constexpr int SAMPLE_THREADS = 256;

template <typename T> __global__ void k_block_sums(const T *sv, uint64_t nblk, int bb, double *bs) {
    __shared__ double sh[SAMPLE_THREADS / 32];
    for (uint64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
        const uint64_t base = b << bb;
        const uint32_t len = 1u << bb;
        double s = 0.0;
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
            const T a = sv[base + i];
            s += (double)a.x * (double)a.x + (double)a.y * (double)a.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < SAMPLE_THREADS / 32; ++w) t += sh[w];
            bs[b] = t;
        }
        __syncthreads();
    }
}

// inclusive prefix of bs[0..nblk) into pre[] by one CTA: thread t owns a
// contiguous chunk; chunk totals are scanned by thread 0 (fixed order)
__global__ void k_block_prefix(const double *bs, uint64_t nblk, double *pre, double *total_out) {
    __shared__ double tot[SAMPLE_THREADS];
    const uint64_t chunk = (nblk + blockDim.x - 1) / blockDim.x;
    const uint64_t b0 = threadIdx.x * chunk, b1 = b0 + chunk < nblk ? b0 + chunk : nblk;
    double s = 0.0;
    for (uint64_t b = b0; b < b1; ++b) s += bs[b];
    tot[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double run = 0.0;
        for (unsigned t = 0; t < blockDim.x; ++t) {
            const double v = tot[t];
            tot[t] = run;
            run += v;
        }
        if (total_out) *total_out = run;
    }
    __syncthreads();
    double run = tot[threadIdx.x];
    for (uint64_t b = b0; b < b1; ++b) {
        run += bs[b];
        pre[b] = run;
    }
}

template <typename T>
__global__ void k_pick(const T *sv, const double *pre, uint64_t nblk, int bb, const double *u, int64_t nshots,
                       int64_t *out) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const double total = pre[nblk - 1];
    const uint32_t len = 1u << bb;
    for (int64_t s = gw; s < nshots; s += nw) {
        const double t = u[s] * total;
        // first block with pre[b] > t (the last block if rounding put t at the top)
        uint64_t lo = 0, hi = nblk - 1;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (pre[mid] > t) hi = mid;
            else lo = mid + 1;
        }
        const uint64_t b = lo;
        double run = b ? pre[b - 1] : 0.0;
        const uint64_t base = b << bb;
        int64_t pick = -1, lastnz = -1;
        for (uint32_t i0 = 0; i0 < len; i0 += 32) {
            double p = 0.0;
            if (i0 + lane < len) {
                const T a = sv[base + i0 + lane];
                p = (double)a.x * (double)a.x + (double)a.y * (double)a.y;
            }
            double ps = p;  // inclusive warp prefix
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double v = __shfl_up_sync(0xffffffffu, ps, o);
                if (lane >= o) ps += v;
            }
            const unsigned nz = __ballot_sync(0xffffffffu, p > 0.0);
            if (nz) lastnz = (int64_t)(base + i0) + (31 - __clz(nz));
            const unsigned hit = __ballot_sync(0xffffffffu, p > 0.0 && run + ps > t);
            if (hit) {
                pick = (int64_t)(base + i0) + (__ffs(hit) - 1);
                break;
            }
            run += __shfl_sync(0xffffffffu, ps, 31);
        }
        if (pick < 0) pick = lastnz >= 0 ? lastnz : (int64_t)base;
        if (lane == 0) out[s] = pick;
    }
}

static uint64_t sample_blocks(int n, int *bb) {
    *bb = n < SAMPLE_BLOCK_BITS ? n : SAMPLE_BLOCK_BITS;
    return 1ull << (n - *bb);
}

}  // namespace desv

using namespace desv;

extern "C" size_t desv_sample_scratch_bytes(int n) {
    if (n < 1 || n > 34) return 0;
    int bb;
    return 2 * sample_blocks(n, &bb) * sizeof(double) + 256;
}

extern "C" int desv_sample_prepare(const void *sv, int n, int dtype, void *scratch, size_t scratch_bytes,
                                   double *total_dev, void *stream) {
    if (!sv || !scratch || n < 1 || n > 34) return fail(DESV_EINVAL, "sample prepare: bad state or scratch");
    if (dtype != DESV_C64 && dtype != DESV_C128) return fail(DESV_EINVAL, "sample prepare: bad dtype");
    if (scratch_bytes < desv_sample_scratch_bytes(n)) return fail(DESV_EINVAL, "sample prepare: scratch too small");
    int bb;
    const uint64_t nblk = sample_blocks(n, &bb);
    double *bs = static_cast<double *>(scratch), *pre = bs + nblk;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = (int)(nblk < (uint64_t)sm_count() * 8 ? nblk : (uint64_t)sm_count() * 8);
    if (dtype == DESV_C64)
        k_block_sums<float2><<<grid, SAMPLE_THREADS, 0, st>>>(static_cast<const float2 *>(sv), nblk, bb, bs);
    else
        k_block_sums<double2><<<grid, SAMPLE_THREADS, 0, st>>>(static_cast<const double2 *>(sv), nblk, bb, bs);
    k_block_prefix<<<1, SAMPLE_THREADS, 0, st>>>(bs, nblk, pre, total_dev);
    return check_launch("sample prepare");
}

extern "C" int desv_sample_pick(const void *sv, int n, int dtype, const void *scratch, size_t scratch_bytes,
                                const double *u_dev, int64_t nshots, int64_t *out_dev, void *stream) {
    if (!sv || !scratch || !u_dev || !out_dev || n < 1 || n > 34 || nshots < 0)
        return fail(DESV_EINVAL, "sample pick: bad arguments");
    if (dtype != DESV_C64 && dtype != DESV_C128) return fail(DESV_EINVAL, "sample pick: bad dtype");
    if (scratch_bytes < desv_sample_scratch_bytes(n)) return fail(DESV_EINVAL, "sample pick: scratch too small");
    if (nshots == 0) return DESV_OK;
    int bb;
    const uint64_t nblk = sample_blocks(n, &bb);
    const double *pre = static_cast<const double *>(scratch) + nblk;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t warps = nshots;
    const int64_t blocks = (warps * 32 + SAMPLE_THREADS - 1) / SAMPLE_THREADS;
    const int grid = (int)(blocks < (int64_t)sm_count() * 16 ? blocks : (int64_t)sm_count() * 16);
    if (dtype == DESV_C64)
        k_pick<float2><<<grid, SAMPLE_THREADS, 0, st>>>(static_cast<const float2 *>(sv), pre, nblk, bb, u_dev, nshots,
                                                         out_dev);
    else
        k_pick<double2><<<grid, SAMPLE_THREADS, 0, st>>>(static_cast<const double2 *>(sv), pre, nblk, bb, u_dev,
                                                          nshots, out_dev);
    return check_launch("sample pick");
}
