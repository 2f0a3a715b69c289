// Bit-reversal permutation of a 2^n array: out[rev_n(i)] = in[i].
//
// The reference keeps amplitudes MSB-first (qubit 0 = most significant index
// bit) and converts to Qiskit / PennyLane's little-endian order with a
// host-side index permutation (interop/qiskit_pennylane.py:115-136).  On the
// device the reversal is a transpose: with the index split as
// hi (top 5 bits) | mid (n-10 bits) | lo (low 5 bits),
// rev(i) = rev5(lo) | rev(mid) | rev5(hi), so a CTA loads the 32 x 32 block
// [hi][lo] of one mid value (32 coalesced rows of 32 elements) into shared
// memory and writes the block [rev5(lo)][rev5(hi)] at rev(mid) (again 32
// coalesced rows).  HBM-bound: one read and one write of the array.
#include "desv_common.cuh"

namespace desv {

__device__ __forceinline__ uint32_t rev5(uint32_t x) { return __brev(x) >> 27; }

template <typename T> __global__ void __launch_bounds__(256) k_bitrev_tiles(const T *in, T *out, int n) {
    __shared__ T tile[32][33];
    const int nm = n - 10;
    const uint64_t nmid = 1ull << nm;
    const uint32_t x = threadIdx.x, y = threadIdx.y;
    for (uint64_t m = blockIdx.x; m < nmid; m += gridDim.x) {
#pragma unroll
        for (uint32_t r = y; r < 32; r += 8) tile[r][x] = in[((uint64_t)r << (n - 5)) | (m << 5) | x];
        __syncthreads();
        const uint64_t rm = nm > 0 ? (__brevll(m) >> (64 - nm)) : 0ull;
        const uint32_t hi = rev5(x);
#pragma unroll
        for (uint32_t r = y; r < 32; r += 8) out[((uint64_t)r << (n - 5)) | (rm << 5) | x] = tile[hi][rev5(r)];
        __syncthreads();
    }
}

// small arrays (n < 10): one element per thread
template <typename T> __global__ void k_bitrev_small(const T *in, T *out, int n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (1u << n)) out[n ? (__brev(i) >> (32 - n)) : 0u] = in[i];
}

template <typename T> static int bitrev(const void *in, void *out, int n, cudaStream_t st) {
    const T *a = static_cast<const T *>(in);
    T *b = static_cast<T *>(out);
    if (n < 10) {
        k_bitrev_small<T><<<((1u << n) + 255) / 256, 256, 0, st>>>(a, b, n);
    } else {
        const uint64_t nmid = 1ull << (n - 10);
        const uint64_t cap = (uint64_t)sm_count() * 8;
        k_bitrev_tiles<T><<<(unsigned)(nmid < cap ? nmid : cap), dim3(32, 8), 0, st>>>(a, b, n);
    }
    return check_launch("bit reversal");
}

}  // namespace desv

using namespace desv;

extern "C" int desv_bit_reverse(const void *in, void *out, int n, int elem, void *stream) {
    if (!in || !out) return fail(DESV_EINVAL, "bit reversal: null array");
    if (in == out) return fail(DESV_EINVAL, "bit reversal: in and out must be distinct arrays");
    if (n < 0 || n > 34) return fail(DESV_EINVAL, "bit reversal: n must be in [0, 34]");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (elem) {
        case DESV_ELEM_F64: return bitrev<double>(in, out, n, st);
        case DESV_ELEM_C64: return bitrev<float2>(in, out, n, st);
        case DESV_ELEM_C128: return bitrev<double2>(in, out, n, st);
        default: return fail(DESV_EINVAL, "bit reversal: element kind must be DESV_ELEM_F64, _C64 or _C128");
    }
}

// ---------------------------------------------------------------------------
// Block swap of two device arrays: a[i] <-> b[i] for i < count (16-byte
// vectors; one read and one write of each element).  The split-state runner
// exchanges the upper half of one chunk with the lower half of its partner
// chunk with it when a chunk-select qubit trades places with the top local
// qubit (both halves are contiguous).
__global__ void __launch_bounds__(256) k_swap16(uint4 *a, uint4 *b, uint64_t count) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint4 x = a[i], y = b[i];
        a[i] = y;
        b[i] = x;
    }
}

extern "C" int desv_swap_blocks(void *a, void *b, size_t bytes, void *stream) {
    if (!a || !b) return fail(DESV_EINVAL, "block swap: null array");
    if (bytes == 0) return DESV_OK;
    if ((reinterpret_cast<uint64_t>(a) | reinterpret_cast<uint64_t>(b) | (uint64_t)bytes) & 15u)
        return fail(DESV_EINVAL, "block swap: arrays and size must be multiples of 16 bytes");
    const uint64_t a0 = reinterpret_cast<uint64_t>(a), b0 = reinterpret_cast<uint64_t>(b);
    if (a0 < b0 + bytes && b0 < a0 + bytes) return fail(DESV_EINVAL, "block swap: the arrays overlap");
    const uint64_t count = bytes / 16;
    const uint64_t blocks = (count + 255) / 256;
    const uint64_t cap = (uint64_t)sm_count() * 8;
    k_swap16<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<uint4 *>(a), static_cast<uint4 *>(b), count);
    return check_launch("block swap");
}
