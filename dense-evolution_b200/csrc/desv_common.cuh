// Shared device helpers of libdesv: complex arithmetic, the sm_90+/sm_100
// bulk-copy (TMA, non-tensor) + mbarrier primitives written as inline PTX,
// bounded waits, and the host-side error plumbing.
#pragma once

#ifdef __CUDACC_RTC__
// Compiled at run time by NVRTC (plan-specialised pass kernels): no host
// headers; the fixed-width types come from here and the status word is the
// module's own, found by name through the driver.
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
extern "C" {
__device__ int desv_rtc_status = 0;
}
#define g_dev_status desv_rtc_status
#define DESV_DEV_TIMEOUT 1
#define DESV_DEV_BADPLAN 2
#include "desv.h"

namespace desv {
#else
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "desv.h"

namespace desv {

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int check_launch(const char *what);
int sm_count();

// Device-side status word: bounded waits set it instead of hanging.  Each
// translation unit has its own copy (no relocatable device code); every unit
// registers a reader with the API layer at load time.
#define DESV_DEV_TIMEOUT 1
#define DESV_DEV_BADPLAN 2
static __device__ int g_dev_status = 0;
void register_status_reader(int (*reader)());
static int tu_status_read_clear() {
    int h = 0;
    if (cudaMemcpyFromSymbol(&h, g_dev_status, sizeof(int)) != cudaSuccess) return 0;
    if (h) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_dev_status, &zero, sizeof(int));
    }
    return h;
}
static const int tu_status_registered = (register_status_reader(&tu_status_read_clear), 0);

// Pauli passes (k_pauli.cu): at most this many terms per tiled pass, and at
// most this many CTAs per SM in the grid of any Pauli pass (tiled or direct),
// so one pass writes at most PAULI_MAX_BLOCKS_PER_SM x SMs partial-sum rows.
constexpr int PAULI_MAX_TERMS = 512;
constexpr int PAULI_MAX_BLOCKS_PER_SM = 8;

// CTAs per row of a rows launch: enough rows x CTAs for about two waves of
// `resident` CTAs, at most one CTA per tile
inline int rows_grid_x(uint64_t tiles_per_row, uint64_t resident, int rows) {
    uint64_t gx = (2 * resident + (uint64_t)rows - 1) / (uint64_t)rows;
    if (gx > tiles_per_row) gx = tiles_per_row;
    return gx < 1 ? 1 : (int)gx;
}
#endif  // __CUDACC_RTC__

// Rows: several states of one qubit count stored back to back, each with its
// own matrix pool, term table and partial sums (one circuit structure run for
// many parameter rows).  A rows launch has one grid row (blockIdx.y) per state;
// its CTAs offset their pointers by blockIdx.y times these strides.  A
// single-state launch passes zeros and one grid row.
struct RowStrides {
    int64_t amps;   // amplitudes from one state to the next
    int64_t mats;   // complex matrix-pool elements from one row's pool to the next
    int64_t terms;  // Pauli term records from one row's table to the next
    int64_t part;   // doubles from one row's partial sums to the next
};

// ---------------------------------------------------------------- complex
template <typename R> struct CT;
template <> struct CT<float> { using T = float2; };
template <> struct CT<double> { using T = double2; };
template <typename R> using cx = typename CT<R>::T;

__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

// acc + a*b
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 acc) {
    return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y)));
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// real coefficient r times a, plus acc
__device__ __forceinline__ float2 rfma(float r, float2 a, float2 acc) {
    return make_float2(fmaf(r, a.x, acc.x), fmaf(r, a.y, acc.y));
}
__device__ __forceinline__ double2 rfma(double r, double2 a, double2 acc) {
    return make_double2(fma(r, a.x, acc.x), fma(r, a.y, acc.y));
}
template <typename T> __device__ __forceinline__ T cneg(T a) { a.x = -a.x; a.y = -a.y; return a; }

__device__ __forceinline__ float2 shfl_xor(float2 v, int m) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ double2 shfl_xor(double2 v, int m) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// insert a zero bit at position p of x
__device__ __forceinline__ uint64_t insert0(uint64_t x, int p) {
    uint64_t lo = x & ((1ull << p) - 1ull);
    return ((x >> p) << (p + 1)) | lo;
}

// ---------------------------------------------------------------- mbarrier / bulk copy (PTX ISA 8.0+, sm_90+)
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after ~`limit` polls (each try_wait itself blocks for a
// hardware-defined slice), records DESV_DEV_TIMEOUT and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit = (1u << 22)) {
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(&g_dev_status, DESV_DEV_TIMEOUT);
    return false;
}
// global -> shared bulk copy, completion counted on `bar` (bytes multiple of 16, both 16B aligned)
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// shared -> global bulk copy in the issuing thread's bulk group
__device__ __forceinline__ void bulk_s2g(void *dst_gmem, const void *src_smem, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem),
                 "r"(smem_addr(src_smem)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace desv
