// desv_pauli_expect_noalloc: <psi|H|psi> without any device allocation.
//
// Some callers cannot hand this library a scratch buffer or let it allocate
// one.  Examples: a host framework whose caching allocator has already
// reserved nearly all of HBM, so a cudaMalloc made behind its back fails or
// breaks its accounting; a plugin that may only allocate at load time; a
// latency-critical loop where cudaMalloc/cudaFree would synchronise the
// device.  This entry point takes only the inputs (psi, passes, terms) and
// the 2-double output.  The per-CTA partial sums of the reduction live in a
// fixed file-scope device array instead.
//
// Limits and rules:
//  * The array holds DESV_NOALLOC_PARTIAL_ROWS partial rows (2 doubles each,
//    256 KiB).  One Pauli pass uses at most PAULI_MAX_BLOCKS_PER_SM (8) x
//    (number of SMs) rows (1184 on a 148-SM B200; k_pauli.cu clamps every
//    Pauli grid to that bound), so a call may run at most 16384 / (8 x SMs)
//    passes with terms (13 on a B200); larger calls, and passes the kernels
//    would refuse (more than PAULI_MAX_TERMS terms, tiles too wide for the
//    precision), are rejected with DESV_EINVAL before any kernel is launched.
//  * Every GPU that loads the library keeps this array until the process exits.
//  * The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current).  Make
//    that first call before any stream capture.
//  * Every call on a device shares the one array, and the array keeps the
//    last call's partial sums.  Each call writes every row it later reads,
//    so no clearing is needed.  Calls that overlap on the GPU (two streams,
//    two host threads) race on the array: serialise them.
#include <mutex>
#include <string>

#include "desv_common.cuh"
#include "tile_pipeline.cuh"

#define DESV_NOALLOC_PARTIAL_ROWS 16384

namespace desv {

int pauli_pass(const void *, void *, int, int, const TileGeom &, const desv_pauli_term *, int, int, double *, int *,
               cudaStream_t);
int pauli_direct(const void *, void *, int, int, int, const desv_pauli_term *, int, int, double *, int *,
                 cudaStream_t);
__global__ void k_sum_rows(const double *, int, int, int, double *);

// Fixed scratch of the allocation-free Pauli expectation (see above).
static __device__ __align__(256) double g_noalloc_partials[2 * DESV_NOALLOC_PARTIAL_ROWS];

static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[64] = {nullptr};

// Device address of g_noalloc_partials on the current device.  The host-side
// name of the array is only a stand-in; the address a kernel may use comes
// from cudaGetSymbolAddress, looked up once per device.
static int noalloc_partials(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("noalloc: cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(DESV_EUNSUPPORTED, "noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p)
            return fail(DESV_ECUDA, std::string("noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return DESV_OK;
}

}  // namespace desv

using namespace desv;

extern "C" int desv_pauli_expect_noalloc(const void *psi, int n, int dtype, const desv_pauli_pass *passes,
                                         int npasses, const desv_pauli_term *terms, double *out, void *stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!psi || !out) return fail(DESV_EINVAL, "noalloc Pauli expectation: null psi or output");
    if (n < 1 || n > 34) return fail(DESV_EINVAL, "noalloc Pauli expectation: n must be in [1, 34]");
    if (dtype != DESV_C64 && dtype != DESV_C128) return fail(DESV_EINVAL, "noalloc Pauli expectation: bad dtype");
    if (reinterpret_cast<uintptr_t>(psi) % 16) return fail(DESV_EINVAL, "noalloc Pauli expectation: psi not 16-byte aligned");
    if (npasses < 0 || (npasses && (!passes || !terms))) return fail(DESV_EINVAL, "noalloc Pauli expectation: null pass arrays");
    // validate every pass and the scratch budget before launching anything
    const size_t rows_per_pass = (size_t)PAULI_MAX_BLOCKS_PER_SM * (size_t)sm_count();
    const int kmax = dtype == DESV_C64 ? 11 : 10;
    size_t budget = 0;
    for (int p = 0; p < npasses; ++p) {
        const desv_pauli_pass &ps = passes[p];
        if (ps.term_begin < 0 || ps.term_end < ps.term_begin)
            return fail(DESV_EINVAL, "noalloc Pauli expectation: term range invalid");
        if (ps.term_end == ps.term_begin) continue;
        if (ps.tile_bits != 0) {
            TileGeom g;
            if (ps.tile_bits > n || ps.tile_bits > kmax || ps.low_bits < (n < 5 ? n : 5) ||
                !make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high))
                return fail(DESV_EINVAL, "noalloc Pauli expectation: invalid tile geometry in pass " + std::to_string(p));
            if (ps.term_end - ps.term_begin > PAULI_MAX_TERMS)
                return fail(DESV_EINVAL, "noalloc Pauli expectation: more than " + std::to_string(PAULI_MAX_TERMS) +
                                             " terms in tiled pass " + std::to_string(p));
        }
        budget += rows_per_pass;
    }
    if (budget > DESV_NOALLOC_PARTIAL_ROWS)
        return fail(DESV_EINVAL, "noalloc Pauli expectation: " + std::to_string(budget / rows_per_pass) +
                                     " passes need more than the fixed " + std::to_string(DESV_NOALLOC_PARTIAL_ROWS) +
                                     " partial rows (at most " +
                                     std::to_string(DESV_NOALLOC_PARTIAL_ROWS / rows_per_pass) +
                                     " passes with terms on this GPU)");
    double *part = nullptr;
    int r = noalloc_partials(&part);
    if (r) return r;
    size_t rows = 0;
    for (int p = 0; p < npasses; ++p) {
        const desv_pauli_pass &ps = passes[p];
        const int nt = ps.term_end - ps.term_begin;
        if (nt == 0) continue;
        int grid = 0;
        if (ps.tile_bits == 0) {
            r = pauli_direct(psi, nullptr, dtype, 0, n, terms + ps.term_begin, nt, 1, part + 2 * rows, &grid, st);
        } else {
            TileGeom g;
            make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high);
            r = pauli_pass(psi, nullptr, dtype, 0, g, terms + ps.term_begin, nt, 1, part + 2 * rows, &grid, st);
        }
        if (r) return r;
        rows += grid;
    }
    if (rows == 0) {
        // no terms: the expectation is 0 (a memset of the caller's output, no allocation)
        if (cudaMemsetAsync(out, 0, 2 * sizeof(double), st) != cudaSuccess) return check_launch("noalloc zero");
        return DESV_OK;
    }
    k_sum_rows<<<1, 256, 0, st>>>(part, (int)rows, 2, 2, out);
    return check_launch("noalloc Pauli reduce");
}
