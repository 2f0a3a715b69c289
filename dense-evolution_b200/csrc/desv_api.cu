// extern "C" entry points of libdesv.so (declared in include/desv.h):
// argument validation, stream plumbing and error reporting.  Nothing here
// allocates device memory; nothing throws across the ABI.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "desv_common.cuh"
#include "tile_pipeline.cuh"

namespace desv {

static thread_local std::string t_last_error;

static std::mutex g_reader_mu;
static int (*g_readers[16])() = {nullptr};
static int g_nreaders = 0;
void register_status_reader(int (*reader)()) {
    std::lock_guard<std::mutex> lk(g_reader_mu);
    if (g_nreaders < 16) g_readers[g_nreaders++] = reader;
}

void set_error(const std::string &msg) { t_last_error = msg; }
int fail(int code, const std::string &msg) {
    set_error(msg);
    return code;
}
int check_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(DESV_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return DESV_OK;
}
int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cache[dev & 63] == 0) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cache[dev & 63] = v > 0 ? v : 1;
    }
    return cache[dev & 63];
}

// implemented in the kernel files
int init_basis(void *, int, int, uint64_t, cudaStream_t);
int scale(void *, int, int, double, double, cudaStream_t);
int probabilities(const void *, int, int, double *, cudaStream_t);
int collapse(void *, int, int, int, int, double, cudaStream_t);
int gate(void *, int, int, int, const int *, uint64_t, uint64_t, const double *, cudaStream_t);
int dot(const void *, const void *, int, int, int, double *, double *, cudaStream_t);
int marginals(const void *, int, int, double *, double *, cudaStream_t);
size_t scratch_bytes(int n);
int fused_pass(void *, int, const TileGeom &, const desv_op *, int, const void *, cudaStream_t);
int pauli_pass(const void *, void *, int, int, const TileGeom &, const desv_pauli_term *, int, int, double *, int *,
               cudaStream_t);
int pauli_direct(const void *, void *, int, int, int, const desv_pauli_term *, int, int, double *, int *,
                 cudaStream_t);
int adjoint_pass(void *, void *, int, const TileGeom &, const desv_op *, int, const void *, int, double *, int *,
                 cudaStream_t);
int grad_reduce(const double *, int, int, const int32_t *, double *, cudaStream_t);
size_t adjoint_scratch_bytes(int);
__global__ void k_sum_rows(const double *, int, int, int, double *);
int jit_pauli_launch(void *handle, const void *psi, void *out, int dtype, int mode, const TileGeom &g, int want_e,
                     double *part, int *grid_out, cudaStream_t st);

static inline cudaStream_t S(void *s) { return static_cast<cudaStream_t>(s); }

static int check_state(const void *sv, int n, int dtype) {
    if (!sv) return fail(DESV_EINVAL, "null statevector pointer");
    if (n < 1 || n > 34) return fail(DESV_EINVAL, "n must be in [1, 34], got " + std::to_string(n));
    if (dtype != DESV_C64 && dtype != DESV_C128) return fail(DESV_EINVAL, "dtype must be DESV_C64 or DESV_C128");
    if (reinterpret_cast<uintptr_t>(sv) % 16) return fail(DESV_EINVAL, "statevector must be 16-byte aligned");
    return DESV_OK;
}

static int check_scratch(const void *scratch, size_t bytes, int n) {
    if (!scratch || bytes < scratch_bytes(n))
        return fail(DESV_EINVAL, "scratch buffer missing or smaller than desv_scratch_bytes(n)");
    return DESV_OK;
}

}  // namespace desv

using namespace desv;

extern "C" {

int desv_abi_version(void) { return DESV_ABI_VERSION; }

int desv_last_error(char *buf, size_t len) {
    if (!buf || !len) return DESV_EINVAL;
    std::snprintf(buf, len, "%s", t_last_error.c_str());
    return DESV_OK;
}

int desv_device_status(void *stream) {
    int h = 0;
    if (cudaStreamSynchronize(S(stream)) != cudaSuccess) return check_launch("device status sync");
    {
        std::lock_guard<std::mutex> lk(g_reader_mu);
        for (int k = 0; k < g_nreaders; ++k) h |= g_readers[k]();
    }
    if (h & DESV_DEV_TIMEOUT) return fail(DESV_ETIMEOUT, "a bounded wait inside a kernel gave up");
    if (h & DESV_DEV_BADPLAN) return fail(DESV_EINVAL, "a kernel skipped a pass whose tile geometry it cannot run");
    return DESV_OK;
}

size_t desv_scratch_bytes(int n, int dtype) {
    (void)dtype;
    if (n < 1) n = 1;
    return scratch_bytes(n);
}

int desv_init_basis(void *sv, int n, int dtype, uint64_t index, void *stream) {
    int r = check_state(sv, n, dtype);
    if (r) return r;
    if (index >> n) return fail(DESV_EINVAL, "basis index out of range");
    return init_basis(sv, n, dtype, index, S(stream));
}

int desv_scale(void *sv, int n, int dtype, double re, double im, void *stream) {
    int r = check_state(sv, n, dtype);
    if (r) return r;
    return scale(sv, n, dtype, re, im, S(stream));
}

int desv_apply_gate(void *sv, int n, int dtype, int ntargets, const int *tb, uint64_t cmask, uint64_t cval,
                    const double *mat, void *stream) {
    int r = check_state(sv, n, dtype);
    if (r) return r;
    if (!tb || !mat) return fail(DESV_EINVAL, "null target or matrix pointer");
    if (ntargets != 1 && ntargets != 2) return fail(DESV_EINVAL, "ntargets must be 1 or 2");
    if (ntargets > n) return fail(DESV_EINVAL, "more targets than qubits");
    uint64_t tmask = 0;
    for (int k = 0; k < ntargets; ++k) {
        if (tb[k] < 0 || tb[k] >= n) return fail(DESV_EINVAL, "target bit out of range");
        if (tmask & (1ull << tb[k])) return fail(DESV_EINVAL, "target bits must differ");
        tmask |= 1ull << tb[k];
    }
    if ((cmask >> n) || (cmask & tmask) || (cval & ~cmask))
        return fail(DESV_EINVAL, "control mask overlaps targets or exceeds n bits");
    return gate(sv, n, dtype, ntargets, tb, cmask, cval, mat, S(stream));
}

int desv_apply_passes(void *sv, int n, int dtype, const desv_pass *passes, int npasses, const desv_op *ops_dev,
                      const void *mats_dev, void *stream) {
    int r = check_state(sv, n, dtype);
    if (r) return r;
    if (npasses < 0 || (npasses && (!passes || !ops_dev || !mats_dev))) return fail(DESV_EINVAL, "null pass arrays");
    for (int p = 0; p < npasses; ++p) {
        const desv_pass &ps = passes[p];
        TileGeom g;
        if (ps.tile_bits > n || ps.low_bits < 5 || ps.tile_bits - ps.low_bits > 16 ||
            !make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high))
            return fail(DESV_EINVAL, "pass " + std::to_string(p) + ": invalid tile geometry");
        if (ps.op_begin < 0 || ps.op_end < ps.op_begin) return fail(DESV_EINVAL, "pass op range invalid");
        if (ps.op_end == ps.op_begin) continue;
        r = fused_pass(sv, dtype, g, ops_dev + ps.op_begin, ps.op_end - ps.op_begin, mats_dev, S(stream));
        if (r) return r;
    }
    return DESV_OK;
}

size_t desv_adjoint_scratch_bytes(int max_params_per_pass) { return adjoint_scratch_bytes(max_params_per_pass); }

int desv_adjoint_passes(void *phi, void *lam, int n, int dtype, const desv_adj_pass *passes, int npasses,
                        const desv_op *ops_dev, const void *mats_dev, const int32_t *map_dev, double *grad_dev,
                        void *scratch, size_t sb, void *stream) {
    int r = check_state(phi, n, dtype);
    if (r) return r;
    if ((r = check_state(lam, n, dtype))) return r;
    if (phi == lam) return fail(DESV_EINVAL, "phi and lambda must be distinct buffers");
    if (npasses < 0 || (npasses && (!passes || !ops_dev || !mats_dev || !map_dev || !grad_dev || !scratch)))
        return fail(DESV_EINVAL, "null adjoint pass arrays");
    for (int p = 0; p < npasses; ++p) {
        const desv_adj_pass &ps = passes[p];
        TileGeom g;
        if (ps.tile_bits > n || ps.low_bits < 5 || !make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high))
            return fail(DESV_EINVAL, "adjoint pass " + std::to_string(p) + ": invalid tile geometry");
        if (ps.op_begin < 0 || ps.op_end < ps.op_begin || ps.nparams < 0 || ps.map_begin < 0)
            return fail(DESV_EINVAL, "adjoint pass ranges invalid");
        if (sb < adjoint_scratch_bytes(ps.nparams)) return fail(DESV_EINVAL, "adjoint scratch too small");
        if (ps.op_end == ps.op_begin) continue;
        int rows = 0;
        r = adjoint_pass(phi, lam, dtype, g, ops_dev + ps.op_begin, ps.op_end - ps.op_begin, mats_dev, ps.nparams,
                         static_cast<double *>(scratch), &rows, S(stream));
        if (r) return r;
        if (ps.nparams > 0) {
            r = grad_reduce(static_cast<const double *>(scratch), rows, ps.nparams, map_dev + ps.map_begin, grad_dev,
                            S(stream));
            if (r) return r;
        }
    }
    return DESV_OK;
}

int desv_norm2(const void *sv, int n, int dtype, double *out, void *scratch, size_t sb, void *stream) {
    int r = check_state(sv, n, dtype);
    if (r) return r;
    if ((r = check_scratch(scratch, sb, n))) return r;
    if (!out) return fail(DESV_EINVAL, "null output");
    return dot(sv, sv, n, dtype, 0, out, static_cast<double *>(scratch), S(stream));
}

int desv_inner(const void *a, const void *b, int n, int dtype, double *out, void *scratch, size_t sb, void *stream) {
    int r = check_state(a, n, dtype);
    if (r) return r;
    if ((r = check_state(b, n, dtype))) return r;
    if ((r = check_scratch(scratch, sb, n))) return r;
    if (!out) return fail(DESV_EINVAL, "null output");
    return dot(a, b, n, dtype, 1, out, static_cast<double *>(scratch), S(stream));
}

int desv_bit_marginals(const void *sv, int n, int dtype, double *out, void *scratch, size_t sb, void *stream) {
    int r = check_state(sv, n, dtype);
    if (r) return r;
    if ((r = check_scratch(scratch, sb, n))) return r;
    if (!out) return fail(DESV_EINVAL, "null output");
    return marginals(sv, n, dtype, out, static_cast<double *>(scratch), S(stream));
}

int desv_probabilities(const void *sv, int n, int dtype, double *out, void *stream) {
    int r = check_state(sv, n, dtype);
    if (r) return r;
    if (!out) return fail(DESV_EINVAL, "null output");
    return probabilities(sv, n, dtype, out, S(stream));
}

int desv_collapse(void *sv, int n, int dtype, int bit, int outcome, double s, void *stream) {
    int r = check_state(sv, n, dtype);
    if (r) return r;
    if (bit < 0 || bit >= n || (outcome != 0 && outcome != 1)) return fail(DESV_EINVAL, "bad bit or outcome");
    return collapse(sv, n, dtype, bit, outcome, s, S(stream));
}

// Side streams of the current device for the <H> passes: they only read psi and
// each writes its own partial rows, so pass p > 0 runs on side stream (p - 1) %
// PAULI_SIDE, forked from and joined back into the caller's stream by events.
// One pass's tail then overlaps the next pass's start.  The mutex is held from the
// fork to the join, so two host threads never interleave their event records.
constexpr int PAULI_SIDE = 3;
struct PauliSide {
    cudaStream_t s[PAULI_SIDE];
    cudaEvent_t fork, join[PAULI_SIDE];
    bool ok;
};
static std::mutex g_side_mu;

static PauliSide *pauli_side() {  // called with g_side_mu held
    static PauliSide side[64];
    static bool made[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return nullptr;
    }
    PauliSide &ps = side[dev];
    if (!made[dev]) {
        made[dev] = true;
        ps.ok = cudaEventCreateWithFlags(&ps.fork, cudaEventDisableTiming) == cudaSuccess;
        for (int k = 0; k < PAULI_SIDE && ps.ok; ++k)
            ps.ok = cudaStreamCreateWithFlags(&ps.s[k], cudaStreamNonBlocking) == cudaSuccess &&
                    cudaEventCreateWithFlags(&ps.join[k], cudaEventDisableTiming) == cudaSuccess;
        if (!ps.ok) cudaGetLastError();
    }
    return ps.ok ? &ps : nullptr;
}

// Whether the <H> passes may fork: not while the caller's stream is being captured
// into a graph (the capture would pull the side streams in), and only with a
// working set of side streams.
static PauliSide *pauli_fork(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (cs != cudaStreamCaptureStatusNone) return nullptr;
    PauliSide *ps = pauli_side();
    if (!ps) return nullptr;
    if (cudaEventRecord(ps->fork, st) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    for (int k = 0; k < PAULI_SIDE; ++k)
        if (cudaStreamWaitEvent(ps->s[k], ps->fork, 0) != cudaSuccess) return nullptr;
    return ps;
}

// handles: NULL, or one specialised kernel (or NULL) per pass (desv_jit_pauli)
static int pauli_common(const void *psi, void *out, int n, int dtype, const desv_pauli_pass *passes, int npasses,
                        const desv_pauli_term *terms, double *expect, void *scratch, size_t sb, bool matvec,
                        void *stream, void *const *handles = nullptr) {
    int r = check_state(psi, n, dtype);
    if (r) return r;
    if (matvec && (r = check_state(out, n, dtype))) return r;
    if (npasses < 0 || (npasses && (!passes || !terms))) return fail(DESV_EINVAL, "null Pauli pass arrays");
    const bool want_e = expect != nullptr;
    if (want_e && (r = check_scratch(scratch, sb, n))) return r;
    double *part = static_cast<double *>(scratch);
    const size_t cap_rows = sb / (2 * sizeof(double));
    size_t rows = 0;
    bool wrote = false;
    for (int p = 0; p < npasses; ++p) {
        const desv_pauli_pass &ps = passes[p];
        if (ps.term_begin < 0 || ps.term_end < ps.term_begin) return fail(DESV_EINVAL, "Pauli term range invalid");
        if (ps.tile_bits != 0) {
            TileGeom g;
            if (ps.tile_bits > n || ps.low_bits < (n < 5 ? n : 5) ||
                !make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high))
                return fail(DESV_EINVAL, "Pauli pass " + std::to_string(p) + ": invalid tile geometry");
        }
    }
    int launching = 0;
    for (int p = 0; p < npasses; ++p) launching += passes[p].term_end > passes[p].term_begin;
    // <H> alone: the passes are independent reads of psi, run concurrently
    std::unique_lock<std::mutex> side_lock(g_side_mu, std::defer_lock);
    PauliSide *side = nullptr;
    if (!matvec && launching > 1) {
        side_lock.lock();
        side = pauli_fork(S(stream));
        if (!side) side_lock.unlock();
    }
    int launched = 0;
    for (int p = 0; p < npasses && !r; ++p) {
        const desv_pauli_pass &ps = passes[p];
        const int nt = ps.term_end - ps.term_begin;
        if (nt == 0 && (!matvec || wrote)) continue;
        if (want_e && rows + 4096 > cap_rows) {
            r = fail(DESV_EINVAL, "scratch too small for this many Pauli passes");
            break;
        }
        const int mode = matvec ? (wrote ? 2 : 1) : 0;
        const cudaStream_t ls = side && launched > 0 ? side->s[(launched - 1) % PAULI_SIDE] : S(stream);
        int grid = 0;
        if (ps.tile_bits == 0) {  // flip masks wider than a tile: global-memory partner reads
            r = pauli_direct(psi, out, dtype, mode, n, terms + ps.term_begin, nt, want_e ? 1 : 0, part + 2 * rows,
                             &grid, ls);
        } else {
            TileGeom g;
            make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high);
            if (handles && handles[p])
                r = jit_pauli_launch(handles[p], psi, out, dtype, mode, g, want_e ? 1 : 0, part + 2 * rows, &grid, ls);
            else
                r = pauli_pass(psi, out, dtype, mode, g, terms + ps.term_begin, nt, want_e ? 1 : 0,
                               part + 2 * rows, &grid, ls);
        }
        if (r) break;
        if (want_e) rows += grid;
        wrote = true;
        ++launched;
    }
    if (side) {  // join every side stream back into the caller's stream, also on an error
        for (int k = 0; k < PAULI_SIDE; ++k) {
            cudaEventRecord(side->join[k], side->s[k]);
            cudaStreamWaitEvent(S(stream), side->join[k], 0);
        }
        side_lock.unlock();
    }
    if (r) return r;
    if (matvec && !wrote) {
        const size_t es = dtype == DESV_C64 ? 8 : 16;
        if (cudaMemsetAsync(out, 0, (1ull << n) * es, S(stream)) != cudaSuccess) return check_launch("matvec zero");
    }
    if (want_e) {
        if (rows == 0) {
            if (cudaMemsetAsync(expect, 0, 2 * sizeof(double), S(stream)) != cudaSuccess) return check_launch("zero");
            return DESV_OK;
        }
        k_sum_rows<<<1, 256, 0, S(stream)>>>(part, (int)rows, 2, 2, expect);
        return check_launch("Pauli reduce");
    }
    return DESV_OK;
}

int desv_pauli_expect(const void *psi, int n, int dtype, const desv_pauli_pass *passes, int npasses,
                      const desv_pauli_term *terms, double *out, void *scratch, size_t sb, void *stream) {
    if (!out) return fail(DESV_EINVAL, "null output");
    return pauli_common(psi, nullptr, n, dtype, passes, npasses, terms, out, scratch, sb, false, stream);
}

int desv_pauli_matvec(const void *psi, void *out, int n, int dtype, const desv_pauli_pass *passes, int npasses,
                      const desv_pauli_term *terms, double *expect, void *scratch, size_t sb, void *stream) {
    if (psi == out) return fail(DESV_EINVAL, "matvec output must not alias the input");
    return pauli_common(psi, out, n, dtype, passes, npasses, terms, expect, scratch, sb, true, stream);
}

int desv_jit_pauli(void *const *handles, const void *psi, void *out, int n, int dtype, const desv_pauli_pass *passes,
                   int npasses, const desv_pauli_term *terms, double *expect, void *scratch, size_t sb, int matvec,
                   void *stream) {
    if (!handles) return fail(DESV_EINVAL, "jit Pauli: null handle array");
    if (matvec) {
        if (psi == out) return fail(DESV_EINVAL, "matvec output must not alias the input");
    } else if (!expect) {
        return fail(DESV_EINVAL, "null output");
    }
    return pauli_common(psi, matvec ? out : nullptr, n, dtype, passes, npasses, terms, expect, scratch, sb,
                        matvec != 0, stream, handles);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batched VQE
namespace desv {
int batch_vqe(int, const desv_batch_args &, int *, int, cudaStream_t);
int batch_max_ctas(int);
int batch_max_params();
int batch_resident_bits();

static void batch_layout(int dtype, int max_n, int max_pool, int ctas, size_t *ws_state, size_t *ws_pool,
                         size_t *pool_stride, uint64_t *ws_amps) {
    const size_t es = dtype == DESV_C64 ? 8 : 16;
    *ws_amps = max_n > batch_resident_bits() ? (1ull << max_n) : 0ull;
    *ws_state = (size_t)ctas * 2 * (size_t)(*ws_amps) * es;
    *pool_stride = (((size_t)max_pool * es) + 255) / 256 * 256;
    *ws_pool = (size_t)ctas * (*pool_stride);
}
}  // namespace desv

extern "C" {

size_t desv_batch_workspace_bytes(int dtype, int max_n, int max_pool_len) {
    if ((dtype != DESV_C64 && dtype != DESV_C128) || max_n < 1 || max_n > 34 || max_pool_len < 0) return 0;
    const int ctas = batch_max_ctas(dtype);
    size_t st, pl, stride;
    uint64_t amps;
    batch_layout(dtype, max_n, max_pool_len, ctas, &st, &pl, &stride, &amps);
    return 256 + st + pl;
}

int desv_batch_vqe(int dtype, int max_n, int max_pool_len, const desv_batch_args *args, void *workspace,
                   size_t workspace_bytes, void *stream) {
    if (dtype != DESV_C64 && dtype != DESV_C128) return fail(DESV_EINVAL, "batch: bad dtype");
    if (!args || !workspace) return fail(DESV_EINVAL, "batch: null args or workspace");
    if (max_n < 9 || max_n > 30) return fail(DESV_EINVAL, "batch: max_n must be in [9, 30]");
    if (args->ncirc < 0) return fail(DESV_EINVAL, "batch: negative circuit count");
    if (args->ncirc == 0) return DESV_OK;
    if (!args->circuits || !args->plans || !args->passes || !args->ops || !args->recipes || !args->cpool ||
        !args->theta || !args->energy || !args->grad)
        return fail(DESV_EINVAL, "batch: null device array in args");
    const int ctas = batch_max_ctas(dtype);
    size_t st, pl, stride;
    uint64_t amps;
    batch_layout(dtype, max_n, max_pool_len, ctas, &st, &pl, &stride, &amps);
    if (workspace_bytes < 256 + st + pl) return fail(DESV_EINVAL, "batch: workspace smaller than desv_batch_workspace_bytes");
    if (reinterpret_cast<uintptr_t>(workspace) % 256) return fail(DESV_EINVAL, "batch: workspace must be 256-byte aligned");
    desv_batch_args a = *args;
    char *w = static_cast<char *>(workspace);
    int *queue = reinterpret_cast<int *>(w);
    a.workspace = w + 256;
    a.ws_amps = amps;
    a.pool_ws = w + 256 + st;
    a.pool_stride_bytes = stride;
    if (cudaMemsetAsync(queue, 0, sizeof(int), S(stream)) != cudaSuccess) return check_launch("batch queue reset");
    int grid = ctas < args->ncirc ? ctas : args->ncirc;
    return batch_vqe(dtype, a, queue, grid, S(stream));
}

}  // extern "C"
