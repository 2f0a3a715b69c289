// extern "C" entry points for rows: one circuit structure evaluated for many
// parameter rows, the rows' states stored back to back as full-width tensors
// (row r at r * 2^n amplitudes) and run by the tiled passes over all SMs, one
// grid row per state.  Replaces the reference's vmap over one circuit shape
// (backends/statevector.py:496-584, run_batch_jit) and, with the Pauli and
// adjoint entry points, energy + gradient per row (solvers/autodiff.py:92-169)
// for the circuits of a batch too wide to live in one CTA's shared memory.
// Argument validation and scratch layout here; kernels in k_fused.cu,
// k_pauli.cu, k_adjoint.cu and k_batch.cu.  Nothing here allocates.
#include <string>

#include "desv_common.cuh"
#include "tile_pipeline.cuh"

namespace desv {
int fused_pass_rows(void *, int, const TileGeom &, const desv_op *, int, const void *, int, const RowStrides &,
                    cudaStream_t);
int pauli_pass_rows(const void *, void *, int, int, const TileGeom &, const desv_pauli_term *, int, int, double *,
                    int *, int, const RowStrides &, cudaStream_t);
int pauli_direct_rows(const void *, void *, int, int, int, const desv_pauli_term *, int, int, double *, int *, int,
                      const RowStrides &, cudaStream_t);
int adjoint_pass_rows(void *, void *, int, const TileGeom &, const desv_op *, int, const void *, int, double *, int *,
                      int, const RowStrides &, cudaStream_t);
int grad_reduce_rows(const double *, int, int, const int32_t *, double *, int, int64_t, cudaStream_t);
int rows_prepare(int, const desv_batch_recipe *, int, const double *, int64_t, const void *, void *, int64_t, void *,
                 int, int, cudaStream_t);
int rows_norm(const void *, int, int, int, double *, double *, cudaStream_t);
int rows_sum(const double *, int64_t, int, int, double *, int, cudaStream_t);
int rows_tangent(void *, int64_t, int, int, const int32_t *, const uint8_t *, const uint32_t *, int64_t, double,
                 const uint8_t *, uint8_t *, cudaStream_t);
int jit_pauli_rows_launch(void *, const void *, void *, int, int, const TileGeom &, int, double *, int *, int,
                          const RowStrides &, const double *, int, cudaStream_t);

// partial-sum slots per state and pass (the rows grid bound of every kernel)
constexpr int ROWS_SLOTS = 64;

static inline cudaStream_t S(void *s) { return static_cast<cudaStream_t>(s); }

static int check_rows(const void *sv, int n, int dtype, int rows) {
    if (!sv) return fail(DESV_EINVAL, "rows: null state pointer");
    if (n < 1 || n > 34) return fail(DESV_EINVAL, "rows: n must be in [1, 34], got " + std::to_string(n));
    if (dtype != DESV_C64 && dtype != DESV_C128) return fail(DESV_EINVAL, "rows: dtype must be DESV_C64 or DESV_C128");
    if (rows < 1 || rows > 65535) return fail(DESV_EINVAL, "rows: row count must be in [1, 65535]");
    if (reinterpret_cast<uintptr_t>(sv) % 16) return fail(DESV_EINVAL, "rows: states must be 16-byte aligned");
    return DESV_OK;
}
}  // namespace desv

using namespace desv;

extern "C" {

size_t desv_rows_scratch_bytes(int rows, int max_params, int max_pauli_passes) {
    if (rows < 1) rows = 1;
    if (max_params < 0) max_params = 0;
    if (max_pauli_passes < 0) max_pauli_passes = 0;
    // Pauli: rows x (passes x SLOTS) x 2 partials + rows x SLOTS norm partials;
    // adjoint: rows x SLOTS x params of one pass (reduced before the next)
    const size_t pauli = (size_t)rows * ROWS_SLOTS * (2 * (size_t)max_pauli_passes + 1);
    const size_t adj = (size_t)rows * ROWS_SLOTS * (size_t)max_params;
    return 8 * (pauli > adj ? pauli : adj) + 256;
}

int desv_rows_prepare(void *states, int n, int dtype, int rows, const desv_batch_recipe *recipes, int nrec,
                      const double *theta, int64_t theta_stride, const void *cpool, void *pools, int64_t pool_stride,
                      void *stream) {
    int r = check_rows(states ? states : pools, n, dtype, rows);
    if (r) return r;
    if (nrec < 0 || (nrec && (!recipes || !theta || !cpool || !pools)))
        return fail(DESV_EINVAL, "rows prepare: null recipe arrays");
    if (theta_stride < 0 || pool_stride < 0) return fail(DESV_EINVAL, "rows prepare: negative stride");
    if (nrec == 0 && !states) return DESV_OK;
    return rows_prepare(dtype, recipes, nrec, theta, theta_stride, cpool, pools, pool_stride, states, n, rows,
                        S(stream));
}

int desv_rows_tangent_prepare(void *pools, int dtype, int rows, int64_t pool_stride, int npasses,
                              const int32_t *ev_begin_dev, const uint8_t *ev_kind_dev, const uint32_t *ev_off_dev,
                              int64_t end_base, double tmax, const uint8_t *allowed_dev, uint8_t *flags_dev,
                              void *stream) {
    if (dtype != DESV_C64) return fail(DESV_EINVAL, "rows tangent: complex64 pools only");
    if (!pools || !ev_begin_dev || !flags_dev || npasses < 0 || rows < 1 || rows > 65535 || pool_stride < 0 ||
        end_base < 0 || end_base + npasses > pool_stride || !(tmax > 0))
        return fail(DESV_EINVAL, "rows tangent: invalid arguments");
    return rows_tangent(pools, pool_stride, rows, npasses, ev_begin_dev, ev_kind_dev, ev_off_dev, end_base, tmax,
                        allowed_dev, flags_dev, S(stream));
}

int desv_apply_passes_rows(void *states, int n, int dtype, int rows, const desv_pass *passes, int npasses,
                           const desv_op *ops_dev, const void *pools, int64_t pool_stride, void *stream) {
    int r = check_rows(states, n, dtype, rows);
    if (r) return r;
    if (npasses < 0 || (npasses && (!passes || !ops_dev || !pools))) return fail(DESV_EINVAL, "rows: null pass arrays");
    if (pool_stride < 0) return fail(DESV_EINVAL, "rows: negative pool stride");
    const RowStrides rs{(int64_t)1 << n, pool_stride, 0, 0};
    for (int p = 0; p < npasses; ++p) {
        const desv_pass &ps = passes[p];
        TileGeom g;
        if (ps.tile_bits > n || ps.low_bits < 5 || ps.tile_bits - ps.low_bits > 16 ||
            !make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high))
            return fail(DESV_EINVAL, "rows pass " + std::to_string(p) + ": invalid tile geometry");
        if (ps.op_begin < 0 || ps.op_end < ps.op_begin) return fail(DESV_EINVAL, "rows pass op range invalid");
        if (ps.op_end == ps.op_begin) continue;
        r = fused_pass_rows(states, dtype, g, ops_dev + ps.op_begin, ps.op_end - ps.op_begin, pools, rows, rs,
                            S(stream));
        if (r) return r;
    }
    return DESV_OK;
}

// handles: NULL, or per pass a specialised rows kernel (or NULL: the
// interpreter runs that pass) reading csym (rows x nsym coefficients)
static int matvec_rows(void *const *handles, const double *csym, int nsym, const void *psi, void *out, int n,
                       int dtype, int rows, const desv_pauli_pass *passes, int npasses, const desv_pauli_term *terms,
                       int64_t term_stride, double *expect, double *norm, void *scratch, size_t sb, void *stream) {
    int r = check_rows(psi, n, dtype, rows);
    if (r) return r;
    if ((r = check_rows(out, n, dtype, rows))) return r;
    if (psi == out) return fail(DESV_EINVAL, "rows matvec: output must not alias the input");
    if (npasses < 0 || (npasses && (!passes || !terms))) return fail(DESV_EINVAL, "rows matvec: null Pauli arrays");
    if (term_stride < 0) return fail(DESV_EINVAL, "rows matvec: negative term stride");
    if ((expect || norm) && (!scratch || sb < desv_rows_scratch_bytes(rows, 0, npasses)))
        return fail(DESV_EINVAL, "rows matvec: scratch smaller than desv_rows_scratch_bytes(rows, 0, npasses)");
    const int64_t slots = (int64_t)ROWS_SLOTS * (npasses > 0 ? npasses : 1);
    double *part = static_cast<double *>(scratch);
    const RowStrides rs{(int64_t)1 << n, 0, term_stride, 2 * slots};
    int used = 0;
    bool wrote = false;
    for (int p = 0; p < npasses; ++p) {
        const desv_pauli_pass &ps = passes[p];
        if (ps.term_begin < 0 || ps.term_end < ps.term_begin) return fail(DESV_EINVAL, "rows matvec: term range invalid");
        const int nt = ps.term_end - ps.term_begin;
        if (nt == 0) continue;
        const int mode = wrote ? 2 : 1;
        int grid = 0;
        double *pp = part ? part + 2 * used : nullptr;
        if (ps.tile_bits == 0) {
            r = pauli_direct_rows(psi, out, dtype, mode, n, terms + ps.term_begin, nt, expect ? 1 : 0, pp, &grid, rows,
                                  rs, S(stream));
        } else {
            TileGeom g;
            if (ps.tile_bits > n || ps.low_bits < (n < 5 ? n : 5) || !make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high))
                return fail(DESV_EINVAL, "rows Pauli pass " + std::to_string(p) + ": invalid tile geometry");
            if (handles && handles[p])
                r = jit_pauli_rows_launch(handles[p], psi, out, dtype, mode, g, expect ? 1 : 0, pp, &grid, rows, rs,
                                          csym, nsym, S(stream));
            else
                r = pauli_pass_rows(psi, out, dtype, mode, g, terms + ps.term_begin, nt, expect ? 1 : 0, pp, &grid,
                                    rows, rs, S(stream));
        }
        if (r) return r;
        if (grid > ROWS_SLOTS) return fail(DESV_EINVAL, "rows matvec: grid above the partial-sum slots");
        used += grid;
        wrote = true;
    }
    if (!wrote) {
        const size_t es = dtype == DESV_C64 ? 8 : 16;
        if (cudaMemsetAsync(out, 0, (size_t)rows * ((size_t)1 << n) * es, S(stream)) != cudaSuccess)
            return check_launch("rows matvec zero");
    }
    if (expect) {
        if (used == 0) {
            if (cudaMemsetAsync(expect, 0, (size_t)rows * 2 * sizeof(double), S(stream)) != cudaSuccess)
                return check_launch("rows matvec: zero expectation");
        } else if ((r = rows_sum(part, 2 * slots, used, 2, expect, rows, S(stream)))) {
            return r;
        }
    }
    if (norm) {
        double *np = part + (size_t)rows * 2 * slots;
        if ((r = rows_norm(psi, n, dtype, rows, np, norm, S(stream)))) return r;
    }
    return DESV_OK;
}

int desv_pauli_matvec_rows(const void *psi, void *out, int n, int dtype, int rows, const desv_pauli_pass *passes,
                           int npasses, const desv_pauli_term *terms, int64_t term_stride, double *expect,
                           double *norm, void *scratch, size_t sb, void *stream) {
    return matvec_rows(nullptr, nullptr, 0, psi, out, n, dtype, rows, passes, npasses, terms, term_stride, expect, norm,
                       scratch, sb, stream);
}

int desv_jit_pauli_matvec_rows(void *const *handles, const double *csym, int nsym, const void *psi, void *out, int n,
                               int dtype, int rows, const desv_pauli_pass *passes, int npasses,
                               const desv_pauli_term *terms, int64_t term_stride, double *expect, double *norm,
                               void *scratch, size_t sb, void *stream) {
    if (!handles) return fail(DESV_EINVAL, "jit rows matvec: null handle array");
    if (nsym < 0 || (nsym > 0 && !csym)) return fail(DESV_EINVAL, "jit rows matvec: null coefficient table");
    return matvec_rows(handles, csym, nsym, psi, out, n, dtype, rows, passes, npasses, terms, term_stride, expect, norm,
                       scratch, sb, stream);
}

int desv_adjoint_passes_rows(void *phi, void *lam, int n, int dtype, int rows, const desv_adj_pass *passes,
                             int npasses, const desv_op *ops_dev, const void *pools, int64_t pool_stride,
                             const int32_t *map_dev, double *grad, int64_t grad_stride, void *scratch, size_t sb,
                             void *stream) {
    int r = check_rows(phi, n, dtype, rows);
    if (r) return r;
    if ((r = check_rows(lam, n, dtype, rows))) return r;
    if (phi == lam) return fail(DESV_EINVAL, "rows adjoint: phi and lambda must be distinct buffers");
    if (npasses < 0 || (npasses && (!passes || !ops_dev || !pools || !map_dev || !grad || !scratch)))
        return fail(DESV_EINVAL, "rows adjoint: null pass arrays");
    if (pool_stride < 0 || grad_stride < 0) return fail(DESV_EINVAL, "rows adjoint: negative stride");
    const RowStrides rs{(int64_t)1 << n, pool_stride, 0, 0};
    for (int p = 0; p < npasses; ++p) {
        const desv_adj_pass &ps = passes[p];
        TileGeom g;
        if (ps.tile_bits > n || ps.low_bits < 5 || !make_geom(g, n, ps.tile_bits, ps.low_bits, ps.high))
            return fail(DESV_EINVAL, "rows adjoint pass " + std::to_string(p) + ": invalid tile geometry");
        if (ps.op_begin < 0 || ps.op_end < ps.op_begin || ps.nparams < 0 || ps.map_begin < 0)
            return fail(DESV_EINVAL, "rows adjoint pass ranges invalid");
        if (sb < desv_rows_scratch_bytes(rows, ps.nparams, 0))
            return fail(DESV_EINVAL, "rows adjoint: scratch smaller than desv_rows_scratch_bytes(rows, params, 0)");
        if (ps.op_end == ps.op_begin) continue;
        int gx = 0;
        r = adjoint_pass_rows(phi, lam, dtype, g, ops_dev + ps.op_begin, ps.op_end - ps.op_begin, pools, ps.nparams,
                              static_cast<double *>(scratch), &gx, rows, rs, S(stream));
        if (r) return r;
        if (gx > ROWS_SLOTS) return fail(DESV_EINVAL, "rows adjoint: grid above the partial-sum slots");
        if (ps.nparams > 0) {
            r = grad_reduce_rows(static_cast<const double *>(scratch), gx, ps.nparams, map_dev + ps.map_begin, grad,
                                 rows, grad_stride, S(stream));
            if (r) return r;
        }
    }
    return DESV_OK;
}

}  // extern "C"
