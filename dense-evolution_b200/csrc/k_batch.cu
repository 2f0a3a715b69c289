// Batched VQE: energy + adjoint gradient of thousands of independent circuits
// of uneven qubit count in ONE persistent launch.
//
// The reference runs one parameter row at a time (run_batch_jit vmaps a single
// circuit structure with one qubit count, backends/statevector.py:496-584;
// energy + jax.grad per circuit, solvers/autodiff.py:92-169).  Here every CTA
// takes the next circuit from an atomic queue (the host orders circuits by
// decreasing cost) and runs, for that circuit alone:
//   1. its matrix pool, computed on the device from theta (recipes),
//   2. the fused forward passes (register-stage interpreter of the fused
//      kernel) on |0...0>,
//   3. lambda = H psi and E = <psi|lambda> (FP64),
//   4. the fused adjoint passes over (psi, lambda) with GRAD probes,
//      accumulating dE/dtheta per warp in FP64.
// Circuits of <= 2^RES amplitudes keep psi and lambda resident in shared memory
// for all four steps (no HBM traffic); larger ones stream tiles of a per-CTA
// workspace in HBM through shared memory pass by pass.
#include <cstdlib>

#include "desv_common.cuh"
#include "stage_ops.cuh"
#include "grad_ops.cuh"
#include "tile_pipeline.cuh"

namespace desv {

constexpr int BATCH_THREADS = 256;  // 2^(12-4): one register stage over a 2^12 tile
constexpr int BATCH_K = 12;         // tile bits of streamed circuits (and the largest resident state)
constexpr int BATCH_MAXP = 320;     // parameters per circuit
constexpr int BATCH_NW = BATCH_THREADS / 32;

template <typename T> __device__ __forceinline__ T cpx(double re, double im) {
    T r;
    r.x = (decltype(r.x))re;
    r.y = (decltype(r.y))im;
    return r;
}

// one recipe entry -> the circuit's pool
template <typename T>
__device__ __forceinline__ void run_recipe(const desv_batch_recipe &r, const double *theta, const T *cpool, T *pool) {
    T *o = pool + r.off;
    const int kind = r.kind & 0xFF;
    if (kind == DESV_RCP_CONST) {
        for (int e = 0; e < r.count; ++e) o[e] = cpool[r.src + e];
        return;
    }
    double th = theta[r.param];
    if (r.kind & DESV_RCP_INVERSE) th = -th;
    double s, c;
    sincos(0.5 * th, &s, &c);
    double s1, c1;
    sincos(th, &s1, &c1);
    switch (kind) {
        case DESV_RCP_RX: o[0] = cpx<T>(c, 0); o[1] = cpx<T>(0, -s); o[2] = cpx<T>(0, -s); o[3] = cpx<T>(c, 0); break;
        case DESV_RCP_RY: o[0] = cpx<T>(c, 0); o[1] = cpx<T>(-s, 0); o[2] = cpx<T>(s, 0); o[3] = cpx<T>(c, 0); break;
        case DESV_RCP_RZ: o[0] = cpx<T>(c, -s); o[1] = cpx<T>(0, 0); o[2] = cpx<T>(0, 0); o[3] = cpx<T>(c, s); break;
        case DESV_RCP_P: o[0] = cpx<T>(1, 0); o[1] = cpx<T>(0, 0); o[2] = cpx<T>(0, 0); o[3] = cpx<T>(c1, s1); break;
        case DESV_RCP_RZ_TAB: o[0] = cpx<T>(c, -s); o[1] = cpx<T>(c, s); o[2] = cpx<T>(c, -s); o[3] = cpx<T>(c, s); break;
        case DESV_RCP_P_TAB: o[0] = cpx<T>(1, 0); o[1] = cpx<T>(c1, s1); o[2] = cpx<T>(1, 0); o[3] = cpx<T>(c1, s1); break;
        case DESV_RCP_CP_VEC: o[0] = cpx<T>(1, 0); o[1] = cpx<T>(1, 0); o[2] = cpx<T>(1, 0); o[3] = cpx<T>(c1, s1); break;
        case DESV_RCP_CRZ_VEC: o[0] = cpx<T>(1, 0); o[1] = cpx<T>(c, -s); o[2] = cpx<T>(1, 0); o[3] = cpx<T>(c, s); break;
        case DESV_RCP_PHASE_VEC: o[0] = o[1] = o[2] = o[3] = cpx<T>(c1, s1); break;
        default: break;
    }
}

// One register stage of a pass over a tile in shared memory (optionally two
// arrays).  Threads >= 2^(K-4) only take part in the barriers.
template <typename T, bool ADJ>
__device__ __forceinline__ void batch_stage(T *s0, T *s1, const desv_op &st, const desv_op *ops, int cnt,
                                            const T *mats, uint64_t tg_base, const uint64_t *ctab, int L,
                                            int active, double *acc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if ((int)threadIdx.x < active) {
        const uint32_t idx = stage_base(threadIdx.x, st.g);
        const uint32_t o0 = 1u << st.g[0], o1 = 1u << st.g[1], o2 = 1u << st.g[2], o3 = 1u << st.g[3];
        T a[16], b[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const uint32_t off = idx + ((j & 1) ? o0 : 0u) + ((j & 2) ? o1 : 0u) + ((j & 4) ? o2 : 0u) + ((j & 8) ? o3 : 0u);
            a[j] = s0[off];
            if (ADJ) b[j] = s1[off];
        }
        const uint64_t tg = tg_base | tl2g(ctab, L, idx);
        if (!ADJ) {
            run_stage_ops(a, ops, cnt, mats, tg, lane);
        } else {
#pragma unroll 1
            for (int q = 0; q < cnt; ++q) {
                const desv_op &op = ops[q];
                if (op.kind == DESV_OP_GRAD) {
                    double v = grad_term(a, b, op, mats + op.mat, tg, lane);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    const int prm = op.param;
                    if (lane == 0 && prm >= 0 && prm < BATCH_MAXP) acc[warp * BATCH_MAXP + prm] += v;
                } else {
                    apply_op_at(a, ops + q, mats, tg, lane);
                    apply_op_at(b, ops + q, mats, tg, lane);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const uint32_t off = idx + ((j & 1) ? o0 : 0u) + ((j & 2) ? o1 : 0u) + ((j & 4) ? o2 : 0u) + ((j & 8) ? o3 : 0u);
            s0[off] = a[j];
            if (ADJ) s1[off] = b[j];
        }
    }
    __syncthreads();
}

// All stages of one pass on one tile already in shared memory.
template <typename T, bool ADJ>
__device__ void batch_tile(T *s0, T *s1, const desv_op *ops, int nops, const T *mats, uint64_t base,
                           const uint64_t *ctab, int K, int L, double *acc) {
    const int active = 1 << (K - 4);
    int k = 0;
    while (k < nops) {
        const desv_op &st = ops[k];
        const int cnt = (int)st.mat;
        batch_stage<T, ADJ>(s0, s1, st, ops + k + 1, cnt, mats, base, ctab, L, active, acc);
        k += 1 + cnt;
    }
}

// one pass over a state (resident: the state is the single tile)
template <typename T, bool ADJ>
__device__ void batch_pass(T *gpsi, T *glam, T *spsi, T *slam, bool resident, const desv_pass &ps, int n,
                           const desv_op *ops, const T *mats, double *acc, uint64_t *ctab) {
    TileGeom g;
    g.n = n;
    g.K = ps.tile_bits;
    g.L = ps.low_bits;
    for (int i = 0; i < g.K - g.L; ++i) g.high[i] = ps.high[i];
    {
        uint64_t tmask = (1ull << g.L) - 1ull;
        for (int i = 0; i < g.K - g.L; ++i) tmask |= 1ull << g.high[i];
        int r = 0;
        for (int b = 0; b < n; ++b)
            if (!((tmask >> b) & 1ull)) g.rest[r++] = (uint8_t)b;
        g.nrest = r;
    }
    const desv_op *pops = ops + ps.op_begin;
    const int nops = ps.op_end - ps.op_begin;
    // tiles must fit the shared-memory buffers and the 4-register-bit stages;
    // a resident state must be exactly one tile (host plans guarantee both)
    if (g.K < 9 || g.K > BATCH_K || (resident && g.K != n) || g.K > n || g.L < 5) {
        if (threadIdx.x == 0) atomicOr(&g_dev_status, DESV_DEV_BADPLAN);
        return;
    }
    // the pass's run table (global offset of each 2^L run of a tile); K - L <= 7
    const uint32_t TILE = 1u << g.K, chunk = 1u << g.L, nch = 1u << (g.K - g.L);
    for (uint32_t c = threadIdx.x; c < nch; c += blockDim.x) ctab[c] = chunk_offset(g, c);
    __syncthreads();
    if (resident) {
        batch_tile<T, ADJ>(spsi, slam, pops, nops, mats, 0, ctab, g.K, g.L, acc);
        __syncthreads();
        return;
    }
    // tile bases by a masked add over the rest bits
    uint64_t rmask = 0;
    for (int r = 0; r < g.nrest; ++r) rmask |= 1ull << g.rest[r];
    const uint64_t one = rmask & (0ull - rmask);  // deposit of tile index 1
    const uint32_t ntiles = 1u << (n - g.K);
    uint64_t base = 0;
    for (uint32_t t = 0; t < ntiles; ++t) {
        for (uint32_t e = threadIdx.x; e < TILE; e += blockDim.x) {
            const uint64_t gi = base + ctab[e >> g.L] + (e & (chunk - 1));
            spsi[e] = gpsi[gi];
            if (ADJ) slam[e] = glam[gi];
        }
        __syncthreads();
        batch_tile<T, ADJ>(spsi, slam, pops, nops, mats, base, ctab, g.K, g.L, acc);
        for (uint32_t e = threadIdx.x; e < TILE; e += blockDim.x) {
            const uint64_t gi = base + ctab[e >> g.L] + (e & (chunk - 1));
            gpsi[gi] = spsi[e];
            if (ADJ) glam[gi] = slam[e];
        }
        __syncthreads();
        base = ((base | ~rmask) + one) & rmask;
    }
}

// MINB: CTAs per SM the register allocation is bounded for (2: 128 registers
// a thread, two CTAs per SM; 1: up to 255 registers, no spills in the adjoint
// stages, one CTA per SM).  DESV_BATCH_MINB picks the instance at run time.
template <typename T, int MINB>
__global__ void __launch_bounds__(BATCH_THREADS, MINB) k_batch_vqe(desv_batch_args args, int *queue) {
    extern __shared__ __align__(128) unsigned char smem[];
    T *sA = reinterpret_cast<T *>(smem);
    T *sB = sA + (1u << BATCH_K);
    double *acc = reinterpret_cast<double *>(sB + (1u << BATCH_K));
    double *red = acc + BATCH_NW * BATCH_MAXP;
    __shared__ uint64_t s_ctab[1u << (BATCH_K - 5)];
    __shared__ int s_c;
    const int tid = threadIdx.x;
    T *wpsi = static_cast<T *>(args.workspace) + (size_t)blockIdx.x * 2 * args.ws_amps;
    T *wlam = wpsi + args.ws_amps;
    T *pool = reinterpret_cast<T *>(static_cast<char *>(args.pool_ws) + (size_t)blockIdx.x * args.pool_stride_bytes);
    const desv_batch_circuit *circs = args.circuits;
    for (;;) {
        if (tid == 0) s_c = atomicAdd(queue, 1);
        __syncthreads();
        const int c = s_c;
        __syncthreads();
        if (c >= args.ncirc) break;
        const desv_batch_circuit cd = circs[c];
        const desv_batch_plan pl = args.plans[cd.plan];
        const int n = pl.n;
        const uint64_t dim = 1ull << n;
        const bool resident = n <= BATCH_K;
        const double *theta = args.theta + cd.theta_off;
        // forward only (run_batch_jit rows): no terms and no adjoint passes; the
        // final state goes to the caller's output row (streamed states are
        // evolved there in place)
        const bool fwd_only = pl.term_end == pl.term_begin && pl.bwd_end == pl.bwd_begin && args.states != nullptr &&
                              cd.state_off >= 0;
        T *out_row = fwd_only ? static_cast<T *>(args.states) + cd.state_off : nullptr;
        // 1. matrices of this circuit
        for (int r = pl.rec_begin + tid; r < pl.rec_end; r += blockDim.x)
            run_recipe<T>(args.recipes[r], theta, static_cast<const T *>(args.cpool), pool);
        for (int i = tid; i < BATCH_NW * BATCH_MAXP; i += blockDim.x) acc[i] = 0.0;
        // 2. |0...0> and the forward passes
        T *gpsi = resident ? sA : (fwd_only ? out_row : wpsi);
        T *glam = resident ? sB : wlam;
        for (uint64_t i = tid; i < dim; i += blockDim.x) gpsi[i] = cpx<T>(i == 0 ? 1.0 : 0.0, 0.0);
        __threadfence_block();
        __syncthreads();
        for (int p = pl.fwd_begin; p < pl.fwd_end; ++p)
            batch_pass<T, false>(gpsi, glam, sA, sB, resident, args.passes[p], n, args.ops, pool, acc, s_ctab);
        if (fwd_only) {
            if (resident)
                for (uint64_t i = tid; i < dim; i += blockDim.x) out_row[i] = sA[i];
            __syncthreads();
            continue;
        }
        // 3. lambda = H psi, E = <psi|lambda>; complex64 circuits divide E (and
        // later the gradient) by the FP64 norm <psi|psi>, which is 1 in exact
        // arithmetic: that removes the first-order effect of the complex64
        // rounding drift of the norm from both
        double ere = 0, nrm = 0;
        for (uint64_t i = tid; i < dim; i += blockDim.x) {
            double2 v = make_double2(0.0, 0.0);
            for (int k = pl.term_begin; k < pl.term_end; ++k) {
                const desv_pauli_term tm = args.terms[k];
                const uint64_t src = i ^ tm.xmask;
                const T pz = gpsi[src];
                const double w = args.coef[cd.coef_off + (k - pl.term_begin)];
                double2 cc = make_double2(tm.cre * w, tm.cim * w);
                if (__popcll(src & tm.zmask) & 1) cc = cneg(cc);
                v = cfma(cc, make_double2((double)pz.x, (double)pz.y), v);
            }
            glam[i] = cpx<T>(v.x, v.y);
            const T a = gpsi[i];
            ere += (double)a.x * v.x + (double)a.y * v.y;
            nrm += (double)a.x * a.x + (double)a.y * a.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ere += __shfl_xor_sync(0xffffffffu, ere, o);
            nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
        }
        if ((tid & 31) == 0) {
            red[tid >> 5] = ere;
            red[BATCH_NW + (tid >> 5)] = nrm;
        }
        __threadfence_block();
        __syncthreads();
        double inv_norm = 1.0;
        if (sizeof(T) == sizeof(float2)) {
            double nn = 0;
            for (int w = 0; w < BATCH_NW; ++w) nn += red[BATCH_NW + w];
            inv_norm = nn > 0 ? 1.0 / nn : 1.0;
        }
        if (tid == 0) {
            double e = 0;
            for (int w = 0; w < BATCH_NW; ++w) e += red[w];
            args.energy[cd.out_index] = e * inv_norm;
        }
        // 4. adjoint sweep over (psi, lambda)
        for (int p = pl.bwd_begin; p < pl.bwd_end; ++p)
            batch_pass<T, true>(gpsi, glam, sA, sB, resident, args.passes[p], n, args.ops, pool, acc, s_ctab);
        __syncthreads();
        for (int q = tid; q < pl.nparams; q += blockDim.x) {
            double s = 0;
            for (int w = 0; w < BATCH_NW; ++w) s += acc[w * BATCH_MAXP + q];
            args.grad[cd.grad_off + q] = 2.0 * s * inv_norm;
        }
        __syncthreads();
    }
}

static size_t batch_smem_bytes(int dtype) {
    const size_t es = dtype == DESV_C64 ? 8 : 16;
    return 2 * ((size_t)1 << BATCH_K) * es + (size_t)BATCH_NW * BATCH_MAXP * 8 + 32 * 8;
}

// CTAs per SM of the register bound (DESV_BATCH_MINB=1 or 2, read once)
static int batch_minb() {
    static int v = 0;
    if (!v) {
        const char *e = getenv("DESV_BATCH_MINB");
        v = (e && e[0] == '1') ? 1 : 2;
    }
    return v;
}

template <typename T, int MINB> static void batch_attrs_t(size_t smem) {
    cudaFuncSetAttribute(k_batch_vqe<T, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

static void batch_attrs(int dtype) {
    static bool done[2][64] = {{false}};
    int dev = 0;
    cudaGetDevice(&dev);
    if (done[dtype][dev & 63]) return;
    const size_t smem = batch_smem_bytes(dtype);
    const bool one = batch_minb() == 1;
    if (dtype == DESV_C64) { if (one) batch_attrs_t<float2, 1>(smem); else batch_attrs_t<float2, 2>(smem); }
    else { if (one) batch_attrs_t<double2, 1>(smem); else batch_attrs_t<double2, 2>(smem); }
    done[dtype][dev & 63] = true;
}

template <typename T, int MINB> static int batch_occ(size_t smem) {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_vqe<T, MINB>, BATCH_THREADS, smem);
    return b;
}

int batch_max_ctas(int dtype) {
    static int cache[2][64] = {{0}};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cache[dtype][dev & 63]) return cache[dtype][dev & 63];
    batch_attrs(dtype);
    const size_t smem = batch_smem_bytes(dtype);
    const bool one = batch_minb() == 1;
    const int b = dtype == DESV_C64 ? (one ? batch_occ<float2, 1>(smem) : batch_occ<float2, 2>(smem))
                                    : (one ? batch_occ<double2, 1>(smem) : batch_occ<double2, 2>(smem));
    cache[dtype][dev & 63] = (b > 0 ? b : 1) * sm_count();
    return cache[dtype][dev & 63];
}

int batch_vqe(int dtype, const desv_batch_args &args, int *queue, int grid, cudaStream_t st) {
    batch_attrs(dtype);
    const size_t smem = batch_smem_bytes(dtype);
    const bool one = batch_minb() == 1;
    if (dtype == DESV_C64) {
        if (one) k_batch_vqe<float2, 1><<<grid, BATCH_THREADS, smem, st>>>(args, queue);
        else k_batch_vqe<float2, 2><<<grid, BATCH_THREADS, smem, st>>>(args, queue);
    } else {
        if (one) k_batch_vqe<double2, 1><<<grid, BATCH_THREADS, smem, st>>>(args, queue);
        else k_batch_vqe<double2, 2><<<grid, BATCH_THREADS, smem, st>>>(args, queue);
    }
    return check_launch("batched VQE");
}

int batch_max_params() { return BATCH_MAXP; }
int batch_resident_bits() { return BATCH_K; }

// ---------------------------------------------------------------------------
// Rows: one circuit structure evaluated for many parameter rows, every row's
// state a full-width tensor of its own (back to back), run by the tiled
// passes over all SMs with one grid row per state (k_fused_pass, k_pauli,
// k_adjoint_pass take RowStrides).  These kernels prepare the rows (matrix
// pools from theta, |0...0>) and reduce per-row partial sums.

// pools[r] <- recipes(theta[r]); states[r] <- |0...0> (states zeroed before)
template <typename T>
__global__ void k_rows_prepare(const desv_batch_recipe *rec, int nrec, const double *theta, int64_t theta_stride,
                               const T *cpool, T *pools, int64_t pool_stride, T *states, int64_t amps) {
    const int r = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nrec) run_recipe<T>(rec[i], theta + (size_t)r * theta_stride, cpool, pools + (size_t)r * pool_stride);
    if (states && i == 0) states[(size_t)r * amps] = cpx<T>(1.0, 0.0);
}

// per-row partial sums of <psi|psi> (FP64): grid (gx, rows)
template <typename T>
__global__ void __launch_bounds__(256) k_rows_norm(const T *sv, uint64_t amps, double *part, int64_t part_stride) {
    sv += blockIdx.y * amps;
    double s = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < amps; i += (uint64_t)gridDim.x * blockDim.x) {
        const T a = sv[i];
        s += (double)a.x * a.x + (double)a.y * a.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double sh[8];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        part[blockIdx.y * part_stride + blockIdx.x] = t;
    }
}

// out[r * width + c] = sum_s part[r * stride + s * width + c] for s < count (fixed order)
__global__ void k_rows_sum(const double *part, int64_t stride, int count, int width, double *out) {
    const int r = blockIdx.x;
    const double *p = part + (size_t)r * stride;
    __shared__ double sh[8];
    for (int c = 0; c < width; ++c) {
        double v = 0;
        for (int s = threadIdx.x; s < count; s += blockDim.x) v += p[(size_t)s * width + c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
            out[(size_t)r * width + c] = t;
        }
    }
}

// Tangent form of the rows' backward passes (the device side of the host's
// TangentPlan.transform, one thread per pass and row): event kinds 0 / 1 are
// the tangent ry / rz records (t from the record's matrix, the running product
// S of the 1/c), 2 / 3 the gradient probes with the generator compiled in /
// read from the pool (their 1/S^2 correction written into the slot / scaled
// into the generator), and the pass-end factor 1/S goes to end_base + pass.
// flags[pass * rows + row] says whether that row runs the pass in tangent form;
// a row whose |t| leaves [0, tmax] or whose S leaves [0, tmax^2] keeps its
// matrices and runs the general kernel.
__global__ void k_rows_tangent(float2 *pools, int64_t pool_stride, int rows, int npass, const int32_t *ev_begin,
                               const uint8_t *ev_kind, const uint32_t *ev_off, int64_t end_base, double tmax,
                               const uint8_t *allowed, uint8_t *flags) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)rows * npass) return;
    const int p = (int)(i / rows), r = (int)(i % rows);
    float2 *pool = pools + (size_t)r * pool_stride;
    const int b = ev_begin[p], e = ev_begin[p + 1];
    bool any = false, ok = true;
    double S = 1.0;
    for (int k = b; k < e && ok; ++k) {
        const int kind = ev_kind[k];
        if (kind > 1) continue;
        const uint32_t off = ev_off[k];
        const double c = pool[off].x;
        const double t = (kind == 0 ? (double)pool[off + 2].x : (double)pool[off].y) / c;
        any = true;
        S /= c;
        if (!(fabs(t) <= tmax) || !(fabs(S) <= tmax * tmax)) ok = false;
    }
    ok = ok && any;
    // allowed (one entry per pass, decided by the caller from the angles with a
    // margin): the caller's choice replaces the check
    if (allowed) ok = allowed[p] != 0 && any;
    flags[(size_t)p * rows + r] = ok ? 1 : 0;
    if (!ok) return;
    S = 1.0;
    for (int k = b; k < e; ++k) {
        const int kind = ev_kind[k];
        const uint32_t off = ev_off[k];
        if (kind <= 1) {
            const double c = pool[off].x;
            const double t = (kind == 0 ? (double)pool[off + 2].x : (double)pool[off].y) / c;
            pool[off] = make_float2((float)t, 0.f);
            S /= c;
        } else {
            const double corr = 1.0 / (S * S);
            if (kind == 2) {
                pool[off] = make_float2((float)corr, 0.f);
            } else {
                for (int q = 0; q < 4; ++q) {
                    pool[off + q].x = (float)((double)pool[off + q].x * corr);
                    pool[off + q].y = (float)((double)pool[off + q].y * corr);
                }
            }
        }
    }
    pool[end_base + p] = make_float2((float)(1.0 / S), 0.f);
}

int rows_tangent(void *pools, int64_t pool_stride, int rows, int npass, const int32_t *ev_begin, const uint8_t *ev_kind,
                 const uint32_t *ev_off, int64_t end_base, double tmax, const uint8_t *allowed, uint8_t *flags,
                 cudaStream_t st) {
    const int64_t total = (int64_t)rows * npass;
    if (total == 0) return DESV_OK;
    k_rows_tangent<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(static_cast<float2 *>(pools), pool_stride, rows,
                                                                     npass, ev_begin, ev_kind, ev_off, end_base, tmax,
                                                                     allowed, flags);
    return check_launch("rows: tangent form");
}

int rows_prepare(int dtype, const desv_batch_recipe *rec, int nrec, const double *theta, int64_t theta_stride,
                 const void *cpool, void *pools, int64_t pool_stride, void *states, int n, int rows, cudaStream_t st) {
    const size_t es = dtype == DESV_C64 ? 8 : 16;
    const uint64_t amps = 1ull << n;
    if (states && cudaMemsetAsync(states, 0, (size_t)rows * amps * es, st) != cudaSuccess)
        return check_launch("rows: zero states");
    const dim3 grid((unsigned)((nrec > 0 ? nrec : 1) + 127) / 128, (unsigned)rows);
    if (dtype == DESV_C64)
        k_rows_prepare<float2><<<grid, 128, 0, st>>>(rec, nrec, theta, theta_stride, static_cast<const float2 *>(cpool),
                                                     static_cast<float2 *>(pools), pool_stride,
                                                     static_cast<float2 *>(states), (int64_t)amps);
    else
        k_rows_prepare<double2><<<grid, 128, 0, st>>>(rec, nrec, theta, theta_stride,
                                                      static_cast<const double2 *>(cpool),
                                                      static_cast<double2 *>(pools), pool_stride,
                                                      static_cast<double2 *>(states), (int64_t)amps);
    return check_launch("rows: prepare");
}

// <psi_r|psi_r> for every row into out[r]; part holds rows x ROWS_NORM_X doubles
constexpr int ROWS_NORM_X = 32;
int rows_norm(const void *sv, int n, int dtype, int rows, double *part, double *out, cudaStream_t st) {
    const uint64_t amps = 1ull << n;
    const uint64_t blocks = (amps + 255) / 256;
    const int gx = (int)(blocks < (uint64_t)ROWS_NORM_X ? blocks : (uint64_t)ROWS_NORM_X);
    if (dtype == DESV_C64)
        k_rows_norm<float2><<<dim3(gx, rows), 256, 0, st>>>(static_cast<const float2 *>(sv), amps, part, ROWS_NORM_X);
    else
        k_rows_norm<double2><<<dim3(gx, rows), 256, 0, st>>>(static_cast<const double2 *>(sv), amps, part, ROWS_NORM_X);
    int r = check_launch("rows: norm");
    if (r) return r;
    k_rows_sum<<<rows, 256, 0, st>>>(part, ROWS_NORM_X, gx, 1, out);
    return check_launch("rows: norm reduce");
}

int rows_sum(const double *part, int64_t stride, int count, int width, double *out, int rows, cudaStream_t st) {
    k_rows_sum<<<rows, 256, 0, st>>>(part, stride, count, width, out);
    return check_launch("rows: reduce");
}

}  // namespace desv
