/*
 * desv.h -- C ABI of libdesv.so, the B200 (sm_100a) dense statevector engine.
 *
 * Every entry point is stream-ordered on a caller-supplied cudaStream_t
 * (passed as void*; NULL = legacy default stream), takes device pointers the
 * caller owns, returns an int status (DESV_OK == 0, negative on error) and
 * never aborts.  desv_last_error() returns the message of the last failure on
 * the calling thread.  No entry point allocates device memory (except the
 * code of a module that desv_jit_load loads): reductions take a
 * caller-provided scratch buffer whose size desv_scratch_bytes() reports.
 *
 * Statevector layout: 2^n amplitudes, complex64 (float2) or complex128
 * (double2), interleaved re/im, MSB-first qubit order -- qubit q is bit
 * (n-1-q) of the amplitude index, as in the reference
 * (dense_evolution/backends/statevector.py:22-33, compiler.py:186-195).
 * All bit arguments below are INDEX BIT positions (0 = least significant);
 * the host library translates qubit -> bit.
 */
#ifndef DESV_H
#define DESV_H

#ifndef __CUDACC_RTC__
#include <stddef.h>
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DESV_ABI_VERSION 1

/* amplitude types */
#define DESV_C64 0
#define DESV_C128 1

/* status codes */
#define DESV_OK 0
#define DESV_EINVAL (-1)
#define DESV_ENOMEM (-2)
#define DESV_ETIMEOUT (-3)
#define DESV_ECUDA (-4)
#define DESV_EUNSUPPORTED (-5)

/* fused-pass op kinds (desv_op.kind) */
#define DESV_OP_STAGE 0 /* start of a register stage: g[0..3] = tile-local bit positions */
#define DESV_OP_M1 1    /* 2x2 on register slot s0 (0..3) or lane bit (s0 = 16 + bit, bit < 5) */
#define DESV_OP_M2 2    /* 4x4 on register slots s0 < s1 (reserved: the host lowers every two-qubit
                           gate to 2x2 / diagonal ops, and the pass kernels reject this kind) */
#define DESV_OP_DIAG 3  /* diagonal on global bits ga, gb: factor d[bit(ga) + 2*bit(gb)] */
#define DESV_OP_GRAD 4  /* adjoint passes only: add Re<lambda|G|phi> to gradient slot `param`;
                           s1 == 0: G = 2x2 generator on s0 (controls as M1),
                           s1 == 1: G = diagonal over ga/gb (as DIAG) */

/* desv_op.flags */
#define DESV_F_REAL 1   /* M1: all entries real */
#define DESV_F_DIAG 2   /* M1: off-diagonal entries zero */
#define DESV_F_PHASE1 4 /* M1: diagonal with m00 == 1 (only |1> rows change) */
#define DESV_F_ANTI 8   /* M1: diagonal entries zero (X, Y, controlled-X/Y) */
#define DESV_F_SIGN 16  /* DIAG: every factor is +1 or -1 */
#define DESV_F_PARAM 32 /* M1/DIAG (adjoint plans): this op carries gradient parameter `param` */

/* One register-stage op of a fused pass (40 bytes, little-endian, packed by
 * the host fusion pass -- dense_evolution/circuits/fusion.py). */
typedef struct desv_op {
    uint8_t kind;
    uint8_t flags;
    int8_t s0, s1;   /* M1 / M2 register slots (see kinds) */
    int8_t cslot;    /* M1: control on register slot (-1: none) */
    uint8_t ga, gb;  /* DIAG: global bit positions (0xFF: absent) */
    int8_t sa, sb;   /* DIAG: register slot holding ga / gb in this stage, -1 if thread-fixed */
    uint8_t g[4];    /* STAGE: tile-local bit positions of register slots 0..3 (ascending, >= 5) */
    uint8_t code[2]; /* host-computed dispatch code, little-endian (0: decode the fields):
                        1+S*5+V register slot S uncontrolled; 21+(S*4+CS)*2+(V!=ANTI) slot S
                        controlled by slot CS; 53+V lane bit uncontrolled; 58+(SA+1)*5+(SB+1)
                        sign-only diagonal; 83+(SA+1)*5+(SB+1) diagonal; |0x8000: cmask/cval
                        predicate applies.  V: 0 general, 1 real, 2 diagonal, 3 phase-on-|1>,
                        4 anti-diagonal (same priority as the flags PHASE1 > DIAG > ANTI > REAL).
                        Grouped ops (forward passes): 120+M general 2x2 on every register slot in
                        the 4-bit mask M, 136+M the same with real matrices (matrices consecutive,
                        ascending slot); 152 a group of s0 +-1 diagonals whose entries are uint32
                        words at the matrix offset: a | b << 8 | pattern << 16 with a, b = register
                        slot 0..3, 0x40 | global bit, or 0xFF (absent), pattern bit k negating
                        amplitudes with bit(a) + 2*bit(b) == k; 160+M general 2x2 on the register
                        slots in M and on the lane bits in the 5-bit mask s1 (slot matrices ascending
                        in packed form: per entry m the pair (re m, re m), (-im m, im m); then the
                        lane matrices ascending, plain), 176+M the same with real matrices stored
                        as (v, v) pairs, 4 elements per matrix; 154 a group of s0 diagonals, 5
                        elements per entry (header word a | b << 8 | kind << 16 | signs << 20, then
                        the 4 factors);
                        192 2x2 on lane bit s0-16 with a register control (cslot) and/or the
                        cmask/cval predicate.  Code 0 is invalid: the kernels skip the op and
                        set the bad-plan device status. */
    uint8_t pad0;
    uint32_t mat;    /* first complex element of this op's matrix in the matrix pool */
    int32_t param;   /* adjoint plans: gradient slot of this op (-1: none) */
    uint64_t cmask;  /* thread-level control: apply iff (index & cmask) == cval */
    uint64_t cval;   /* (cmask never covers this stage's register bits) */
} desv_op;

/* One fused pass: a tile of 2^tile_bits amplitudes = the low_bits contiguous
 * index bits plus the high[] bits; all ops [op_begin, op_end) run on the tile
 * in shared memory between one HBM read and one HBM write. */
typedef struct desv_pass {
    int32_t tile_bits; /* K, 9..12 (complex64) / 9..11 (complex128) */
    int32_t low_bits;  /* L >= 5 */
    int32_t op_begin, op_end;
    uint8_t high[16];  /* K - L global bit positions >= L, ascending */
} desv_pass;

/* One fused pass of the adjoint backward sweep over (phi, lambda): like
 * desv_pass, plus the gradient slots its GRAD ops use -- slot s adds into
 * grad[map[map_begin + s]]. */
typedef struct desv_adj_pass {
    int32_t tile_bits, low_bits, op_begin, op_end;
    uint8_t high[16];
    int32_t nparams, map_begin;
    int32_t pad[2];
} desv_adj_pass;

/* A Pauli term group of the fused Pauli kernels: all terms sharing one flip mask. */
typedef struct desv_pauli_term {
    uint64_t xmask; /* X|Y index bits: (P psi)[i] = psi[i ^ xmask] * ... */
    uint64_t zmask; /* Y|Z index bits: sign (-1)^popcount((i ^ xmask) & zmask) */
    double cre, cim; /* coefficient times i^(number of Y) */
} desv_pauli_term;

/* One tile pass of the Pauli kernels: terms [term_begin, term_end) whose flip
 * masks lie inside the tile (low_bits contiguous bits + high[]).  tile_bits
 * == 0 marks a direct pass for flip masks wider than any tile: partners are
 * then read straight from global memory. */
typedef struct desv_pauli_pass {
    int32_t tile_bits, low_bits, term_begin, term_end;
    uint8_t high[16];
} desv_pauli_pass;

/* ---- library ---------------------------------------------------------- */
int desv_abi_version(void);
int desv_last_error(char *buf, size_t len);
/* Reads (and clears) the device-side status word that bounded waits inside
 * kernels set instead of hanging; synchronizes `stream`. */
int desv_device_status(void *stream);
/* Bytes of scratch the reductions of an n-qubit state need. */
size_t desv_scratch_bytes(int n, int dtype);

/* ---- state (replaces DenseSVSimulator._reset_sv / set_initial_state,
 *      backends/statevector.py:101-137) ------------------------------------ */
int desv_init_basis(void *sv, int n, int dtype, uint64_t index, void *stream);
/* sv *= (re + i im)  (normalize, statevector.py:141-147) */
int desv_scale(void *sv, int n, int dtype, double re, double im, void *stream);

/* ---- gates (replaces apply_gate_1q/_2q, apply_cx/cz/rx/ry/rz,
 *      statevector.py:167-268, and one row of the compiled step
 *      _apply_gate_fast_step, circuits/compiler.py:136-315) -------------- */
/* ntargets 1 or 2; target_bits[0] is the LOW bit of the matrix index for 2
 * targets (row = 2*bit(target_bits[1]) + bit(target_bits[0])); mat is
 * row-major interleaved re,im doubles (8 or 32 values). */
int desv_apply_gate(void *sv, int n, int dtype, int ntargets, const int *target_bits,
                    uint64_t ctrl_mask, uint64_t ctrl_val, const double *mat, void *stream);

/* ---- fused passes (replaces the lax.scan over gate rows,
 *      circuits/compiler.py:318-355) ---------------------------------------- */
/* ops_dev / mats_dev: device arrays of desv_op and complex (float2 for C64,
 * double2 for C128); passes: HOST array. */
int desv_apply_passes(void *sv, int n, int dtype, const desv_pass *passes, int npasses,
                      const desv_op *ops_dev, const void *mats_dev, void *stream);

/* ---- adjoint gradient (replaces jax.grad through the lax.scan of
 *      solvers/autodiff.py:136-166) ----------------------------------------- */
size_t desv_adjoint_scratch_bytes(int max_params_per_pass);
/* Runs the backward passes in place on phi (circuit output, un-applied back
 * to the input) and lambda (H psi); grad_dev[map[...]] += 2 Re<lambda|G|phi>
 * per GRAD op (grad_dev is NOT zeroed here). */
int desv_adjoint_passes(void *phi, void *lam, int n, int dtype, const desv_adj_pass *passes, int npasses,
                        const desv_op *ops_dev, const void *mats_dev, const int32_t *map_dev, double *grad_dev,
                        void *scratch, size_t scratch_bytes, void *stream);

/* ---- batched VQE (replaces run_batch_jit's vmap over one circuit shape,
 *      backends/statevector.py:496-584, plus energy_fn + jax.grad per circuit,
 *      solvers/autodiff.py:92-169): energy and adjoint gradient of thousands of
 *      circuits of different qubit counts in one persistent launch. ------------ */

/* recipe kinds: how a record's matrix is made from theta on the device */
#define DESV_RCP_CONST 0     /* copy `count` complex values from cpool[src] */
#define DESV_RCP_RX 1        /* 2x2 RX(theta) */
#define DESV_RCP_RY 2        /* 2x2 RY(theta) */
#define DESV_RCP_RZ 3        /* 2x2 RZ(theta) */
#define DESV_RCP_P 4         /* 2x2 diag(1, e^{i theta}) */
#define DESV_RCP_RZ_TAB 5    /* 1-bit diagonal table of RZ(theta) */
#define DESV_RCP_P_TAB 6     /* 1-bit diagonal table of P(theta) */
#define DESV_RCP_CP_VEC 7    /* diagonal (1, 1, 1, e^{i theta}) */
#define DESV_RCP_CRZ_VEC 8   /* diagonal (1, e^{-i theta/2}, 1, e^{i theta/2}) */
#define DESV_RCP_PHASE_VEC 9 /* scalar e^{i theta} as a 4-entry diagonal */
#define DESV_RCP_INVERSE 0x100 /* use -theta (inverse gate) */

typedef struct desv_batch_recipe {
    uint32_t off;   /* destination in the circuit's pool (complex elements) */
    int32_t param;  /* theta index within the circuit (-1 for constants) */
    uint16_t kind;  /* DESV_RCP_* (| DESV_RCP_INVERSE) */
    uint16_t count; /* complex values written (constants) */
    uint32_t src;   /* constants: first value in cpool */
} desv_batch_recipe;

/* one circuit structure: forward passes, adjoint passes, recipes, Hamiltonian terms */
typedef struct desv_batch_plan {
    int32_t n;                   /* qubits, 9..34 */
    int32_t fwd_begin, fwd_end;  /* desv_pass rows of the forward circuit */
    int32_t bwd_begin, bwd_end;  /* desv_pass rows of the adjoint sweep (GRAD param = theta index) */
    int32_t rec_begin, rec_end;  /* recipes filling the circuit's pool */
    int32_t term_begin, term_end;/* Pauli terms (coefficient = cre/cim x the circuit's coef[k]) */
    int32_t nparams, pool_len, pad;
} desv_batch_plan;

typedef struct desv_batch_circuit {
    int32_t plan, out_index;     /* plan row; energy index */
    int64_t theta_off;           /* first parameter in theta */
    int64_t coef_off;            /* first term coefficient in coef */
    int64_t grad_off;            /* first gradient entry in grad */
    int64_t state_off;           /* forward-only plans (no terms, no adjoint passes): the circuit's
                                    final state goes to states + state_off (amplitudes); -1: none */
} desv_batch_circuit;

/* device pointers of one batch; workspace fields are filled by desv_batch_vqe */
typedef struct desv_batch_args {
    int32_t ncirc, pad;
    const desv_batch_circuit *circuits; /* processed in array order: sort by decreasing cost */
    const desv_batch_plan *plans;
    const desv_pass *passes;
    const desv_op *ops;
    const desv_batch_recipe *recipes;
    const void *cpool;                  /* float2 / double2 constants */
    const double *theta, *coef;
    const desv_pauli_term *terms;
    double *energy, *grad;
    void *workspace;
    uint64_t ws_amps;
    void *pool_ws;
    uint64_t pool_stride_bytes;
    void *states;                       /* forward-only circuits' output states (may be NULL) */
} desv_batch_args;

size_t desv_batch_workspace_bytes(int dtype, int max_n, int max_pool_len);
/* One persistent launch over every circuit of `args` (host struct of device
 * pointers).  Circuits of <= 12 qubits run in shared memory; larger ones
 * stream a per-CTA slice of `workspace`.  Capturable in a CUDA graph after a
 * first (warm-up) call.  Forward-only circuits (a plan without terms and
 * adjoint passes, state_off >= 0, args->states set: run_batch_jit's rows)
 * write their final state to args->states + state_off and, when wider than
 * 12 qubits, are evolved there in place, so max_n (which sizes the per-CTA
 * state slices) only has to cover the other circuits. */
int desv_batch_vqe(int dtype, int max_n, int max_pool_len, const desv_batch_args *args, void *workspace,
                   size_t workspace_bytes, void *stream);

/* ---- rows: one circuit structure for many parameter rows (replaces
 *      run_batch_jit's vmap over one circuit shape, backends/statevector.py:
 *      496-584, and energy_fn + jax.grad per row, solvers/autodiff.py:92-169,
 *      for circuits too wide for one CTA's shared memory).  The rows' states
 *      are full-width tensors back to back (row r at r * 2^n amplitudes); every
 *      pass covers all rows in one launch over all SMs, one grid row per state.
 *      rows is in [1, 65535]; pools, term tables and gradients are per row at
 *      the given strides. ------------------------------------------------------ */
/* scratch for the Pauli and adjoint rows calls below */
size_t desv_rows_scratch_bytes(int rows, int max_params_per_pass, int max_pauli_passes);
/* pools + r * pool_stride <- the recipes applied to theta + r * theta_stride
 * (pool_stride in complex elements); if states != NULL, every row's state is
 * set to |0...0>. */
int desv_rows_prepare(void *states, int n, int dtype, int rows, const desv_batch_recipe *recipes_dev, int nrec,
                      const double *theta_dev, int64_t theta_stride, const void *cpool_dev, void *pools_dev,
                      int64_t pool_stride, void *stream);
/* desv_apply_passes on every row, row r with the pool at pools + r * pool_stride */
int desv_apply_passes_rows(void *states, int n, int dtype, int rows, const desv_pass *passes, int npasses,
                           const desv_op *ops_dev, const void *pools_dev, int64_t pool_stride, void *stream);
/* out_r = H_r psi_r with row r's terms at terms + r * term_stride (records);
 * expect_dev[2r..2r+1] = <psi_r|H_r psi_r> and norm_dev[r] = <psi_r|psi_r>
 * when those pointers are not NULL (both overwritten). */
int desv_pauli_matvec_rows(const void *psi, void *out, int n, int dtype, int rows, const desv_pauli_pass *passes,
                           int npasses, const desv_pauli_term *terms_dev, int64_t term_stride, double *expect_dev,
                           double *norm_dev, void *scratch, size_t scratch_bytes, void *stream);
/* desv_pauli_matvec_rows with the tiled passes that have a specialised rows
 * kernel (handles[p] != NULL, desv_jit_load kind 3 / 4 for the first / later
 * passes, compiled with per-row coefficient symbols): such a kernel reads row
 * r's coefficients from csym_dev + r * nsym; the other passes run on the
 * interpreter from the term tables. */
int desv_jit_pauli_matvec_rows(void *const *handles, const double *csym_dev, int nsym, const void *psi, void *out,
                               int n, int dtype, int rows, const desv_pauli_pass *passes, int npasses,
                               const desv_pauli_term *terms_dev, int64_t term_stride, double *expect_dev,
                               double *norm_dev, void *scratch, size_t scratch_bytes, void *stream);
/* Tangent form of the rows' backward passes (complex64): per pass p and row r,
 * walks events [ev_begin[p], ev_begin[p+1]) -- kind 0 / 1: a tangent ry / rz
 * record at pool offset ev_off (its matrix replaced by t = s / c), kind 2 / 3:
 * a gradient probe whose generator is compiled in / read from the pool (the
 * probe's 1/S^2 correction written into its slot / scaled into its generator)
 * -- and writes the pass-end factor 1/S to end_base + p.  flags_dev[p * rows +
 * r] = 1 where row r runs pass p in tangent form; a row whose |t| leaves
 * [0, tmax] or whose S leaves [0, tmax^2] is left untouched (flag 0) and runs
 * the general kernel.  allowed_dev (NULL, or one byte per pass, the caller's
 * choice from the angles) replaces that check. */
int desv_rows_tangent_prepare(void *pools_dev, int dtype, int rows, int64_t pool_stride, int npasses,
                              const int32_t *ev_begin_dev, const uint8_t *ev_kind_dev, const uint32_t *ev_off_dev,
                              int64_t end_base, double tmax, const uint8_t *allowed_dev, uint8_t *flags_dev,
                              void *stream);
/* One rows backward pass with the row's form chosen per row: the tangent kernel
 * runs the rows whose rflag_dev entry is 1, the general kernel the others (both
 * launched, on one grid), then the per-row gradient reduction. */
int desv_jit_adjoint_rows_split(void *handle_tangent, void *handle_general, const unsigned char *rflag_dev,
                                void *phi, void *lam, int n, int dtype, int rows, const desv_adj_pass *pass,
                                const desv_op *ops_dev, const void *pools_dev, int64_t pool_stride,
                                const int32_t *map_dev, double *grad_dev, int64_t grad_stride, void *scratch,
                                size_t scratch_bytes, void *stream);
/* desv_adjoint_passes on every row: grad_dev[r * grad_stride + map[...]] +=
 * 2 Re<lambda_r|G|phi_r> (not zeroed here). */
int desv_adjoint_passes_rows(void *phi, void *lam, int n, int dtype, int rows, const desv_adj_pass *passes,
                             int npasses, const desv_op *ops_dev, const void *pools_dev, int64_t pool_stride,
                             const int32_t *map_dev, double *grad_dev, int64_t grad_stride, void *scratch,
                             size_t scratch_bytes, void *stream);

/* ---- reductions (FP64 accumulation; statevector.py:141-147,272-358,599-607,
 *      utils/measurement.py:71-94) ------------------------------------------ */
/* out_dev[0] = sum |a_i|^2 (double, device) */
int desv_norm2(const void *sv, int n, int dtype, double *out_dev, void *scratch, size_t scratch_bytes,
               void *stream);
/* out_dev[0..1] = <a|b> (re, im) */
int desv_inner(const void *a, const void *b, int n, int dtype, double *out_dev, void *scratch,
               size_t scratch_bytes, void *stream);
/* out_dev[b] = sum_i |a_i|^2 * bit_b(i) for every bit b < n, out_dev[n] = sum_i |a_i|^2 */
int desv_bit_marginals(const void *sv, int n, int dtype, double *out_dev, void *scratch,
                       size_t scratch_bytes, void *stream);
/* probs_dev[i] = |a_i|^2 (double) */
int desv_probabilities(const void *sv, int n, int dtype, double *probs_dev, void *stream);
/* measurement collapse: zero amplitudes whose bit `bit` != outcome, scale the rest by `scale` */
int desv_collapse(void *sv, int n, int dtype, int bit, int outcome, double scale, void *stream);

/* ---- finite-shot sampling (replaces the host path of sample_counts,
 *      utils/measurement.py:17-68: rng.choice over |a|^2) ------------------- */
size_t desv_sample_scratch_bytes(int n);
/* Block sums and CDF of |a_i|^2 in scratch (FP64); *total_dev = sum |a_i|^2. */
int desv_sample_prepare(const void *sv, int n, int dtype, void *scratch, size_t scratch_bytes, double *total_dev,
                        void *stream);
/* out_dev[s] = first index i with cumsum(|a|^2)[i] > u_dev[s] * total (numpy's
 * searchsorted(cdf, u, 'right')); needs the scratch of desv_sample_prepare. */
int desv_sample_pick(const void *sv, int n, int dtype, const void *scratch, size_t scratch_bytes,
                     const double *u_dev, int64_t nshots, int64_t *out_dev, void *stream);

/* ---- plan-specialised fused passes (the same work as desv_apply_passes for
 *      one pass, with the pass's op list compiled in).  The source is CUDA
 *      written against csrc/jit_pass.cuh; it is compiled with NVRTC for
 *      sm_100a and loaded into `device`'s primary context.  NVRTC and the
 *      driver are opened with dlopen on first use. ---------------------------- */
/* 1 if NVRTC and the CUDA driver could be opened; else 0 and the reason in why */
int desv_jit_available(char *why, size_t len);
/* Compile + load one pass kernel (entry point "desv_jit_kernel", tile shape
 * tile_bits / nbuf ring slots); kind 0: a fused pass (desv_jit_pass), kind 1:
 * an adjoint backward pass (desv_jit_adjoint), kind 2 + mode: a Pauli pass
 * (desv_jit_pauli).  include_dirs: directories
 * separated by ':'.  The NVRTC log goes to log (may be NULL). */
int desv_jit_load(const char *src, const char *include_dirs, int kind, int tile_bits, int nbuf, int dtype,
                  int device, void **handle, char *log, size_t loglen);
int desv_jit_free(void *handle);
/* Compile a pass source with NVRTC for sm_100a without loading it (needs no
 * GPU): DESV_OK or DESV_EINVAL with the compiler log in log. */
int desv_jit_compile_check(const char *src, const char *include_dirs, char *log, size_t loglen);
/* Run the loaded kernel over one pass (its tile geometry must match the
 * compiled tile_bits); mats_dev is the same matrix pool desv_apply_passes reads. */
int desv_jit_pass(void *handle, void *sv, int n, int dtype, const desv_pass *pass, const void *mats_dev,
                  void *stream);
/* desv_jit_pass on `rows` states back to back (row r at r * 2^n amplitudes),
 * row r with its pool at pools_dev + r * pool_stride (complex elements): the
 * specialised form of desv_apply_passes_rows for one pass. */
int desv_jit_pass_rows(void *handle, void *states, int n, int dtype, int rows, const desv_pass *pass,
                       const void *pools_dev, int64_t pool_stride, void *stream);
/* desv_pauli_expect (matvec == 0) or desv_pauli_matvec (matvec != 0) with the
 * tiled passes that have a specialised kernel (handles[p] != NULL, loaded with
 * kind 2 + the mode the pass runs in: 0 <H>; 1 the first H psi pass, 2 the
 * later ones) run through it; the other passes through the interpreter. */
int desv_jit_pauli(void *const *handles, const void *psi, void *out, int n, int dtype, const desv_pauli_pass *passes,
                   int npasses, const desv_pauli_term *terms, double *expect, void *scratch, size_t scratch_bytes,
                   int matvec, void *stream);
/* ---- interop (replaces _to_qiskit_bit_order, interop/qiskit_pennylane.py:115-136) */
/* element kinds of desv_bit_reverse */
#define DESV_ELEM_F64 0  /* probabilities */
#define DESV_ELEM_C64 1  /* complex64 amplitudes */
#define DESV_ELEM_C128 2 /* complex128 amplitudes */
/* out[rev_n(i)] = in[i] for i < 2^n: MSB-first (this engine, the reference)
 * <-> little-endian (Qiskit, PennyLane) index order.  Out of place; both
 * arrays on the device. */
int desv_bit_reverse(const void *in, void *out, int n, int elem, void *stream);

/* ---- split states (replaces the chunk-select exchange of
 *      backends/chunk/kernels.py:300-330, a ppermute per gate) -------------- */
/* a[i] <-> b[i] over `bytes` bytes (multiples of 16, non-overlapping device
 * arrays): the exchange of a chunk's upper half with its partner chunk's
 * lower half when a chunk-select qubit trades places with the top local
 * qubit. */
int desv_swap_blocks(void *a, void *b, size_t bytes, void *stream);

/* Rotation passes (complex64 forward passes of circuits lowered to real
 * rotations and diagonals; replaces the per-gate scan step of
 * circuits/compiler.py:136-355 like desv_jit_pass).  desv_rot_load compiles
 * one pass's generated source (entry point desv_rot_kernel, 2^(tile_bits-5)
 * threads, nbuf ring slots (1, 2 or 3, as the source was generated for), a
 * by-value parameter block of param_floats floats) for sm_100a;
 * desv_rot_pass runs it over the 2^n complex64 state sv with the pass's tile
 * geometry (tile_bits, low_bits, high[]; op_begin / op_end are not used) and
 * the per-call values params[0..param_floats) (host memory, copied by the
 * launch). */
int desv_rot_load(const char *src, const char *include_dirs, int tile_bits, int nbuf, int param_floats, int device,
                  void **handle, char *log, size_t loglen);
int desv_rot_pass(void *handle, void *sv, int n, const desv_pass *pass, const float *params, int param_floats,
                  void *stream);
/* One adjoint backward pass (the work of desv_adjoint_passes for that pass,
 * including the gradient reduction into grad_dev[map_dev[map_begin + p]]);
 * ops_dev is the whole op array (the compiled source indexes it absolutely). */
int desv_jit_adjoint(void *handle, void *phi, void *lam, int n, int dtype, const desv_adj_pass *pass,
                     const desv_op *ops_dev, const void *mats_dev, const int32_t *map_dev, double *grad_dev,
                     void *scratch, size_t scratch_bytes, void *stream);
/* desv_jit_adjoint on `rows` (phi, lambda) pairs back to back: the specialised
 * form of desv_adjoint_passes_rows for one pass (pools at pool_stride, row r's
 * gradient at grad_dev + r * grad_stride; scratch of desv_rows_scratch_bytes). */
int desv_jit_adjoint_rows(void *handle, void *phi, void *lam, int n, int dtype, int rows, const desv_adj_pass *pass,
                          const desv_op *ops_dev, const void *pools_dev, int64_t pool_stride,
                          const int32_t *map_dev, double *grad_dev, int64_t grad_stride, void *scratch,
                          size_t scratch_bytes, void *stream);

/* ---- Pauli sums (replaces pauli_sum_expectation / pauli_sum_matvec,
 *      physics/observables.py:63-186,250-308) ------------------------------- */
/* out_dev[0..1] = sum_k <psi|c_k P_k|psi> (re, im), FP64 accumulation.  The
 * passes only read psi and write disjoint partial rows, so pass p > 0 runs on
 * one of three library-owned side streams of the current device, forked from
 * `stream` and joined back into it by events before the final reduction: work
 * queued on `stream` afterwards sees the result as usual.  While `stream` is
 * being captured into a CUDA graph the passes run on `stream` in order.  The
 * same holds for desv_jit_pauli with matvec = 0. */
int desv_pauli_expect(const void *psi, int n, int dtype, const desv_pauli_pass *passes, int npasses,
                      const desv_pauli_term *terms_dev, double *out_dev, void *scratch,
                      size_t scratch_bytes, void *stream);
/* Allocation-free variant of desv_pauli_expect (no counterpart in the
 * reference: an addition for callers that cannot allocate device memory or
 * pass a scratch buffer, e.g. hosts whose allocator already owns all of HBM,
 * plugins that may not allocate after load, latency-critical loops).  Same
 * inputs and output minus the scratch: the per-CTA partial sums use a fixed
 * 256 KiB device array inside the library, held by every GPU that loads it
 * until exit.  At most 16384 / (8 x SMs) passes with terms (13 on a 148-SM
 * B200); more are rejected with DESV_EINVAL before any launch.  The first
 * call on a device looks the array up (cudaGetSymbolAddress): make it before
 * any stream capture.  Calls share the array: calls that overlap on the GPU
 * race and must be serialised. */
int desv_pauli_expect_noalloc(const void *psi, int n, int dtype, const desv_pauli_pass *passes, int npasses,
                              const desv_pauli_term *terms_dev, double *out_dev, void *stream);
/* out = H psi (overwrites out); if expect_dev != NULL also accumulates
 * <psi|H psi> into expect_dev[0..1] like desv_pauli_expect. */
int desv_pauli_matvec(const void *psi, void *out, int n, int dtype, const desv_pauli_pass *passes,
                      int npasses, const desv_pauli_term *terms_dev, double *expect_dev, void *scratch,
                      size_t scratch_bytes, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* DESV_H */
